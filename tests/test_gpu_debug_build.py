"""The debug build of the library (bounds checks in the kernels, canary words
after every scratch allocation) on small parity cases: every output equals
the oracle's and no check fires.  compute-sanitizer is not available on this
GPU pool, so these checks stand in for it.  A canary overwrite planted from
the host (an in-bounds memset of the workspace, never a faulting access)
must be reported."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_FAILED = 10
CANARY_TAG = 0x0C000000


def _run(code_or_module, env_extra, timeout=900):
    env = dict(os.environ, MKF_B200_LIB="debug", **env_extra)
    args = [sys.executable, "-m", code_or_module] if not code_or_module.startswith("-c") else \
        [sys.executable, "-c", code_or_module[2:]]
    r = subprocess.run(args, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_debug_build_parity_and_clean_checks():
    res = _run("tests.debug_cases", {})
    for name, r in res.items():
        assert r["parity"], f"{name}: output differs from the oracle"
        assert r["status"] == 0 and r["report"][0] == 0, f"{name}: check failed {r['report']}"


PLANT = """
import ctypes, json
from mkf_b200 import capi, params
from mkf_b200 import evaluator as ev
from tests import helpers as H
lit = params.small("ckks", log_n=12, n_q=4, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                   scale_bits=45)
case = H.mkf_ckks_case(lit, 2, 3)
P = ev.Parameters(lit, "ckks")
E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
E.MulRelinNew(ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale),
              ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale)).download()
rep = (ctypes.c_uint64 * 4)()
st = capi.lib().mkf_debug_status(0, rep)
print(json.dumps({"status": st, "report": [int(x) for x in rep]}))
"""


def test_debug_build_reports_a_planted_canary_overwrite():
    r = _run("-c" + PLANT, {"MKF_DEBUG_PLANT_CANARY": "1"})
    assert r["status"] == CHECK_FAILED
    assert r["report"][0] >= 1 and (r["report"][1] & 0xFF000000) == CANARY_TAG
