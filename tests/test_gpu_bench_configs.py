"""Bit-exact parity at the sizes the benchmark times and the serving trace
serves, word for word against the oracle (mod q, as the reference's
testbench compares: hardware/u55c/hls/tb/tb_par1_mkf_ckks.cpp:46-63):

* the benchmarked product, MKF-CKKS mult+relin+rescale+materialize at
  logN 16, k = 8, 24 Q limbs (top level) and 9 (level 8)
  (software/mkf/mkf_cpu/ckks.go:102-166);
* KKLSS-CKKS mult+relin+rescale at k = 8 on the serving rings of logN 14, 15
  and 16 (software/kklss/mkckks/evaluator.go:419-446);
* KKLSS-BFV mult+relin at k = 8 on the logN 14, 15 and 16 serving rings
  and at k = 4 on C2 (the logN 15 chain of fifteen 58-bit primes)
  (software/kklss/mkbfv/evaluator.go:85-152).

The oracle runs in spawned worker processes (one case each) while the test
process builds the same seeded case and runs it on the GPU.
"""
import concurrent.futures as cf
import multiprocessing as mp
import os

import numpy as np
import pytest

from mkf_b200 import autotune
from mkf_b200 import evaluator as ev
from oracle import keygen as kg
from tests import bench_cases as BC
from tests import helpers as H
from tests.test_gpu_parity import _kklss_rlkset, assert_eq_mod

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_results():
    """Every case's oracle output, computed in parallel in spawned workers."""
    workers = max(1, min(len(BC.CASES), (os.cpu_count() or 2) - 1, 9))
    ex = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"))
    futs = {name: ex.submit(BC.oracle_output, name) for name in BC.CASES}
    yield futs
    ex.shutdown(wait=True, cancel_futures=True)


_CTX = {}


def _params(lit, scheme):
    key = (lit.name, scheme)
    if key not in _CTX:
        _CTX.clear()  # one large context at a time
        _CTX[key] = ev.Parameters(lit, scheme)
    return _CTX[key]


@pytest.mark.parametrize("name", ["mkf_ckks_c3_k8_top", "mkf_ckks_c3_k8_l8"])
def test_mkf_ckks_c3_k8_bitexact(name, oracle_results):
    case = BC.build(name)
    lit = case.lit
    P = _params(lit, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    left = ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale)
    right = ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale)
    want, lv, sc = oracle_results[name].result()
    # both inner-product forms the autotuner chooses between: stand-alone,
    # and fused into the digits' row pass (the benchmark's choice)
    for fuse in (0, 1):
        autotune.set_tuning(P, fuse_ip=fuse)
        out = E.MulRelinNew(left, right, materialize=True)
        got = out.download()
        assert out.Level() == lv == case.level - 1
        assert abs(out.Scale - sc) <= 1e-9 * sc
        assert got.shape[0] == case.k + 1
        # the materialized form: C0, then Gamma once per party
        assert_eq_mod(got[:2], want, lit.q[: lv + 1])
        for i in range(2, case.k + 1):
            assert np.array_equal(got[i], got[1])
    assert kg.precision_bits(H.mkf_ckks_decode(case, got, lv, sc), case.want) > 20


@pytest.mark.parametrize("name", ["kklss_ckks_s14_k8_top", "kklss_ckks_s15_k8_l9",
                                  "kklss_ckks_s16_k8_top"])
def test_kklss_ckks_serving_rings_bitexact(name, oracle_results):
    case = BC.build(name)
    lit, k = case.lit, case.k
    P = _params(lit, "ckks")
    rs = _kklss_rlkset(P, case, range(k))
    a = ev.Ciphertext.from_array(P, case.op0, False, ids=list(range(k)), scale=lit.scale)
    b = ev.Ciphertext.from_array(P, case.op1, False, ids=list(range(k)), scale=lit.scale)
    out = ev.Evaluator(P).MulRelinNew(a, b, rs)
    got = out.download()
    want, lv, sc = oracle_results[name].result()
    assert out.Level() == lv and out.ids == list(range(k))
    assert_eq_mod(got, want, lit.q[: lv + 1])
    assert kg.precision_bits(H.kklss_ckks_decode(case, got, lv, sc), case.want) > 15


@pytest.mark.parametrize("name", ["kklss_bfv_s14_k8", "kklss_bfv_c2_k4", "kklss_bfv_s15_k8",
                                  "kklss_bfv_s16_k8"])
def test_kklss_bfv_serving_rings_bitexact(name, oracle_results):
    case = BC.build(name)
    lit, k = case.lit, case.k
    P = _params(lit, "bfv")
    rs = _kklss_rlkset(P, case, range(k))
    a = ev.Ciphertext.from_array(P, case.op0, False, ids=list(range(k)))
    b = ev.Ciphertext.from_array(P, case.op1, False, ids=list(range(k)))
    got = ev.Evaluator(P).MulRelinNew(a, b, rs).download()
    want, _, _ = oracle_results[name].result()
    assert_eq_mod(got, want, lit.q)
    # the messages are sparse, so the exact plaintext product is known
    assert np.array_equal(H.kklss_bfv_decrypt(case, got), case.want)
