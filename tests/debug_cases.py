"""Small parity cases run through the debug build of the library
(libmkf_b200_debug.so: bounds checks in the kernels, canary words after every
scratch allocation).  Run as a child process with MKF_B200_LIB=debug:

    MKF_B200_LIB=debug python -m tests.debug_cases

Each case is compared word for word with the oracle; after each one the
library's check records must be clean.  Prints one JSON line.
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from mkf_b200 import autotune, capi, params  # noqa: E402
from mkf_b200 import evaluator as ev  # noqa: E402
from oracle import keygen as kg  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402
from tests import helpers as H  # noqa: E402


def status():
    rep = (ctypes.c_uint64 * 4)()
    st = capi.lib().mkf_debug_status(0, rep)
    return st, [int(x) for x in rep]


def same(a, b, moduli):
    return bool(np.array_equal(H.canon(a, moduli), H.canon(b, moduli)))


def case_ntt():
    ok = True
    for log_n in (10, 12, 13, 14, 15, 16):
        lit = params.small("ckks", log_n=log_n, n_q=3, n_p=2, q_bits=50, first_bits=60, p_bits=55)
        P = ev.Parameters(lit, "ckks")
        o = Oracle.from_literal(lit)
        x = kg.uniform(kg.rng(log_n), lit.q, o.n)
        ok &= same(ev.ntt(P, x), o.ntt(x, "Q"), lit.q)
        ok &= same(ev.ntt(P, x, inverse=True), o.intt(x, "Q"), lit.q)
    return ok


def case_decompose():
    ok = True
    for log_n in (12, 13, 16):
        lit = params.small("ckks", log_n=log_n, n_q=7, n_p=4, q_bits=50, first_bits=60, p_bits=60)
        P = ev.Parameters(lit, "ckks")
        o = Oracle.from_literal(lit)
        for gamma in (1, 2):
            for level in (6, 3):
                x = kg.uniform(kg.rng(level), lit.q[: level + 1], o.n)
                ok &= same(ev.decompose(P, gamma, level, x), o.decompose(gamma, level, x),
                           list(lit.q[: level + 1]) + list(lit.p))
    return ok


def case_mkf_ckks():
    ok = True
    lit = params.small("ckks", log_n=13, n_q=6, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                       scale_bits=45)
    case = H.mkf_ckks_case(lit, 3, 5)
    want, lv, _ = case.o.mkf_ckks_mulrelin(3, 5, case.left, case.right, case.keys.fold,
                                           case.keys.relin, True, lit.scale, lit.scale ** 2)
    P = ev.Parameters(lit, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    L = ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale)
    R = ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale)
    for fuse in (0, 1):
        for width in (1, 2):
            autotune.set_tuning(P, fuse_ip=fuse, ip_width=width, col_split=2 if fuse else 8)
            ok &= same(E.MulRelinNew(L, R).download(), want, lit.q[: lv + 1])
    return ok


def case_kklss_ckks():
    lit = params.small("ckks", log_n=13, n_q=6, n_p=4, q_bits=50, first_bits=60, p_bits=60,
                       scale_bits=50)
    k, level = 3, 5
    case = H.kklss_ckks_case(lit, k, level, has0=[1, 1, 0], has1=[0, 1, 1])
    want, lv, _ = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                             case.keys.rlk, case.keys.crs_u, lit.scale, lit.scale,
                                             lit.scale)
    P = ev.Parameters(lit, "ckks")
    rs = ev.RelinearizationKeySet(P, case.keys.crs_u)
    for i in range(k):
        rs.AddRelinearizationKey(i, case.keys.rlk[i])
    a = ev.Ciphertext.from_array(P, case.op0[[0, 1, 2]], False, ids=[0, 1], scale=lit.scale)
    b = ev.Ciphertext.from_array(P, case.op1[[0, 2, 3]], False, ids=[1, 2], scale=lit.scale)
    return same(ev.Evaluator(P).MulRelinNew(a, b, rs).download(), want, lit.q[: lv + 1])


def case_bfv():
    ok = True
    lit = params.small("bfv", log_n=12, n_q=4, n_p=2, q_bits=54, p_bits=60)
    P = ev.Parameters(lit, "bfv")
    c = H.kklss_bfv_case(lit, 2)
    want = c.o.kklss_bfv_mulrelin(2, c.has0, c.has1, c.op0, c.op1, c.keys.rlk, c.keys.crs_u, lit.t)
    rs = ev.RelinearizationKeySet(P, c.keys.crs_u)
    for i in range(2):
        rs.AddRelinearizationKey(i, c.keys.rlk[i])
    got = ev.Evaluator(P).MulRelinNew(ev.Ciphertext.from_array(P, c.op0, False, ids=[0, 1]),
                                      ev.Ciphertext.from_array(P, c.op1, False, ids=[0, 1]),
                                      rs).download()
    ok &= same(got, want, lit.q)
    m = H.mkf_bfv_case(lit, 2)
    want = m.o.mkf_bfv_mulrelin(2, m.left, m.right, m.keys.fold, m.keys.relin, lit.t)
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(m.keys.fold), m.keys.relin))
    got = E.MulRelinNew(ev.Ciphertext.from_array(P, m.left, False),
                        ev.Ciphertext.from_array(P, m.right, False)).download()
    ok &= same(got, want, lit.q)
    return ok


def case_batch_and_server():
    """A graph-captured batch plan and the serving loop (both guarded per job)."""
    lit = params.small("ckks", log_n=13, n_q=5, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                       scale_bits=45)
    case = H.mkf_ckks_case(lit, 2, 4)
    want, lv, _ = case.o.mkf_ckks_mulrelin(2, 4, case.left, case.right, case.keys.fold,
                                           case.keys.relin, True, lit.scale, lit.scale ** 2)
    P = ev.Parameters(lit, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    L = ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale)
    R = ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale)
    outs = [ev.Ciphertext(P, 2, lv, True) for _ in range(3)]
    jobs = [("mkf", E, L, R, o, True, False) for o in outs]
    E.MulRelinNew(L, R)  # sizes the context's workspaces before the capture
    b = ev.Batch(P, jobs, lanes=2, graph=True)
    b.launch()
    b.close()
    ok = all(same(o.download(), want, lit.q[: lv + 1]) for o in outs)
    srv = ev.Server(device=0, scratch_bytes=1 << 30, slots=2)
    for j in jobs:
        srv.submit(j)
    srv.drain()
    srv.close()
    ok &= all(same(o.download(), want, lit.q[: lv + 1]) for o in outs)
    return ok


CASES = [case_ntt, case_decompose, case_mkf_ckks, case_kklss_ckks, case_bfv, case_batch_and_server]


def main():
    assert capi.LIB_PATH.endswith("libmkf_b200_debug.so"), capi.LIB_PATH
    res = {}
    for fn in CASES:
        ok = fn()
        st, rep = status()
        res[fn.__name__] = {"parity": bool(ok), "status": st, "report": rep}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
