"""GPU parity at ring degrees 2^13..2^16 (the fused decomposition + NTT path)
and at the benchmark configurations C1 (CKKS logN=14, k=2), C2 (BFV logN=15,
k=4) and C3 (CKKS logN=16) with two parties, bit-exact against the oracle.
The k = 8 products at C3 and on the serving rings are compared word for word
in test_gpu_bench_configs.py."""
import numpy as np
import pytest

from mkf_b200 import params
from mkf_b200 import evaluator as ev
from oracle import keygen as kg
from oracle.oracle import Oracle
from tests import helpers as H
from tests.test_gpu_parity import assert_eq_mod, gpu, _kklss_rlkset

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [13, 14, 15, 16])
@pytest.mark.parametrize("gamma", [1, 2])
def test_fused_decompose_ntt(log_n, gamma):
    lit = params.small("ckks", log_n=log_n, n_q=7, n_p=4, q_bits=50, first_bits=60, p_bits=60)
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    for level in (6, 4, 3):
        x = kg.uniform(kg.rng(log_n * 10 + level), lit.q[: level + 1], o.n)
        want = o.decompose(gamma, level, x)
        got = ev.decompose(P, gamma, level, x)
        assert_eq_mod(got, want, list(lit.q[: level + 1]) + list(lit.p))


def _mkf_ckks(lit, k, level):
    case = H.mkf_ckks_case(lit, k, level)
    want, lv, sc = case.o.mkf_ckks_mulrelin(k, level, case.left, case.right, case.keys.fold,
                                            case.keys.relin, True, lit.scale, lit.scale ** 2)
    P = gpu(lit, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    out = E.MulRelinNew(ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale),
                        ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale))
    got = out.download()
    assert_eq_mod(got, want, lit.q[: lv + 1])
    return case, got, lv, sc


def test_mkf_ckks_logn13():
    lit = params.small("ckks", log_n=13, n_q=5, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                       scale_bits=45)
    case, got, lv, sc = _mkf_ckks(lit, 3, 4)
    assert kg.precision_bits(H.mkf_ckks_decode(case, got, lv, sc), case.want) > 20


def test_mkf_ckks_c1():
    """Benchmark configuration C1: CKKS logN=14, Q = 55b + 7x40b, P = 2x45b, k=2, scale 2^40."""
    lit = params.get("ckks", "C1")
    case, got, lv, sc = _mkf_ckks(lit, 2, lit.max_level)
    prec = kg.precision_bits(H.mkf_ckks_decode(case, got, lv, sc), case.want)
    assert prec > 12, prec


def test_mkf_ckks_c3_k2_bitexact():
    """Benchmark configuration C3 parameters (logN=16, 24 Q limbs, 4 P limbs) at k=2, top level
    and level 8."""
    lit = params.get("ckks", "C3")
    for level in (lit.max_level, 8):
        case, got, lv, sc = _mkf_ckks(lit, 2, level)
        assert lv == level - 1
        assert kg.precision_bits(H.mkf_ckks_decode(case, got, lv, sc), case.want) > 25


def test_mkf_bfv_c2_k4_bitexact():
    """Benchmark configuration C2: BFV logN=15, fifteen 58-bit Q, two 60-bit P, t=65537, k=4."""
    lit = params.get("bfv", "C2")
    case = H.mkf_bfv_case(lit, 4, sparse=True)
    want = case.o.mkf_bfv_mulrelin(4, case.left, case.right, case.keys.fold, case.keys.relin, lit.t)
    P = gpu(lit, "bfv")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    got = E.MulRelinNew(ev.Ciphertext.from_array(P, case.left, False),
                        ev.Ciphertext.from_array(P, case.right, False)).download()
    assert_eq_mod(got, want, lit.q)
    assert np.array_equal(H.mkf_bfv_decrypt(case, got), case.want)


def test_kklss_ckks_logn13_masks():
    lit = params.small("ckks", log_n=13, n_q=6, n_p=4, q_bits=50, first_bits=60, p_bits=60,
                       scale_bits=50)
    k, level = 3, 5
    case = H.kklss_ckks_case(lit, k, level, has0=[1, 1, 0], has1=[0, 1, 1])
    want, lv, sc = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                              case.keys.rlk, case.keys.crs_u, lit.scale, lit.scale,
                                              lit.scale)
    P = gpu(lit, "ckks")
    rs = _kklss_rlkset(P, case, range(k))
    a = ev.Ciphertext.from_array(P, case.op0[[0, 1, 2]], False, ids=[0, 1], scale=lit.scale)
    b = ev.Ciphertext.from_array(P, case.op1[[0, 2, 3]], False, ids=[1, 2], scale=lit.scale)
    got = ev.Evaluator(P).MulRelinNew(a, b, rs).download()
    assert_eq_mod(got, want, lit.q[: lv + 1])
    assert kg.precision_bits(H.kklss_ckks_decode(case, got, lv, sc), case.want) > 20


def test_kklss_bfv_logn14():
    lit = params.small("bfv", log_n=14, n_q=4, n_p=2, q_bits=56, p_bits=60)
    case = H.kklss_bfv_case(lit, 2, sparse=True)
    want = case.o.kklss_bfv_mulrelin(2, case.has0, case.has1, case.op0, case.op1, case.keys.rlk,
                                     case.keys.crs_u, lit.t)
    P = gpu(lit, "bfv")
    rs = _kklss_rlkset(P, case, range(2))
    got = ev.Evaluator(P).MulRelinNew(ev.Ciphertext.from_array(P, case.op0, False, ids=[0, 1]),
                                      ev.Ciphertext.from_array(P, case.op1, False, ids=[0, 1]),
                                      rs).download()
    assert_eq_mod(got, want, lit.q)
    assert np.array_equal(H.kklss_bfv_decrypt(case, got), case.want)
