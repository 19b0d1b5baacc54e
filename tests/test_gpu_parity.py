"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the
same seeded inputs.  Integer work, so the bar is bit-exact (compared mod q,
as the reference's testbench does: hardware/u55c/hls/tb/tb_par1_mkf_ckks.cpp:
46-63)."""
import numpy as np
import pytest

from mkf_b200 import capi, params
from mkf_b200 import evaluator as ev
from oracle import keygen as kg
from oracle.oracle import Oracle
from tests import helpers as H

pytestmark = pytest.mark.gpu

CK = params.small("ckks", log_n=10, n_q=6, n_p=4, q_bits=50, first_bits=60, p_bits=60, scale_bits=50)
CK2 = params.small("ckks", log_n=11, n_q=5, n_p=2, q_bits=40, first_bits=55, p_bits=45, scale_bits=40)
BF = params.small("bfv", log_n=10, n_q=4, n_p=2, q_bits=54, p_bits=60)
BF3 = params.small("bfv", log_n=11, n_q=5, n_p=2, q_bits=58, p_bits=60)


_CTX = {}


def gpu(lit, scheme):
    # keyed by the whole literal: small chains of one name can differ in
    # their prime sizes
    key = (lit, scheme)
    if key not in _CTX:
        _CTX[key] = ev.Parameters(lit, scheme)
    return _CTX[key]


def assert_eq_mod(a, b, moduli):
    a = H.canon(a, moduli)
    b = H.canon(b, moduli)
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        raise AssertionError(f"{len(bad)} words differ, first at {bad[0].tolist()}")


# ---------------------------------------------------------------------------
# NTT
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16])
def test_ntt_matches_oracle(log_n):
    lit = params.small("ckks", log_n=log_n, n_q=3, n_p=2, q_bits=50, first_bits=60, p_bits=60)
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    g = kg.rng(log_n)
    for basis in ("Q", "P"):
        x = kg.uniform(g, o.moduli(basis), o.n)
        want = o.ntt(x, basis)
        got = ev.ntt(P, x, basis)
        assert_eq_mod(got, want, o.moduli(basis))
        back = ev.ntt(P, got, basis, inverse=True)
        assert np.array_equal(back, x)
        assert np.array_equal(ev.ntt(P, x, basis, inverse=True), o.intt(x, basis))


def test_ntt_qmul_basis_and_subrange():
    P = gpu(BF3, "bfv")
    o = Oracle.from_literal(BF3)
    x = kg.uniform(kg.rng(3), BF3.q_mul[2:4], o.n)
    got = ev.ntt(P, x, "QM", first=2)
    want = o.ntt(x, "QM", first=2)
    assert np.array_equal(got, want)


def test_ntt_edge_values():
    """0, q-1 and a constant polynomial (whose NTT is constant)."""
    lit = params.small("ckks", log_n=14, n_q=2, n_p=1, q_bits=50, first_bits=60, p_bits=60)
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    x = np.zeros((2, o.n), np.uint64)
    x[:, 0] = 7
    x[0, 1:] = lit.q[0] - 1
    assert np.array_equal(ev.ntt(P, x), o.ntt(x, "Q"))
    c = np.zeros((1, o.n), np.uint64)
    c[0, 0] = 5
    assert np.all(ev.ntt(P, c, first=0)[0] == 5)


# ---------------------------------------------------------------------------
# gadget decomposition, key switch, rescale
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("gamma", [1, 2])
@pytest.mark.parametrize("level", [5, 4, 2, 1, 0])
def test_decompose_matches_oracle(gamma, level):
    P = gpu(CK, "ckks")
    o = Oracle.from_literal(CK)
    x = kg.uniform(kg.rng(100 + level), CK.q[: level + 1], o.n)
    want = o.decompose(gamma, level, x)
    got = ev.decompose(P, gamma, level, x)
    mods = list(CK.q[: level + 1]) + list(CK.p)
    assert_eq_mod(got, want, mods)


def test_decompose_float_correction_boundary():
    """Coefficients near the CRT wrap (x = Q_digit - 1, 0, 1) exercise the
    float64 correction of reconstructRNS."""
    P = gpu(CK, "ckks")
    o = Oracle.from_literal(CK)
    x = np.zeros((6, o.n), np.uint64)
    for i in range(6):
        x[i, 0] = CK.q[i] - 1
        x[i, 1] = 0
        x[i, 2] = 1
        x[i, 3] = CK.q[i] // 2
    want = o.decompose(1, 5, x)
    got = ev.decompose(P, 1, 5, x)
    assert_eq_mod(got, want, list(CK.q) + list(CK.p))


@pytest.mark.parametrize("ntt_output", [True, False])
@pytest.mark.parametrize("level", [5, 2])
def test_switch_one_matches_oracle(ntt_output, level):
    P = gpu(CK, "ckks")
    o = Oracle.from_literal(CK)
    R = kg.RNS(o)
    keys = kg.mkf_keygen(R, 1, 11)
    x = kg.uniform(kg.rng(12), CK.q[: level + 1], o.n)
    w0, w1 = o.mkf_switch_one(level, x, keys.fold[0], in_ntt=True, ntt_output=ntt_output)
    g0, g1 = ev.switch_one(P, level, x, keys.fold[0], in_ntt=True, ntt_output=ntt_output)
    mods = CK.q[: level + 1]
    assert_eq_mod(g0, w0, mods)
    assert_eq_mod(g1, w1, mods)


@pytest.mark.parametrize("ntt", [True, False])
def test_rescale_matches_oracle(ntt):
    P = gpu(CK, "ckks")
    o = Oracle.from_literal(CK)
    x = kg.uniform(kg.rng(21), CK.q, o.n)
    ct = ev.Ciphertext.from_array(P, x[None], is_ntt=ntt, scale=CK.scale * CK.q[5])
    E = ev.Evaluator(P)
    out = E.RescaleNew(ct, CK.scale)
    assert out.Level() == 4
    assert_eq_mod(out.download()[0], o.rescale(5, x, ntt), CK.q[:5])


# ---------------------------------------------------------------------------
# full products
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("lit,k,level", [(CK, 2, 5), (CK, 3, 3), (CK2, 2, 4), (CK2, 4, 2)])
def test_mkf_ckks_product_bitexact(lit, k, level):
    case = H.mkf_ckks_case(lit, k, level)
    want, lv, sc = case.o.mkf_ckks_mulrelin(k, level, case.left, case.right, case.keys.fold,
                                            case.keys.relin, True, lit.scale, lit.scale ** 2)
    P = gpu(lit, "ckks")
    ks = ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin)
    E = ev.MKFEvaluator(P, ks)
    L = ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale)
    Rr = ev.Ciphertext.from_array(P, case.right, True, scale=lit.scale)
    out = E.MulRelinNew(L, Rr, rescale=True)
    assert out.Level() == lv and abs(out.Scale - sc) <= 1e-9 * sc
    got = out.download()
    assert_eq_mod(got, want, lit.q[: lv + 1])
    assert H.mkf_ckks_decode(case, got, lv, sc) is not None


def test_mkf_ckks_materialized_output():
    case = H.mkf_ckks_case(CK, 3, 4)
    P = gpu(CK, "ckks")
    ks = ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin)
    E = ev.MKFEvaluator(P, ks)
    L = ev.Ciphertext.from_array(P, case.left, True)
    Rr = ev.Ciphertext.from_array(P, case.right, True)
    compact = E.MulRelinNew(L, Rr).download()
    full = E.MulRelinNew(L, Rr, materialize=True).download()
    assert full.shape[0] == 4
    assert np.array_equal(full[0], compact[0])
    for i in range(1, 4):
        assert np.array_equal(full[i], compact[1])


def test_mkf_ckks_without_rescale():
    case = H.mkf_ckks_case(CK, 2, 5)
    want, lv, _ = case.o.mkf_ckks_mulrelin(2, 5, case.left, case.right, case.keys.fold,
                                           case.keys.relin, False)
    P = gpu(CK, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    out = E.MulRelinNew(ev.Ciphertext.from_array(P, case.left, True),
                        ev.Ciphertext.from_array(P, case.right, True), rescale=False)
    assert_eq_mod(out.download(), want, CK.q)


@pytest.mark.parametrize("lit,k", [(BF, 2), (BF, 1), (BF3, 3)])
def test_mkf_bfv_product_bitexact(lit, k):
    case = H.mkf_bfv_case(lit, k)
    want = case.o.mkf_bfv_mulrelin(k, case.left, case.right, case.keys.fold, case.keys.relin, lit.t)
    P = gpu(lit, "bfv")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    out = E.MulRelinNew(ev.Ciphertext.from_array(P, case.left, False),
                        ev.Ciphertext.from_array(P, case.right, False))
    got = out.download()
    assert_eq_mod(got, want, lit.q)
    if case.want is not None:
        assert np.array_equal(H.mkf_bfv_decrypt(case, got), case.want)


def _kklss_rlkset(P, case, ids):
    rs = ev.RelinearizationKeySet(P, case.keys.crs_u)
    for i in ids:
        rs.AddRelinearizationKey(i, case.keys.rlk[i])
    return rs


@pytest.mark.parametrize("lit,k,level", [(CK, 2, 5), (CK, 3, 3), (CK2, 2, 4)])
def test_kklss_ckks_product_bitexact(lit, k, level):
    case = H.kklss_ckks_case(lit, k, level)
    want, lv, sc = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                              case.keys.rlk, case.keys.crs_u, lit.scale, lit.scale,
                                              lit.scale)
    P = gpu(lit, "ckks")
    rs = _kklss_rlkset(P, case, range(k))
    E = ev.Evaluator(P)
    a = ev.Ciphertext.from_array(P, case.op0, False, ids=list(range(k)), scale=lit.scale)
    b = ev.Ciphertext.from_array(P, case.op1, False, ids=list(range(k)), scale=lit.scale)
    out = E.MulRelinNew(a, b, rs)
    assert out.Level() == lv and out.ids == list(range(k))
    assert_eq_mod(out.download(), want, lit.q[: lv + 1])


def test_kklss_ckks_different_id_sets():
    """op0 over parties {0,1}, op1 over {1,2}: output over the union {0,1,2}
    (mkrlwe/keyswitch_hoisted.go handles absent components by skipping them)."""
    k, level = 3, 4
    case = H.kklss_ckks_case(CK, k, level, has0=[1, 1, 0], has1=[0, 1, 1])
    want, lv, sc = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                              case.keys.rlk, case.keys.crs_u, CK.scale, CK.scale,
                                              CK.scale)
    P = gpu(CK, "ckks")
    rs = _kklss_rlkset(P, case, range(k))
    a = ev.Ciphertext.from_array(P, case.op0[[0, 1, 2]], False, ids=[0, 1], scale=CK.scale)
    b = ev.Ciphertext.from_array(P, case.op1[[0, 2, 3]], False, ids=[1, 2], scale=CK.scale)
    out = ev.Evaluator(P).MulRelinNew(a, b, rs)
    assert out.ids == [0, 1, 2]
    assert_eq_mod(out.download(), want, CK.q[: lv + 1])
    got = H.kklss_ckks_decode(case, out.download(), lv, sc)
    assert kg.precision_bits(got, case.want) > 15


@pytest.mark.parametrize("lit,k", [(BF, 2), (BF3, 3)])
def test_kklss_bfv_product_bitexact(lit, k):
    case = H.kklss_bfv_case(lit, k)
    want = case.o.kklss_bfv_mulrelin(k, case.has0, case.has1, case.op0, case.op1, case.keys.rlk,
                                     case.keys.crs_u, lit.t)
    P = gpu(lit, "bfv")
    rs = _kklss_rlkset(P, case, range(k))
    a = ev.Ciphertext.from_array(P, case.op0, False, ids=list(range(k)))
    b = ev.Ciphertext.from_array(P, case.op1, False, ids=list(range(k)))
    got = ev.Evaluator(P).MulRelinNew(a, b, rs).download()
    assert_eq_mod(got, want, lit.q)
    if case.want is not None:
        assert np.array_equal(H.kklss_bfv_decrypt(case, got), case.want)


# ---------------------------------------------------------------------------
# error behaviour (the reference panics / returns errors)
# ---------------------------------------------------------------------------
def test_missing_relinearization_key():
    case = H.kklss_ckks_case(CK, 2, 3)
    P = gpu(CK, "ckks")
    rs = _kklss_rlkset(P, case, [0])
    a = ev.Ciphertext.from_array(P, case.op0, False, ids=[0, 1], scale=CK.scale)
    with pytest.raises(capi.MissingKeyError):
        ev.Evaluator(P).MulRelinNew(a, a, rs)


def test_rescale_at_level_zero_errors():
    P = gpu(CK, "ckks")
    ct = ev.Ciphertext(P, 1, 0, True, scale=CK.scale)
    with pytest.raises(capi.LevelError):
        ev.Evaluator(P).RescaleNew(ct, CK.scale)


def test_wrong_key_size_rejected():
    P = gpu(CK, "ckks")
    with pytest.raises(capi.MKFError):
        ev.SwitchingKey(P, np.zeros(10, np.uint64))
