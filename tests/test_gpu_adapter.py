"""The paper-facing (n+1)-component interface (mkf_b200.adapter, the
reference's paperMKFLattigoAdapter) and the primitives under it: fold alone,
repeated-Gamma materialization, component-wise add/sub and public products,
bit-exact against the oracle; a public-mask product followed by rescale
decrypts to the expected slots."""
import numpy as np
import pytest

from mkf_b200 import capi
from mkf_b200 import evaluator as ev
from mkf_b200.adapter import PaperMKFAdapter
from oracle import keygen as kg
from tests import helpers as H
from tests.fixture_cases import BF, CK
from tests.test_gpu_parity import assert_eq_mod, gpu

pytestmark = pytest.mark.gpu


def _oracle_fold(o, side, fold, k, level, ntt):
    a0, a1 = side[0].copy(), np.zeros_like(side[0])
    for i in range(k):
        s0, s1 = o.mkf_switch_one(level, side[i + 1], fold[i], ntt, ntt)
        a0, a1 = o.add(a0, s0), o.add(a1, s1)
    return a0, a1


@pytest.fixture(scope="module")
def ckks_case():
    k, level = 3, CK.max_level
    case = H.mkf_ckks_case(CK, k, level)
    P = gpu(CK, "ckks")
    keys = ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin)
    return case, P, keys


def test_fold_and_materialize_ckks(ckks_case):
    case, P, keys = ckks_case
    A = PaperMKFAdapter(P, keys)
    ct = ev.Ciphertext.from_array(P, case.left, True, scale=CK.scale)
    compact = A.FoldToAggregate(ct)
    want = _oracle_fold(case.o, case.left, case.keys.fold, case.k, case.level, True)
    got = compact.download()
    qs = CK.q[: case.level + 1]
    assert_eq_mod(got[0], want[0], qs)
    assert_eq_mod(got[1], want[1], qs)
    full = A.MaterializeAggregate(compact).download()
    assert full.shape[0] == case.k + 1
    assert np.array_equal(full[0], got[0])
    for j in range(1, case.k + 1):
        assert np.array_equal(full[j], got[1])


def test_fold_bfv():
    k = 2
    case = H.mkf_bfv_case(BF, k)
    P = gpu(BF, "bfv")
    keys = ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin)
    ct = ev.Ciphertext.from_array(P, case.left, False)
    out = ev.Ciphertext(P, 2, BF.max_level, False)
    capi.check(P.handle, capi.lib().mkf_mkf_fold(P.handle, ct.handle, keys.handle, out.handle, None))
    want = _oracle_fold(case.o, case.left, case.keys.fold, k, BF.max_level, False)
    got = out.download()
    assert_eq_mod(got[0], want[0], BF.q)
    assert_eq_mod(got[1], want[1], BF.q)


def test_componentwise_ops(ckks_case):
    case, P, keys = ckks_case
    A = PaperMKFAdapter(P, keys)
    o = case.o
    a = ev.Ciphertext.from_array(P, case.left, True, scale=CK.scale)
    b = ev.Ciphertext.from_array(P, case.right, True, scale=CK.scale)
    qs = CK.q[: case.level + 1]
    s, d = A.AddNew(a, b).download(), A.SubNew(a, b).download()
    for c in range(case.k + 1):
        assert_eq_mod(s[c], o.add(case.left[c], case.right[c]), qs)
        assert_eq_mod(d[c], o.sub(case.left[c], case.right[c]), qs)
    pt = case.right[1]
    ptc = ev.Ciphertext.from_array(P, pt[None], True, scale=2.0)
    m = A.MulNew(a, ptc)
    assert m.Scale == CK.scale * 2.0
    got = m.download()
    for c in range(case.k + 1):
        assert_eq_mod(got[c], o.mul(case.left[c], pt), qs)
    with pytest.raises(capi.MKFError, match="party ids|components"):
        other = ev.Ciphertext.from_array(P, case.right[:3], True, scale=CK.scale)
        A.AddNew(a, other)


def test_paper_mulrelin_matches_oracle_and_decrypts(ckks_case):
    case, P, keys = ckks_case
    A = PaperMKFAdapter(P, keys)
    a = ev.Ciphertext.from_array(P, case.left, True, scale=CK.scale)
    b = ev.Ciphertext.from_array(P, case.right, True, scale=CK.scale)
    out = A.MulRelinNew(a, b)
    assert out.n_comp == case.k + 1 and out.Level() == case.level
    want, lv, sc = case.o.mkf_ckks_mulrelin(case.k, case.level, case.left, case.right, case.keys.fold,
                                            case.keys.relin, False, CK.scale, CK.scale ** 2)
    got = out.download()
    qs = CK.q[: lv + 1]
    assert_eq_mod(got[0], want[0], qs)
    for j in range(1, case.k + 1):
        assert_eq_mod(got[j], want[1], qs)
    # rescale the carrier, then decrypt with the aggregate secret
    r = A.RescaleNew(out)
    d = H.mkf_ckks_decode(case, r.download()[:2], r.Level(), r.Scale)
    assert kg.precision_bits(d, case.want) > 20


def test_public_mask_then_rescale_decrypts(ckks_case):
    case, P, keys = ckks_case
    A = PaperMKFAdapter(P, keys)
    o, N = case.o, CK.n
    g = np.random.default_rng(5)
    mask = (g.uniform(-1, 1, N // 2) + 1j * g.uniform(-1, 1, N // 2))
    enc = kg.CKKSEncoder(CK.log_n)
    pt = o.ntt(o.from_int(enc.encode(mask, CK.scale), "Q", 0, case.level + 1), "Q")
    a = ev.Ciphertext.from_array(P, case.left, True, scale=CK.scale)
    m = A.MulNew(a, ev.Ciphertext.from_array(P, pt[None], True, scale=CK.scale))
    compact = A.FoldToAggregate(A.RescaleNew(m))
    got = compact.download()
    # decrypt c0 + c1 s_E; the left operand encrypts sum_i z_i
    s = o.ntt(o.from_int(case.keys.aggregate, "Q", 0, compact.Level() + 1), "Q")
    ph = o.intt(o.add(got[0], o.mul(got[1], s)), "Q")
    dec = enc.decode(kg.crt_centered(ph, CK.q[: compact.Level() + 1]), compact.Scale)
    left_slots = H.mkf_ckks_decode(case, np.stack(_oracle_fold(o, case.left, case.keys.fold, case.k,
                                                               case.level, True)),
                                   case.level, CK.scale)
    assert kg.precision_bits(dec, left_slots * mask) > 18
