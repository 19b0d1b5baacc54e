"""Rotations and conjugation on the GPU, bit-exact against the oracle and
decrypting to rotated / conjugated slots: KKLSS RotateHoisted and Conjugate
(software/kklss/mkrlwe/keyswitch_hoisted.go:198-249, keyswitch.go:301-343),
MKF paper RotateNew (software/mkf/mkf_cpu/true_mkf_ckks.go:321-353)."""
import numpy as np
import pytest

from mkf_b200 import capi, params
from mkf_b200 import evaluator as ev
from mkf_b200.adapter import PaperMKFAdapter
from oracle import keygen as kg
from tests import helpers as H
from tests.test_gpu_parity import assert_eq_mod, gpu

pytestmark = pytest.mark.gpu

CK = params.small("ckks", log_n=10, n_q=4, n_p=2, q_bits=45, first_bits=55, p_bits=55, scale_bits=45)
CK14 = params.small("ckks", log_n=14, n_q=4, n_p=2, q_bits=45, first_bits=55, p_bits=55, scale_bits=45)


def _fold(o, side, fold, k, level):
    a0, a1 = side[0].copy(), np.zeros_like(side[0])
    for i in range(k):
        s0, s1 = o.mkf_switch_one(level, side[i + 1], fold[i], True, True)
        a0, a1 = o.add(a0, s0), o.add(a1, s1)
    return np.stack([a0, a1])


@pytest.mark.parametrize("lit,r", [(CK, 5), (CK, -3), (CK14, 7)])
def test_mkf_rotation(lit, r):
    k, level = 2, lit.max_level
    case = H.mkf_ckks_case(lit, k, level)
    o = case.o
    gal = o.galois_element(r)
    rk = kg.mkf_rotation_keys(kg.RNS(o), case.keys, gal, 21)
    want = o.mkf_rotate(level, case.left, rk, gal)
    P = gpu(lit, "ckks")
    assert ev.galois_element(P, r) == gal
    rot = ev.MKFKeySet(P, list(rk), None)
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    ct = ev.Ciphertext.from_array(P, case.left, True, scale=lit.scale)
    got = E.RotateNew(ct, gal, rot).download()
    qs = lit.q[: level + 1]
    assert_eq_mod(got[0], want[0], qs)
    for j in range(1, k + 1):
        assert_eq_mod(got[j], want[1], qs)
    if lit is CK:
        before = H.mkf_ckks_decode(case, _fold(o, case.left, case.keys.fold, k, level), level, lit.scale)
        after = H.mkf_ckks_decode(case, got[:2], level, lit.scale)
        assert kg.precision_bits(after, np.roll(before, -r)) > 20


def test_adapter_rotation_and_missing_keys():
    k, level, r = 2, CK.max_level, 4
    case = H.mkf_ckks_case(CK, k, level)
    o = case.o
    gal = o.galois_element(r)
    rk = kg.mkf_rotation_keys(kg.RNS(o), case.keys, gal, 22)
    P = gpu(CK, "ckks")
    A = PaperMKFAdapter(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin),
                        {gal: ev.MKFKeySet(P, list(rk), None)})
    ct = ev.Ciphertext.from_array(P, case.left, True, scale=CK.scale)
    out = A.RotateNew(ct, r).download()
    want = o.mkf_rotate(level, case.left, rk, gal)
    assert_eq_mod(out[0], want[0], CK.q[: level + 1])
    with pytest.raises(capi.MissingKeyError):
        A.RotateNew(ct, r + 1)
    with pytest.raises(capi.MissingKeyError, match="relinearization"):
        ev.MKFEvaluator(P, A.rotations[gal]).MulRelinNew(ct, ct)


@pytest.mark.parametrize("lit,r", [(CK, 3), (CK14, -5)])
def test_kklss_rotation(lit, r):
    k, level = 2, lit.max_level
    case = H.kklss_ckks_case(lit, k, level)
    o = case.o
    gal = o.galois_element(r)
    keys, crs = kg.kklss_galois_keys(kg.RNS(o), case.keys, gal, 31)
    want = o.kklss_rotate(level, case.op0, keys, crs, gal)
    P = gpu(lit, "ckks")
    gks = ev.GaloisKeySet(P, gal, crs)
    for i in range(k):
        gks.AddKey(i, keys[i])
    ct = ev.Ciphertext.from_array(P, case.op0, False, ids=list(range(k)), scale=lit.scale)
    out = ev.Evaluator(P).RotateNew(ct, r, gks)
    assert out.ids == list(range(k))
    got = out.download()
    assert_eq_mod(got, want, lit.q[: level + 1])
    if lit is CK:
        before = H.kklss_ckks_decode(case, case.op0, level, lit.scale)
        after = H.kklss_ckks_decode(case, got, level, lit.scale)
        assert kg.precision_bits(after, np.roll(before, -r)) > 18


def test_kklss_conjugation_and_missing_key():
    k, level = 2, CK.max_level
    case = H.kklss_ckks_case(CK, k, level)
    o = case.o
    gc = o.conjugation_element()
    keys, crs = kg.kklss_galois_keys(kg.RNS(o), case.keys, gc, 32, conjugation=True)
    want = o.kklss_conjugate(level, case.op0, keys, crs, gc)
    P = gpu(CK, "ckks")
    assert ev.conjugation_element(P) == gc
    gks = ev.GaloisKeySet(P, gc, crs, conjugation=True)
    gks.AddKey(0, keys[0])
    ct = ev.Ciphertext.from_array(P, case.op0, False, ids=[0, 1], scale=CK.scale)
    with pytest.raises(capi.MissingKeyError, match="id 1"):
        ev.Evaluator(P).ConjugateNew(ct, gks)
    gks.AddKey(1, keys[1])
    got = ev.Evaluator(P).ConjugateNew(ct, gks).download()
    assert_eq_mod(got, want, CK.q[: level + 1])
    before = H.kklss_ckks_decode(case, case.op0, level, CK.scale)
    after = H.kklss_ckks_decode(case, got, level, CK.scale)
    assert kg.precision_bits(after, np.conj(before)) > 18
