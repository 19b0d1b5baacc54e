"""Oracle self-validation of the rotation and conjugation key switches
(KKLSS RotateHoisted / Conjugate, software/kklss/mkrlwe/keyswitch_hoisted.go:
198-249 and keyswitch.go:301-343; MKF paper RotateNew, software/mkf/mkf_cpu/
true_mkf_ckks.go:323-353): with valid Galois keys the results decrypt to the
rotated / conjugated slots."""
import numpy as np

from mkf_b200 import params
from oracle import keygen as kg
from tests import helpers as H

CK = params.small("ckks", log_n=10, n_q=4, n_p=2, q_bits=45, first_bits=55, p_bits=55, scale_bits=45)


def _mkf_fold(o, side, fold, k, level):
    a0, a1 = side[0].copy(), np.zeros_like(side[0])
    for i in range(k):
        s0, s1 = o.mkf_switch_one(level, side[i + 1], fold[i], True, True)
        a0, a1 = o.add(a0, s0), o.add(a1, s1)
    return np.stack([a0, a1])


def test_automorphism_composes():
    case = H.mkf_ckks_case(CK, 1, 2)
    o = case.o
    x = case.left[0]
    g3, g5 = o.galois_element(3), o.galois_element(5)
    a = o.automorphism(2, o.automorphism(2, x, g3), g5)
    b = o.automorphism(2, x, o.galois_element(8))
    assert np.array_equal(a, b)
    # the NTT-domain form is the coefficient form moved through the NTT
    y = o.automorphism_ntt(2, o.ntt(x, "Q"), g3)
    assert np.array_equal(o.intt(y, "Q"), o.automorphism(2, x, g3))


def test_mkf_rotation_decrypts():
    k, level, r = 2, CK.max_level, 5
    case = H.mkf_ckks_case(CK, k, level)
    o = case.o
    gal = o.galois_element(r)
    rk = kg.mkf_rotation_keys(kg.RNS(o), case.keys, gal, 21)
    rot = o.mkf_rotate(level, case.left, rk, gal)
    before = H.mkf_ckks_decode(case, _mkf_fold(o, case.left, case.keys.fold, k, level), level, CK.scale)
    after = H.mkf_ckks_decode(case, rot, level, CK.scale)
    assert kg.precision_bits(after, np.roll(before, -r)) > 20


def test_kklss_rotation_and_conjugation_decrypt():
    k, level, r = 2, CK.max_level, 3
    case = H.kklss_ckks_case(CK, k, level)
    o = case.o
    R = kg.RNS(o)
    before = H.kklss_ckks_decode(case, case.op0, level, CK.scale)
    gal = o.galois_element(r)
    rk, crs = kg.kklss_galois_keys(R, case.keys, gal, 31)
    rot = o.kklss_rotate(level, case.op0, rk, crs, gal)
    after = H.kklss_ckks_decode(case, rot, level, CK.scale)
    assert kg.precision_bits(after, np.roll(before, -r)) > 18
    gc = o.conjugation_element()
    ck, crs2 = kg.kklss_galois_keys(R, case.keys, gc, 32, conjugation=True)
    conj = o.kklss_conjugate(level, case.op0, ck, crs2, gc)
    after = H.kklss_ckks_decode(case, conj, level, CK.scale)
    assert kg.precision_bits(after, np.conj(before)) > 18
