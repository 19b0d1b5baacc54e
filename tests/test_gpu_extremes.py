"""GPU parity on the words at the edges of the float64 residue path.

Limbs below 2^50 run their NTTs, multSum and key products on the float64
pipe with lazy reductions placed by compile-time schedules; the schedules are
correct only if the bounds they assume hold for every input.  These tests
feed the words that push those bounds hardest -- all q-1, alternating 0 and
q-1, and the two words whose centered representatives have the largest
magnitude, (q-1)/2 and (q+1)/2 -- to every limb (float64 limbs of 50-bit
primes, the tightest case, and integer limbs of 55- and 60-bit primes), and
compare with the oracle word for word:

* forward and inverse NTT phases (the lazy butterflies of Lattigo's
  ring.NTT / InvNTT, restated at hardware/u55c/hls/kernels/
  par1_mkf_ckks_kernel.cpp:93-162), logN 13-16;
* the digit column pass, whose multSum words are rebuilt from digits
  y_i = x_i (Q/q_i)^-1 mod q_i chosen at their extremes (reconstructRNS and
  multSum, software/kklss/mkrlwe/basis_extension.go:537-646), logN 13-16;
* the fused row pass + key inner product, through full MKF products whose
  fold and relinearization keys hold one extreme word everywhere
  (KeyswitchHoistedNoModDown, software/mkf/mkf_cpu/common.go:79-107),
  logN 13-16 and the six-digit C3 chain.
"""
import numpy as np
import pytest

from mkf_b200 import params
from mkf_b200 import evaluator as ev
from oracle.oracle import Oracle
from tests.test_gpu_parity import assert_eq_mod, gpu

pytestmark = pytest.mark.gpu

PATTERNS = ("q-1", "0,q-1", "(q-1)/2", "(q-1)/2,(q+1)/2")


def pattern_limb(q, n, pattern):
    q = int(q)
    w = np.empty(n, np.uint64)
    if pattern == "q-1":
        w[:] = q - 1
    elif pattern == "0,q-1":
        w[0::2], w[1::2] = 0, q - 1
    elif pattern == "(q-1)/2":
        w[:] = (q - 1) // 2
    elif pattern == "(q-1)/2,(q+1)/2":
        w[0::2], w[1::2] = (q - 1) // 2, (q + 1) // 2
    else:
        raise ValueError(pattern)
    return w


def pattern_poly(moduli, n, pattern):
    return np.stack([pattern_limb(q, n, pattern) for q in moduli])


def chain(log_n):
    # Q: one 60-bit (integer, Harvey butterflies) and six 50-bit primes
    # (float64); P: 55-bit primes (integer, lazy butterflies)
    return params.small("ckks", log_n=log_n, n_q=7, n_p=4, q_bits=50, first_bits=60, p_bits=55,
                        scale_bits=50)


@pytest.mark.parametrize("log_n", [13, 14, 15, 16])
def test_ntt_extreme_words(log_n):
    lit = chain(log_n)
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    for basis in ("Q", "P"):
        mods = o.moduli(basis)
        for pattern in PATTERNS:
            x = pattern_poly(mods, o.n, pattern)
            assert_eq_mod(ev.ntt(P, x, basis), o.ntt(x, basis), mods)
            assert_eq_mod(ev.ntt(P, x, basis, inverse=True), o.intt(x, basis), mods)


def digit_sources(lit, gamma, level):
    alpha = len(lit.p) // gamma
    return [list(range(s, min(s + alpha, level + 1))) for s in range(0, level + 1, alpha)]


def coeffs_with_digits(lit, gamma, level, n, pattern):
    """Coefficient-domain words whose reconstruction digits
    y_i = x_i (Q_d/q_i)^-1 mod q_i follow `pattern` in every digit d."""
    x = np.zeros((level + 1, n), np.uint64)
    for src in digit_sources(lit, gamma, level):
        qs = [int(lit.q[j]) for j in src]
        Qd = 1
        for q in qs:
            Qd *= q
        for j, q in zip(src, qs):
            y = pattern_limb(q, n, pattern)
            c = (Qd // q) % q
            # a pattern holds at most two distinct words: map each once
            vals, inv = np.unique(y, return_inverse=True)
            x[j] = np.array([(int(v) * c) % q for v in vals], dtype=np.uint64)[inv]
    return x


@pytest.mark.parametrize("log_n", [13, 14, 15, 16])
@pytest.mark.parametrize("gamma", [1, 2])
def test_decompose_extreme_digits(log_n, gamma):
    lit = chain(log_n)
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    level = lit.max_level
    mods = list(lit.q[: level + 1]) + list(lit.p)
    for pattern in PATTERNS:
        x = coeffs_with_digits(lit, gamma, level, o.n, pattern)
        assert_eq_mod(ev.decompose(P, gamma, level, x), o.decompose(gamma, level, x), mods)
    # the coefficient words themselves at their extremes
    for pattern in ("q-1", "(q-1)/2,(q+1)/2"):
        x = pattern_poly(lit.q[: level + 1], o.n, pattern)
        assert_eq_mod(ev.decompose(P, gamma, level, x), o.decompose(gamma, level, x), mods)


def extreme_key(lit, pattern):
    """A switching key [beta][2][nQ+nP][N] holding one extreme word per limb."""
    beta = (len(lit.q) + len(lit.p) - 1) // len(lit.p)
    limb = pattern_poly(list(lit.q) + list(lit.p), lit.n, pattern)
    return np.ascontiguousarray(np.broadcast_to(limb, (beta, 2) + limb.shape))


@pytest.mark.parametrize("lit_name", ["n13", "n14", "n15", "n16", "C3"])
def test_fused_inner_product_extreme_keys(lit_name):
    lit = params.get("ckks", "C3") if lit_name == "C3" else chain(int(lit_name[1:]))
    k, level = 2, lit.max_level
    P = gpu(lit, "ckks")
    o = Oracle.from_literal(lit)
    from mkf_b200 import autotune
    autotune.set_tuning(P, fuse_ip=1)
    n = o.n
    for kp, op_pat in (("q-1", "q-1"), ("(q-1)/2", "(q-1)/2,(q+1)/2"),
                       ("(q-1)/2,(q+1)/2", "(q-1)/2")):
        fold = [extreme_key(lit, kp) for _ in range(k)]
        relin = extreme_key(lit, kp)
        ops = []
        for side in range(2):
            ops.append(np.ascontiguousarray(
                np.stack([pattern_poly(lit.q[: level + 1], n, op_pat)] * (k + 1))))
        want, lv, sc = o.mkf_ckks_mulrelin(k, level, ops[0], ops[1], fold, relin, True, lit.scale,
                                           lit.scale ** 2)
        E = ev.MKFEvaluator(P, ev.MKFKeySet(P, fold, relin))
        got = E.MulRelinNew(ev.Ciphertext.from_array(P, ops[0], True, scale=lit.scale),
                            ev.Ciphertext.from_array(P, ops[1], True, scale=lit.scale)).download()
        assert_eq_mod(got, want, lit.q[: lv + 1])
