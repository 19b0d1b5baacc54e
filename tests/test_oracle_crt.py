"""Independent big-integer checks of the oracle's basis conversions.

The oracle restates Lattigo's and the KKLSS fork's RNS arithmetic word by
word (Montgomery constants, lazy representatives, a float64 correction).
These tests restate what that arithmetic computes in plain Python integers
on CRT-reconstructed coefficients, at small ring degrees:

* ModUp (modUpExact / reconstructRNS + multSum,
  software/kklss/mkrlwe/basis_extension.go:337-357, 537-646): the canonical
  integer X in [0, Q) of the source residues, reduced into each target
  modulus -- exactly, with the correction v = floor(sum y_i / q_i) evaluated
  in float64 in the reference's order;
* ModDown (ModDownQPtoQ[NTT], basis_extension.go:192-288): floor(X / P) for
  X the CRT integer of the QP residues;
* rescale (DivRoundByLastModulus[NTT], called from
  software/kklss/mkckks/evaluator.go:391): floor((X + h) / q_L) with
  h = (q_L - 1) / 2, i.e. X / q_L rounded;
* the gadget decomposition (DecomposeAndSplit, basis_extension.go:428-535):
  per digit, the digit's own limbs kept and the CRT integer of its source
  limbs reduced into every other limb.
"""
import numpy as np
import pytest

from mkf_b200 import params
from oracle import keygen as kg
from oracle.oracle import Oracle

LITS = [
    params.small("ckks", log_n=6, n_q=5, n_p=2, q_bits=50, first_bits=60, p_bits=60),
    params.small("ckks", log_n=7, n_q=6, n_p=4, q_bits=40, first_bits=55, p_bits=45),
]


def prod(xs):
    r = 1
    for x in xs:
        r *= int(x)
    return r


def crt(residues, moduli):
    """Per-coefficient CRT integer in [0, prod(moduli)) of [L][N] residues."""
    M = prod(moduli)
    out = [0] * residues.shape[1]
    for r, q in zip(residues, moduli):
        q = int(q)
        Mi = M // q
        c = Mi * pow(Mi % q, -1, q)
        for x in range(residues.shape[1]):
            out[x] += int(r[x]) * c
    return [v % M for v in out]


def modup_reference(residues, src, tgt):
    """The reference's exact ModUp of residues over `src` into `tgt`:
    sum_i y_i (Q/q_i) - v Q with y_i = x_i (Q/q_i)^-1 mod q_i and
    v = floor(sum_i y_i / q_i) summed in float64 in source order."""
    Q = prod(src)
    n = residues.shape[1]
    out = np.zeros((len(tgt), n), np.uint64)
    for x in range(n):
        acc, vf = 0, 0.0
        for i, q in enumerate(src):
            q = int(q)
            y = int(residues[i][x]) * pow((Q // q) % q, -1, q) % q
            acc += y * (Q // q)
            vf += float(y) / float(q)
        X = acc - int(vf) * Q
        for j, p in enumerate(tgt):
            out[j][x] = X % int(p)
    return out


def canon(a, moduli):
    a = np.array(a, dtype=np.uint64, copy=True)
    for i, q in enumerate(moduli):
        a[i] %= np.uint64(q)
    return a


@pytest.mark.parametrize("lit", LITS, ids=lambda l: l.name)
def test_modup_q_to_p_is_crt(lit):
    o = Oracle.from_literal(lit)
    for level in (lit.max_level, 1):
        src = lit.q[: level + 1]
        x = kg.uniform(kg.rng(level), src, o.n)
        got = canon(o.modup_q_to_p(level, x), lit.p)
        assert np.array_equal(got, modup_reference(x, src, lit.p))
        X = crt(x, src)
        exact = np.array([[v % p for v in X] for p in lit.p], dtype=np.uint64)
        assert np.array_equal(got, exact)


@pytest.mark.parametrize("lit", LITS, ids=lambda l: l.name)
def test_modup_p_to_q_is_crt(lit):
    o = Oracle.from_literal(lit)
    level = lit.max_level
    x = kg.uniform(kg.rng(5), lit.p, o.n)
    got = canon(o.modup_p_to_q(level, x), lit.q[: level + 1])
    X = crt(x, lit.p)
    exact = np.array([[v % q for v in X] for q in lit.q[: level + 1]], dtype=np.uint64)
    assert np.array_equal(got, exact)


def test_modup_float_correction_semantics():
    """Source words whose y_i sum to just below an integer: the float64
    correction may round up, and the oracle must then follow the reference
    (a result off by Q), not the exact CRT."""
    lit = LITS[0]
    o = Oracle.from_literal(lit)
    level = 2
    src = [int(q) for q in lit.q[: level + 1]]
    Q = prod(src)
    x = np.zeros((level + 1, o.n), np.uint64)
    # X = Q - 1, Q - 2, 0, 1, ...: y_i / q_i sums to (almost) an integer
    for c in range(o.n):
        X = (Q - 1 - c) % Q if c < o.n // 2 else c - o.n // 2
        for i, q in enumerate(src):
            x[i][c] = X % q
    got = canon(o.modup_q_to_p(level, x), lit.p)
    assert np.array_equal(got, modup_reference(x, src, lit.p))


@pytest.mark.parametrize("lit", LITS, ids=lambda l: l.name)
@pytest.mark.parametrize("ntt", [False, True])
def test_moddown_is_floor_div_p(lit, ntt):
    o = Oracle.from_literal(lit)
    for level in (lit.max_level, 2):
        qs = list(lit.q[: level + 1])
        x = np.concatenate([kg.uniform(kg.rng(level + 7), qs, o.n),
                            kg.uniform(kg.rng(level + 8), lit.p, o.n)])
        P = prod(lit.p)
        X = crt(x, qs + list(lit.p))
        want = np.array([[(v // P) % q for v in X] for q in qs], dtype=np.uint64)
        if ntt:
            xn = np.concatenate([o.ntt(x[: level + 1], "Q"), o.ntt(x[level + 1:], "P")])
            got = o.intt(canon(o.moddown(level, xn, True), qs), "Q")
        else:
            got = o.moddown(level, x, False)
        assert np.array_equal(canon(got, qs), want)


@pytest.mark.parametrize("lit", LITS, ids=lambda l: l.name)
@pytest.mark.parametrize("ntt", [False, True])
def test_rescale_is_rounded_division(lit, ntt):
    o = Oracle.from_literal(lit)
    for level in (lit.max_level, 1):
        qs = list(lit.q[: level + 1])
        x = kg.uniform(kg.rng(level + 3), qs, o.n)
        qL = int(qs[-1])
        h = (qL - 1) // 2
        X = crt(x, qs)
        want = np.array([[((v + h) // qL) % int(q) for v in X] for q in qs[:-1]], dtype=np.uint64)
        if ntt:
            got = o.intt(canon(o.rescale(level, o.ntt(x, "Q"), True), qs[:-1]), "Q")
        else:
            got = o.rescale(level, x, False)
        assert np.array_equal(canon(got, qs[:-1]), want)


@pytest.mark.parametrize("lit", LITS, ids=lambda l: l.name)
@pytest.mark.parametrize("gamma", [1, 2])
def test_decompose_digits_are_crt(lit, gamma):
    o = Oracle.from_literal(lit)
    alpha = len(lit.p) // gamma
    for level in (lit.max_level, 2):
        qs = list(lit.q[: level + 1])
        mods = qs + list(lit.p)
        x = kg.uniform(kg.rng(level + 11), qs, o.n)
        out = o.decompose(gamma, level, x)
        for d in range(out.shape[0]):
            src = list(range(d * alpha, min(d * alpha + alpha, level + 1)))
            coeff = np.concatenate([o.intt(out[d][: level + 1], "Q"),
                                    o.intt(out[d][level + 1:], "P")])
            coeff = canon(coeff, mods)
            X = crt(x[src], [qs[j] for j in src])
            for j, m in enumerate(mods):
                want = x[j] if j in src else np.array([v % int(m) for v in X], dtype=np.uint64)
                assert np.array_equal(coeff[j], want % np.uint64(m)), (d, j)
