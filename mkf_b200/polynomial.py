"""Polynomial evaluation over MKF paper carriers.

Restates paperMKFCKKSEvaluator.EvaluatePoly
(software/mkf/mkf_cpu/true_mkf_ckks_polynomial.go:79-273): Lattigo v2.3's
balanced power basis and baby-step/giant-step recursion, with every
ciphertext product routed through the MKF mult+relin (no rescale) and every
rescale, addition and constant through the carrier operations.  The host
schedule below follows the reference function by function; the device work
is the library's (mkf_mkf_mulrelin, mkf_rescale, mkf_add/sub, mkf_ct_copy,
mkf_slot_const).

The schedule talks to a backend (`CarrierBackend` for the GPU) so that the
same code can drive any implementation of the carrier operations.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from typing import Dict, List, Sequence

import numpy as np

from . import capi

NEGLIGIBLE = 1e-14  # Lattigo ckks.IsNegligbleThreshold


@dataclass
class Polynomial:
    """ckks.Polynomial: coefficients in the standard or Chebyshev basis.
    For the Chebyshev basis the caller maps x -> (2x - a - b)/(b - a) first,
    as with Lattigo's EvaluatePoly."""
    coeffs: List[complex]
    max_deg: int = -1
    lead: bool = True
    basis: str = "standard"
    a: float = -1.0
    b: float = 1.0

    def __post_init__(self):
        self.coeffs = [complex(c) for c in self.coeffs]
        if self.max_deg < 0:
            self.max_deg = len(self.coeffs) - 1

    def degree(self) -> int:
        return len(self.coeffs) - 1

    def depth(self) -> int:
        return self.degree().bit_length()

    def copy(self) -> "Polynomial":
        return Polynomial(list(self.coeffs), self.max_deg, self.lead, self.basis, self.a, self.b)


def not_negligible(c: complex) -> bool:
    return abs(c.real) > NEGLIGIBLE or abs(c.imag) > NEGLIGIBLE


def odd_or_even(coeffs: List[complex]):
    """paperMKFOddOrEven (true_mkf_ckks_polynomial.go:40-62): parity of the
    polynomial; zeroes the vanishing half."""
    odd, even = True, True
    for i, c in enumerate(coeffs):
        nz = not_negligible(c)
        odd = odd and not (i % 2 == 0 and nz)
        even = even and not (i % 2 == 1 and nz)
        if not odd and not even:
            break
    if odd or even:
        start = 1 if even else 0
        for i in range(start, len(coeffs), 2):
            coeffs[i] = 0j
    return odd, even


def split_coefficients(p: Polynomial, split: int):
    """paperMKFSplitCoefficients (:156-178)."""
    rem = Polynomial([0j] * split, basis=p.basis)
    if p.max_deg == p.degree():
        rem.max_deg = split - 1
    else:
        rem.max_deg = p.max_deg - (p.degree() - split + 1)
    rem.coeffs[:] = p.coeffs[:split]
    quo = Polynomial([0j] * (p.degree() - split + 1), max_deg=p.max_deg, basis=p.basis)
    quo.coeffs[0] = p.coeffs[split]
    if p.basis == "standard":
        quo.coeffs[1:] = p.coeffs[split + 1:]
    else:
        offset = 1
        for index in range(split + 1, p.degree() + 1):
            quo.coeffs[index - split] = 2 * p.coeffs[index]
            rem.coeffs[split - offset] -= p.coeffs[index]
            offset += 1
    quo.lead = p.lead
    rem.lead = False
    return quo, rem


# ---------------------------------------------------------------------------
# integer encodings of constants (Lattigo's scaleUpExact and Gaussian integers)
# ---------------------------------------------------------------------------
def scale_up_exact(value: float, n: float, q: int) -> int:
    """Lattigo scaleUpExact: round(|value| * n) (float64 product, +0.5 at
    53-bit precision, truncated), reduced mod q, negated for value < 0."""
    neg = value < 0
    x = (-n * value) if neg else (n * value)
    r = int(math.floor(x + 0.5)) % q
    return (q - r) % q if neg else r


def gaussian_integers(value: complex, scale: float):
    """The big integers evaluateFromPowerBasis multiplies with (:247-251):
    real and imaginary parts times scale, exact 106-bit products truncated
    toward zero."""
    cs = Fraction(scale)
    return int(Fraction(value.real) * cs), int(Fraction(value.imag) * cs)


class Schedule:
    """The reference's EvaluatePoly over a backend."""

    def __init__(self, backend):
        self.be = backend

    def evaluate(self, x, poly: Polynomial, target_scale: float):
        be = self.be
        if not poly.coeffs:
            raise ValueError("polynomial is empty")
        p = poly.copy()
        if be.level(x) < p.depth():
            raise ValueError(f"{be.level(x)} levels < {p.depth()} polynomial depth")
        powers: Dict[int, object] = {1: be.copy(x)}
        log_degree = p.degree().bit_length()
        log_split = log_degree >> 1
        odd, even = odd_or_even(p.coeffs)
        for degree in range(2, 1 << log_split):
            if not (even or odd) or (degree % 2 == 0 and even) or (degree % 2 == 1 and odd):
                self._power(degree, powers, target_scale, p.basis)
        for index in range(log_split, log_degree):
            self._power(1 << index, powers, target_scale, p.basis)
        res = self._recurse(target_scale, log_split, log_degree, p, powers)
        return be.with_scale(res, target_scale)

    def _power(self, degree, powers, scale, basis):
        be = self.be
        if degree in powers:
            return
        sub = 0
        if degree & (degree - 1) == 0:
            left = right = degree // 2
        else:
            k = int(math.ceil(math.log2(degree))) - 1
            left = (1 << k) - 1
            right = degree + 1 - (1 << k)
            if basis == "chebyshev":
                sub = abs(left - right)
        self._power(left, powers, scale, basis)
        self._power(right, powers, scale, basis)
        prod = be.mul_relin(powers[left], powers[right])
        powers[degree] = be.rescale(prod, scale)
        if basis == "chebyshev":
            powers[degree] = be.add(powers[degree], powers[degree])
            if sub == 0:
                powers[degree] = be.add_const(powers[degree], -1.0)
            else:
                self._power(sub, powers, scale, basis)
                powers[degree] = be.sub(powers[degree], powers[sub])

    def _recurse(self, target_scale, log_split, log_degree, p: Polynomial, powers):
        be = self.be
        if p.degree() < (1 << log_split):
            if p.lead and log_split > 1 and p.max_deg % (1 << (log_split + 1)) > (1 << (log_split - 1)):
                log_degree = p.degree().bit_length()
                log_split = log_degree >> 1
                return self._recurse(target_scale, log_split, log_degree, p, powers)
            return self._from_power_basis(target_scale, p, powers)
        next_power = 1 << log_split
        while next_power < (p.degree() >> 1) + 1:
            next_power <<= 1
        quo, rem = split_coefficients(p, next_power)
        level = be.level(powers[next_power]) - 1
        if quo.max_deg >= (1 << (log_degree - 1)) and quo.lead:
            level += 1
        qi = float(be.q[level])
        left = self._recurse(target_scale * qi / be.scale(powers[next_power]), log_split, log_degree,
                             quo, powers)
        right = self._recurse(target_scale, log_split, log_degree, rem, powers)
        if be.level(left) > be.level(right):
            while be.level(left) != be.level(right) + 1:
                left = be.drop_level(left, 1)
        left = be.mul_relin(left, powers[next_power])
        if be.level(left) > be.level(right):
            left = be.rescale(left, target_scale)
            return be.add(left, right)
        left = be.add(left, right)
        return be.rescale(left, target_scale)

    def _from_power_basis(self, target_scale, p: Polynomial, powers):
        be = self.be
        minimum = 0
        for degree in range(p.degree(), 0, -1):
            if not_negligible(p.coeffs[degree]):
                minimum = degree
                break
        constant = p.coeffs[0]
        if minimum == 0:
            res = be.zero(be.level(powers[1]), target_scale)
            if not_negligible(constant):
                return be.add_const(res, constant)
            return res
        minimum = p.degree()
        qi = float(be.q[be.level(powers[minimum])])
        res = be.zero(be.level(powers[minimum]), target_scale * qi)
        if not_negligible(constant):
            res = be.add_const(res, constant)
        for degree in range(p.degree(), 0, -1):
            c = p.coeffs[degree]
            if not not_negligible(c):
                continue
            re, im = gaussian_integers(c, target_scale * qi / be.scale(powers[degree]))
            res = be.mult_gauss_add(powers[degree], re, im, res)
        return be.rescale(res, target_scale)


# ---------------------------------------------------------------------------
# constants per limb and half of the NTT slots
# ---------------------------------------------------------------------------
def add_const_residues(value: complex, scale: float, q: Sequence[int], iq: Sequence[int], nl: int):
    """AddConst: re_s + im_s*i on the first half, re_s - im_s*i on the
    second, re_s/im_s = scaleUpExact(part, scale, q)."""
    out = np.zeros((nl, 2), np.uint64)
    for l in range(nl):
        qi = int(q[l])
        r = scale_up_exact(value.real, scale, qi) if value.real != 0 else 0
        i = (scale_up_exact(value.imag, scale, qi) * int(iq[l])) % qi if value.imag != 0 else 0
        out[l, 0] = (r + i) % qi
        out[l, 1] = (r - i) % qi
    return out


def gauss_residues(re: int, im: int, q: Sequence[int], iq: Sequence[int], nl: int):
    """MultByGaussianIntegerAndAdd: (re + im*i) mod q on the first half,
    (re - im*i) mod q on the second (Euclidean residues of the big integers)."""
    out = np.zeros((nl, 2), np.uint64)
    for l in range(nl):
        qi = int(q[l])
        r, i = re % qi, (im % qi) * int(iq[l]) % qi
        out[l, 0] = (r + i) % qi
        out[l, 1] = (r - i) % qi
    return out


def lattigo_add_scales(s0: float, s1: float):
    """Lattigo v2.3 evaluateInPlace: the smaller-scale operand is multiplied
    by uint64(larger / smaller) when that is above 1; the result carries the
    larger scale.  Returns (factor0, factor1, out_scale)."""
    if s0 > s1:
        return 1, max(1, int(s0 / s1)), s0
    if s1 > s0:
        return max(1, int(s1 / s0)), 1, s1
    return 1, 1, s0


class CarrierBackend:
    """GPU carrier operations of a PaperMKFAdapter for the schedule."""

    def __init__(self, adapter):
        from . import evaluator as ev
        self.ev = ev
        self.A = adapter
        P = adapter.params
        self.P = P
        self.q = list(P.literal.q)
        # the fourth root of unity of each limb, as the library's NTT sees it:
        # slot 0 of NTT(X^(N/2))
        x = np.zeros((len(self.q), P.N), np.uint64)
        x[:, P.N // 2] = 1
        self.iq = [int(v) for v in ev.ntt(P, x)[:, 0]]

    def level(self, ct):
        return ct.Level()

    def scale(self, ct):
        return ct.Scale

    def copy(self, ct):
        out = self.A.NewCiphertext(ct.Level(), ct.Scale)
        capi.check(self.P.handle, capi.lib().mkf_ct_copy(self.P.handle, ct.handle, out.handle, None))
        return out

    def with_scale(self, ct, scale):
        capi.lib().mkf_ct_set_scale(ct.handle, float(scale))
        return ct

    def zero(self, level, scale):
        return self.A.NewCiphertext(level, scale)

    def drop_level(self, ct, n):
        out = self.A.NewCiphertext(ct.Level() - n, ct.Scale)
        capi.check(self.P.handle, capi.lib().mkf_ct_copy(self.P.handle, ct.handle, out.handle, None))
        return out

    def mul_relin(self, a, b):
        return self.A.MulRelinNew(a, b)

    def rescale(self, ct, target):
        return self.A.RescaleNew(ct, target)

    def _slot(self, ct, consts, mode, out):
        capi.check(self.P.handle, capi.lib().mkf_slot_const(
            self.P.handle, ct.handle, capi.ptr(np.ascontiguousarray(consts)), mode, out.handle, None))

    def add(self, a, b):
        return self.A.AddNew(a, b)  # Lattigo's scale handling is in mkf_add

    def sub(self, a, b):
        return self.A.SubNew(a, b)

    def add_const(self, ct, value):
        out = self.A.NewCiphertext(ct.Level(), ct.Scale)
        nl = ct.Level() + 1
        self._slot(ct, add_const_residues(complex(value), ct.Scale, self.q, self.iq, nl),
                   capi.SLOT_ADD_C0, out)
        return out

    def mult_gauss_add(self, ct, re, im, target):
        # limbs above the input's level keep their values, as in Lattigo
        nl = target.Level() + 1
        if ct.Level() + 1 < nl:
            raise ValueError("the accumulator is above the input's level")
        self._slot(ct, gauss_residues(re, im, self.q, self.iq, nl), capi.SLOT_MUL_ADD, target)
        return target


def EvaluatePoly(adapter, x, poly: Polynomial, target_scale: float):
    """paperMKFCKKSEvaluator.EvaluatePoly on the GPU."""
    return Schedule(CarrierBackend(adapter)).evaluate(x, poly, target_scale)
