"""Parameter sets for the multi-key mult+relin path.

This mirrors the parameter literals the reference evaluators are built from
(``ckks.ParametersLiteral`` / ``bfv.ParametersLiteral`` /
``mkbfv.ParametersLiteral``): a ring degree, the Q chain, the special primes P,
the BFV auxiliary chain QMul and the scheme constants.

* ``P1``/``P2`` are the exact chains of the reference
  (software/mkf/mkf_cpu/params.go:15-101, identical to the KKLSS test literals
  PN14QP439/PN15QP880 in software/kklss/mkckks/mkckks_test.go:51-91 and
  software/kklss/mkbfv/mkbfv_test.go:28-110).
* ``C1``/``C2``/``C3`` are the benchmark configurations: every prime is the
  largest NTT-friendly prime (q = 1 mod 2N) below 2^b that has not been used
  earlier in the same set, assigned in the order Q, QMul, P.
* ``S14``/``S15``/``S16`` are the serving-trace chains at logN 14/15/16 that
  carry both a CKKS and a BFV view (the BFV view uses the same Q as QMul-twin).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

# --------------------------------------------------------------------------
# primes
# --------------------------------------------------------------------------


def _is_prime(n: int) -> bool:
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def ntt_primes_below(bits: int, log_n: int, count: int, skip: int = 0) -> List[int]:
    """The `count` largest primes q < 2^bits with q = 1 mod 2N, after skipping
    the first `skip` of them (so that groups of equal bit size stay disjoint)."""
    step = 2 << log_n
    q = ((1 << bits) - 1) // step * step + 1
    if q >= 1 << bits:
        q -= step
    out: List[int] = []
    seen = 0
    while len(out) < count:
        if q < (1 << (bits - 1)):
            raise ValueError(f"not enough {bits}-bit NTT primes for logN={log_n}")
        if _is_prime(q):
            if seen >= skip:
                out.append(q)
            seen += 1
        q -= step
    return out


class _PrimeAllocator:
    """Hands out primes largest-first per bit size, never twice."""

    def __init__(self, log_n: int):
        self.log_n = log_n
        self.used = {}

    def take(self, bits: int, count: int) -> List[int]:
        skip = self.used.get(bits, 0)
        self.used[bits] = skip + count
        return ntt_primes_below(bits, self.log_n, count, skip)


# --------------------------------------------------------------------------
# parameter literal
# --------------------------------------------------------------------------


@dataclass(frozen=True)
class ParametersLiteral:
    """Unchecked parameters (reference: ckks/bfv/mkbfv ParametersLiteral)."""

    name: str
    log_n: int
    q: Tuple[int, ...]
    p: Tuple[int, ...]
    q_mul: Tuple[int, ...] = ()
    log_slots: int = 0
    scale: float = 0.0
    t: int = 0
    sigma: float = 3.2

    @property
    def n(self) -> int:
        return 1 << self.log_n

    @property
    def max_level(self) -> int:
        return len(self.q) - 1

    def with_name(self, name: str) -> "ParametersLiteral":
        return ParametersLiteral(name, self.log_n, self.q, self.p, self.q_mul,
                                 self.log_slots, self.scale, self.t, self.sigma)


def _lit(name, log_n, q, p, q_mul=(), log_slots=0, scale=0.0, t=0):
    return ParametersLiteral(name, log_n, tuple(q), tuple(p), tuple(q_mul),
                             log_slots, float(scale), int(t))


# exact reference chains ---------------------------------------------------
CKKS_P1 = _lit("P1", 14,
               [0x7ffffffffe70001, 0xffffffff00001, 0xfffffffe40001,
                0xfffffffe20001, 0xfffffffbe0001, 0xfffffffa60001],
               [0xffffffffffc0001, 0xfffffffff840001], log_slots=13, scale=2.0 ** 52)
CKKS_P2 = _lit("P2", 15,
               [0xfffffffff6a0001, 0x3fffffffd60001, 0x3fffffffca0001,
                0x3fffffff6d0001, 0x3fffffff5d0001, 0x3fffffff550001,
                0x3fffffff390001, 0x3fffffff360001, 0x3fffffff2a0001,
                0x3fffffff000001, 0x3ffffffefa0001, 0x3ffffffef40001,
                0x3ffffffed70001, 0x3ffffffed30001],
               [0x7ffffffffe70001, 0x7ffffffffe10001], log_slots=14, scale=2.0 ** 54)
BFV_P1 = _lit("P1", 14,
              [0x1fffffffe30001, 0x1fffffffd10001, 0x1fffffffbf0001,
               0x1fffffffb60001, 0x1fffffff920001, 0x3fffffffd60001],
              [0xffffffffffc0001, 0xfffffffff840001],
              q_mul=[0x1fffffffd80001, 0x1fffffffc50001, 0x1fffffffb90001,
                     0x1fffffffa50001, 0x1fffffff900001, 0x3fffffffca0001],
              t=65537)
BFV_P2 = _lit("P2", 15,
              [0x3fffffffd60001, 0x3fffffff6d0001, 0x3fffffff550001,
               0x3fffffff360001, 0x3fffffff000001, 0x3ffffffef40001,
               0x3ffffffed30001, 0x3ffffffe970001, 0x3ffffffe800001,
               0x3ffffffe410001, 0x7fffffffe90001, 0x7fffffffbd0001,
               0x7fffffffaa0001, 0x7fffffff9f0001],
              [0xffffffffffc0001, 0xfffffffff840001],
              q_mul=[0x3fffffffca0001, 0x3fffffff5d0001, 0x3fffffff390001,
                     0x3fffffff2a0001, 0x3ffffffefa0001, 0x3ffffffed70001,
                     0x3ffffffeaa0001, 0x3ffffffe920001, 0x3ffffffe790001,
                     0x3ffffffe320001, 0x7fffffffbf0001, 0x7fffffffba0001,
                     0x7fffffffa50001, 0x7fffffff7e0001],
              t=65537)


def _gen_ckks(name, log_n, first_bits, n_rest, rest_bits, n_p, p_bits, scale_bits):
    a = _PrimeAllocator(log_n)
    q = a.take(first_bits, 1) + a.take(rest_bits, n_rest)
    p = a.take(p_bits, n_p)
    return _lit(name, log_n, q, p, log_slots=log_n - 1, scale=2.0 ** scale_bits)


def _gen_bfv(name, log_n, n_q, q_bits, n_p, p_bits, t=65537):
    a = _PrimeAllocator(log_n)
    q = a.take(q_bits, n_q)
    q_mul = a.take(q_bits, n_q)
    p = a.take(p_bits, n_p)
    return _lit(name, log_n, q, p, q_mul=q_mul, t=t)


_CACHE = {}


def get(scheme: str, name: str) -> ParametersLiteral:
    """Named parameter set: scheme in {"ckks", "bfv"}."""
    key = (scheme.lower(), name.upper())
    if key in _CACHE:
        return _CACHE[key]
    s, n = key
    if s == "ckks":
        table = {
            "P1": lambda: CKKS_P1,
            "P2": lambda: CKKS_P2,
            # C1: one 55-bit + seven 40-bit Q, two 45-bit P, scale 2^40
            "C1": lambda: _gen_ckks("C1", 14, 55, 7, 40, 2, 45, 40),
            # C3: one 60-bit + twenty-three 50-bit Q, four 60-bit P, scale 2^50
            "C3": lambda: _gen_ckks("C3", 16, 60, 23, 50, 4, 60, 50),
            # batched / serving chains
            "S14": lambda: _gen_ckks("S14", 14, 55, 7, 40, 2, 45, 40),
            "S15": lambda: _gen_ckks("S15", 15, 60, 15, 50, 4, 60, 50),
            "S16": lambda: _gen_ckks("S16", 16, 60, 23, 50, 4, 60, 50),
        }
    elif s == "bfv":
        table = {
            "P1": lambda: BFV_P1,
            "P2": lambda: BFV_P2,
            # C2: fifteen 58-bit Q (+ fifteen 58-bit QMul), two 60-bit P, t=65537
            "C2": lambda: _gen_bfv("C2", 15, 15, 58, 2, 60),
            "S14": lambda: _gen_bfv("S14", 14, 6, 54, 2, 60),
            "S15": lambda: _gen_bfv("S15", 15, 15, 58, 2, 60),
            "S16": lambda: _gen_bfv("S16", 16, 15, 58, 2, 60),
        }
    else:
        raise ValueError(f"unknown scheme {scheme!r}")
    if n not in table:
        raise ValueError(f"unknown {s} parameter set {name!r}")
    lit = table[n]()
    _CACHE[key] = lit
    return lit


def small(scheme: str, log_n: int = 10, n_q: int = 4, n_p: int = 2,
          q_bits: int = 50, first_bits: Optional[int] = None, p_bits: int = 60,
          scale_bits: Optional[int] = None, t: int = 65537) -> ParametersLiteral:
    """Small chains used by the parity tests (same construction rules)."""
    a = _PrimeAllocator(log_n)
    fb = first_bits or q_bits
    if scheme == "ckks":
        q = a.take(fb, 1) + a.take(q_bits, n_q - 1)
        p = a.take(p_bits, n_p)
        return _lit(f"ckks-n{log_n}-q{n_q}-p{n_p}", log_n, q, p,
                    log_slots=log_n - 1, scale=2.0 ** (scale_bits or q_bits))
    q = a.take(q_bits, n_q)
    q_mul = a.take(q_bits, n_q)
    p = a.take(p_bits, n_p)
    return _lit(f"bfv-n{log_n}-q{n_q}-p{n_p}", log_n, q, p, q_mul=q_mul, t=t)


def alpha_beta(lit: ParametersLiteral, level: int, gamma: int) -> Tuple[int, int]:
    """Gadget shape: alpha = |P|/gamma limbs per digit, beta digits at level
    (mkrlwe/params.go:63-71; gamma = 1 is Lattigo's rlwe decomposition)."""
    alpha = len(lit.p) // gamma
    return alpha, (level + alpha) // alpha
