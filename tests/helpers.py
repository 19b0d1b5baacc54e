"""Shared builders for the parity tests: seeded keys and ciphertexts from the
oracle's test-side generator, in the C-ABI layout."""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from oracle import keygen as kg
from oracle.oracle import Oracle


def bfv_plain(lit, m, nl):
    """Delta*m mod each q (Delta = floor(Q/t)), coefficient domain."""
    Q = 1
    for q in lit.q:
        Q *= q
    delta = Q // lit.t
    out = np.zeros((nl, len(m)), np.uint64)
    mi = [int(x) for x in m]
    for i, q in enumerate(lit.q[:nl]):
        d = delta % q
        out[i] = np.array([(x * d) % q for x in mi], dtype=np.uint64)
    return out


def bfv_decrypt(lit, ph_coeff):
    Q = 1
    for q in lit.q:
        Q *= q
    c = kg.crt_centered(ph_coeff, lit.q)
    return np.array([((lit.t * x + Q // 2) // Q) % lit.t for x in c], dtype=object)


def negacyclic_mod(a, b, t):
    r = kg.negacyclic_mul_int(np.array(a, dtype=object), np.array(b, dtype=object))
    return np.array([int(x) % t for x in r], dtype=object)


@dataclass
class MKFCase:
    lit: object
    o: Oracle
    k: int
    level: int
    keys: kg.MKFKeys
    left: np.ndarray
    right: np.ndarray
    want: object  # expected slots (CKKS) or plaintext poly (BFV)


def mkf_ckks_case(lit, k, level, seed=3) -> MKFCase:
    o = Oracle.from_literal(lit)
    R = kg.RNS(o)
    N = o.n
    keys = kg.mkf_keygen(R, k, seed)
    enc = kg.CKKSEncoder(lit.log_n)
    g = kg.rng(seed + 77)
    nl = level + 1
    cts, sums = [], []
    for _ in range(2):
        zs = [(g.uniform(-1, 1, N // 2) + 1j * g.uniform(-1, 1, N // 2)) / k for _ in range(k)]
        sums.append(np.sum(zs, axis=0))
        C0 = np.zeros((nl, N), np.uint64)
        comps = []
        for i in range(k):
            m = o.ntt(o.from_int(enc.encode(zs[i], lit.scale), "Q", 0, nl), "Q")
            c0, c1 = kg.pk_encrypt_ntt(o, keys.public[i], m, level, g)
            C0 = o.add(C0, c0)
            comps.append(c1)
        cts.append(np.ascontiguousarray(np.stack([C0] + comps)))
    return MKFCase(lit, o, k, level, keys, cts[0], cts[1], sums[0] * sums[1])


def mkf_ckks_decode(case: MKFCase, out, lv, scale):
    o, lit = case.o, case.lit
    s = o.ntt(o.from_int(case.keys.aggregate, "Q", 0, lv + 1), "Q")
    ph = o.intt(o.add(out[0][: lv + 1], o.mul(out[1][: lv + 1], s)), "Q")
    return kg.CKKSEncoder(lit.log_n).decode(kg.crt_centered(ph, lit.q[: lv + 1]), scale)


def sparse_message(g, n, t, nnz=8):
    m = np.zeros(n, dtype=np.int64)
    m[g.choice(n, nnz, replace=False)] = g.integers(0, t, nnz)
    return m


def sparse_negacyclic_mod(a, b, t):
    n = len(a)
    out = [0] * n
    ia = [i for i in range(n) if a[i]]
    ib = [j for j in range(n) if b[j]]
    for i in ia:
        for j in ib:
            k = i + j
            v = int(a[i]) * int(b[j])
            if k >= n:
                out[k - n] -= v
            else:
                out[k] += v
    return np.array([x % t for x in out], dtype=object)


def mkf_bfv_case(lit, k, seed=5, sparse=False) -> MKFCase:
    o = Oracle.from_literal(lit)
    R = kg.RNS(o)
    N = o.n
    nq = len(lit.q)
    keys = kg.mkf_keygen(R, k, seed)
    g = kg.rng(seed + 1)
    cts, sums = [], []
    for _ in range(2):
        ms = [sparse_message(g, N, lit.t) if sparse else g.integers(0, lit.t, N) for _ in range(k)]
        sums.append(np.sum(ms, axis=0) % lit.t)
        C0 = np.zeros((nq, N), np.uint64)
        comps = []
        for i in range(k):
            m = o.ntt(bfv_plain(lit, ms[i], nq), "Q")
            c0, c1 = kg.pk_encrypt_ntt(o, keys.public[i], m, nq - 1, g)
            C0 = o.add(C0, o.intt(c0, "Q"))
            comps.append(o.intt(c1, "Q"))
        cts.append(np.ascontiguousarray(np.stack([C0] + comps)))
    if sparse:
        want = sparse_negacyclic_mod(sums[0], sums[1], lit.t)
    else:
        want = negacyclic_mod(sums[0], sums[1], lit.t) if N <= 4096 else None
    return MKFCase(lit, o, k, nq - 1, keys, cts[0], cts[1], want)


def mkf_bfv_decrypt(case: MKFCase, out):
    o, lit = case.o, case.lit
    s = o.ntt(o.from_int(case.keys.aggregate, "Q"), "Q")
    ph = o.add(out[0], o.intt(o.mul(o.ntt(out[1], "Q"), s), "Q"))
    return bfv_decrypt(lit, ph)


@dataclass
class KKLSSCase:
    lit: object
    o: Oracle
    k: int
    level: int
    keys: kg.KKLSSKeys
    op0: np.ndarray
    op1: np.ndarray
    has0: List[int]
    has1: List[int]
    want: object


def kklss_ckks_case(lit, k, level, seed=7, has0=None, has1=None) -> KKLSSCase:
    o = Oracle.from_literal(lit)
    R = kg.RNS(o)
    N = o.n
    nl = level + 1
    keys = kg.kklss_keygen(R, k, seed)
    enc = kg.CKKSEncoder(lit.log_n)
    g = kg.rng(seed + 2)
    has = [has0 or [1] * k, has1 or [1] * k]
    cts, sums = [], []
    for side in range(2):
        ct = np.zeros((k + 1, nl, N), np.uint64)
        tot = np.zeros(N // 2, complex)
        for i in range(k):
            if not has[side][i]:
                continue
            z = (g.uniform(-1, 1, N // 2) + 1j * g.uniform(-1, 1, N // 2)) / k
            tot += z
            m = o.from_int(enc.encode(z, lit.scale), "Q", 0, nl)
            c0, c1 = kg.kklss_encrypt(o, keys.public[i], m, level, g)
            ct[0] = o.add(ct[0], c0)
            ct[i + 1] = c1
        cts.append(ct)
        sums.append(tot)
    return KKLSSCase(lit, o, k, level, keys, cts[0], cts[1], has[0], has[1], sums[0] * sums[1])


def kklss_ckks_decode(case: KKLSSCase, out, lv, scale, ids=None):
    o, lit = case.o, case.lit
    ids = ids if ids is not None else list(range(case.k))
    ph = out[0][: lv + 1].copy()
    for c, pid in enumerate(ids):
        s = o.ntt(o.from_int(case.keys.secrets[pid], "Q", 0, lv + 1), "Q")
        ph = o.add(ph, o.intt(o.mul(o.ntt(out[c + 1][: lv + 1], "Q"), s), "Q"))
    return kg.CKKSEncoder(lit.log_n).decode(kg.crt_centered(ph, lit.q[: lv + 1]), scale)


def kklss_bfv_case(lit, k, seed=9, sparse=False) -> KKLSSCase:
    o = Oracle.from_literal(lit)
    R = kg.RNS(o)
    N = o.n
    nq = len(lit.q)
    keys = kg.kklss_keygen(R, k, seed, bfv_t=lit.t)
    g = kg.rng(seed + 3)
    cts, sums = [], []
    for _ in range(2):
        ct = np.zeros((k + 1, nq, N), np.uint64)
        tot = np.zeros(N, dtype=object)
        for i in range(k):
            m = sparse_message(g, N, lit.t) if sparse else g.integers(0, lit.t, N)
            tot = (tot + m) % lit.t
            c0, c1 = kg.kklss_encrypt(o, keys.public[i], bfv_plain(lit, m, nq), nq - 1, g)
            ct[0] = o.add(ct[0], c0)
            ct[i + 1] = c1
        cts.append(ct)
        sums.append(tot)
    if sparse:
        want = sparse_negacyclic_mod(sums[0], sums[1], lit.t)
    else:
        want = negacyclic_mod(sums[0], sums[1], lit.t) if N <= 4096 else None
    return KKLSSCase(lit, o, k, nq - 1, keys, cts[0], cts[1], [1] * k, [1] * k, want)


def kklss_bfv_decrypt(case: KKLSSCase, out):
    o, lit = case.o, case.lit
    ph = out[0].copy()
    for i in range(case.k):
        s = o.ntt(o.from_int(case.keys.secrets[i], "Q"), "Q")
        ph = o.add(ph, o.intt(o.mul(o.ntt(out[i + 1], "Q"), s), "Q"))
    return bfv_decrypt(lit, ph)


def canon(a, moduli):
    """Reduce an [.., L, N] array limb-wise (compare mod q like the
    reference's testbench, hardware/u55c/hls/tb/tb_par1_mkf_ckks.cpp:46-63)."""
    a = np.array(a, dtype=np.uint64, copy=True)
    for i, q in enumerate(moduli):
        a[..., i, :] %= np.uint64(q)
    return a
