"""TEST INFRASTRUCTURE ONLY: seeded key material, encryption, decryption and
encoding for the parity and precision tests.

The reference samples everything from an unseeded crypto PRNG
(software/kklss/mkrlwe/params.go:28, keygen.go:26, encryptor.go:32), so its
keys cannot be reproduced from a seed; parity is established by feeding the
same key and ciphertext words to the oracle and to the product.  The
generators below reproduce the reference's key *algebra* (which relation each
key satisfies, in which domain and Montgomery form it is stored) so that the
products also decrypt correctly:

* Lattigo rlwe.GenSwitchingKey(s_in, s_out) as used by MKF
  (software/mkf/mkf_cpu/common.go:44-51): b_i = e_i - a_i*s_out + P*s_in*g_i,
  stored MForm/NTT over QP, digits of alpha = |P| limbs.
* KKLSS GenRelinearizationKey (software/kklss/mkrlwe/keygen.go:137-187):
  b = -s*a + e, d = -r*a + P*s*g + e, v = -(s*u + P*r*g + e).
* KKLSS BFV halves (software/kklss/mkbfv/keygen.go:107-244) with the big
  integer gadget G_i = floor(Q*QMul/Q_i * t * T_i * P / QMul).

Secrets are uniform ternary, errors a rounded Gaussian with sigma = 3.2
bounded at 6 sigma (software/kklss/mkrlwe/keygen.go:35).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .oracle import Oracle

SIGMA = 3.2


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def ternary(g: np.random.Generator, n: int) -> np.ndarray:
    return g.integers(-1, 2, size=n, dtype=np.int64)


def gaussian(g: np.random.Generator, n: int, sigma: float = SIGMA) -> np.ndarray:
    e = np.rint(g.normal(0.0, sigma, size=n)).astype(np.int64)
    b = int(6 * sigma)
    return np.clip(e, -b, b)


def uniform(g: np.random.Generator, moduli: Sequence[int], n: int) -> np.ndarray:
    out = np.empty((len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[i] = g.integers(0, int(q), size=n, dtype=np.uint64)
    return out


def negacyclic_mul_int(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Exact negacyclic product of two small integer polynomials (object ints)."""
    n = len(a)
    full = np.convolve(a.astype(object), b.astype(object))
    out = full[:n].copy()
    out[: n - 1] -= full[n:]
    return out


class RNS:
    """Helpers over the oracle's Q/P/QMul/R bases."""

    def __init__(self, orc: Oracle):
        self.o = orc
        self.n = orc.n
        self.nq, self.np_ = len(orc.q), len(orc.p)
        self.P = 1
        for p in orc.p:
            self.P *= p

    # a QP polynomial is a pair (Q part [nq][n], P part [np][n])
    def qp_from_int(self, v, nq=None):
        nq = self.nq if nq is None else nq
        return (self.o.from_int(v, "Q", 0, nq), self.o.from_int(v, "P", 0, self.np_))

    def qp_ntt(self, a):
        return (self.o.ntt(a[0], "Q"), self.o.ntt(a[1], "P"))

    def qp_mform(self, a):
        return (self.o.mform(a[0], "Q"), self.o.mform(a[1], "P"))

    def qp_mul(self, a, b):
        return (self.o.mul(a[0], b[0], "Q"), self.o.mul(a[1], b[1], "P"))

    def qp_add(self, a, b):
        return (self.o.add(a[0], b[0], "Q"), self.o.add(a[1], b[1], "P"))

    def qp_sub(self, a, b):
        return (self.o.sub(a[0], b[0], "Q"), self.o.sub(a[1], b[1], "P"))

    def qp_neg(self, a):
        z = (np.zeros_like(a[0]), np.zeros_like(a[1]))
        return self.qp_sub(z, a)

    def qp_uniform(self, g):
        return (uniform(g, self.o.q, self.n), uniform(g, self.o.p, self.n))

    def qp_pack(self, a):
        return np.concatenate([a[0], a[1]], axis=0)

    def qp_error_ntt(self, g):
        return self.qp_ntt(self.qp_from_int(gaussian(g, self.n)))

    def qp_secret_ntt(self, s):
        return self.qp_ntt(self.qp_from_int(s))


# ----------------------------------------------------------------------------
# MKF (Lattigo rlwe) switching keys
# ----------------------------------------------------------------------------


def mkf_switching_key(R: RNS, s_in_ntt, s_out_ntt, g) -> np.ndarray:
    """[betaMax][2][nQ+nP][N]: key digit i = (b_i, a_i) in MForm/NTT with
    b_i + a_i*s_out = e_i + P*s_in*g_i (alpha = |P| limbs per digit)."""
    o = R.o
    alpha = R.np_
    beta = (R.nq + alpha - 1) // alpha
    key = np.zeros((beta, 2, R.nq + R.np_, R.n), np.uint64)
    p_mod = [R.P % q for q in o.q]
    ps_in = o.scalar(s_in_ntt[0], p_mod, "Q")
    for i in range(beta):
        a = R.qp_uniform(g)
        e = R.qp_error_ntt(g)
        b = R.qp_sub(e, R.qp_mul(a, s_out_ntt))
        bq = b[0].copy()
        for j in range(i * alpha, min((i + 1) * alpha, R.nq)):
            bq[j] = o.add(bq[j], ps_in[j], "Q", j)
        b = (bq, b[1])
        key[i, 0] = R.qp_pack(R.qp_mform(b))
        key[i, 1] = R.qp_pack(R.qp_mform(a))
    return key


@dataclass
class MKFKeys:
    secrets: List[np.ndarray]      # ternary coefficient vectors
    aggregate: np.ndarray           # sum of the secrets
    fold: np.ndarray                # [k][betaMax][2][nQ+nP][N]
    relin: np.ndarray               # [betaMax][2][nQ+nP][N]
    public: list                    # per party (pk0, pk1) over Q, NTT


def mkf_keygen(R: RNS, k: int, seed: int) -> MKFKeys:
    """software/mkf/mkf_cpu/common.go:32-51 (aggregateSecret, generateOnlineKeys)."""
    o = R.o
    secrets = [ternary(rng(seed * 1000 + i), R.n) for i in range(k)]
    agg = np.sum(secrets, axis=0).astype(np.int64)
    agg_ntt = R.qp_secret_ntt(agg)
    fold = np.zeros((k,) + (0,), np.uint64)
    folds = []
    for i in range(k):
        s_ntt = R.qp_secret_ntt(secrets[i])
        folds.append(mkf_switching_key(R, s_ntt, agg_ntt, rng(seed * 1000 + 100 + i)))
    fold = np.stack(folds)
    sq = R.qp_mul(agg_ntt, agg_ntt)
    relin = mkf_switching_key(R, sq, agg_ntt, rng(seed * 1000 + 999))
    public = []
    for i in range(k):
        g = rng(seed * 1000 + 500 + i)
        a = uniform(g, o.q, R.n)
        e = o.ntt(o.from_int(gaussian(g, R.n), "Q"), "Q")
        s_ntt = o.ntt(o.from_int(secrets[i], "Q"), "Q")
        public.append((o.sub(e, o.mul(a, s_ntt)), a))
    return MKFKeys(secrets, agg, fold, relin, public)


def pk_encrypt_ntt(o: Oracle, pk, m_ntt: np.ndarray, level: int, g):
    """Lattigo public-key encryption in the NTT domain at `level`:
    (v*pk0 + e0 + m, v*pk1 + e1)."""
    nl = level + 1
    v = o.ntt(o.from_int(ternary(g, o.n), "Q", 0, nl), "Q")
    e0 = o.ntt(o.from_int(gaussian(g, o.n), "Q", 0, nl), "Q")
    e1 = o.ntt(o.from_int(gaussian(g, o.n), "Q", 0, nl), "Q")
    c0 = o.add(o.add(o.mul(v, pk[0][:nl]), e0), m_ntt[:nl])
    c1 = o.add(o.mul(v, pk[1][:nl]), e1)
    return c0, c1


# ----------------------------------------------------------------------------
# KKLSS keys
# ----------------------------------------------------------------------------


def kklss_switch_part(R: RNS, s_ntt_q, g, gadget_q: Optional[List[List[int]]] = None,
                      gadget_p: Optional[List[List[int]]] = None, gamma: int = 2):
    """KKLSS GenSwitchingKey (keygen.go:270-327): per digit e + P*s*g_i (true
    value, NTT).  With gadget_q/gadget_p the BFV gadget residues G_i replace
    P*g_i on every limb (mkbfv/keygen.go:174-244)."""
    o = R.o
    alpha = R.np_ // gamma
    beta = (R.nq + alpha - 1) // alpha
    out = []
    for i in range(beta):
        e = R.qp_error_ntt(g)
        if gadget_q is None:
            add_q = np.zeros((R.nq, R.n), np.uint64)
            p_mod = [R.P % q for q in o.q]
            ps = o.scalar(s_ntt_q[0], p_mod, "Q")
            for j in range(i * alpha, min((i + 1) * alpha, R.nq)):
                add_q[j] = ps[j]
            part = (o.add(e[0], add_q, "Q"), e[1])
        else:
            gq = o.scalar(s_ntt_q[0], gadget_q[i], "Q")
            gp = o.scalar(s_ntt_q[1], gadget_p[i], "P")
            part = (o.add(e[0], gq, "Q"), o.add(e[1], gp, "P"))
        out.append(part)
    return out


@dataclass
class KKLSSKeys:
    secrets: List[np.ndarray]
    r: List[np.ndarray]
    crs_a: np.ndarray     # [betaMax][nQ+nP][N] MForm (CRS[0])
    crs_u: np.ndarray     # [betaMax][nQ+nP][N] MForm (CRS[-1])
    crs_a2: Optional[np.ndarray]  # CRS[-3] for BFV
    rlk: np.ndarray       # CKKS: [k][3][beta][nQ+nP][N]; BFV: [k][2][3][beta][nQ+nP][N]
    public: list          # per party (pk0, pk1) over Q NTT, true values


def _crs(R: RNS, beta: int, g):
    """CRS digits: uniform, stored in MForm (mkrlwe/params.go:49-58)."""
    true = [R.qp_uniform(g) for _ in range(beta)]
    stored = np.stack([R.qp_pack(R.qp_mform(t)) for t in true])
    return true, stored


def bfv_gadgets(R: RNS, t: int, gamma: int = 2):
    """G residues of mkbfv/keygen.go:174-244 for both halves."""
    o = R.o
    alpha = R.np_ // gamma
    beta = (R.nq + alpha - 1) // alpha
    Q = 1
    for q in o.q:
        Q *= q
    QM = 1
    for q in o.q_mul:
        QM *= q
    QQM = Q * QM
    halves = []
    for moduli in (o.q, o.q_mul):
        gq, gp = [], []
        for i in range(beta):
            Qi = 1
            for j in range(alpha):
                Qi *= moduli[i * alpha + j]
            Gi = QQM // Qi
            Ti = pow((QQM // Qi) % Qi, -1, Qi)
            Gi = Gi * t * Ti * R.P // QM
            gq.append([Gi % q for q in o.q])
            gp.append([Gi % p for p in o.p])
        halves.append((gq, gp))
    return halves


def kklss_keygen(R: RNS, k: int, seed: int, bfv_t: int = 0) -> KKLSSKeys:
    o = R.o
    gamma = 2
    alpha = R.np_ // gamma
    beta = (R.nq + alpha - 1) // alpha
    g0 = rng(seed * 7919 + 1)
    a_true, crs_a = _crs(R, beta, g0)
    u_true, crs_u = _crs(R, beta, g0)
    a2_true, crs_a2 = (None, None)
    if bfv_t:
        a2_true, crs_a2 = _crs(R, beta, g0)
        gad = bfv_gadgets(R, bfv_t, gamma)
    secrets, rs, rlks, public = [], [], [], []
    for i in range(k):
        g = rng(seed * 7919 + 100 + i)
        s, r = ternary(g, R.n), ternary(g, R.n)
        secrets.append(s)
        rs.append(r)
        s_ntt, r_ntt = R.qp_secret_ntt(s), R.qp_secret_ntt(r)
        v_part = kklss_switch_part(R, r_ntt, g, gamma=gamma)
        v = [R.qp_neg(R.qp_add(v_part[j], R.qp_mul(u_true[j], s_ntt))) for j in range(beta)]
        V = np.stack([R.qp_pack(R.qp_mform(x)) for x in v])
        if not bfv_t:
            b = [R.qp_sub(R.qp_error_ntt(g), R.qp_mul(a_true[j], s_ntt)) for j in range(beta)]
            d_part = kklss_switch_part(R, s_ntt, g, gamma=gamma)
            d = [R.qp_sub(d_part[j], R.qp_mul(a_true[j], r_ntt)) for j in range(beta)]
            B = np.stack([R.qp_pack(R.qp_mform(x)) for x in b])
            D = np.stack([R.qp_pack(R.qp_mform(x)) for x in d])
            rlks.append(np.stack([B, D, V]))
        else:
            halves = []
            for h, a_h in enumerate((a_true, a2_true)):
                b = [R.qp_sub(R.qp_error_ntt(g), R.qp_mul(a_h[j], s_ntt)) for j in range(beta)]
                gq, gp = gad[h]
                d_part = kklss_switch_part(R, s_ntt, g, gq, gp, gamma)
                d = [R.qp_sub(d_part[j], R.qp_mul(a_h[j], r_ntt)) for j in range(beta)]
                B = np.stack([R.qp_pack(R.qp_mform(x)) for x in b])
                D = np.stack([R.qp_pack(R.qp_mform(x)) for x in d])
                halves.append(np.stack([B, D, V if h == 0 else np.zeros_like(V)]))
            rlks.append(np.stack(halves))
        # public key (mkrlwe/keygen.go:88-109): a = CRS[0] digit 0 over Q
        e = o.ntt(o.from_int(gaussian(g, R.n), "Q"), "Q")
        a0 = a_true[0][0]
        public.append((o.sub(e, o.mul(a0, s_ntt[0])), a0))
    return KKLSSKeys(secrets, rs, crs_a, crs_u, crs_a2, np.stack(rlks), public)


def kklss_encrypt(o: Oracle, pk, m_coeff_q: np.ndarray, level: int, g):
    """mkrlwe/encryptor.go:95-158, coefficient-domain output:
    (InvNTT(v*pk0) + e0 + m, InvNTT(v*pk1) + e1)."""
    nl = level + 1
    v = o.ntt(o.from_int(ternary(g, o.n), "Q", 0, nl), "Q")
    c0 = o.intt(o.mul(v, pk[0][:nl]), "Q")
    c1 = o.intt(o.mul(v, pk[1][:nl]), "Q")
    c0 = o.add(o.add(c0, o.from_int(gaussian(g, o.n), "Q", 0, nl)), m_coeff_q[:nl])
    c1 = o.add(c1, o.from_int(gaussian(g, o.n), "Q", 0, nl))
    return c0, c1


# ----------------------------------------------------------------------------
# CRT / encoding / decoding
# ----------------------------------------------------------------------------


def crt_centered(residues: np.ndarray, moduli: Sequence[int]) -> List[int]:
    """Exact CRT reconstruction of [L][N] residues, centered in (-Q/2, Q/2]."""
    Q = 1
    for q in moduli:
        Q *= int(q)
    basis = []
    for q in moduli:
        q = int(q)
        Qi = Q // q
        basis.append(Qi * pow(Qi % q, -1, q))
    n = residues.shape[1]
    cols = [[int(x) for x in residues[i]] for i in range(len(moduli))]
    out = []
    half = Q // 2
    for x in range(n):
        v = 0
        for i in range(len(moduli)):
            v += cols[i][x] * basis[i]
        v %= Q
        if v > half:
            v -= Q
        out.append(v)
    return out


class CKKSEncoder:
    """Canonical-embedding encoder with slots at the roots zeta^(5^j)."""

    def __init__(self, log_n: int):
        self.n = 1 << log_n
        n = self.n
        self.zeta = np.exp(1j * np.pi * np.arange(n) / n)
        exps = np.ones(n // 2, dtype=np.int64)
        for j in range(1, n // 2):
            exps[j] = exps[j - 1] * 5 % (2 * n)
        self.k_pos = (exps - 1) // 2
        self.k_neg = (2 * n - exps - 1) // 2

    def encode(self, z: np.ndarray, scale: float) -> np.ndarray:
        n = self.n
        vals = np.zeros(n, np.complex128)
        vals[self.k_pos] = z
        vals[self.k_neg] = np.conj(z)
        m = np.fft.fft(vals) / n * np.conj(self.zeta)
        return np.rint(m.real * scale).astype(np.int64)

    def decode(self, coeffs: Sequence[int], scale: float) -> np.ndarray:
        c = np.array([float(x) / scale for x in coeffs])
        vals = self.n * np.fft.ifft(c * self.zeta)
        return vals[self.k_pos]


def precision_bits(got: np.ndarray, want: np.ndarray) -> float:
    err = np.max(np.abs(got - want))
    return float(-np.log2(err)) if err > 0 else 64.0


# ----------------------------------------------------------------------------
# Galois keys (rotations / conjugation)
# ----------------------------------------------------------------------------


def automorphism_int(s: np.ndarray, galois: int) -> np.ndarray:
    """X -> X^galois on a signed coefficient vector (Lattigo ring.Permute)."""
    n = len(s)
    out = np.zeros(n, dtype=np.int64)
    for i in range(n):
        raw = i * galois
        v = int(s[i])
        out[raw % n] = -v if (raw // n) % 2 else v
    return out


def mkf_rotation_keys(R: RNS, keys: MKFKeys, galois: int, seed: int) -> np.ndarray:
    """One sigma(s_i) -> s_E switching key per party (the paper evaluator's
    rotation keys, software/mkf/mkf_cpu/true_mkf_ckks.go:321-360)."""
    agg_ntt = R.qp_secret_ntt(keys.aggregate)
    out = []
    for i, s in enumerate(keys.secrets):
        ss = R.qp_secret_ntt(automorphism_int(s, galois))
        out.append(mkf_switching_key(R, ss, agg_ntt, rng(seed * 1000 + 300 + i)))
    return np.stack(out)


def kklss_galois_keys(R: RNS, keys: KKLSSKeys, galois: int, seed: int, conjugation: bool = False):
    """KKLSS GenRotationKey / GenConjugationKey (software/kklss/mkrlwe/
    keygen.go:190-268) for every party, with a fresh CRS vector (CRS[rot] or
    CRS[-2]).  Rotation: rk = e + P s g - a sigma^-1(s); conjugation:
    ck = e + P sigma(s) g - a s.  Returns (keys [k][beta][nQ+nP][N] MForm,
    CRS stored [beta][nQ+nP][N])."""
    alpha = R.np_ // 2
    beta = (R.nq + alpha - 1) // alpha
    g0 = rng(seed * 7919 + 17)
    a_true, crs = _crs(R, beta, g0)
    n2 = 2 * R.n
    out = []
    for i, s in enumerate(keys.secrets):
        g = rng(seed * 7919 + 400 + i)
        s_ntt = R.qp_secret_ntt(s)
        if conjugation:
            gad = kklss_switch_part(R, R.qp_secret_ntt(automorphism_int(s, galois)), g, gamma=2)
            sub = s_ntt
        else:
            gad = kklss_switch_part(R, s_ntt, g, gamma=2)
            sub = R.qp_secret_ntt(automorphism_int(s, pow(galois, -1, n2)))
        k_ = [R.qp_sub(gad[j], R.qp_mul(a_true[j], sub)) for j in range(beta)]
        out.append(np.stack([R.qp_pack(R.qp_mform(x)) for x in k_]))
    return np.stack(out), crs
