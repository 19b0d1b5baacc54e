"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle.c).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker or as the timed CPU
baseline.  The product (``mkf_b200``) never imports it.  See oracle.h for the
parity status (psi/twiddle tables unpinned, P1 constants pinned).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build() -> str:
    """Compile oracle.c with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = ctypes.CDLL(_LIB_PATH)
    vp = ctypes.c_void_p
    i = ctypes.c_int
    d = ctypes.c_double
    L.oracle_ctx_new.restype = vp
    L.oracle_ctx_new.argtypes = [i, _u64p, i, _u64p, i, _u64p, i]
    L.oracle_ctx_free.argtypes = [vp]
    L.oracle_ring_consts.argtypes = [vp, i, i, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p]
    L.oracle_rescale_const.restype = ctypes.c_uint64
    L.oracle_rescale_const.argtypes = [vp, i, i]
    L.oracle_modup_consts.argtypes = [_u64p, i, _u64p, i, _u64p, _u64p, _u64p]
    L.oracle_moddown_consts.argtypes = [_u64p, i, _u64p, i, _u64p]
    L.oracle_ntt.argtypes = [vp, i, i, i, _u64p, _u64p, i]
    L.oracle_decompose.argtypes = [vp, i, i, _u64p, _u64p]
    L.oracle_modup_q_to_p.argtypes = [vp, i, _u64p, _u64p]
    L.oracle_modup_p_to_q.argtypes = [vp, i, _u64p, _u64p]
    L.oracle_moddown.argtypes = [vp, i, i, _u64p, _u64p]
    L.oracle_rescale.argtypes = [vp, i, i, _u64p, _u64p]
    L.oracle_mkf_switch_one.argtypes = [vp, i, i, _u64p, _u64p, i, _u64p, _u64p]
    L.oracle_mkf_ckks_mulrelin.restype = i
    L.oracle_mkf_ckks_mulrelin.argtypes = [vp, i, i, _u64p, _u64p, _u64p, _u64p, i, d,
                                           ctypes.POINTER(d), _u64p]
    L.oracle_mkf_bfv_mulrelin.restype = i
    L.oracle_mkf_bfv_mulrelin.argtypes = [vp, i, _u64p, _u64p, _u64p, _u64p,
                                          ctypes.c_uint64, _u64p]
    L.oracle_kklss_ckks_mulrelin.restype = i
    L.oracle_kklss_ckks_mulrelin.argtypes = [vp, i, i, _u8p, _u8p, _u64p, _u64p, _u64p,
                                             _u64p, d, d, d, ctypes.POINTER(d), _u64p]
    L.oracle_kklss_bfv_mulrelin.restype = i
    L.oracle_kklss_bfv_mulrelin.argtypes = [vp, i, _u8p, _u8p, _u64p, _u64p, _u64p,
                                            _u64p, ctypes.c_uint64, _u64p]
    L.oracle_automorphism.argtypes = [vp, i, _u64p, ctypes.c_uint64, _u64p]
    L.oracle_kklss_external_product.argtypes = [vp, i, _u64p, _u64p, _u64p]
    L.oracle_mform.restype = ctypes.c_uint64
    L.oracle_mform.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    for name in ("oracle_poly_mul", "oracle_poly_add", "oracle_poly_sub"):
        getattr(L, name).argtypes = [vp, i, i, i, _u64p, _u64p, _u64p]
    L.oracle_poly_mform.argtypes = [vp, i, i, i, _u64p, _u64p]
    L.oracle_poly_scalar.argtypes = [vp, i, i, i, _u64p, _u64p, _u64p]
    L.oracle_poly_from_i64.argtypes = [vp, i, i, i, _i64p, _u64p]
    _lib = L
    return L


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_u64p)


def _arr(v: Sequence[int]) -> np.ndarray:
    return np.ascontiguousarray(np.array([int(x) for x in v], dtype=np.uint64))


WHICH = {"Q": 0, "P": 1, "QM": 2, "R": 3}


class Oracle:
    """One parameter context of the oracle."""

    def __init__(self, log_n: int, q: Sequence[int], p: Sequence[int],
                 q_mul: Sequence[int] = ()):
        self.L = lib()
        self.log_n = log_n
        self.n = 1 << log_n
        self.q = [int(x) for x in q]
        self.p = [int(x) for x in p]
        self.q_mul = [int(x) for x in q_mul]
        self._q, self._pp, self._qm = _arr(self.q), _arr(self.p), _arr(self.q_mul or [1])
        self.ctx = self.L.oracle_ctx_new(log_n, _p(self._q), len(self.q), _p(self._pp),
                                         len(self.p), _p(self._qm), len(self.q_mul))

    @classmethod
    def from_literal(cls, lit) -> "Oracle":
        return cls(lit.log_n, lit.q, lit.p, lit.q_mul)

    def close(self):
        if self.ctx:
            self.L.oracle_ctx_free(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # moduli ----------------------------------------------------------------
    def moduli(self, which: str):
        return {"Q": self.q, "P": self.p, "QM": self.q_mul, "R": self.q + self.q_mul}[which]

    def beta_max(self, gamma: int) -> int:
        alpha = len(self.p) // gamma
        return (len(self.q) + alpha - 1) // alpha

    # tables ----------------------------------------------------------------
    def ring_consts(self, which: str, idx: int):
        q, qinv, ninv, g = (ctypes.c_uint64() for _ in range(4))
        psi = np.zeros(self.n, np.uint64)
        psiinv = np.zeros(self.n, np.uint64)
        self.L.oracle_ring_consts(self.ctx, WHICH[which], idx, ctypes.byref(q), ctypes.byref(qinv),
                                  ctypes.byref(ninv), _p(psi), _p(psiinv), ctypes.byref(g))
        return dict(q=q.value, qinv=qinv.value, ninv=ninv.value, g=g.value, psi=psi, psiinv=psiinv)

    def rescale_const(self, i: int, j: int) -> int:
        return int(self.L.oracle_rescale_const(self.ctx, i, j))

    @staticmethod
    def modup_consts(src: Sequence[int], tgt: Sequence[int]):
        L = lib()
        s, t = _arr(src), _arr(tgt)
        inv = np.zeros(len(src), np.uint64)
        qmod = np.zeros((len(tgt), len(src)), np.uint64)
        vq = np.zeros((len(tgt), len(src) + 1), np.uint64)
        L.oracle_modup_consts(_p(s), len(src), _p(t), len(tgt), _p(inv), _p(qmod), _p(vq))
        return inv, qmod, vq

    @staticmethod
    def moddown_consts(Q: Sequence[int], P: Sequence[int]):
        L = lib()
        out = np.zeros((len(P), len(Q)), np.uint64)
        L.oracle_moddown_consts(_p(_arr(Q)), len(Q), _p(_arr(P)), len(P), _p(out))
        return out

    # elementwise / NTT -------------------------------------------------------
    def ntt(self, a: np.ndarray, which: str = "Q", first: int = 0, inverse: bool = False) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64)
        nl = a.size // self.n
        out = np.empty_like(a)
        self.L.oracle_ntt(self.ctx, WHICH[which], first, nl, _p(a), _p(out), int(inverse))
        return out

    def intt(self, a, which="Q", first=0):
        return self.ntt(a, which, first, inverse=True)

    def _ew(self, fn, a, b, which, first):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = np.empty_like(a)
        fn(self.ctx, WHICH[which], first, a.size // self.n, _p(a), _p(b), _p(out))
        return out

    def mul(self, a, b, which="Q", first=0):
        return self._ew(self.L.oracle_poly_mul, a, b, which, first)

    def add(self, a, b, which="Q", first=0):
        return self._ew(self.L.oracle_poly_add, a, b, which, first)

    def sub(self, a, b, which="Q", first=0):
        return self._ew(self.L.oracle_poly_sub, a, b, which, first)

    def mform(self, a, which="Q", first=0):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.empty_like(a)
        self.L.oracle_poly_mform(self.ctx, WHICH[which], first, a.size // self.n, _p(a), _p(out))
        return out

    def scalar(self, a, residues, which="Q", first=0):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.empty_like(a)
        s = _arr(residues)
        self.L.oracle_poly_scalar(self.ctx, WHICH[which], first, a.size // self.n, _p(a), _p(s), _p(out))
        return out

    def from_int(self, v: np.ndarray, which="Q", first=0, nlimbs: Optional[int] = None) -> np.ndarray:
        v = np.ascontiguousarray(v, dtype=np.int64)
        if nlimbs is None:
            nlimbs = len(self.moduli(which)) - first
        out = np.empty((nlimbs, self.n), np.uint64)
        self.L.oracle_poly_from_i64(self.ctx, WHICH[which], first, nlimbs, v.ctypes.data_as(_i64p), _p(out))
        return out

    # path primitives --------------------------------------------------------------
    def decompose(self, gamma: int, level: int, coeff: np.ndarray) -> np.ndarray:
        alpha = len(self.p) // gamma
        beta = (level + alpha) // alpha
        coeff = np.ascontiguousarray(coeff, dtype=np.uint64)
        out = np.zeros((beta, level + 1 + len(self.p), self.n), np.uint64)
        self.L.oracle_decompose(self.ctx, gamma, level, _p(coeff), _p(out))
        return out

    def modup_q_to_p(self, level, a):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros((len(self.p), self.n), np.uint64)
        self.L.oracle_modup_q_to_p(self.ctx, level, _p(a), _p(out))
        return out

    def modup_p_to_q(self, level, a):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros((level + 1, self.n), np.uint64)
        self.L.oracle_modup_p_to_q(self.ctx, level, _p(a), _p(out))
        return out

    def moddown(self, level, qp, ntt: bool):
        qp = np.ascontiguousarray(qp, dtype=np.uint64)
        out = np.zeros((level + 1, self.n), np.uint64)
        self.L.oracle_moddown(self.ctx, level, int(ntt), _p(qp), _p(out))
        return out

    def rescale(self, level, a, ntt: bool):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros((level, self.n), np.uint64)
        self.L.oracle_rescale(self.ctx, level, int(ntt), _p(a), _p(out))
        return out

    def mkf_switch_one(self, level, x, key, in_ntt=True, ntt_output=True):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        key = np.ascontiguousarray(key, dtype=np.uint64)
        o0 = np.zeros((level + 1, self.n), np.uint64)
        o1 = np.zeros_like(o0)
        self.L.oracle_mkf_switch_one(self.ctx, level, int(in_ntt), _p(x), _p(key), int(ntt_output),
                                     _p(o0), _p(o1))
        return o0, o1

    def mkf_ckks_mulrelin(self, k, level, left, right, fold_keys, relin, rescale=True,
                          target_scale=1.0, scale_in=1.0):
        left = np.ascontiguousarray(left, dtype=np.uint64)
        right = np.ascontiguousarray(right, dtype=np.uint64)
        fk = np.ascontiguousarray(fold_keys, dtype=np.uint64)
        rk = np.ascontiguousarray(relin, dtype=np.uint64)
        out = np.zeros((2, level + 1, self.n), np.uint64)
        sc = ctypes.c_double(scale_in)
        lv = self.L.oracle_mkf_ckks_mulrelin(self.ctx, k, level, _p(left), _p(right), _p(fk), _p(rk),
                                             int(rescale), float(target_scale), ctypes.byref(sc), _p(out))
        if lv < 0:
            raise ValueError("oracle MKF CKKS mult+relin failed")
        return np.ascontiguousarray(out.reshape(-1)[: 2 * (lv + 1) * self.n].reshape(2, lv + 1, self.n)), lv, sc.value

    def mkf_bfv_mulrelin(self, k, left, right, fold_keys, relin, t):
        out = np.zeros((2, len(self.q), self.n), np.uint64)
        self.L.oracle_mkf_bfv_mulrelin(self.ctx, k, _p(np.ascontiguousarray(left)), _p(np.ascontiguousarray(right)),
                                       _p(np.ascontiguousarray(fold_keys)), _p(np.ascontiguousarray(relin)), int(t), _p(out))
        return out

    def kklss_ckks_mulrelin(self, k, level, has0, has1, op0, op1, rlk, crs_u, scale0, scale1, target_scale):
        h0 = np.ascontiguousarray(np.array(has0, np.uint8))
        h1 = np.ascontiguousarray(np.array(has1, np.uint8))
        out = np.zeros((k + 1, level + 1, self.n), np.uint64)
        so = ctypes.c_double(0.0)
        lv = self.L.oracle_kklss_ckks_mulrelin(
            self.ctx, k, level, h0.ctypes.data_as(_u8p), h1.ctypes.data_as(_u8p),
            _p(np.ascontiguousarray(op0)), _p(np.ascontiguousarray(op1)), _p(np.ascontiguousarray(rlk)),
            _p(np.ascontiguousarray(crs_u)), float(scale0), float(scale1), float(target_scale),
            ctypes.byref(so), _p(out))
        flat = out.reshape(-1)[: (k + 1) * (lv + 1) * self.n]
        return np.ascontiguousarray(flat.reshape(k + 1, lv + 1, self.n)), lv, so.value

    # Galois automorphisms and rotations -----------------------------------
    def galois_element(self, rotation: int) -> int:
        """Lattigo GaloisElementForColumnRotationBy: 5^r mod 2N, r taken mod N/2."""
        return pow(5, rotation % (self.n // 2), 2 * self.n)

    def conjugation_element(self) -> int:
        """GaloisElementForRowRotation: 2N - 1."""
        return 2 * self.n - 1

    def automorphism(self, level, a, galois):
        """X -> X^galois on the coefficient domain of Q limbs [0, level]."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.empty_like(a)
        for c in range(a.size // ((level + 1) * self.n)):
            x = np.ascontiguousarray(a.reshape(-1, level + 1, self.n)[c])
            y = np.empty_like(x)
            self.L.oracle_automorphism(self.ctx, level, _p(x), int(galois), _p(y))
            out.reshape(-1, level + 1, self.n)[c] = y
        return out

    def automorphism_ntt(self, level, a, galois):
        """mkfAutomorphismNTT (true_mkf_ckks.go:307-320): InvNTT, permute, NTT."""
        return self.ntt(self.automorphism(level, self.intt(a, "Q"), galois), "Q")

    def kklss_external_product(self, level, a_coeff, bg):
        a = np.ascontiguousarray(a_coeff, dtype=np.uint64)
        out = np.zeros((level + 1, self.n), np.uint64)
        self.L.oracle_kklss_external_product(self.ctx, level, _p(a), _p(np.ascontiguousarray(bg)), _p(out))
        return out

    def kklss_rotate(self, level, ct, rot_keys, crs, galois):
        """KKLSS rotation (RotateHoisted, software/kklss/mkrlwe/keyswitch_hoisted.go:
        198-249): c0 += sum_i Ext(c_i, rk_i); c_i = Ext(c_i, CRS[rot]); then
        every component permuted.  ct: [k+1][level+1][N] coefficient domain."""
        k = ct.shape[0] - 1
        out = np.empty_like(ct)
        c0 = ct[0].copy()
        for i in range(k):
            c0 = self.add(c0, self.kklss_external_product(level, ct[i + 1], rot_keys[i]))
            out[i + 1] = self.kklss_external_product(level, ct[i + 1], crs)
        out[0] = c0
        return self.automorphism(level, out, galois)

    def kklss_conjugate(self, level, ct, conj_keys, crs, galois):
        """KKLSS conjugation (Conjugate, keyswitch.go:301-343, with the gadget
        product of keyswitch_hoisted.go:11-45): every component permuted, then
        c0 += sum_i Ext(c_i, ck_i); c_i = Ext(c_i, CRS[-2])."""
        k = ct.shape[0] - 1
        p = self.automorphism(level, ct, galois)
        out = p.copy()
        for i in range(k):
            out[0] = self.add(out[0], self.kklss_external_product(level, p[i + 1], conj_keys[i]))
            out[i + 1] = self.kklss_external_product(level, p[i + 1], crs)
        return out

    def mkf_rotate(self, level, ct, rot_keys, galois):
        """MKF paper RotateNew (true_mkf_ckks.go:323-353): sigma(C0) + sum_i
        switchOne(sigma(c_i), rk_i)[0], and sum_i switchOne(...)[1]; NTT domain.
        Returns the compact pair."""
        k = ct.shape[0] - 1
        a0 = self.automorphism_ntt(level, ct[0], galois)
        a1 = np.zeros_like(a0)
        for i in range(k):
            u0, u1 = self.mkf_switch_one(level, self.automorphism_ntt(level, ct[i + 1], galois),
                                         rot_keys[i], True, True)
            a0, a1 = self.add(a0, u0), self.add(a1, u1)
        return np.stack([a0, a1])

    def kklss_bfv_mulrelin(self, k, has0, has1, op0, op1, rlk, crs_u, t):
        h0 = np.ascontiguousarray(np.array(has0, np.uint8))
        h1 = np.ascontiguousarray(np.array(has1, np.uint8))
        out = np.zeros((k + 1, len(self.q), self.n), np.uint64)
        self.L.oracle_kklss_bfv_mulrelin(
            self.ctx, k, h0.ctypes.data_as(_u8p), h1.ctypes.data_as(_u8p),
            _p(np.ascontiguousarray(op0)), _p(np.ascontiguousarray(op1)), _p(np.ascontiguousarray(rlk)),
            _p(np.ascontiguousarray(crs_u)), int(t), _p(out))
        return out
