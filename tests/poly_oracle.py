"""The polynomial schedule (mkf_b200.polynomial.Schedule) over carrier
operations built from the oracle: the reference for the GPU backend."""
from dataclasses import dataclass

import numpy as np

from mkf_b200.polynomial import add_const_residues, gauss_residues, lattigo_add_scales


@dataclass
class OCt:
    a: np.ndarray  # [k+1][level+1][N], NTT domain
    scale: float

    @property
    def level(self):
        return self.a.shape[1] - 1


class OracleBackend:
    def __init__(self, o, fold, relin, k):
        self.o, self.fold, self.relin, self.k = o, fold, relin, k
        self.q = list(o.q)
        x = np.zeros((len(self.q), o.n), np.uint64)
        x[:, o.n // 2] = 1
        self.iq = [int(v) for v in o.ntt(x, "Q")[:, 0]]

    def level(self, ct):
        return ct.level

    def scale(self, ct):
        return ct.scale

    def copy(self, ct):
        return OCt(ct.a.copy(), ct.scale)

    def with_scale(self, ct, s):
        return OCt(ct.a, s)

    def zero(self, level, scale):
        return OCt(np.zeros((self.k + 1, level + 1, self.o.n), np.uint64), scale)

    def drop_level(self, ct, n):
        return OCt(np.ascontiguousarray(ct.a[:, : ct.level + 1 - n]), ct.scale)

    def _fold(self, a):
        o, L = self.o, a.shape[1] - 1
        f0, f1 = a[0].copy(), np.zeros_like(a[0])
        for i in range(self.k):
            s0, s1 = o.mkf_switch_one(L, a[i + 1], self.fold[i], True, True)
            f0, f1 = o.add(f0, s0), o.add(f1, s1)
        return f0, f1

    def mul_relin(self, x, y):
        o = self.o
        lv = min(x.level, y.level)
        l0, l1 = (v[: lv + 1] for v in self._fold(x.a))
        r0, r1 = (v[: lv + 1] for v in self._fold(y.a))
        mu0, mu2 = o.mul(l0, r0), o.mul(l1, r1)
        mu1 = o.sub(o.sub(o.mul(o.add(l0, l1), o.add(r0, r1)), mu0), mu2)
        u0, u1 = o.mkf_switch_one(lv, mu2, self.relin, True, True)
        c0, g = o.add(mu0, u0), o.add(mu1, u1)
        return OCt(np.stack([c0] + [g] * self.k), x.scale * y.scale)

    def rescale(self, ct, target):
        o = self.o
        a, s = ct.a, ct.scale
        lv = ct.level
        if lv == 0:
            raise ValueError("cannot rescale at level 0")
        while lv > 0 and s / float(self.q[lv]) >= target / 2:
            a = np.stack([o.rescale(lv, a[u], True) for u in range(a.shape[0])])
            s /= float(self.q[lv])
            lv -= 1
        return OCt(a, s)

    def _mulc(self, a, residues):
        o, N = self.o, self.o.n
        c = np.zeros((a.shape[1], N), np.uint64)
        c[:, : N // 2] = residues[:, 0:1]
        c[:, N // 2:] = residues[:, 1:2]
        return np.stack([o.mul(a[u], c) for u in range(a.shape[0])])

    def _addsub(self, x, y, sub):
        fa, fb, sc = lattigo_add_scales(x.scale, y.scale)
        lv = min(x.level, y.level)
        a, b = x.a[:, : lv + 1], y.a[:, : lv + 1]
        if fa > 1:
            a = self._mulc(a, gauss_residues(fa, 0, self.q, self.iq, lv + 1))
        if fb > 1:
            b = self._mulc(b, gauss_residues(fb, 0, self.q, self.iq, lv + 1))
        fn = self.o.sub if sub else self.o.add
        return OCt(np.stack([fn(a[u], b[u]) for u in range(a.shape[0])]), sc)

    def add(self, x, y):
        return self._addsub(x, y, False)

    def sub(self, x, y):
        return self._addsub(x, y, True)

    def add_const(self, ct, value):
        o, N = self.o, self.o.n
        r = add_const_residues(complex(value), ct.scale, self.q, self.iq, ct.level + 1)
        c = np.zeros((ct.level + 1, N), np.uint64)
        c[:, : N // 2] = r[:, 0:1]
        c[:, N // 2:] = r[:, 1:2]
        a = ct.a.copy()
        a[0] = o.add(a[0], c)
        return OCt(a, ct.scale)

    def mult_gauss_add(self, ct, re, im, target):
        nl = target.level + 1
        prod = self._mulc(ct.a[:, :nl], gauss_residues(re, im, self.q, self.iq, nl))
        return OCt(np.stack([self.o.add(target.a[u], prod[u]) for u in range(prod.shape[0])]),
                   target.scale)


def decode_carrier(case, a, level, scale):
    """Decrypts an (n+1)-component carrier: c0 + sum_i c_i s_i (each party's
    own secret), then CKKS-decodes."""
    from oracle import keygen as kg
    o, lit = case.o, case.lit
    ph = a[0][: level + 1].copy()
    for i, s in enumerate(case.keys.secrets):
        sn = o.ntt(o.from_int(s, "Q", 0, level + 1), "Q")
        ph = o.add(ph, o.mul(a[i + 1][: level + 1], sn))
    ph = o.intt(ph, "Q")
    return kg.CKKSEncoder(lit.log_n).decode(kg.crt_centered(ph, lit.q[: level + 1]), scale)
