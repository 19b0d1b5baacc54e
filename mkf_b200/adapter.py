"""The paper-facing (n+1)-component interface over the GPU path.

Mirrors paperMKFLattigoAdapter (software/mkf/mkf_cpu/true_mkf_ckks_adapter.go:
13-252) and paperMKFCKKSEvaluator (true_mkf_ckks.go:227-304): a k-party
MK-CKKS ciphertext is carried as c0 plus one component per party, all in the
NTT domain, so that code written against the carrier interface (packing,
linear layers, products) runs unchanged.

* MulRelinNew / MulRelin: the MKF product without rescale, output
  materialized to n+1 components (true_mkf_ckks.go:253-304);
* MulNew / Mul: a public NTT-domain plaintext applied to every component
  (adapter MulNew, :80-127);
* AddNew / SubNew / Add / Sub: component-wise linear operations (the
  embedded Lattigo evaluator's job in the reference);
* Rescale / RescaleNew (true_mkf_ckks.go RescaleNew; Lattigo Rescale);
* FoldToAggregate / MaterializeAggregate (foldCarrierToAggregate,
  materializeAggregate, :190-222).

* RotateNew / Rotate / RotateHoistedNew: the paper rotation with one
  sigma(s_i) -> s_E key per party and Galois element (:130-160,
  true_mkf_ckks.go:321-353), keys given per Galois element.

* EvaluatePoly: the reference's baby-step/giant-step schedule
  (true_mkf_ckks_polynomial.go) over these operations (mkf_b200.polynomial).

The collective refresh protocol is out of scope.
"""
from __future__ import annotations

from typing import Dict, Optional

from . import capi
from .evaluator import (Ciphertext, Evaluator, MKFEvaluator, MKFKeySet, Parameters,
                        galois_element)


class PaperMKFAdapter:
    def __init__(self, params: Parameters, keys: MKFKeySet,
                 rotations: Optional[Dict[int, MKFKeySet]] = None):
        """rotations: Galois element -> key set of the k sigma(s_i) -> s_E keys."""
        if params.scheme != "ckks":
            raise ValueError("the paper interface is MK-CKKS")
        self.params, self.keys = params, keys
        self.rotations = dict(rotations or {})
        self.parties = keys.k
        self._mkf = MKFEvaluator(params, keys)
        self._ev = Evaluator(params)

    # carriers -------------------------------------------------------------
    def NewCiphertext(self, level: int, scale: Optional[float] = None) -> Ciphertext:
        return Ciphertext(self.params, self.parties + 1, level, True,
                          scale=self.params.Scale() if scale is None else scale)

    def _check_carrier(self, ct: Ciphertext, what: str):
        if ct.n_comp != self.parties + 1:
            raise ValueError(f"{what}: expected a {self.parties + 1}-component carrier, got {ct.n_comp}")

    # products -------------------------------------------------------------
    def MulRelinNew(self, left: Ciphertext, right: Ciphertext) -> Ciphertext:
        self._check_carrier(left, "MulRelin")
        self._check_carrier(right, "MulRelin")
        return self._mkf.MulRelinNew(left, right, rescale=False, materialize=True)

    def MulRelin(self, left: Ciphertext, right: Ciphertext, out: Ciphertext):
        self._check_carrier(out, "MulRelin output")
        self._mkf.MulRelin(left, right, out, rescale=False, materialize=True)

    def MulNew(self, carrier: Ciphertext, public: Ciphertext) -> Ciphertext:
        self._check_carrier(carrier, "Mul")
        out = Ciphertext(self.params, carrier.n_comp, min(carrier.Level(), public.Level()), True)
        self.Mul(carrier, public, out)
        return out

    def Mul(self, carrier: Ciphertext, public: Ciphertext, out: Ciphertext):
        capi.check(self.params.handle, capi.lib().mkf_mul_plain(
            self.params.handle, carrier.handle, public.handle, out.handle, None))

    # linear -----------------------------------------------------------------
    def _ew(self, fn, a, b, out):
        capi.check(self.params.handle, fn(self.params.handle, a.handle, b.handle, out.handle, None))

    def AddNew(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        out = Ciphertext(self.params, a.n_comp, min(a.Level(), b.Level()), True)
        self._ew(capi.lib().mkf_add, a, b, out)
        return out

    def SubNew(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        out = Ciphertext(self.params, a.n_comp, min(a.Level(), b.Level()), True)
        self._ew(capi.lib().mkf_sub, a, b, out)
        return out

    def Add(self, a, b, out):
        self._ew(capi.lib().mkf_add, a, b, out)

    def Sub(self, a, b, out):
        self._ew(capi.lib().mkf_sub, a, b, out)

    # rescale ----------------------------------------------------------------
    def RescaleNew(self, ct: Ciphertext, minScale: Optional[float] = None) -> Ciphertext:
        return self._ev.RescaleNew(ct, self.params.Scale() if minScale is None else minScale)

    def Rescale(self, ct: Ciphertext, minScale: float, out: Ciphertext):
        self._ev.Rescale(ct, minScale, out)

    # aggregate form ---------------------------------------------------------
    def FoldToAggregate(self, carrier: Ciphertext) -> Ciphertext:
        """The compact (c0, Gamma) pair under the aggregate secret."""
        self._check_carrier(carrier, "fold")
        out = Ciphertext(self.params, 2, carrier.Level(), True)
        capi.check(self.params.handle, capi.lib().mkf_mkf_fold(
            self.params.handle, carrier.handle, self.keys.handle, out.handle, None))
        return out

    def MaterializeAggregate(self, compact: Ciphertext) -> Ciphertext:
        """c0, then Gamma once per party."""
        out = Ciphertext(self.params, self.parties + 1, compact.Level(), True)
        capi.check(self.params.handle, capi.lib().mkf_mkf_materialize(
            self.params.handle, compact.handle, out.handle, None))
        return out

    # not provided -----------------------------------------------------------
    def RotateNew(self, ct: Ciphertext, rotation: int) -> Ciphertext:
        self._check_carrier(ct, "Rotate")
        if rotation % (self.params.N // 2) == 0:
            out = self.NewCiphertext(ct.Level(), ct.Scale)
            out.upload(ct.download())
            return out
        g = galois_element(self.params, rotation)
        keys = self.rotations.get(g)
        if keys is None or keys.k != self.parties:
            raise capi.MissingKeyError(
                5, f"party-specific Galois keys missing for rotation {rotation} (element {g})")
        return self._mkf.RotateNew(ct, g, keys, materialize=True)

    def Rotate(self, ct: Ciphertext, rotation: int, out: Ciphertext):
        out.upload(self.RotateNew(ct, rotation).download())

    def RotateHoistedNew(self, ct: Ciphertext, rotations):
        return {r: self.RotateNew(ct, r) for r in rotations}

    def EvaluatePoly(self, ct: Ciphertext, polynomial, targetScale: float) -> Ciphertext:
        """paperMKFCKKSEvaluator.EvaluatePoly (true_mkf_ckks_polynomial.go:79-111):
        `polynomial` is a mkf_b200.polynomial.Polynomial in the standard or
        Chebyshev basis (input already mapped for the latter)."""
        from .polynomial import EvaluatePoly
        self._check_carrier(ct, "EvaluatePoly")
        return EvaluatePoly(self, ct, polynomial, targetScale)
