"""Products at the benchmarked and served sizes, built from fixed seeds so that
a worker process and the test process build the same inputs.

``oracle_output(name)`` runs the oracle on the case ``name`` and returns its
output reduced mod q; the GPU tests compute these in a pool of spawned worker
processes while they build the same case themselves and run it on the GPU.
"""
from __future__ import annotations

import numpy as np

from mkf_b200 import params
from tests import helpers as H

# name -> (construction, scheme, parameter set, parties, level (-1: top))
CASES = {
    # MKF-CKKS C3 (logN 16, 60b + 23 x 50b, P = 4 x 60b), k = 8: the product
    # the benchmark times, at the top level and at level 8
    "mkf_ckks_c3_k8_top": ("mkf", "ckks", "C3", 8, -1),
    "mkf_ckks_c3_k8_l8": ("mkf", "ckks", "C3", 8, 8),
    # KKLSS-CKKS on the serving rings, k = 8
    "kklss_ckks_s14_k8_top": ("kklss", "ckks", "S14", 8, -1),
    "kklss_ckks_s15_k8_l9": ("kklss", "ckks", "S15", 8, 9),
    "kklss_ckks_s16_k8_top": ("kklss", "ckks", "S16", 8, -1),
    # KKLSS-BFV on the serving rings (S15 is the C2 chain), full level
    "kklss_bfv_s14_k8": ("kklss", "bfv", "S14", 8, -1),
    "kklss_bfv_c2_k4": ("kklss", "bfv", "C2", 4, -1),
    "kklss_bfv_s15_k8": ("kklss", "bfv", "S15", 8, -1),
    "kklss_bfv_s16_k8": ("kklss", "bfv", "S16", 8, -1),
}

SEED = {"mkf": 31, "kklss": 41}


def literal(name):
    _, scheme, pset, _, _ = CASES[name]
    return params.get(scheme, pset)


def build(name):
    """The seeded case (keys, operands, expected plaintext or slots)."""
    cons, scheme, _, k, level = CASES[name]
    lit = literal(name)
    lv = lit.max_level if level < 0 else level
    if cons == "mkf":
        return H.mkf_ckks_case(lit, k, lv, seed=SEED[cons])
    if scheme == "ckks":
        return H.kklss_ckks_case(lit, k, lv, seed=SEED[cons])
    return H.kklss_bfv_case(lit, k, seed=SEED[cons], sparse=True)


def run_oracle(name, case):
    """Oracle output (canonical) and, for CKKS, its level and scale."""
    cons, scheme, _, k, _ = CASES[name]
    lit = case.lit
    o = case.o
    if cons == "mkf":
        want, lv, sc = o.mkf_ckks_mulrelin(k, case.level, case.left, case.right, case.keys.fold,
                                           case.keys.relin, True, lit.scale, lit.scale ** 2)
        return H.canon(want, lit.q[: lv + 1]), lv, sc
    if scheme == "ckks":
        want, lv, sc = o.kklss_ckks_mulrelin(k, case.level, case.has0, case.has1, case.op0,
                                             case.op1, case.keys.rlk, case.keys.crs_u, lit.scale,
                                             lit.scale, lit.scale)
        return H.canon(want, lit.q[: lv + 1]), lv, sc
    want = o.kklss_bfv_mulrelin(k, case.has0, case.has1, case.op0, case.op1, case.keys.rlk,
                                case.keys.crs_u, lit.t)
    return H.canon(want, lit.q), lit.max_level, 0.0


def oracle_output(name):
    """Worker entry point: build the case and run the oracle on it."""
    case = build(name)
    out, lv, sc = run_oracle(name, case)
    return np.ascontiguousarray(out), lv, sc
