"""Fixture directories written from the oracle in the reference's exporter
format (mkf_b200.fixtures), with the stage dumps the MKF exporter writes."""
import os

import numpy as np

from mkf_b200 import fixtures, params
from tests import helpers as H

CK = params.small("ckks", log_n=10, n_q=6, n_p=4, q_bits=50, first_bits=60, p_bits=60, scale_bits=50)
CK2 = params.small("ckks", log_n=11, n_q=5, n_p=2, q_bits=40, first_bits=55, p_bits=45, scale_bits=40)
BF = params.small("bfv", log_n=10, n_q=4, n_p=2, q_bits=54, p_bits=60)


def mkf_ckks_fixture(d, lit=CK, k=2, stages=True):
    level = lit.max_level
    case = H.mkf_ckks_case(lit, k, level)
    o = case.o
    out, lv, sc = o.mkf_ckks_mulrelin(k, level, case.left, case.right, case.keys.fold,
                                      case.keys.relin, True, lit.scale, lit.scale ** 2)
    fixtures.export_mkf(d, "MKF-CKKS", lit.name, lit, case.left, case.right, case.keys.fold,
                        case.keys.relin, out, lv)
    if stages:
        x = case.left[1]
        dec = o.decompose(1, level, o.intt(x, "Q"))
        fixtures._write_words(os.path.join(d, "debug_switch0_decomposition_qp.bin"), dec)
        o0, o1 = o.mkf_switch_one(level, x, case.keys.fold[0], True, True)
        fixtures._write_words(os.path.join(d, "debug_switch0_moddown_q.bin"), o0, o1)
        folds = []
        for side in (case.left, case.right):
            a0, a1 = side[0].copy(), np.zeros_like(side[0])
            for i in range(k):
                s0, s1 = o.mkf_switch_one(level, side[i + 1], case.keys.fold[i], True, True)
                a0, a1 = o.add(a0, s0), o.add(a1, s1)
            folds += [a0, a1]
        fixtures._write_words(os.path.join(d, "stage_fold_q.bin"), *folds)
    return case, out, lv


def mkf_bfv_fixture(d, lit=BF, k=2):
    case = H.mkf_bfv_case(lit, k)
    out = case.o.mkf_bfv_mulrelin(k, case.left, case.right, case.keys.fold, case.keys.relin, lit.t)
    fixtures.export_mkf(d, "MKF-BFV", lit.name, lit, case.left, case.right, case.keys.fold,
                        case.keys.relin, out, lit.max_level)
    return case, out


def kklss_ckks_fixture(d, lit=CK2, k=2):
    level = lit.max_level
    case = H.kklss_ckks_case(lit, k, level)
    out, lv, sc = case.o.kklss_ckks_mulrelin(k, level, case.has0, case.has1, case.op0, case.op1,
                                             case.keys.rlk, case.keys.crs_u, lit.scale, lit.scale,
                                             lit.scale)
    fixtures.export_kklss(d, "KKLSS-CKKS", lit.name, lit, case.op0, case.op1, list(case.keys.rlk),
                          case.keys.crs_u, out, lv)
    return case, out, lv
