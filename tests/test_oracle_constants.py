"""Pin the oracle's precompute layer against the reference's P1 known-answer
constants (tests/golden/p1_constants.json, extracted from
hardware/u55c/hls/include/par1_{ckks,bfv}_hls_constants.hpp by
tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from mkf_b200 import params
from oracle.oracle import Oracle

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "p1_constants.json")))


def vals(scheme, name):
    return GOLD[scheme][name]["values"]


@pytest.fixture(scope="module")
def ckks():
    lit = params.get("ckks", "P1")
    return lit, Oracle.from_literal(lit)


@pytest.fixture(scope="module")
def bfv():
    lit = params.get("bfv", "P1")
    return lit, Oracle.from_literal(lit)


def test_p1_chains_match_reference(ckks, bfv):
    assert list(ckks[0].q) == vals("ckks", "Q")
    assert list(ckks[0].p) == vals("ckks", "P")
    assert list(bfv[0].q) == vals("bfv", "Q")
    assert list(bfv[0].q_mul) == vals("bfv", "QM")
    assert list(bfv[0].p) == vals("bfv", "P")


@pytest.mark.parametrize("scheme", ["ckks", "bfv"])
def test_montgomery_and_ninv(scheme, ckks, bfv):
    lit, o = ckks if scheme == "ckks" else bfv
    for which, name, ninv in (("Q", "MRED_Q", "N_INV_Q"), ("P", "MRED_P", "N_INV_P")):
        mods = o.moduli(which)
        for i in range(len(mods)):
            c = o.ring_consts(which, i)
            assert c["qinv"] == vals(scheme, name)[i]
            assert c["ninv"] == vals(scheme, ninv)[i]
            assert (c["q"] * c["qinv"]) % (1 << 64) == 1
    if scheme == "bfv":
        for i in range(len(lit.q_mul)):
            c = o.ring_consts("QM", i)
            assert c["qinv"] == vals("bfv", "MRED_QM")[i]
            assert c["ninv"] == vals("bfv", "N_INV_QM")[i]


def test_r2(ckks):
    lit, _ = ckks
    for q, r2 in zip(lit.q, vals("ckks", "R2_Q")):
        assert pow(2, 128, q) == r2


@pytest.mark.parametrize("scheme", ["ckks", "bfv"])
def test_decomposition_modup_tables(scheme, ckks, bfv):
    """DECOMP_INV / DECOMP_QSTAR / DECOMP_MINUS_Q are Lattigo's basis-extension
    tables for each alpha=2 digit onto every QP target (fpga_constants_test.go:
    138-141, modUpFor)."""
    lit, o = ckks if scheme == "ckks" else bfv
    qp = list(lit.q) + list(lit.p)
    beta = GOLD[scheme]["BETA"]
    inv_g = np.array(vals(scheme, "DECOMP_INV"), dtype=object).reshape(beta, 2)
    qs_g = np.array(vals(scheme, "DECOMP_QSTAR"), dtype=object).reshape(beta, len(qp), 2)
    mq_g = np.array(vals(scheme, "DECOMP_MINUS_Q"), dtype=object).reshape(beta, len(qp))
    for d in range(beta):
        src = list(lit.q[2 * d: 2 * d + 2])
        inv, qmod, vq = Oracle.modup_consts(src, qp)
        assert [int(x) for x in inv] == list(inv_g[d])
        for t in range(len(qp)):
            if t in (2 * d, 2 * d + 1):
                continue  # own limbs are copied, not extended
            assert [int(x) for x in qmod[t]] == list(qs_g[d, t]), (d, t)
            assert int(vq[t, 1]) == mq_g[d, t], (d, t)


@pytest.mark.parametrize("scheme", ["ckks", "bfv"])
def test_moddown_tables(scheme, ckks, bfv):
    lit, o = ckks if scheme == "ckks" else bfv
    inv, qmod, vq = Oracle.modup_consts(list(lit.p), list(lit.q))
    assert [int(x) for x in inv] == vals(scheme, "P2Q_INV")
    g = np.array(vals(scheme, "P2Q_QSTAR"), dtype=object).reshape(len(lit.q), len(lit.p))
    for t in range(len(lit.q)):
        assert [int(x) for x in qmod[t]] == list(g[t])
        assert int(vq[t, 1]) == vals(scheme, "P2Q_MINUS_P")[t]
    md = Oracle.moddown_consts(list(lit.q), list(lit.p))
    assert [int(x) for x in md[-1]] == vals(scheme, "P_INV_Q")


def test_rescale_table(ckks):
    lit, o = ckks
    want = vals("ckks", "RESCALE_5_TO_4")
    got = [o.rescale_const(5, j) for j in range(5)]
    assert got == want


def test_bfv_q_qmul_tables(bfv):
    lit, o = bfv
    inv, qmod, vq = Oracle.modup_consts(list(lit.q), list(lit.q_mul))
    assert [int(x) for x in inv] == vals("bfv", "Q2M_INV")
    g = np.array(vals("bfv", "Q2M_QSTAR"), dtype=object).reshape(len(lit.q_mul), len(lit.q))
    for t in range(len(lit.q_mul)):
        assert [int(x) for x in qmod[t]] == list(g[t])
        assert int(vq[t, 1]) == vals("bfv", "Q2M_MINUS_Q")[t]
    inv, qmod, vq = Oracle.modup_consts(list(lit.q_mul), list(lit.q))
    assert [int(x) for x in inv] == vals("bfv", "M2Q_INV")
    g = np.array(vals("bfv", "M2Q_QSTAR"), dtype=object).reshape(len(lit.q), len(lit.q_mul))
    for t in range(len(lit.q)):
        assert [int(x) for x in qmod[t]] == list(g[t])
        assert int(vq[t, 1]) == vals("bfv", "M2Q_MINUS_M")[t]
