"""NTT phase splits (Parameters(..., ntt_row_log=)): a context built with the
other split of its ring degree computes the same transform and the same
products, word for word, as the default split."""
import numpy as np
import pytest

from mkf_b200 import autotune, capi, params
from mkf_b200 import evaluator as ev

pytestmark = pytest.mark.gpu


def _lit(log_n):
    return params.small("ckks", log_n=log_n, n_q=6, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                        scale_bits=45)


def _limbs(g, moduli, n, lead=()):
    out = np.empty(tuple(lead) + (len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = g.integers(0, q, size=tuple(lead) + (n,), dtype=np.uint64)
    return out


@pytest.mark.parametrize("log_n", [14, 15])
def test_other_split_gives_the_same_products(log_n):
    lit = _lit(log_n)
    default, other = autotune.split_options(log_n)
    ctxs = [ev.Parameters(lit, "ckks", ntt_row_log=rl) for rl in (default, other)]
    g = np.random.default_rng(log_n)
    qp = list(lit.q) + list(lit.p)
    beta = (len(lit.q) - 1 + len(lit.p)) // len(lit.p)
    k = 3
    fold = [_limbs(g, qp, lit.n, (beta, 2)) for _ in range(k)]
    relin = _limbs(g, qp, lit.n, (beta, 2))
    level = lit.max_level
    ops = [_limbs(g, lit.q[: level + 1], lit.n, (k + 1,)) for _ in range(2)]
    outs = []
    for P in ctxs:
        E = ev.MKFEvaluator(P, ev.MKFKeySet(P, fold, relin))
        left, right = (ev.Ciphertext.from_array(P, o, True, scale=lit.scale) for o in ops)
        got = []
        for fuse_ip in (0, 1):
            autotune.set_tuning(P, fuse_ip=fuse_ip)
            got.append(E.MulRelinNew(left, right, True, True).download())
        assert np.array_equal(got[0], got[1])
        outs.append(got[0])
    assert np.array_equal(outs[0], outs[1]), f"logN {log_n}: split {other} differs from {default}"


@pytest.mark.parametrize("log_n", [14, 15])
def test_other_split_ntt_matches(log_n):
    lit = _lit(log_n)
    default, other = autotune.split_options(log_n)
    g = np.random.default_rng(100 + log_n)
    x = _limbs(g, lit.q, lit.n)
    res = []
    for rl in (default, other):
        P = ev.Parameters(lit, "ckks", ntt_row_log=rl)
        L = capi.lib()
        r = []
        for inverse in (0, 1):
            out = np.empty_like(x)
            capi.check(P.handle, L.mkf_ntt_host(P.handle, 0, 0, len(lit.q), capi.ptr(x), capi.ptr(out),
                                                inverse))
            r.append(out)
        res.append(r)
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])


def test_unbuilt_split_is_refused():
    with pytest.raises(capi.MKFError):
        ev.Parameters(_lit(14), "ckks", ntt_row_log=9)
