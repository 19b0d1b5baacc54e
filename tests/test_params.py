"""Parameter sets: the reference's chains verbatim, and the benchmark chains
built by the stated rule (largest NTT-friendly primes below 2^b)."""
import pytest

from mkf_b200 import params
from oracle.oracle import Oracle


def _is_prime(n):
    return params._is_prime(n)


@pytest.mark.parametrize("scheme,name", [("ckks", "C1"), ("ckks", "C3"), ("bfv", "C2"),
                                         ("ckks", "S15"), ("bfv", "S16")])
def test_generated_chains(scheme, name):
    lit = params.get(scheme, name)
    allm = list(lit.q) + list(lit.q_mul) + list(lit.p)
    assert len(set(allm)) == len(allm)
    for m in allm:
        assert _is_prime(m) and (m - 1) % (2 * lit.n) == 0 and m < 2 ** 61


def test_c3_shape():
    lit = params.get("ckks", "C3")
    assert lit.log_n == 16 and len(lit.q) == 24 and len(lit.p) == 4
    assert lit.q[0].bit_length() == 60 and all(q.bit_length() == 50 for q in lit.q[1:])
    assert all(p.bit_length() == 60 for p in lit.p)
    assert lit.scale == 2.0 ** 50
    # largest below 2^b: no larger NTT prime of that size is skipped
    step = 2 * lit.n
    q = (1 << 50) - 1
    q = q - (q - 1) % step
    first = None
    while first is None:
        if _is_prime(q):
            first = q
        q -= step
    assert lit.q[1] == first


def test_c2_shape():
    lit = params.get("bfv", "C2")
    assert lit.log_n == 15 and len(lit.q) == 15 and len(lit.q_mul) == 15 and len(lit.p) == 2
    assert lit.t == 65537


def test_c1_shape():
    lit = params.get("ckks", "C1")
    assert lit.log_n == 14 and len(lit.q) == 8 and len(lit.p) == 2
    assert lit.q[0].bit_length() == 55 and all(q.bit_length() == 40 for q in lit.q[1:])
    assert all(p.bit_length() == 45 for p in lit.p)


def test_alpha_beta():
    lit = params.get("ckks", "C3")
    assert params.alpha_beta(lit, 23, 1) == (4, 6)
    assert params.alpha_beta(lit, 23, 2) == (2, 12)
    assert params.alpha_beta(lit, 8, 1) == (4, 3)
