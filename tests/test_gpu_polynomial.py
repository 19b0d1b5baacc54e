"""Polynomial evaluation over MKF paper carriers (the reference's
paperMKFCKKSEvaluator.EvaluatePoly schedule, software/mkf/mkf_cpu/
true_mkf_ckks_polynomial.go:79-273) on the GPU: every carrier it returns
equals, word for word, the same schedule run over oracle operations, and
decrypts to p(x) slot by slot."""
import numpy as np
import pytest

from mkf_b200 import params
from mkf_b200 import evaluator as ev
from mkf_b200.adapter import PaperMKFAdapter
from mkf_b200.polynomial import Polynomial, Schedule, CarrierBackend
from oracle import keygen as kg
from tests import helpers as H
from tests.poly_oracle import OCt, OracleBackend, decode_carrier
from tests.test_gpu_parity import assert_eq_mod, gpu

pytestmark = pytest.mark.gpu

LIT = params.small("ckks", log_n=11, n_q=7, n_p=2, q_bits=40, first_bits=55, p_bits=55, scale_bits=40)


@pytest.fixture(scope="module")
def setup():
    k = 2
    case = H.mkf_ckks_case(LIT, k, LIT.max_level)
    P = gpu(LIT, "ckks")
    A = PaperMKFAdapter(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    return case, P, A


@pytest.mark.parametrize("coeffs,basis", [
    ([0.5, 0.3, -0.2, 0.1, 0, 0.05, 0, 0.02], "standard"),
    ([0, 1, 0, 0.5, 0, 0.25], "standard"),
    ([0.25, 0, 0.5, 0, 0.125], "standard"),
    ([0.1, 0.4, -0.3, 0.2, 0.1, -0.05], "chebyshev"),
    ([0.3 + 0.1j, -0.2j, 0.1], "standard"),
])
def test_evaluate_poly(setup, coeffs, basis):
    case, P, A = setup
    poly = Polynomial(coeffs, basis=basis)
    ob = OracleBackend(case.o, case.keys.fold, case.keys.relin, case.k)
    want = Schedule(ob).evaluate(OCt(case.left, LIT.scale), poly, LIT.scale)
    x = ev.Ciphertext.from_array(P, case.left, True, scale=LIT.scale)
    got = Schedule(CarrierBackend(A)).evaluate(x, poly, LIT.scale)
    assert got.Level() == want.level and got.n_comp == case.k + 1
    g = got.download()
    assert_eq_mod(g, want.a, LIT.q[: want.level + 1])
    xs = decode_carrier(case, case.left, LIT.max_level, LIT.scale)
    ref = sum(c * xs ** i for i, c in enumerate(coeffs)) if basis == "standard" else \
        np.polynomial.chebyshev.chebval(xs, coeffs)
    assert kg.precision_bits(decode_carrier(case, g, got.Level(), got.Scale), ref) > 20


def test_depth_check(setup):
    case, P, A = setup
    x = ev.Ciphertext.from_array(P, case.left[:, :3], True, scale=LIT.scale)
    with pytest.raises(ValueError, match="polynomial depth"):
        Schedule(CarrierBackend(A)).evaluate(x, Polynomial([0.1] * 9), LIT.scale)
