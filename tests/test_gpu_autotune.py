"""Every launch choice the autotuner can set computes the same words, and
tuning leaves the fastest choice on the context."""
import numpy as np
import pytest

from mkf_b200 import autotune, params
from mkf_b200 import evaluator as ev
from tests import helpers as H
from tests.test_gpu_parity import gpu

pytestmark = pytest.mark.gpu

LIT = params.small("ckks", log_n=14, n_q=6, n_p=2, q_bits=45, first_bits=55, p_bits=55, scale_bits=45)


def test_all_choices_compute_the_same_words(tmp_path):
    k = 3
    case = H.mkf_ckks_case(LIT, k, LIT.max_level)
    P = gpu(LIT, "ckks")
    E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(case.keys.fold), case.keys.relin))
    a = ev.Ciphertext.from_array(P, case.left, True, scale=LIT.scale)
    b = ev.Ciphertext.from_array(P, case.right, True, scale=LIT.scale)
    ref = None
    for cnd in autotune.candidates():
        autotune.set_tuning(P, **cnd)
        got = E.MulRelinNew(a, b, rescale=True, materialize=True).download()
        if ref is None:
            ref = got
        assert np.array_equal(got, ref), f"{cnd} differs"
    cache = str(tmp_path / "tune.json")
    res = autotune.tune_mkf(P, k, operands=(E, a, b), cache_path=cache)
    assert res["best"] == autotune.get_tuning(P) and len(res["ms"]) >= 10
    again = autotune.tune_mkf(P, k, operands=(E, a, b), cache_path=cache)
    assert again["cached"] and again["best"] == res["best"]
