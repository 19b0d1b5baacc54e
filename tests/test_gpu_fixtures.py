"""GPU path against fixture directories in the reference's exporter format:
oracle-written MKF-CKKS (with the first switch's decomposition/ModDown and
the fold stage dumps), MKF-BFV and KKLSS-CKKS fixtures must match word for
word; a planted wrong word must be reported."""
import os

import pytest

from mkf_b200 import fixtures
from tests import fixture_cases as F

pytestmark = pytest.mark.gpu


def test_mkf_ckks_fixture_with_stages(tmp_path):
    d = str(tmp_path / "mkf_ckks")
    F.mkf_ckks_fixture(d)
    rep = fixtures.run(fixtures.load(d))
    assert rep["output_mismatches"] == 0, rep
    assert rep["stages"]["debug_switch0_decomposition_qp.bin"] == 0
    assert rep["stages"]["debug_switch0_moddown_q.bin"] == 0
    assert rep["stages"]["stage_fold_q.bin"] == 0
    assert rep["match"]


def test_mkf_bfv_fixture(tmp_path):
    d = str(tmp_path / "mkf_bfv")
    F.mkf_bfv_fixture(d)
    rep = fixtures.run(fixtures.load(d))
    assert rep["match"], rep


def test_kklss_ckks_fixture(tmp_path):
    d = str(tmp_path / "kklss")
    F.kklss_ckks_fixture(d)
    rep = fixtures.run(fixtures.load(d))
    assert rep["match"], rep


def test_planted_error_is_reported(tmp_path):
    d = str(tmp_path / "mkf_ckks")
    F.mkf_ckks_fixture(d, stages=False)
    path = os.path.join(d, fixtures.MKF_FILES["output"])
    with open(path, "r+b") as f:
        f.seek(8 * 5)
        b = f.read(1)
        f.seek(8 * 5)
        f.write(bytes([b[0] ^ 1]))
    rep = fixtures.run(fixtures.load(d, check_hashes=False))
    assert rep["output_mismatches"] == 1 and not rep["match"]
