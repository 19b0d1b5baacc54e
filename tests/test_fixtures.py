"""Fixture ingest/export in the reference's exporter format
(software/mkf/mkf_cpu/fpga_fixture_test.go, software/kklss/mkckks/
fpga_fixture_test.go): round trip of every file, SHA-256 checks, manifest
fields and the parameter literal recovered from a manifest."""
import json
import os

import numpy as np
import pytest

from mkf_b200 import fixtures
from tests import fixture_cases as F


def test_mkf_ckks_round_trip(tmp_path):
    d = str(tmp_path / "mkf_ckks")
    case, out, lv = F.mkf_ckks_fixture(d)
    m = fixtures.read_manifest(d)
    assert m["scheme"] == "MKF-CKKS" and m["parties"] == 2
    assert m["input_level_q"] == F.CK.max_level and m["output_level_q"] == lv
    assert set(m["sha256"]) == set(fixtures.MKF_FILES.values())
    fx = fixtures.load(d)
    assert np.array_equal(fx.left, case.left) and np.array_equal(fx.right, case.right)
    assert np.array_equal(fx.fold, np.stack(case.keys.fold)) and np.array_equal(fx.relin, case.keys.relin)
    # c0, gamma, then gamma once per party
    assert fx.expected.shape[0] == 2 + 2
    assert np.array_equal(fx.expected[0], out[0])
    for j in range(1, 4):
        assert np.array_equal(fx.expected[j], out[1])
    assert fx.lit.q == F.CK.q and fx.lit.p == F.CK.p
    assert fx.lit.scale == float(F.CK.q[F.CK.max_level])  # unnamed set: one rescale


def test_mkf_bfv_and_kklss_round_trip(tmp_path):
    d = str(tmp_path / "mkf_bfv")
    case, out = F.mkf_bfv_fixture(d)
    fx = fixtures.load(d)
    assert fx.scheme == "MKF-BFV" and fx.lit.q_mul == F.BF.q_mul and fx.lit.t == F.BF.t
    assert np.array_equal(fx.expected[1], out[1])
    d = str(tmp_path / "kklss")
    case, out, lv = F.kklss_ckks_fixture(d)
    fx = fixtures.load(d)
    m = fixtures.read_manifest(d)
    assert m["ciphertext_order"] == ["0", "user0", "user1"]
    assert np.array_equal(fx.expected, out)
    assert np.array_equal(fx.rlk[1], case.keys.rlk[1].reshape(-1))
    assert np.array_equal(fx.crs_u, case.keys.crs_u.reshape(-1))


def test_hash_mismatch_is_reported(tmp_path):
    d = str(tmp_path / "mkf_ckks")
    F.mkf_ckks_fixture(d, stages=False)
    path = os.path.join(d, fixtures.MKF_FILES["output"])
    with open(path, "r+b") as f:
        f.seek(8)
        b = f.read(1)
        f.seek(8)
        f.write(bytes([b[0] ^ 1]))
    assert fixtures.verify_hashes(d, fixtures.read_manifest(d)) == [fixtures.MKF_FILES["output"]]
    with pytest.raises(ValueError, match="SHA-256"):
        fixtures.load(d)
    fixtures.load(d, check_hashes=False)


def test_named_parameter_set_is_recognised():
    from mkf_b200 import params
    c1 = params.get("ckks", "C1")
    m = {"scheme": "MKF-CKKS", "parameter": "C1", "polynomial_degree": c1.n, "q": list(c1.q),
         "p": list(c1.p), "input_level_q": c1.max_level}
    assert fixtures.literal_from_manifest(json.loads(json.dumps(m))) is c1


def test_wrong_file_size_is_rejected(tmp_path):
    d = str(tmp_path / "mkf_ckks")
    F.mkf_ckks_fixture(d, stages=False)
    path = os.path.join(d, fixtures.MKF_FILES["inputs"])
    with open(path, "ab") as f:
        f.write(b"\0" * 8)
    with pytest.raises(ValueError, match="words, expected"):
        fixtures.load(d, check_hashes=False)
