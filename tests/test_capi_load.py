"""The C-ABI library loads and exports every entry point include/mkf_b200.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os

import pytest

from mkf_b200 import capi


def test_library_built():
    assert os.path.exists(capi.LIB_PATH), "run python -m mkf_b200.build"


def test_exports_every_declared_symbol():
    L = ctypes.CDLL(capi.LIB_PATH)
    declared = capi.declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_declarations():
    L = capi.lib()
    for s in capi.declared_symbols():
        assert getattr(L, s).restype is not None or s.endswith("destroy"), s


def test_version_and_launch_counter():
    L = capi.lib()
    assert b"sm_100a" in L.mkf_version()
    L.mkf_launch_count(1)
    assert L.mkf_launch_count(0) == 0


def test_ctx_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from mkf_b200 import params
    from mkf_b200.evaluator import Parameters
    with pytest.raises(capi.MKFError):
        Parameters(params.small("ckks", 10, 3, 2), "ckks")
