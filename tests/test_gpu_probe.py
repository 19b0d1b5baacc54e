"""The butterfly-throughput probe behind the bench's compute roofline runs on
the GPU and reports a positive, finite rate for both arithmetic kinds, and
rejects an unknown kind."""
import ctypes
import math

import pytest

from mkf_b200 import capi

pytestmark = pytest.mark.gpu


def test_probe_reports_both_kinds():
    L = capi.lib()
    for kind in (0, 1):
        v = ctypes.c_double(0.0)
        assert L.mkf_probe_butterflies(0, kind, ctypes.byref(v)) == 0
        assert math.isfinite(v.value) and v.value > 1.0
    v = ctypes.c_double(0.0)
    assert L.mkf_probe_butterflies(0, 7, ctypes.byref(v)) != 0
