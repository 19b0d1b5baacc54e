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


def test_python_constants_match_the_header():
    """The Python binding's copies of the header's constants (status codes,
    flags, job kinds, batch flags, slot ops) have the header's values, and
    the parameter descriptor has the header's fields in order."""
    import re
    from mkf_b200 import capi
    text = open(capi.HEADER).read()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (MKF_\w+) (\d+)", text)}
    enums = {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(MKF_(?:ERR_\w+|OK|FLAG_\w+))\s*=\s*(\d+)", text)}
    for name, value in enums.items():
        if name.startswith("MKF_ERR_") or name == "MKF_OK":
            assert capi.STATUS[value] == name
    assert capi.FLAG_RESCALE == enums["MKF_FLAG_RESCALE"]
    assert capi.FLAG_MATERIALIZE == enums["MKF_FLAG_MATERIALIZE"]
    for short in ("BATCH_GRAPH", "BATCH_FUSE_KEYS", "BATCH_PERSISTENT", "BATCH_TEST_STALL",
                  "JOB_MKF", "JOB_KKLSS", "SLOT_MUL_ADD", "SLOT_ADD_C0", "SLOT_MUL"):
        assert getattr(capi, short) == defines["MKF_" + short], short
    for cname, pycls in (("mkf_params_desc", capi.ParamsDesc), ("mkf_tuning", capi.Tuning),
                         ("mkf_job", capi.Job), ("mkf_server_config", capi.ServerConfig)):
        body = text[text.index("typedef struct %s {" % cname):text.index("} %s;" % cname)]
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in re.findall(r"([^;{]+);", body):
            # "const mkf_ct *a, *b" declares two fields
            fields += [re.split(r"[\s*]+", part.strip())[-1] for part in decl.split(",")]
        assert fields == [f for f, _ in pycls._fields_], cname
