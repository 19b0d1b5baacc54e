"""ctypes binding of libmkf_b200.so (the C ABI in include/mkf_b200.h).

The library is required: importing this module without the built extension
raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# MKF_B200_LIB=debug selects the debug build (bounds checks and canaries)
LIB_PATH = os.path.join(HERE, "_lib", "libmkf_b200_debug.so"
                        if os.environ.get("MKF_B200_LIB") == "debug" else "libmkf_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mkf_b200.h")

u64p = ctypes.POINTER(ctypes.c_uint64)
i32p = ctypes.POINTER(ctypes.c_int32)
vp = ctypes.c_void_p

OK = 0
STATUS = {
    0: "MKF_OK", 1: "MKF_ERR_INVALID_ARG", 2: "MKF_ERR_CUDA", 3: "MKF_ERR_OOM",
    4: "MKF_ERR_UNSUPPORTED", 5: "MKF_ERR_MISSING_KEY", 6: "MKF_ERR_LEVEL",
    7: "MKF_ERR_TIMEOUT", 8: "MKF_ERR_BUSY", 9: "MKF_ERR_CANCELLED", 10: "MKF_ERR_CHECK",
}
SCHEME = {"ckks": 0, "bfv": 1}
KEY_SWITCHING, KEY_KKLSS_RLK, KEY_KKLSS_BFV_RLK, KEY_GADGET = 1, 2, 3, 4
FLAG_RESCALE, FLAG_MATERIALIZE = 1, 2


class MKFError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class MissingKeyError(MKFError):
    pass


class LevelError(MKFError):
    pass


class ParamsDesc(ctypes.Structure):
    _fields_ = [
        ("scheme", ctypes.c_int), ("log_n", ctypes.c_int),
        ("q", u64p), ("n_q", ctypes.c_int),
        ("p", u64p), ("n_p", ctypes.c_int),
        ("q_mul", u64p), ("n_q_mul", ctypes.c_int),
        ("scale", ctypes.c_double), ("t", ctypes.c_uint64), ("device", ctypes.c_int),
        ("ntt_row_log", ctypes.c_int),
    ]


SLOT_MUL_ADD, SLOT_ADD_C0, SLOT_MUL = 0, 1, 2
JOB_MKF, JOB_KKLSS = 1, 2
BATCH_GRAPH = 1
BATCH_FUSE_KEYS = 2
BATCH_PERSISTENT = 4
BATCH_TEST_STALL = 256


class Job(ctypes.Structure):
    """struct mkf_job: one product of a batch."""
    _fields_ = [
        ("kind", ctypes.c_int), ("a", vp), ("b", vp),
        ("mkf_keys", vp), ("kklss_keys", vp),
        ("flags", ctypes.c_int), ("out", vp), ("status", ctypes.c_int),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("fuse_ip", ctypes.c_int), ("ip_block", ctypes.c_int), ("modup_chunk", ctypes.c_int),
                ("col_split", ctypes.c_int), ("ip_width", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("scratch_bytes", ctypes.c_size_t),
                ("slots", ctypes.c_int), ("queue_cap", ctypes.c_int), ("fuse_max", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("span_s", ctypes.c_double), ("scratch_peak_bytes", ctypes.c_size_t),
                ("inflight_peak", ctypes.c_int)]


_lib = None


def declared_symbols():
    """Entry points declared in include/mkf_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mkf_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mkf_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    i, d, sz = ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    sig = {
        "mkf_version": (ctypes.c_char_p, []),
        "mkf_launch_count": (ctypes.c_uint64, [i]),
        "mkf_probe_butterflies": (i, [i, i, ctypes.POINTER(d)]),
        "mkf_ntt_f64_schedule": (ctypes.c_uint, [i, i, i, i, i]),
        "mkf_debug_status": (i, [i, ctypes.POINTER(ctypes.c_uint64)]),
        "mkf_ctx_create": (i, [ctypes.POINTER(ParamsDesc), ctypes.POINTER(vp)]),
        "mkf_ctx_destroy": (None, [vp]),
        "mkf_last_error": (i, [vp, ctypes.c_char_p, sz]),
        "mkf_ctx_beta": (i, [vp, i, i]),
        "mkf_key_words": (sz, [vp, i]),
        "mkf_key_upload": (i, [vp, i, u64p, sz, ctypes.POINTER(vp)]),
        "mkf_key_destroy": (None, [vp]),
        "mkf_ct_create": (i, [vp, i, i, i, ctypes.POINTER(vp)]),
        "mkf_ct_destroy": (None, [vp]),
        "mkf_ct_set_parties": (i, [vp, i32p, i]),
        "mkf_ct_get_parties": (i, [vp, i32p, i, ctypes.POINTER(i)]),
        "mkf_ct_set_scale": (i, [vp, d]),
        "mkf_ct_scale": (d, [vp]),
        "mkf_ct_level": (i, [vp]),
        "mkf_ct_ncomp": (i, [vp]),
        "mkf_ct_upload": (i, [vp, u64p, sz, vp]),
        "mkf_ct_download": (i, [vp, u64p, sz, vp]),
        "mkf_ct_upload_async": (i, [vp, u64p, sz, vp]),
        "mkf_ct_download_async": (i, [vp, u64p, sz, vp]),
        "mkf_mkf_keyset_create": (i, [vp, ctypes.POINTER(vp), i, vp, ctypes.POINTER(vp)]),
        "mkf_mkf_keyset_destroy": (None, [vp]),
        "mkf_mkf_mulrelin": (i, [vp, vp, vp, vp, i, vp, vp]),
        "mkf_kklss_keyset_create": (i, [vp, vp, ctypes.POINTER(vp)]),
        "mkf_kklss_keyset_add": (i, [vp, ctypes.c_int32, vp]),
        "mkf_kklss_keyset_destroy": (None, [vp]),
        "mkf_kklss_union": (i, [vp, vp, i32p, i, ctypes.POINTER(i)]),
        "mkf_kklss_mulrelin": (i, [vp, vp, vp, vp, vp, vp]),
        "mkf_rescale": (i, [vp, vp, d, vp, vp]),
        "mkf_ntt_host": (i, [vp, i, i, i, u64p, u64p, i]),
        "mkf_decompose_host": (i, [vp, i, i, u64p, u64p]),
        "mkf_switch_one_host": (i, [vp, i, i, u64p, u64p, i, u64p, u64p]),
        "mkf_rescale_noalloc": (i, [vp, ctypes.c_void_p, ctypes.c_void_p, i, i, i, vp]),
        "mkf_batch_create": (i, [vp, ctypes.POINTER(Job), i, i, i, ctypes.POINTER(vp)]),
        "mkf_batch_launch": (i, [vp, vp]),
        "mkf_batch_destroy": (None, [vp]),
        "mkf_batch_kernels": (ctypes.c_uint64, [vp]),
        "mkf_batch_check": (i, [vp]),
        "mkf_mulrelin_batch": (i, [vp, ctypes.POINTER(Job), i, vp]),
        "mkf_mkf_fold": (i, [vp, vp, vp, vp, vp]),
        "mkf_mkf_materialize": (i, [vp, vp, vp, vp]),
        "mkf_add": (i, [vp, vp, vp, vp, vp]),
        "mkf_sub": (i, [vp, vp, vp, vp, vp]),
        "mkf_mul_plain": (i, [vp, vp, vp, vp, vp]),
        "mkf_galois_element": (ctypes.c_uint64, [vp, i]),
        "mkf_conjugation_element": (ctypes.c_uint64, [vp]),
        "mkf_galois_keyset_create": (i, [vp, ctypes.c_uint64, vp, i, ctypes.POINTER(vp)]),
        "mkf_galois_keyset_add": (i, [vp, ctypes.c_int32, vp]),
        "mkf_galois_keyset_destroy": (None, [vp]),
        "mkf_kklss_rotate": (i, [vp, vp, vp, vp, vp]),
        "mkf_mkf_rotate": (i, [vp, vp, vp, ctypes.c_uint64, vp, vp]),
        "mkf_ct_copy": (i, [vp, vp, vp, vp]),
        "mkf_slot_const": (i, [vp, vp, u64p, i, vp, vp]),
        "mkf_ctx_get_tuning": (i, [vp, ctypes.POINTER(Tuning)]),
        "mkf_ctx_set_tuning": (i, [vp, ctypes.POINTER(Tuning)]),
        "mkf_server_create": (i, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
        "mkf_job_scratch": (i, [ctypes.POINTER(Job), ctypes.POINTER(sz)]),
        "mkf_server_submit": (i, [vp, ctypes.POINTER(Job), ctypes.POINTER(ctypes.c_uint64)]),
        "mkf_server_wait": (i, [vp, ctypes.c_uint64, d, ctypes.POINTER(i), ctypes.POINTER(d)]),
        "mkf_server_drain": (i, [vp, d]),
        "mkf_server_pause": (i, [vp, i]),
        "mkf_server_stats_get": (i, [vp, ctypes.POINTER(ServerStats)]),
        "mkf_server_stats_reset": (i, [vp]),
        "mkf_server_destroy": (None, [vp]),
        "mkf_profile_enable": (i, [vp, i]),
        "mkf_profile_kinds": (i, []),
        "mkf_profile_kind_name": (ctypes.c_char_p, [i]),
        "mkf_profile_read": (i, [vp, ctypes.POINTER(d), ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(d)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def ptr(a: np.ndarray):
    if a.dtype != np.uint64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous uint64 array")
    return a.ctypes.data_as(u64p)


def check(ctx_handle, status: int):
    if status == OK:
        return
    buf = ctypes.create_string_buffer(512)
    if ctx_handle:
        lib().mkf_last_error(ctx_handle, buf, 512)
    msg = buf.value.decode(errors="replace")
    if status == 5:
        raise MissingKeyError(status, msg)
    if status == 6:
        raise LevelError(status, msg)
    raise MKFError(status, msg)
