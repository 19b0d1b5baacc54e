"""Host-side mirror of the reference evaluator API for the mult+relin path.

Names and argument meaning follow the reference's Go API:

* ``Evaluator.MulRelinNew(op0, op1, rlkSet)`` and ``Evaluator.Rescale`` --
  mkckks.Evaluator (software/kklss/mkckks/evaluator.go:360-446) and
  mkbfv.Evaluator (software/kklss/mkbfv/evaluator.go:85-91), KKLSS
  construction with per-party relinearization keys;
* ``MKFEvaluator.MulRelinNew(left, right)`` -- the MKF aggregate-fold
  product of CKKSCase.Run / BFVCase.Run (software/mkf/mkf_cpu/ckks.go:102-166,
  bfv.go:212-252) and paperMKFCKKSEvaluator.MulRelinNew
  (true_mkf_ckks.go:253-304);
* ``RelinearizationKeySet.AddRelinearizationKey`` (mkrlwe/keys.go:263-281).

Errors: the reference panics on a missing key or a level mismatch and returns
an error from Rescale; here both raise (MissingKeyError, LevelError, MKFError).
Everything runs through libmkf_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import capi
from .params import ParametersLiteral


class Parameters:
    """A parameter literal instantiated on one GPU (tables resident in HBM).
    ntt_row_log: row stages of the NTT split (0: ceil(logN/2); logN 14 also
    takes 8, logN 15 also 7); the transform's results do not depend on it."""

    def __init__(self, literal: ParametersLiteral, scheme: str, device: int = 0,
                 ntt_row_log: int = 0):
        L = capi.lib()
        self.literal = literal
        self.scheme = scheme.lower()
        self.device = device
        self._q = np.array(literal.q, dtype=np.uint64)
        self._p = np.array(literal.p, dtype=np.uint64)
        self._qm = np.array(literal.q_mul or (0,), dtype=np.uint64)
        d = capi.ParamsDesc()
        d.scheme = capi.SCHEME[self.scheme]
        d.log_n = literal.log_n
        d.q, d.n_q = capi.ptr(self._q), len(literal.q)
        d.p, d.n_p = capi.ptr(self._p), len(literal.p)
        if self.scheme == "bfv":
            d.q_mul, d.n_q_mul = capi.ptr(self._qm), len(literal.q_mul)
        d.scale = literal.scale
        d.t = literal.t
        d.device = device
        d.ntt_row_log = ntt_row_log
        self.ntt_row_log = ntt_row_log
        h = ctypes.c_void_p()
        st = L.mkf_ctx_create(ctypes.byref(d), ctypes.byref(h))
        if st != capi.OK:
            raise capi.MKFError(st, f"mkf_ctx_create failed for {literal.name}")
        self.handle = h.value

    def close(self):
        if getattr(self, "handle", None):
            capi.lib().mkf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def N(self) -> int:
        return self.literal.n

    def MaxLevel(self) -> int:
        return self.literal.max_level

    def Scale(self) -> float:
        return self.literal.scale

    def T(self) -> int:
        return self.literal.t

    def beta(self, level: int, gamma: int) -> int:
        return capi.lib().mkf_ctx_beta(self.handle, level, gamma)

    def key_words(self, kind: int) -> int:
        return int(capi.lib().mkf_key_words(self.handle, kind))


class Key:
    """Key material resident in HBM (Lattigo layout: MForm, NTT, Q then P)."""

    def __init__(self, params: Parameters, kind: int, words: np.ndarray):
        words = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
        h = ctypes.c_void_p()
        capi.check(params.handle, capi.lib().mkf_key_upload(
            params.handle, kind, capi.ptr(words), words.size, ctypes.byref(h)))
        self.params, self.kind, self.handle = params, kind, h.value

    def __del__(self):
        try:
            if self.handle:
                capi.lib().mkf_key_destroy(self.handle)
        except Exception:
            pass


def SwitchingKey(params, words):
    return Key(params, capi.KEY_SWITCHING, words)


class Ciphertext:
    """HBM-resident multi-key ciphertext: component 0 then one per party."""

    def __init__(self, params: Parameters, n_comp: int, level: int, is_ntt: bool,
                 ids: Optional[Sequence[int]] = None, scale: Optional[float] = None):
        h = ctypes.c_void_p()
        capi.check(params.handle, capi.lib().mkf_ct_create(params.handle, n_comp, level, int(is_ntt),
                                                           ctypes.byref(h)))
        self.params, self.handle = params, h.value
        if ids is not None:
            self.set_ids(ids)
        if scale is not None:
            capi.lib().mkf_ct_set_scale(self.handle, float(scale))

    @classmethod
    def from_array(cls, params, arr: np.ndarray, is_ntt: bool, ids=None, scale=None):
        arr = np.ascontiguousarray(arr, dtype=np.uint64)
        ct = cls(params, arr.shape[0], arr.shape[1] - 1, is_ntt, ids, scale)
        ct.upload(arr)
        return ct

    def __del__(self):
        try:
            if self.handle:
                capi.lib().mkf_ct_destroy(self.handle)
        except Exception:
            pass

    def set_ids(self, ids):
        a = (ctypes.c_int32 * len(ids))(*[int(x) for x in ids])
        capi.check(self.params.handle, capi.lib().mkf_ct_set_parties(self.handle, a, len(ids)))

    @property
    def ids(self) -> List[int]:
        n = ctypes.c_int()
        buf = (ctypes.c_int32 * 128)()
        capi.lib().mkf_ct_get_parties(self.handle, buf, 128, ctypes.byref(n))
        return list(buf[: n.value])

    def Level(self) -> int:
        return capi.lib().mkf_ct_level(self.handle)

    @property
    def n_comp(self) -> int:
        return capi.lib().mkf_ct_ncomp(self.handle)

    @property
    def Scale(self) -> float:
        return capi.lib().mkf_ct_scale(self.handle)

    def shape(self):
        return (self.n_comp, self.Level() + 1, self.params.N)

    def upload(self, arr: np.ndarray, stream=None):
        arr = np.ascontiguousarray(arr, dtype=np.uint64)
        capi.check(self.params.handle, capi.lib().mkf_ct_upload(self.handle, capi.ptr(arr), arr.size, stream))

    def download(self, out: Optional[np.ndarray] = None, stream=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape(), np.uint64)
        capi.check(self.params.handle, capi.lib().mkf_ct_download(self.handle, capi.ptr(out), out.size, stream))
        return out


class RelinearizationKeySet:
    """KKLSS per-party (b, d, v) keys plus the CRS vector u."""

    def __init__(self, params: Parameters, crs_u: np.ndarray):
        self.params = params
        self.u = Key(params, capi.KEY_GADGET, crs_u)
        h = ctypes.c_void_p()
        capi.check(params.handle, capi.lib().mkf_kklss_keyset_create(params.handle, self.u.handle,
                                                                     ctypes.byref(h)))
        self.handle = h.value
        self.keys: Dict[int, Key] = {}

    def AddRelinearizationKey(self, party_id: int, rlk_words: np.ndarray):
        kind = capi.KEY_KKLSS_BFV_RLK if self.params.scheme == "bfv" else capi.KEY_KKLSS_RLK
        k = Key(self.params, kind, rlk_words)
        capi.check(self.params.handle, capi.lib().mkf_kklss_keyset_add(self.handle, int(party_id), k.handle))
        self.keys[int(party_id)] = k

    def __del__(self):
        try:
            if self.handle:
                capi.lib().mkf_kklss_keyset_destroy(self.handle)
        except Exception:
            pass


class MKFKeySet:
    """MKF online keys of one party subset: fold keys s_i -> s_E and relin."""

    def __init__(self, params: Parameters, fold: Sequence[np.ndarray], relin: Optional[np.ndarray]):
        """relin = None: a bundle of k keys used only to fold or rotate (for
        instance one sigma(s_i) -> s_E key per party)."""
        self.params = params
        self.fold = [SwitchingKey(params, f) for f in fold]
        self.relin = SwitchingKey(params, relin) if relin is not None else None
        arr = (ctypes.c_void_p * len(self.fold))(*[f.handle for f in self.fold])
        h = ctypes.c_void_p()
        capi.check(params.handle, capi.lib().mkf_mkf_keyset_create(
            params.handle, arr, len(self.fold), self.relin.handle if self.relin else None,
            ctypes.byref(h)))
        self.handle = h.value
        self.k = len(self.fold)

    def __del__(self):
        try:
            if self.handle:
                capi.lib().mkf_mkf_keyset_destroy(self.handle)
        except Exception:
            pass


def galois_element(params: Parameters, rotation: int) -> int:
    """5^r mod 2N (Lattigo GaloisElementForColumnRotationBy)."""
    return int(capi.lib().mkf_galois_element(params.handle, int(rotation)))


def conjugation_element(params: Parameters) -> int:
    return int(capi.lib().mkf_conjugation_element(params.handle))


class GaloisKeySet:
    """KKLSS rotation or conjugation keys of one Galois element
    (RotationKeySet / ConjugationKeySet): the CRS vector they were made with
    and one gadget key per party."""

    def __init__(self, params: Parameters, galois: int, crs: np.ndarray, conjugation: bool = False):
        self.params, self.galois, self.conjugation = params, int(galois), conjugation
        self.crs = Key(params, capi.KEY_GADGET, crs)
        h = ctypes.c_void_p()
        capi.check(params.handle, capi.lib().mkf_galois_keyset_create(
            params.handle, self.galois, self.crs.handle, int(conjugation), ctypes.byref(h)))
        self.handle = h.value
        self.keys: Dict[int, Key] = {}

    def AddKey(self, party_id: int, words: np.ndarray):
        k = Key(self.params, capi.KEY_GADGET, words)
        capi.check(self.params.handle, capi.lib().mkf_galois_keyset_add(self.handle, party_id, k.handle))
        self.keys[party_id] = k

    def __del__(self):
        try:
            if self.handle:
                capi.lib().mkf_galois_keyset_destroy(self.handle)
        except Exception:
            pass


def _rescale_count(params: Parameters, level: int, min_scale: float, scale: float):
    q = params.literal.q
    nb = 0
    while level - nb >= 0 and scale / float(q[level - nb]) >= min_scale / 2:
        scale /= float(q[level - nb])
        nb += 1
    return nb, scale


class Evaluator:
    """KKLSS evaluator (mkckks.Evaluator / mkbfv.Evaluator)."""

    def __init__(self, params: Parameters):
        self.params = params

    def MulRelinNew(self, op0: Ciphertext, op1: Ciphertext, rlkSet: RelinearizationKeySet,
                    stream=None) -> Ciphertext:
        L = capi.lib()
        n = ctypes.c_int()
        L.mkf_kklss_union(op0.handle, op1.handle, None, 0, ctypes.byref(n))
        level = min(op0.Level(), op1.Level())
        if self.params.scheme == "ckks":
            if level == 0:
                raise capi.LevelError(6, "cannot rescale: input already at level 0")
            nb, _ = _rescale_count(self.params, level, self.params.Scale(), op0.Scale * op1.Scale)
            level -= nb
        out = Ciphertext(self.params, n.value + 1, level, False)
        capi.check(self.params.handle, L.mkf_kklss_mulrelin(self.params.handle, op0.handle, op1.handle,
                                                            rlkSet.handle, out.handle, stream))
        return out

    def Galois(self, ctIn: Ciphertext, keys: GaloisKeySet, ctOut: Ciphertext, stream=None):
        capi.check(self.params.handle, capi.lib().mkf_kklss_rotate(
            self.params.handle, ctIn.handle, keys.handle, ctOut.handle, stream))

    def RotateNew(self, ctIn: Ciphertext, rotation: int, keys: GaloisKeySet) -> Ciphertext:
        """mkckks.Evaluator.RotateHoistedNew (mkckks/evaluator.go:590-621):
        slots rotated left by `rotation`."""
        if rotation % (self.params.N // 2) == 0:
            out = Ciphertext(self.params, ctIn.n_comp, ctIn.Level(), False, ctIn.ids, ctIn.Scale)
            out.upload(ctIn.download())
            return out
        if keys.conjugation or keys.galois != galois_element(self.params, rotation):
            raise capi.MissingKeyError(5, f"no rotation keys for rotation {rotation}")
        out = Ciphertext(self.params, ctIn.n_comp, ctIn.Level(), False)
        self.Galois(ctIn, keys, out)
        return out

    def ConjugateNew(self, ctIn: Ciphertext, keys: GaloisKeySet) -> Ciphertext:
        """mkckks.Evaluator.ConjugateNew (mkckks/evaluator.go:533-544)."""
        if not keys.conjugation:
            raise capi.MissingKeyError(5, "no conjugation keys")
        out = Ciphertext(self.params, ctIn.n_comp, ctIn.Level(), False)
        self.Galois(ctIn, keys, out)
        return out

    def Rescale(self, ctIn: Ciphertext, minScale: float, ctOut: Ciphertext, stream=None):
        capi.check(self.params.handle, capi.lib().mkf_rescale(self.params.handle, ctIn.handle,
                                                              float(minScale), ctOut.handle, stream))

    def RescaleNew(self, ctIn: Ciphertext, minScale: float) -> Ciphertext:
        if minScale <= 0:
            raise capi.LevelError(6, "cannot Rescale: minScale is 0")
        if ctIn.Level() == 0:
            raise capi.LevelError(6, "cannot Rescale: input Ciphertext already at level 0")
        nb, _ = _rescale_count(self.params, ctIn.Level(), minScale, ctIn.Scale)
        out = Ciphertext(self.params, ctIn.n_comp, ctIn.Level() - nb, False)
        self.Rescale(ctIn, minScale, out)
        return out


class MKFEvaluator:
    """MKF aggregate-fold mult+relin for one party subset."""

    def __init__(self, params: Parameters, keys: MKFKeySet):
        self.params, self.keys = params, keys

    def output_level(self, left: Ciphertext, right: Ciphertext, rescale: bool) -> int:
        level = min(left.Level(), right.Level())
        if self.params.scheme == "ckks" and rescale:
            nb, _ = _rescale_count(self.params, level, self.params.Scale(), left.Scale * right.Scale)
            level -= nb
        return level

    def MulRelinNew(self, left: Ciphertext, right: Ciphertext, rescale: bool = True,
                    materialize: bool = False, stream=None) -> Ciphertext:
        lvl = self.output_level(left, right, rescale)
        n_out = self.keys.k + 1 if materialize else 2
        out = Ciphertext(self.params, n_out, lvl, self.params.scheme == "ckks")
        self.MulRelin(left, right, out, rescale, materialize, stream)
        return out

    def RotateNew(self, ct: Ciphertext, galois: int, rot_keys: "MKFKeySet",
                  materialize: bool = True) -> Ciphertext:
        """Paper RotateNew (true_mkf_ckks.go:321-353) with one
        sigma(s_i) -> s_E key per party in rot_keys."""
        out = Ciphertext(self.params, ct.n_comp if materialize else 2, ct.Level(), True)
        capi.check(self.params.handle, capi.lib().mkf_mkf_rotate(
            self.params.handle, ct.handle, rot_keys.handle, int(galois), out.handle, None))
        return out

    def MulRelin(self, left, right, out, rescale=True, materialize=False, stream=None):
        flags = (capi.FLAG_RESCALE if rescale else 0) | (capi.FLAG_MATERIALIZE if materialize else 0)
        capi.check(self.params.handle, capi.lib().mkf_mkf_mulrelin(
            self.params.handle, left.handle, right.handle, self.keys.handle, flags, out.handle, stream))


class Batch:
    """A batch plan (mkf_batch_create): many products over concurrent lanes,
    optionally captured into one CUDA graph.  Jobs are
    ("mkf", MKFEvaluator, left, right, out, rescale, materialize) or
    ("kklss", RelinearizationKeySet, op0, op1, out); outputs are shaped as for
    the single calls (see MKFEvaluator.output_level / Evaluator.MulRelinNew).
    fuse_keys: MKF-CKKS jobs that share a key bundle, flags and level run as
    fused calls (each key read once per group; MKF_BATCH_FUSE_KEYS).
    persistent: the whole plan runs as one launch of the persistent executor
    (MKF_BATCH_PERSISTENT); check() then reports whether its bounded waits
    all completed."""

    def __init__(self, params: Parameters, jobs, lanes: int = 8, graph: bool = True,
                 fuse_keys: bool = False, persistent: bool = False, extra_flags: int = 0):
        self.params = params
        self._keep = list(jobs)  # handles must outlive the plan
        arr = (capi.Job * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            if j[0] == "mkf":
                _, ev, left, right, out, rescale, materialize = j
                arr[i].kind = capi.JOB_MKF
                arr[i].mkf_keys = ev.keys.handle
                arr[i].flags = (capi.FLAG_RESCALE if rescale else 0) | \
                    (capi.FLAG_MATERIALIZE if materialize else 0)
            else:
                _, rlk, left, right, out = j
                arr[i].kind = capi.JOB_KKLSS
                arr[i].kklss_keys = rlk.handle
            arr[i].a, arr[i].b, arr[i].out = left.handle, right.handle, out.handle
        self.jobs = arr
        h = ctypes.c_void_p()
        flags = (capi.BATCH_GRAPH if graph else 0) | (capi.BATCH_FUSE_KEYS if fuse_keys else 0) | \
            (capi.BATCH_PERSISTENT if persistent else 0) | extra_flags
        st = capi.lib().mkf_batch_create(params.handle, arr, len(jobs), lanes, flags,
                                        ctypes.byref(h))
        capi.check(params.handle, st)
        self.handle = h

    def statuses(self):
        return [int(self.jobs[i].status) for i in range(len(self._keep))]

    def launch(self, stream=None):
        capi.check(self.params.handle, capi.lib().mkf_batch_launch(self.handle, stream))

    @property
    def kernels(self) -> int:
        return int(capi.lib().mkf_batch_kernels(self.handle))

    def check(self):
        """Waits for the last launch; raises MKFError (MKF_ERR_TIMEOUT when a
        persistent plan's bounded wait ran out)."""
        capi.check(self.params.handle, capi.lib().mkf_batch_check(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            capi.lib().mkf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_job(job) -> "capi.Job":
    """struct mkf_job from ("mkf", MKFEvaluator, left, right, out, rescale,
    materialize) or ("kklss", RelinearizationKeySet, op0, op1, out)."""
    j = capi.Job()
    if job[0] == "mkf":
        _, ev_, left, right, out, rescale, materialize = job
        j.kind, j.mkf_keys = capi.JOB_MKF, ev_.keys.handle
        j.flags = (capi.FLAG_RESCALE if rescale else 0) | (capi.FLAG_MATERIALIZE if materialize else 0)
    else:
        _, rlk, left, right, out = job
        j.kind, j.kklss_keys = capi.JOB_KKLSS, rlk.handle
    j.a, j.b, j.out = left.handle, right.handle, out.handle
    return j


def job_scratch_bytes(job) -> int:
    j = make_job(job)
    n = ctypes.c_size_t()
    st = capi.lib().mkf_job_scratch(ctypes.byref(j), ctypes.byref(n))
    capi.check(job[2].params.handle, st)
    return int(n.value)


class Server:
    """The serving loop (mkf_server_*): submit products as they arrive,
    wait for tickets, read p50/p99 latency and throughput."""

    def __init__(self, device: int = 0, scratch_bytes: int = 8 << 30, slots: int = 8,
                 queue_cap: int = 4096, fuse_max: int = 0):
        """fuse_max > 1: an admitted MKF-CKKS request takes up to fuse_max - 1
        queued requests that share its key bundle into one fused call."""
        cfg = capi.ServerConfig(device, scratch_bytes, slots, queue_cap, fuse_max)
        h = ctypes.c_void_p()
        st = capi.lib().mkf_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != capi.OK:
            raise capi.MKFError(st, "mkf_server_create failed")
        self.handle = h
        self._live = {}

    def submit(self, job) -> int:
        """Queues one job; returns its ticket or raises MKFError (BUSY, OOM,
        validation errors with the job's own status)."""
        j = make_job(job)
        t = ctypes.c_uint64()
        st = capi.lib().mkf_server_submit(self.handle, ctypes.byref(j), ctypes.byref(t))
        if st != capi.OK:
            capi.check(job[2].params.handle, st)
        self._live[t.value] = job  # keep the handles alive until waited
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0):
        """Returns (job status, latency ms); raises MKFError(TIMEOUT) when the
        ticket has not completed within timeout_s."""
        js, lat = ctypes.c_int(), ctypes.c_double()
        st = capi.lib().mkf_server_wait(self.handle, ticket, float(timeout_s), ctypes.byref(js),
                                        ctypes.byref(lat))
        if st != capi.OK:
            raise capi.MKFError(st, f"ticket {ticket}")
        self._live.pop(ticket, None)
        return int(js.value), float(lat.value)

    def drain(self, timeout_s: float = -1.0):
        st = capi.lib().mkf_server_drain(self.handle, float(timeout_s))
        if st != capi.OK:
            raise capi.MKFError(st, "drain")

    def pause(self, paused: bool = True):
        capi.lib().mkf_server_pause(self.handle, int(paused))

    def stats(self) -> dict:
        s = capi.ServerStats()
        capi.lib().mkf_server_stats_get(self.handle, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in capi.ServerStats._fields_}

    def reset_stats(self):
        capi.lib().mkf_server_stats_reset(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            capi.lib().mkf_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# stage-level primitives ------------------------------------------------------

def ntt(params: Parameters, arr: np.ndarray, basis: str = "Q", first: int = 0, inverse=False):
    arr = np.ascontiguousarray(arr, dtype=np.uint64)
    out = np.empty_like(arr)
    b = {"Q": 0, "P": 1, "QM": 2}[basis]
    capi.check(params.handle, capi.lib().mkf_ntt_host(params.handle, b, first, arr.size // params.N,
                                                      capi.ptr(arr), capi.ptr(out), int(inverse)))
    return out


def decompose(params: Parameters, gamma: int, level: int, coeff: np.ndarray) -> np.ndarray:
    coeff = np.ascontiguousarray(coeff, dtype=np.uint64)
    beta = params.beta(level, gamma)
    out = np.empty((beta, level + 1 + len(params.literal.p), params.N), np.uint64)
    capi.check(params.handle, capi.lib().mkf_decompose_host(params.handle, gamma, level, capi.ptr(coeff),
                                                            capi.ptr(out)))
    return out


def switch_one(params: Parameters, level: int, x: np.ndarray, key: np.ndarray, in_ntt=True,
               ntt_output=True):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    key = np.ascontiguousarray(key, dtype=np.uint64)
    o0 = np.empty((level + 1, params.N), np.uint64)
    o1 = np.empty_like(o0)
    capi.check(params.handle, capi.lib().mkf_switch_one_host(params.handle, level, int(in_ntt), capi.ptr(x),
                                                             capi.ptr(key), int(ntt_output), capi.ptr(o0),
                                                             capi.ptr(o1)))
    return o0, o1


def launch_count(reset: bool = False) -> int:
    return int(capi.lib().mkf_launch_count(int(reset)))
