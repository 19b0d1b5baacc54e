"""Launch autotuner: picks, per context and workload, the launch choices that
make a product fastest on the device at hand.

The choices (mkf_tuning) never change the words computed, only the time:

* ``fuse_ip``: the key-switch inner products fused into the digits' row
  pass, or run as their own memory-bound kernel;
* ``ip_block`` and ``ip_width``: the key-switch tile of that kernel, threads
  per block and coefficients per thread (2: 16-byte loads);
* ``col_split``: limbs per block of the digit column pass (the blocks of a
  column tile share its limb walk, ceil(limbs / col_split) limbs each);
* ``modup_chunk``: target limbs per thread of the party-summed ModUp.

The NTT runs as a column phase and a row phase; each phase is radix-8
passes (three butterfly stages on eight words held in registers) plus one
pass of radix 2^(stages mod 3), so the phase split sets the radix
composition: at logN 15, 7 + 8 stages (8*8*2 and 8*8*4) or 8 + 7; at
logN 14, 7 + 7 or 6 + 8.  The split is a context creation choice
(Parameters(..., ntt_row_log=)), picked by ``tune_split``, which times one
product on a context of each split.

The tuner times a product per candidate with CUDA events (after a warm-up)
in a coordinate descent over the axes (each axis swept with the others held
at their best so far, twice over), keeps the fastest, sets it on the
context, and can keep the result in a JSON cache keyed by device and
workload shape (ring degree, limbs, digits, parties).
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
from typing import Callable, Dict, Iterable, List, Optional, Tuple

import numpy as np

from . import capi

AXES = {"fuse_ip": (0, 1), "ip_block": (128, 256, 512), "modup_chunk": (8, 12, 24),
        "col_split": (1, 2, 4, 8), "ip_width": (1, 2)}


def candidates(axes: Dict[str, Iterable] = AXES) -> List[dict]:
    keys = list(axes)
    return [dict(zip(keys, vals)) for vals in itertools.product(*(axes[k] for k in keys))]


def get_tuning(params) -> dict:
    t = capi.Tuning()
    capi.check(params.handle, capi.lib().mkf_ctx_get_tuning(params.handle, ctypes.byref(t)))
    return {f: getattr(t, f) for f, _ in capi.Tuning._fields_}


def set_tuning(params, **kw):
    cur = get_tuning(params)
    cur.update(kw)
    t = capi.Tuning(**{f: int(cur[f]) for f, _ in capi.Tuning._fields_})
    capi.check(params.handle, capi.lib().mkf_ctx_set_tuning(params.handle, ctypes.byref(t)))


def search(cands: List[dict], time_fn: Callable[[dict], float],
           rounds: int = 2) -> Tuple[dict, Dict[str, float]]:
    """Times every candidate `rounds` times, sweeping the whole grid each
    round so that drifts hit all candidates alike (time_fn sets a candidate
    and returns ms), and returns the one with the lowest best time together
    with the table of best times."""
    table: Dict[str, float] = {}
    for _ in range(max(1, rounds)):
        for cnd in cands:
            k = json.dumps(cnd, sort_keys=True)
            table[k] = min(table.get(k, float("inf")), float(time_fn(cnd)))
    best_key = min(table, key=table.get)
    return json.loads(best_key), table


def descend(axes: Dict[str, Iterable], time_fn: Callable[[dict], float], start: dict,
            rounds: int = 2) -> Tuple[dict, Dict[str, float]]:
    """Coordinate descent: sweeps one axis at a time with the other axes at
    their best value so far, `rounds` times over all axes.  Every point is
    timed once per visit and keeps its best time; returns the best point and
    the table of best times of every point visited."""
    table: Dict[str, float] = {}
    cur = dict(start)

    def t(cnd):
        k = json.dumps(cnd, sort_keys=True)
        table[k] = min(table.get(k, float("inf")), float(time_fn(cnd)))
        return table[k]

    for _ in range(max(1, rounds)):
        for ax, vals in axes.items():
            best_v, best_t = cur[ax], None
            for v in vals:
                cnd = dict(cur, **{ax: v})
                tv = t(cnd)
                if best_t is None or tv < best_t:
                    best_v, best_t = v, tv
            cur[ax] = best_v
    best_key = min(table, key=table.get)
    return json.loads(best_key), table


def split_options(log_n: int) -> List[int]:
    """Row-phase stage counts (ntt_row_log) the kernels are built for at
    log_n, the default first; [] below logN 13 (one tile holds a limb)."""
    return {13: [7], 14: [7, 8], 15: [8, 7], 16: [8]}.get(log_n, [])


def tune_split(literal, scheme: str, k: int, level: Optional[int] = None, device: int = 0,
               reps: int = 4) -> Tuple[int, Dict[int, float]]:
    """Times one MKF mult+relin(+rescale) of k parties on a context of each
    NTT split of the ring (random keys and operands, default launch choices
    otherwise) and returns (the fastest ntt_row_log, {row_log: ms})."""
    import torch
    from . import evaluator as ev
    opts = split_options(literal.log_n)
    if len(opts) < 2:
        return (opts[0] if opts else 0), {}
    level = literal.max_level if level is None else level
    g = np.random.default_rng(11)
    qmin = min(min(literal.q), min(literal.p))
    nQ, nP, N = len(literal.q), len(literal.p), literal.n
    beta = (nQ + nP - 1) // nP
    kimg = g.integers(0, qmin, size=(beta, 2, nQ + nP, N), dtype=np.uint64)
    cimg = [g.integers(0, qmin, size=(k + 1, level + 1, N), dtype=np.uint64) for _ in range(2)]
    ckks = scheme == "ckks"
    table = {}
    for rl in opts:
        P = ev.Parameters(literal, scheme, device=device, ntt_row_log=rl)
        E = ev.MKFEvaluator(P, ev.MKFKeySet(P, [kimg] * k, kimg))
        left, right = (ev.Ciphertext.from_array(P, c, ckks, scale=literal.scale) for c in cimg)
        out = ev.Ciphertext(P, k + 1, E.output_level(left, right, ckks), ckks)
        st = torch.cuda.Stream(device=device)
        cs = ctypes.c_void_p(st.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        E.MulRelin(left, right, out, rescale=ckks, materialize=True, stream=cs)  # warm-up
        e0.record(st)
        for _ in range(reps):
            E.MulRelin(left, right, out, rescale=ckks, materialize=True, stream=cs)
        e1.record(st)
        e1.synchronize()
        table[rl] = e0.elapsed_time(e1) / reps
        del out, left, right, E, P
    return min(table, key=table.get), table


def _cache_key(params, k: int, level: int) -> str:
    import torch
    lit = params.literal
    name = torch.cuda.get_device_name(params.device) if torch.cuda.is_available() else "cpu"
    beta = (level + len(lit.p)) // len(lit.p)
    return (f"{name}|mkf-{params.scheme}|logN{lit.log_n}|Q{len(lit.q)}|P{len(lit.p)}|"
            f"L{level + 1}|beta{beta}|k{k}")


def tune_mkf(params, k: int, level: Optional[int] = None, reps: int = 4, keys=None, operands=None,
             cache_path: Optional[str] = None, cands: Optional[List[dict]] = None) -> dict:
    """Tunes the MKF mult+relin(+rescale) of k parties at `level` on this
    context and leaves the fastest choice set.  keys/operands: an
    (MKFEvaluator, left, right) triple to time on; random ones are made
    otherwise.  Returns {"best": ..., "ms": {candidate: ms}, "cached": bool}."""
    import torch
    from . import evaluator as ev
    lit = params.literal
    level = lit.max_level if level is None else level
    key = _cache_key(params, k, level)
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            set_tuning(params, **cache[key]["best"])
            return dict(cache[key], cached=True)
    if operands is None:
        g = np.random.default_rng(7)
        qmin = min(min(lit.q), min(lit.p))
        nQ, nP, N = len(lit.q), len(lit.p), lit.n
        beta = (nQ + nP - 1) // nP
        kimg = g.integers(0, qmin, size=(beta, 2, nQ + nP, N), dtype=np.uint64)
        E = ev.MKFEvaluator(params, ev.MKFKeySet(params, [kimg] * k, kimg))
        cts = [ev.Ciphertext.from_array(params, g.integers(0, qmin, size=(k + 1, level + 1, N),
                                                           dtype=np.uint64),
                                        params.scheme == "ckks", scale=lit.scale) for _ in range(2)]
        operands = (E, cts[0], cts[1])
    E, left, right = operands
    ckks = params.scheme == "ckks"
    out = ev.Ciphertext(params, k + 1, E.output_level(left, right, ckks), ckks)
    st = torch.cuda.Stream(device=params.device)
    cs = ctypes.c_void_p(st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_fn(cnd):
        set_tuning(params, **cnd)
        E.MulRelin(left, right, out, rescale=ckks, materialize=True, stream=cs)  # warm-up
        e0.record(st)
        for _ in range(reps):
            E.MulRelin(left, right, out, rescale=ckks, materialize=True, stream=cs)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    if cands is not None:
        best, table = search(cands, time_fn)
    else:
        best, table = descend(AXES, time_fn, get_tuning(params))
    set_tuning(params, **best)
    res = {"best": best, "ms": table, "cached": False}
    if cache_path:
        cache = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        cache[key] = {"best": best, "ms": table}
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1)
    return res
