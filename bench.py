#!/usr/bin/env python
"""Benchmark of the multi-key mult+relin path on B200.

Workload (one "product" = one MKF-CKKS mult+relin+rescale+materialize, the
timed region of CKKSCase.Run, software/mkf/mkf_cpu/ckks.go:241-292):
logN=16, k=8 parties, Q = one 60-bit + twenty-three 50-bit primes, P = four
60-bit primes, scale 2^50, top level (24 limbs), operands in the NTT domain.
Synthetic data: uniformly random key and ciphertext words (the keys of the
reference are pseudo-random; their values do not change the work).

A step = `--batch` products.  `value` is the batched form (the products of a
step spread over `--streams` CUDA streams, each with its own workspace);
`plain` is one product at a time on one stream.  Latency percentiles are the
plain per-product device times.  Inputs (1.6 GB of keys) exceed the 126 MB L2.

`--impl reference` times the reference algorithm's CPU restatement (the
oracle; the reference's Go + Lattigo v2.3.0 is not installable here) on all
host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mult+relin ops/s at logN=16,k=8: batched/served vs plain GPU; p50/p99 latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mkf_b200", choices=["mkf_b200", "reference"])
    ap.add_argument("--config", default="C3")
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--level", type=int, default=-1)
    ap.add_argument("--batch", type=int, default=48,
                    help="products per step (48: at 20 steps the timed region lasts about 3 s)")
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--mix", type=int, default=512,
                    help="products in the mixed batch (k in {2,4,8,16}, logN in {14,15}, "
                         "level uniform over [1,L]); 0 skips it")
    ap.add_argument("--lanes", default="4,8,16", help="lane counts the batch autotuner tries")
    ap.add_argument("--plan-lanes", default="1,2",
                    help="lane counts tried for the headline key-fused plan")
    ap.add_argument("--plan-forms", default="graph,persistent",
                    help="batch plan forms tried: graph (the lanes' kernels in a CUDA graph), "
                         "persistent (one launch of the persistent executor)")
    ap.add_argument("--tuning", default="",
                    help='launch choices as JSON, e.g. {"fuse_ip": 1, "ip_block": 256, '
                         '"modup_chunk": 24}, instead of autotuning (profiling runs)')
    ap.add_argument("--serve-seconds", type=float, default=6.0,
                    help="length of each open-loop Poisson trace; 0 skips serving")
    ap.add_argument("--serve-rate", type=float, default=1000.0,
                    help="offered load (req/s) of the trace at load factor 1 when it is below "
                         "the measured capacity; otherwise the capacity")
    ap.add_argument("--serve-loads", default="0.8",
                    help="load factors (x the offered load above) of the traces, e.g. "
                         "0.5,0.8,1.0,1.2")
    ap.add_argument("--serve-parties16", type=int, default=64,
                    help="party-pool size of the logN=16 rings")
    ap.add_argument("--serve-templates", type=int, default=96)
    ap.add_argument("--serve-hbm-gb", type=float, default=150.0,
                    help="HBM budget of the serving trace: key pool plus request scratch")
    ap.add_argument("--serve-slots", type=int, default=8,
                    help="requests the serving loop runs concurrently (slot streams)")
    ap.add_argument("--served-seconds", type=float, default=3.0,
                    help="open-loop trace of the headline product through the serving loop; "
                         "0 skips it")
    ap.add_argument("--served-slots", type=int, default=4)
    ap.add_argument("--served-fuse", type=int, default=8,
                    help="requests of one key bundle the serving loop fuses per call (0: off)")
    ap.add_argument("--served-fuse-slots", type=int, default=2)
    ap.add_argument("--profile-products", type=int, default=0,
                    help="profiling run: after --warmup products, run this many plain products of "
                         "the headline workload (one stream) and exit; for ncu captures")
    ap.add_argument("--profile-persistent", action="store_true",
                    help="with --profile-products: run them as one persistent plan instead")
    ap.add_argument("--configs", type=int, default=1,
                    help="1: also time C1 and C2 (plain GPU, oracle on one core)")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the KKLSS serving traces (no headline line)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


from mkf_b200.replicas import Replicas, dist_env  # noqa: E402


def ncu_figures():
    """Per-kernel figures of the committed ncu capture (profiles/ncu_kernels.json):
    DRAM bytes per launch unit (dram__bytes_read.sum + dram__bytes_write.sum)
    and pipe utilisation, with the command and commit that produced them."""
    p = os.path.join(ROOT, "profiles", "ncu_kernels.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def digits_col_compute(L, device, lit, k, L1, nP, kinds):
    """Compute roofline of the digit column pass: its radix-8 butterflies per
    second against the ceiling measured on this GPU by mkf_probe_butterflies
    (a register-resident loop of the transform's own butterflies), float64
    for moduli below 2^50 and integer for the others.  A product runs the
    column pass over 2k+1 polynomials (fold of both operands, then the
    relinearization digit) of beta digits; each digit transforms every limb
    but its own (level+1+nP limbs, N/2 * n1 butterflies each).  The multSum
    words rebuilt on the way are extra work, not counted."""
    if "ntt_digits_col" not in kinds:
        return None
    import ctypes
    peaks = []
    for kind in (0, 1):
        v = ctypes.c_double(0.0)
        if L.mkf_probe_butterflies(device, kind, ctypes.byref(v)) != 0:
            return None
        peaks.append(v.value)
    N, logN = lit.n, lit.log_n
    n1 = logN - (logN + 1) // 2 if logN > 12 else logN
    mods = list(lit.q[:L1]) + list(lit.p)
    beta = (L1 + nP - 1) // nP
    n_fp = n_int = 0
    for d in range(beta):
        own = set(range(d * nP, min((d + 1) * nP, L1)))
        for li, q in enumerate(mods):
            if li in own:
                continue
            if q < (1 << 50):
                n_fp += 1
            else:
                n_int += 1
    per_limb = N // 2 * n1
    polys = 2 * k + 1
    bfly_fp, bfly_int = polys * n_fp * per_limb, polys * n_int * per_limb
    ms = kinds["ntt_digits_col"]["ms"] / kinds["ntt_digits_col"]["launches"] * 2
    achieved = (bfly_fp + bfly_int) / (ms / 1e3) / 1e9
    peak = (bfly_fp + bfly_int) / (bfly_fp / peaks[1] + bfly_int / peaks[0])
    return {"unit": "G butterfly/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "peak_int": peaks[0], "peak_fp64": peaks[1], "fp64_share": bfly_fp / (bfly_fp + bfly_int),
            "peak_source": "mkf_probe_butterflies on this GPU",
            "counted": "column-pass butterflies per product (2 launches); the fused multSum is extra"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline (the oracle: test infrastructure, timed here as the baseline)
# ---------------------------------------------------------------------------
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


_CPU_CASE = {}


def _cpu_case(config, k, level, seed):
    """Random keys and operands of one product (kept per worker process)."""
    key_ = (config, k, level, seed)
    if key_ in _CPU_CASE:
        return _CPU_CASE[key_]
    sys.path.insert(0, ROOT)
    from mkf_b200 import params
    from oracle.oracle import Oracle
    from oracle import keygen as kg
    lit = params.get("ckks", config)
    o = Oracle.from_literal(lit)
    N = o.n
    nQ, nP = len(lit.q), len(lit.p)
    beta = (nQ + nP - 1) // nP
    g = kg.rng(seed)
    L1 = level + 1
    key = np.stack([np.stack([np.concatenate([kg.uniform(g, lit.q, N), kg.uniform(g, lit.p, N)])
                              for _ in range(2)]) for _ in range(beta)])
    left = np.stack([kg.uniform(g, lit.q[:L1], N) for _ in range(k + 1)])
    right = np.stack([kg.uniform(g, lit.q[:L1], N) for _ in range(k + 1)])
    fold = np.ascontiguousarray(np.stack([key] * k))
    _CPU_CASE.clear()
    _CPU_CASE[key_] = (lit, o, key, fold, left, right)
    return _CPU_CASE[key_]


def _cpu_product_worker(args):
    """One full MKF-CKKS mult+relin+rescale (fold of both operands with k
    distinct fold-key slots, Karatsuba tensor, relinearization, rescale) by
    the oracle on this process's core; 'switch' runs one switchOne only
    (warm-up).  Returns the seconds it took."""
    config, k, level, what, seed = args
    lit, o, key, fold, left, right = _cpu_case(config, k, level, seed)
    if what == "switch":
        t0 = time.perf_counter()
        o.mkf_switch_one(level, left[1], key, True, True)
        return time.perf_counter() - t0
    t0 = time.perf_counter()
    o.mkf_ckks_mulrelin(k, level, left, right, fold, key, True, lit.scale, lit.scale ** 2)
    return time.perf_counter() - t0


def cpu_baseline(config, k, level, repeats=3):
    """Full products on one core, the median of `repeats` (about 25 s)."""
    times = [_cpu_product_worker((config, k, level, "product", 7)) for _ in range(repeats)]
    t = statistics.median(times)
    return {"value": 1.0 / t, "unit": "mult+relin ops/s", "cores": 1, "kind": "port",
            "cpu": cpu_model(), "repeats": repeats, "seconds": times,
            "sample": f"one full MKF-CKKS mult+relin+rescale ({config}, k={k}, level {level}) by "
                      f"the C oracle on one core, median of {repeats}: {t:.2f} s"}


def _worker_count():
    cores = os.cpu_count() or 1
    try:
        # each worker holds about 4 GB (keys, operands, the oracle's buffers)
        mem_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES") / 1e9
        return max(1, min(cores, int(mem_gb // 4)))
    except (ValueError, OSError):
        return cores


def run_reference(a):
    """--impl reference: the reference algorithm's CPU restatement (the
    oracle) on every host core.  A timed step runs one full product on each
    worker process concurrently and lasts as long as the slowest of them;
    warm-up steps run one switchOne per worker."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    from mkf_b200 import params
    lit = params.get("ckks", a.config)
    level = lit.max_level if a.level < 0 else a.level
    workers = _worker_count()
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for _ in range(max(1, a.warmup)):
            pool.map(_cpu_product_worker, [(a.config, a.k, level, "switch", 10 + i)
                                           for i in range(workers)], chunksize=1)
        times = []
        for s in range(a.steps):
            t0 = time.perf_counter()
            pool.map(_cpu_product_worker, [(a.config, a.k, level, "product", 10 + i)
                                           for i in range(workers)], chunksize=1)
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = workers * a.steps / total
    sample = (f"each step: one full MKF-CKKS mult+relin+rescale ({a.config}, k={a.k}, level "
              f"{level}) on each of {workers} worker processes at once, wall time of the step")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "mult+relin ops/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"MKF-CKKS mult+relin+rescale {a.config} logN=16 k={a.k} "
                                   f"level {level}", "parties": a.k, "level": level},
            "cpu_baseline": {"value": value, "unit": "mult+relin ops/s", "cores": workers,
                             "kind": "port", "cpu": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": "mult+relin ops/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "Go and Lattigo v2.3.0 are absent on this box; the reference algorithm is "
                    "timed through its C restatement (oracle/)."}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def random_limbs(g, moduli, n, count=1):
    out = np.empty((count, len(moduli), n), np.uint64)
    for c in range(count):
        for i, q in enumerate(moduli):
            out[c, i] = g.integers(0, int(q), size=n, dtype=np.uint64)
    return out


def best_plan(ev, P, jobs, lanes_arg, cs, stream, reps=3, forms="graph"):
    """The key-fused batch plan (replayed from a CUDA graph) with the fastest
    lane count of `lanes_arg` and form of `forms` ("graph": the lanes' kernels
    in the graph; "persistent": the plan as one launch of the persistent
    executor); returns (plan, label, {label: ms per launch})."""
    tried, best = {}, None
    cands = [(int(x), f) for f in forms.split(",") if f for x in lanes_arg.split(",") if x]
    for lanes, form in cands:
        label = f"{lanes}{' persistent' if form == 'persistent' else ''}"
        b = ev.Batch(P, jobs, lanes=lanes, graph=True, fuse_keys=True,
                     persistent=form == "persistent")
        b.launch(cs)
        b.check()
        e0, e1 = __import__("torch").cuda.Event(enable_timing=True), \
            __import__("torch").cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            b.launch(cs)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        b.check()
        tried[label] = ms
        if best is None or ms < best[1]:
            if best is not None:
                best[0].close()
            best = (b, ms, label)
        else:
            b.close()
    return best[0], best[2], tried


def run_c3(a, reps, ws, rank, local):
    """The headline workload's sections (plain, streams, key-fused plan,
    kernel breakdown, e2e, level 8, served).  Every device buffer of the
    headline context is freed when this returns."""
    import torch
    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev

    lit = params.get("ckks", a.config)
    level = lit.max_level if a.level < 0 else a.level
    k = a.k
    N = lit.n
    P = ev.Parameters(lit, "ckks", device=local)
    g = np.random.Generator(np.random.PCG64(1234 + rank))
    nQ, nP = len(lit.q), len(lit.p)
    beta = (nQ + nP - 1) // nP
    qp = list(lit.q) + list(lit.p)

    def key():
        return np.ascontiguousarray(random_limbs(g, qp, N, 2 * beta).reshape(beta, 2, nQ + nP, N))

    ks = ev.MKFKeySet(P, [key() for _ in range(k)], key())
    E = ev.MKFEvaluator(P, ks)
    L1 = level + 1
    streams = [torch.cuda.Stream() for _ in range(max(1, a.streams))]
    # operand pairs cycled through by the products of a step; each stream
    # writes its own output (its products run in order)
    nin = max(8, len(streams))
    ins = []
    for _ in range(nin):
        l = ev.Ciphertext.from_array(P, random_limbs(g, lit.q[:L1], N, k + 1), True, scale=lit.scale)
        r = ev.Ciphertext.from_array(P, random_limbs(g, lit.q[:L1], N, k + 1), True, scale=lit.scale)
        ins.append((l, r))
    # launch choices: time every candidate on this workload, keep the fastest
    from mkf_b200 import autotune
    if a.tuning:
        fixed = json.loads(a.tuning)
        autotune.set_tuning(P, **fixed)
        tuned = {"best": autotune.get_tuning(P), "ms": {}}
    else:
        tuned = autotune.tune_mkf(P, k, level, operands=(E, ins[0][0], ins[0][1]))
    lout = E.output_level(ins[0][0], ins[0][1], True)
    outs = [ev.Ciphertext(P, k + 1, lout, True) for _ in range(len(streams))]
    sidx = {s.cuda_stream: i for i, s in enumerate(streams)}

    def product(i, s):
        l, r = ins[i % nin]
        E.MulRelin(l, r, outs[sidx[s.cuda_stream]], rescale=True, materialize=True,
                   stream=ctypes_stream(s))

    barrier = reps.barrier
    max_over_ranks = reps.max_over_ranks

    if a.profile_products > 0:
        if a.profile_persistent:
            # the products as one persistent plan (one lane), launched
            # --warmup times and then once more
            pouts = [ev.Ciphertext(P, k + 1, lout, True) for _ in range(a.profile_products)]
            pj = [("mkf", E, ins[j % nin][0], ins[j % nin][1], pouts[j], True, True)
                  for j in range(a.profile_products)]
            plan = ev.Batch(P, pj, lanes=1, graph=False, persistent=True)
            cs0 = ctypes_stream(streams[0])
            for _ in range(a.warmup + 1):
                plan.launch(cs0)
            plan.check()
            plan.close()
        else:
            for i in range(a.warmup):
                product(i, streams[0])
            torch.cuda.synchronize()
            for i in range(a.profile_products):
                product(i, streams[0])
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_products": a.profile_products, "tuning": tuned["best"],
                              "config": a.config, "k": k, "level": level}), flush=True)
        return None

    # ---- plain: one product at a time on one stream -------------------------
    L = capi.lib()
    s0 = streams[0]
    for i in range(a.warmup):
        product(i, s0)
    barrier()
    lat = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    plain_steps = max(a.steps, 5)
    t_plain = 0.0
    for i in range(plain_steps):
        ev0.record(s0)
        product(i, s0)
        ev1.record(s0)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        lat.append(ms)
        t_plain += ms
    barrier()
    plain_ops = ws * plain_steps / (max_over_ranks(t_plain) / 1e3)
    # per-kernel breakdown: the same products again with the library's event
    # profiler on (its events are kept out of the timed loop above)
    L.mkf_profile_enable(P.handle, 1)
    for i in range(plain_steps):
        product(i, s0)
    torch.cuda.synchronize()
    nk = L.mkf_profile_kinds()
    pms = (ctypes.c_double * nk)()
    pcnt = (ctypes.c_uint64 * nk)()
    pby = (ctypes.c_double * nk)()
    L.mkf_profile_read(P.handle, pms, pcnt, pby)
    L.mkf_profile_enable(P.handle, 0)

    # ---- batched: `batch` products per step over `streams` streams -------------
    # Steps are pipelined: stream j%streams issues product j of every step in
    # order (reusing its own operands and outputs), so a step's products start
    # as soon as their stream is free instead of waiting for the whole
    # previous step; the streams fork from and join into streams[0] around the
    # timed region only.
    def fork():
        start = torch.cuda.Event()
        start.record(streams[0])
        for s in streams[1:]:
            s.wait_event(start)

    def join():
        for s in streams[1:]:
            e = torch.cuda.Event()
            e.record(s)
            streams[0].wait_event(e)

    def batched_step(step):
        for j in range(a.batch):
            product(step * a.batch + j, streams[j % len(streams)])

    fork()
    for i in range(a.warmup):
        batched_step(i)
    join()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(streams[0])
    fork()
    for step in range(a.steps):
        batched_step(step)
    join()
    t1.record(streams[0])
    t1.synchronize()
    barrier()
    streams_ms = max_over_ranks(t0.elapsed_time(t1))
    streams_res = {"value": ws * a.steps * a.batch / (streams_ms / 1e3), "unit": "mult+relin ops/s",
                   "ms_per_step": streams_ms / a.steps, "streams": len(streams),
                   "form": "one call per product, products spread over the streams"}

    # ---- batched (headline): the step's products as one key-fused plan ----------
    # The products share the key bundle, so the plan runs them as fused calls
    # (every stage one launch per group of products, every key read once per
    # group), spread over lanes and replayed from one CUDA graph per step.
    cs0 = ctypes_stream(s0)
    pouts = [ev.Ciphertext(P, k + 1, lout, True) for _ in range(a.batch)]
    pjobs = [("mkf", E, ins[j % nin][0], ins[j % nin][1], pouts[j], True, True)
             for j in range(a.batch)]
    plan, plan_lanes, plan_tried = best_plan(ev, P, pjobs, a.plan_lanes, cs0, s0,
                                             forms=a.plan_forms)
    for _ in range(a.warmup):
        plan.launch(cs0)
    torch.cuda.synchronize()
    barrier()
    L.mkf_launch_count(1)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    t0.record(s0)
    for step in range(a.steps):
        plan.launch(cs0)
    t1.record(s0)
    t1.synchronize()
    barrier()
    clk = clocks.stop()
    launches = int(L.mkf_launch_count(0))
    total_ms = max_over_ranks(t0.elapsed_time(t1))
    value = ws * a.steps * a.batch / (total_ms / 1e3)
    plan.check()
    plan_res = {"lanes": int(plan_lanes.split()[0]), "kernels_per_step": plan.kernels, "graph": True,
                "fuse_keys": True, "persistent": plan_lanes.endswith("persistent"),
                "lanes_ms_per_step": plan_tried}
    plan.close()
    del pouts, pjobs

    kinds = {}
    for i in range(nk):
        nm = L.mkf_profile_kind_name(i).decode()
        if pcnt[i]:
            kinds[nm] = {"ms": pms[i], "launches": int(pcnt[i]), "bytes": pby[i]}
    top = max(kinds.items(), key=lambda kv: kv[1]["ms"])
    peak, peak_kind = measured_peaks()
    tk = top[1]
    avg_ms = tk["ms"] / tk["launches"]
    bytes_per_launch = tk["bytes"] / tk["launches"]
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    traffic, pipes, traffic_src = None, None, None
    nf = ncu_figures()
    fig = (nf or {}).get("kernels", {}).get(top[0])
    if fig and fig.get("shape") == [lit.log_n, L1, nP] and "dram_bytes_per_unit" in fig:
        # DRAM traffic grows with the launch's units (source polynomials of the
        # digit kernels); the fold launch (2k) and the relinearization launch
        # (one) alternate, so a launch averages (2k+1)/2 of them
        units = (2 * k + 1) / 2 if top[0].startswith("ntt_digits") else 1
        traffic = fig["dram_bytes_per_unit"] * units
        pipes = fig.get("pipes")
        traffic_src = {"capture": nf.get("capture"), "scaled_by_units": units}
    roofline = {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_ms,
                "share": tk["ms"] / sum(v["ms"] for v in kinds.values()),
                "limiter": "float64 and integer multiply pipes, not HBM",
                "pipes_ncu": pipes, "traffic_source": traffic_src,
                "compute": digits_col_compute(L, local, lit, k, L1, nP, kinds),
                "timed_in": "profiled replay of the plain loop (one stream, no overlap)"}

    # ---- e2e through the C ABI with pinned host buffers -------------------------
    e2e = None
    if not a.no_e2e:
        words_in = (k + 1) * L1 * N
        words_out = (k + 1) * (lout + 1) * N
        ns = len(streams)
        # pinned host operands (two per stream, cycled) and one pinned output
        # buffer and one set of device operands per stream
        hin = [torch.empty(words_in, dtype=torch.int64, pin_memory=True) for _ in range(2 * ns)]
        for h in hin:
            h.numpy().view(np.uint64)[:] = g.integers(0, int(lit.q[-1]), size=words_in, dtype=np.uint64)
        hout = [torch.empty(words_out, dtype=torch.int64, pin_memory=True) for _ in range(ns)]
        e_ins = [(ev.Ciphertext(P, k + 1, level, True, scale=lit.scale),
                  ev.Ciphertext(P, k + 1, level, True, scale=lit.scale)) for _ in range(ns)]
        e_outs = [ev.Ciphertext(P, k + 1, lout, True) for _ in range(ns)]

        def e2e_step():
            for j in range(a.batch):
                si = j % ns
                cs = ctypes_stream(streams[si])
                l, r = e_ins[si]
                capi.check(P.handle, L.mkf_ct_upload_async(
                    l.handle, ctypes.cast(hin[2 * si].data_ptr(), capi.u64p), words_in, cs))
                capi.check(P.handle, L.mkf_ct_upload_async(
                    r.handle, ctypes.cast(hin[2 * si + 1].data_ptr(), capi.u64p), words_in, cs))
                E.MulRelin(l, r, e_outs[si], rescale=True, materialize=True, stream=cs)
                capi.check(P.handle, L.mkf_ct_download_async(
                    e_outs[si].handle, ctypes.cast(hout[si].data_ptr(), capi.u64p), words_out, cs))

        fork()
        for _ in range(a.warmup):
            e2e_step()
        join()
        torch.cuda.synchronize()
        barrier()
        t0.record(streams[0])
        fork()
        for _ in range(a.steps):
            e2e_step()
        join()
        t1.record(streams[0])
        t1.synchronize()
        barrier()
        e_ms = max_over_ranks(t0.elapsed_time(t1))
        e2e = {"value": ws * a.steps * a.batch / (e_ms / 1e3), "unit": "mult+relin ops/s",
               "h2d_bytes_per_step": 2 * a.batch * words_in * 8,
               "d2h_bytes_per_step": a.batch * words_out * 8}

    # the same workload at level 8 (L1 = 9 limbs, beta = 3): plain and batched
    lvl8 = None
    if level > 8:
        l8 = 8
        ins8 = [(ev.Ciphertext.from_array(P, random_limbs(g, lit.q[: l8 + 1], N, k + 1), True,
                                          scale=lit.scale),
                 ev.Ciphertext.from_array(P, random_limbs(g, lit.q[: l8 + 1], N, k + 1), True,
                                          scale=lit.scale)) for _ in range(nin)]
        lo8 = E.output_level(ins8[0][0], ins8[0][1], True)
        outs8 = [ev.Ciphertext(P, k + 1, lo8, True) for _ in range(len(streams))]

        def product8(i, s):
            l, r = ins8[i % nin]
            E.MulRelin(l, r, outs8[sidx[s.cuda_stream]], rescale=True, materialize=True,
                       stream=ctypes_stream(s))

        for i in range(a.warmup):
            product8(i, s0)
        barrier()
        lat8 = []
        for i in range(plain_steps):
            ev0.record(s0)
            product8(i, s0)
            ev1.record(s0)
            ev1.synchronize()
            lat8.append(ev0.elapsed_time(ev1))
        barrier()

        def batched8(step):
            for j in range(a.batch):
                product8(step * a.batch + j, streams[j % len(streams)])

        fork()
        for i in range(a.warmup):
            batched8(i)
        join()
        torch.cuda.synchronize()
        barrier()
        t0.record(streams[0])
        fork()
        for step in range(a.steps):
            batched8(step)
        join()
        t1.record(streams[0])
        t1.synchronize()
        barrier()
        ms8 = max_over_ranks(t0.elapsed_time(t1))
        pouts8 = [ev.Ciphertext(P, k + 1, lo8, True) for _ in range(a.batch)]
        pjobs8 = [("mkf", E, ins8[j % nin][0], ins8[j % nin][1], pouts8[j], True, True)
                  for j in range(a.batch)]
        plan8, lanes8, tried8 = best_plan(ev, P, pjobs8, a.plan_lanes, cs0, s0, forms=a.plan_forms)
        for _ in range(a.warmup):
            plan8.launch(cs0)
        torch.cuda.synchronize()
        barrier()
        t0.record(s0)
        for step in range(a.steps):
            plan8.launch(cs0)
        t1.record(s0)
        t1.synchronize()
        barrier()
        pms8 = max_over_ranks(t0.elapsed_time(t1))
        plan8.close()
        del pouts8, pjobs8
        lat8.sort()
        lvl8 = {"level": l8, "plain": ws * plain_steps / (max_over_ranks(sum(lat8)) / 1e3),
                "batched": ws * a.steps * a.batch / (pms8 / 1e3), "plan": lanes8,
                "plan_ms_per_step": tried8,
                "streams": ws * a.steps * a.batch / (ms8 / 1e3), "unit": "mult+relin ops/s",
                "latency_ms": {"p50": lat8[len(lat8) // 2],
                               "p99": lat8[min(len(lat8) - 1, int(0.99 * len(lat8)))]}}

    served = run_served(a, local, P, E, ins, lout, k, plain_ops) if a.served_seconds > 0 else None
    lat_sorted = sorted(lat)
    return {
        "value": value, "ms_per_step": total_ms / a.steps, "k": k, "level": level,
        "streams": len(streams), "plain": {"value": plain_ops, "unit": "mult+relin ops/s"},
        "batched_over_plain": value / plain_ops, "batched_form": plan_res, "streams_res": streams_res,
        "latency_ms": {"p50": lat_sorted[len(lat) // 2],
                       "p99": lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))]},
        "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "level8": lvl8,
        "autotune": {"best": tuned["best"], "ms_per_product": tuned["ms"]},
        "served": served, "kernels": kinds, "clocks": clk,
    }


def run_gpu(a):
    import gc

    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    reps = Replicas("nccl", timeout_s=300)
    if a.serve_only:
        serve = run_serve(a, local, rank)
        if rank == 0:
            print(json.dumps({"metric": "KKLSS serving trace", "serving": serve}), flush=True)
        reps.close()
        return
    c3 = run_c3(a, reps, ws, rank, local)
    if c3 is None:  # profiling run
        reps.close()
        return
    gc.collect()
    torch.cuda.synchronize()
    barrier, max_over_ranks = reps.barrier, reps.max_over_ranks
    mix = run_mix(a, local, rank, barrier, max_over_ranks) if a.mix > 0 else None
    gc.collect()
    configs = run_configs(a, local) if a.configs and rank == 0 else None
    gc.collect()
    serve = run_serve(a, local, rank) if a.serve_seconds > 0 else None

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a.config, c3["k"], c3["level"])

    if rank == 0:
        k, level = c3["k"], c3["level"]
        line = {
            "metric": METRIC, "value": c3["value"], "unit": "mult+relin ops/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": c3["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (uniform random key and ciphertext words)",
            "config": {"workload": f"MKF-CKKS mult+relin+rescale+materialize {a.config}: logN=16, "
                                   f"k={k}, Q=1x60b+23x50b, P=4x60b, level {level}",
                       "parties": k, "level": level, "batch_per_step": a.batch,
                       "form": "key-fused batch plan replayed from a CUDA graph",
                       "l2": "inputs (keys 1.6 GB) larger than L2",
                       "parallelism": "replicas" if ws > 1 else "single GPU"},
            "plain": c3["plain"],
            "batched_over_plain": c3["batched_over_plain"],
            "batched_form": c3["batched_form"],
            "streams": c3["streams_res"],
            "latency_ms": c3["latency_ms"],
            "e2e": c3["e2e"],
            "gpu_launches": c3["gpu_launches"],
            "roofline": c3["roofline"],
            "level8": c3["level8"],
            "autotune": c3["autotune"],
            "served": c3["served"],
            "batched_mix": mix,
            "other_configs": configs,
            "serving": serve,
            "kernels": c3["kernels"],
            "clocks": c3["clocks"],
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    reps.close()


import ctypes  # noqa: E402


def run_mix(a, local, rank, barrier, max_over_ranks):
    """The mixed batch: `a.mix` MK-CKKS products (MKF construction, rescale and
    materialize), k uniform over {2,4,8,16}, ring uniform over the logN=14
    and logN=15 sets, level uniform over [1,L].  Plain = one product per call
    on one stream; batched = the plan replayed from its CUDA graph, lanes
    picked by timing each candidate.  Synthetic uniform words (values below
    every modulus of the ring), keys shared per (ring, k)."""
    import torch
    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev
    from mkf_b200 import autotune
    g = np.random.Generator(np.random.PCG64(777 + rank))
    rings, splits = {}, {}
    for name in ("S14", "S15"):
        lit = params.get("ckks", name)
        # the NTT phase split of the ring, by timing a k = 8 top-level product
        rl, split_ms = autotune.tune_split(lit, "ckks", 8, device=local, reps=3)
        splits[name] = {"row_log": rl, "col_log": lit.log_n - rl,
                        "ms_per_product": {str(k_): v for k_, v in split_ms.items()}}
        P = ev.Parameters(lit, "ckks", device=local, ntt_row_log=rl)
        nQ, nP, N = len(lit.q), len(lit.p), lit.n
        qmin = min(min(lit.q), min(lit.p))
        beta = (nQ + nP - 1) // nP
        key = g.integers(0, qmin, size=(beta, 2, nQ + nP, N), dtype=np.uint64)
        evs = {k: ev.MKFEvaluator(P, ev.MKFKeySet(P, [key] * k, key)) for k in (2, 4, 8, 16)}
        ctbuf = g.integers(0, qmin, size=17 * nQ * N, dtype=np.uint64)
        rings[name] = (lit, P, evs, ctbuf)
    items, shapes = [], []
    for _ in range(a.mix):
        name = ("S14", "S15")[int(g.integers(2))]
        lit, P, evs, ctbuf = rings[name]
        k = int(g.choice([2, 4, 8, 16]))
        level = int(g.integers(1, lit.max_level + 1))
        words = (k + 1) * (level + 1) * lit.n
        ops = []
        for _ in range(2):
            c = ev.Ciphertext(P, k + 1, level, True, scale=lit.scale)
            c.upload(ctbuf[:words].reshape(k + 1, level + 1, lit.n))
            ops.append(c)
        E = evs[k]
        out = ev.Ciphertext(P, k + 1, E.output_level(ops[0], ops[1], True), True)
        items.append(("mkf", E, ops[0], ops[1], out, True, True))
        shapes.append((name, k, level))
    P0 = rings["S14"][1]
    s0 = torch.cuda.Stream()
    cs = ctypes_stream(s0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L = capi.lib()

    def plain_pass():
        for it in items:
            it[1].MulRelin(it[2], it[3], it[4], rescale=True, materialize=True, stream=cs)

    def timed(fn, reps):
        for _ in range(max(1, a.warmup)):
            fn()
        barrier()
        e0.record(s0)
        for _ in range(reps):
            fn()
        e1.record(s0)
        e1.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)) / reps

    reps = max(2, a.steps // 2)
    plain_ms = timed(plain_pass, reps)
    # autotune the lane count: time each candidate plan, keep the fastest
    tried = {}
    best = None
    forms = [f for f in a.plan_forms.split(",") if f]
    for lanes in [int(x) for x in a.lanes.split(",") if x]:
        for fuse in (False, True):
            for form in forms:
                pers = form == "persistent"
                b = ev.Batch(P0, items, lanes=lanes, graph=True, fuse_keys=fuse, persistent=pers)
                ms = timed(lambda: b.launch(cs), reps)
                b.check()
                tried[f"{lanes}{' fused' if fuse else ''}{' persistent' if pers else ''}"] = ms
                if best is None or ms < best[1]:
                    if best is not None:
                        best[0].close()
                    best = (b, ms, lanes, fuse, pers)
                else:
                    b.close()
    b, batch_ms, lanes, fuse, pers = best
    L.mkf_launch_count(1)
    batch_ms = timed(lambda: b.launch(cs), reps)
    kernels = int(L.mkf_launch_count(0)) // (reps + max(1, a.warmup))
    n = len(items)
    # the same comparison per (ring, k) bucket: which products batching helps
    buckets = {}
    for name in ("S14", "S15"):
        for kb in (2, 4, 8, 16):
            sub = [it for it, sh in zip(items, shapes) if sh[0] == name and sh[1] == kb]
            if not sub:
                continue

            def plain_sub(sub=sub):
                for it in sub:
                    it[1].MulRelin(it[2], it[3], it[4], rescale=True, materialize=True, stream=cs)

            p_ms = timed(plain_sub, reps)
            bb = ev.Batch(P0, sub, lanes=lanes, graph=True, fuse_keys=fuse, persistent=pers)
            b_ms = timed(lambda: bb.launch(cs), reps)
            bb.check()
            bb.close()
            buckets[f"{name}_k{kb}"] = {"products": len(sub), "plain_ms": p_ms, "batched_ms": b_ms,
                                        "batched_over_plain": p_ms / b_ms}
            if "persistent" in forms and not pers:
                # the bucket as one persistent launch, beside the chosen form
                bp = ev.Batch(P0, sub, lanes=lanes, graph=True, fuse_keys=fuse, persistent=True)
                pp_ms = timed(lambda: bp.launch(cs), reps)
                bp.check()
                bp.close()
                buckets[f"{name}_k{kb}"]["persistent_ms"] = pp_ms
    res = {"workload": f"{n} MK-CKKS mult+relin+rescale+materialize products, k uniform over "
                       "{2,4,8,16}, logN uniform over {14 (S14: 55b+7x40b, P 2x45b), "
                       "15 (S15: 60b+15x50b, P 4x60b)}, level uniform over [1,L]",
           "products": n,
           "plain": {"value": n / (plain_ms / 1e3), "unit": "mult+relin ops/s", "ms": plain_ms},
           "batched": {"value": n / (batch_ms / 1e3), "unit": "mult+relin ops/s", "ms": batch_ms,
                       "lanes": lanes, "graph": True, "fuse_keys": fuse, "persistent": pers,
                       "kernels_per_launch": kernels},
           "batched_over_plain": plain_ms / batch_ms,
           "autotune_plan_ms": tried,
           "ntt_split": splits,
           "buckets": buckets,
           "mix": {f"k{k}": sum(1 for s in shapes if s[1] == k) for k in (2, 4, 8, 16)}}
    b.close()
    return res


def poisson_trace(srv, templates, rate, seconds, g):
    """Open-loop Poisson arrivals at `rate` req/s for `seconds` through the
    serving loop; returns its statistics (latency: submit -> result complete
    on the device)."""
    srv.reset_stats()
    n_req = max(1, int(rate * seconds))
    gaps = g.exponential(1.0 / rate, size=n_req)
    picks = g.integers(0, len(templates), size=n_req)
    busy = 0
    t_start = time.perf_counter()
    t_next = t_start
    for i in range(n_req):
        t_next += gaps[i]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        try:
            srv.submit(templates[picks[i]][i % len(templates[picks[i]])])
        except Exception as e:  # MKF_ERR_BUSY: the queue is full
            if getattr(e, "status", None) != 8:
                raise
            busy += 1
    srv.drain()
    wall = time.perf_counter() - t_start
    st = srv.stats()
    return {"offered_req_s": rate, "seconds": seconds, "requests": n_req, "busy_rejected": busy,
            "throughput_req_s": st["completed"] / wall if wall > 0 else None,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
            "inflight_peak": st["inflight_peak"],
            "scratch_peak_gb": st["scratch_peak_bytes"] / 1e9}


def run_served(a, local, P, E, ins, lout, k, plain_ops):
    """The served form twice: requests fused per key bundle by the serving
    loop (`--served-fuse` products per call on `--served-fuse-slots` slots),
    and one call per request on `--served-slots` slots."""
    fused = run_served_one(a, local, P, E, ins, lout, k, plain_ops, a.served_fuse_slots,
                           a.served_fuse) if a.served_fuse > 1 else None
    single = run_served_one(a, local, P, E, ins, lout, k, plain_ops, a.served_slots, 0)
    best = fused if fused and fused["value"] > single["value"] else single
    return dict(best, unfused=single if best is fused else None,
                fused=fused if best is single else None)


def run_served_one(a, local, P, E, ins, lout, k, plain_ops, slots, fuse_max):
    """The headline product (MKF-CKKS C3, k parties) through the serving loop
    (mkf_server_*): a closed burst measures the served throughput with the
    loop saturated, then an open-loop Poisson trace at 0.8 x that rate gives
    p50/p99 latency.  Requests run on `--served-slots` slot streams with
    scratch carved from one pool sized for that many products."""
    from mkf_b200 import evaluator as ev
    g = np.random.Generator(np.random.PCG64(4242))
    slots = max(1, slots)
    per_slot = max(1, fuse_max)
    T = 2 * slots * per_slot
    outs = [ev.Ciphertext(P, k + 1, lout, True) for _ in range(T)]
    templates = [[("mkf", E, ins[i % len(ins)][0], ins[i % len(ins)][1], outs[i], True, True)]
                 for i in range(T)]
    need = ev.job_scratch_bytes(templates[0][0])
    pool = need * slots * per_slot + (256 << 20)
    srv = ev.Server(device=local, scratch_bytes=pool, slots=slots, queue_cap=4096,
                    fuse_max=fuse_max)
    try:
        for i in range(T):
            srv.submit(templates[i][0])
        srv.drain()
        srv.reset_stats()
        burst = 256
        t0 = time.perf_counter()
        for i in range(burst):
            srv.submit(templates[i % T][0])
        srv.drain()
        capacity = burst / (time.perf_counter() - t0)
        bst = srv.stats()
        trace = poisson_trace(srv, templates, 0.8 * capacity, a.served_seconds, g)
    finally:
        srv.close()
    return {"workload": "the headline product through the serving loop",
            "value": capacity, "unit": "mult+relin ops/s", "slots": slots, "fuse_max": fuse_max,
            "scratch_pool_gb": pool / 1e9,
            "burst": {"requests": burst, "p50_ms": bst["p50_ms"], "p99_ms": bst["p99_ms"]},
            "served_over_plain": capacity / plain_ops,
            "open_loop": trace}


def run_configs(a, local):
    """The other benchmark configurations, one product per call on one stream
    (plain) and, for reference, the C oracle on one core: C1 (CKKS logN 14,
    k 2, 55b + 7x40b, P 2x45b) and C2 (BFV logN 15, k 4, fifteen 58-bit Q and
    QMul, P 2x60b, t 65537), in both constructions (MKF aggregate fold and
    KKLSS per-party keys).  Synthetic uniform words."""
    import torch
    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev
    from oracle.oracle import Oracle
    res = {}
    g = np.random.Generator(np.random.PCG64(31337))
    st = torch.cuda.Stream()
    cs = ctypes_stream(st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for cfg, scheme, k in (("C1", "ckks", 2), ("C2", "bfv", 4)):
        lit = params.get(scheme, cfg)
        P = ev.Parameters(lit, scheme, device=local)
        nQ, nP, N = len(lit.q), len(lit.p), lit.n
        qmin = min(min(lit.q), min(lit.p), min(lit.q_mul) if lit.q_mul else 1 << 62)
        beta1 = (nQ + nP - 1) // nP
        key = g.integers(0, qmin, size=(beta1, 2, nQ + nP, N), dtype=np.uint64)
        level = lit.max_level
        ops = g.integers(0, qmin, size=(2, k + 1, level + 1, N), dtype=np.uint64)
        ckks = scheme == "ckks"
        E = ev.MKFEvaluator(P, ev.MKFKeySet(P, [key] * k, key))
        l = ev.Ciphertext.from_array(P, ops[0], ckks, scale=lit.scale if ckks else None)
        r = ev.Ciphertext.from_array(P, ops[1], ckks, scale=lit.scale if ckks else None)
        out = ev.Ciphertext(P, 2, E.output_level(l, r, ckks), ckks)
        kind = capi.KEY_KKLSS_RLK if ckks else capi.KEY_KKLSS_BFV_RLK
        rlk = ev.RelinearizationKeySet(P, g.integers(0, qmin, size=P.key_words(capi.KEY_GADGET),
                                                      dtype=np.uint64))
        img = g.integers(0, qmin, size=P.key_words(kind), dtype=np.uint64)
        for pid in range(k):
            rlk.AddRelinearizationKey(pid, img)
        kl = ev.Ciphertext.from_array(P, ops[0], False, ids=list(range(k)),
                                      scale=lit.scale if ckks else None)
        kr = ev.Ciphertext.from_array(P, ops[1], False, ids=list(range(k)),
                                      scale=lit.scale if ckks else None)
        kout = ev.Evaluator(P).MulRelinNew(kl, kr, rlk)  # output shape; reused below
        Lb = capi.lib()

        def kklss():
            capi.check(P.handle, Lb.mkf_kklss_mulrelin(P.handle, kl.handle, kr.handle, rlk.handle,
                                                       kout.handle, cs))
        row = {}
        for name, fn in (("mkf", lambda: E.MulRelin(l, r, out, rescale=ckks, stream=cs)),
                         ("kklss", kklss)):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            n = 20
            e0.record(st)
            for _ in range(n):
                fn()
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / n
            row[name] = {"plain_ops_s": 1e3 / ms, "ms": ms}
        # the oracle, one core, one MKF product
        o = Oracle.from_literal(lit)
        fold = np.ascontiguousarray(np.stack([key] * k))
        t0 = time.perf_counter()
        if ckks:
            o.mkf_ckks_mulrelin(k, level, ops[0], ops[1], fold, key, True, lit.scale, lit.scale ** 2)
        else:
            o.mkf_bfv_mulrelin(k, ops[0], ops[1], fold, key, lit.t)
        row["mkf"]["cpu_oracle_s"] = time.perf_counter() - t0
        row["workload"] = f"{scheme.upper()} {cfg}: logN {lit.log_n}, k {k}, level {level}"
        res[cfg] = row
        del E, l, r, out, kl, kr, kout, rlk, P
    return res


def run_serve(a, local, rank):
    """Open-loop serving traces through the serving loop (mkf_server_*): KKLSS
    mult+relin requests, scheme 50/50 CKKS/BFV, ring uniform over logN
    {14,15,16}, k uniform over {2..16} parties drawn from a per-ring key pool
    (64 parties at logN 14/15, `--serve-parties16` at 16), level uniform.
    Per-party relinearization keys are distinct HBM buffers.  Requests are
    drawn from `--serve-templates` prepared operand sets.  First a closed burst
    measures capacity; then Poisson arrivals at each load factor of
    `--serve-loads` times min(rate, capacity)."""
    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev
    g = np.random.Generator(np.random.PCG64(999 + rank))
    rings = []
    key_bytes = 0
    for scheme in ("ckks", "bfv"):
        for name, npart in (("S14", 64), ("S15", 64), ("S16", a.serve_parties16)):
            lit = params.get(scheme, name)
            P = ev.Parameters(lit, scheme, device=local)
            qmin = min(min(lit.q), min(lit.p), min(lit.q_mul) if lit.q_mul else 1 << 62)
            kind = capi.KEY_KKLSS_RLK if scheme == "ckks" else capi.KEY_KKLSS_BFV_RLK
            img = g.integers(0, qmin, size=P.key_words(kind), dtype=np.uint64)
            rlk = ev.RelinearizationKeySet(P, g.integers(0, qmin, size=P.key_words(capi.KEY_GADGET),
                                                          dtype=np.uint64))
            for pid in range(npart):
                rlk.AddRelinearizationKey(pid, img)
            key_bytes += 8 * npart * img.size
            N, nq = lit.n, len(lit.q)
            buf = g.integers(0, qmin, size=17 * nq * N, dtype=np.uint64)
            rings.append((scheme, name, lit, P, rlk, npart, buf))
    E = {}
    templates = []
    for _ in range(a.serve_templates):
        scheme, name, lit, P, rlk, npart, buf = rings[int(g.integers(len(rings)))]
        k = int(g.integers(2, 17))
        level = int(g.integers(1, lit.max_level + 1)) if scheme == "ckks" else lit.max_level
        ids = [int(x) for x in g.choice(npart, size=k, replace=False)]
        words = (k + 1) * (level + 1) * lit.n
        ops = []
        for _ in range(2):
            c = ev.Ciphertext(P, k + 1, level, False, ids=ids, scale=lit.scale if scheme == "ckks" else None)
            c.upload(buf[:words].reshape(k + 1, level + 1, lit.n))
            ops.append(c)
        ev_ = E.setdefault(id(P), ev.Evaluator(P))
        ref_level = level - 1 if scheme == "ckks" else level
        outs = [ev.Ciphertext(P, k + 1, ref_level, False) for _ in range(2)]
        templates.append([("kklss", rlk, ops[0], ops[1], o) for o in outs])
    need = max(ev.job_scratch_bytes(t[0]) for t in templates)
    slots = max(1, a.serve_slots)
    # keys and request scratch share the HBM budget of the trace
    pool = int(min(max(need * 3, 8 << 30), 40 << 30, a.serve_hbm_gb * 1e9 - key_bytes))
    if pool < need:
        raise SystemExit(f"serving: {key_bytes / 1e9:.1f} GB of keys leave no room for a "
                         f"{need / 1e9:.1f} GB request under {a.serve_hbm_gb} GB")
    srv = ev.Server(device=local, scratch_bytes=pool, slots=slots, queue_cap=4096)
    # closed burst: capacity
    burst = [templates[i % len(templates)][i % 2] for i in range(2 * len(templates))]
    for j in burst[: len(templates)]:
        srv.submit(j)
    srv.drain()
    srv.reset_stats()
    t0 = time.perf_counter()
    for j in burst:
        srv.submit(j)
    srv.drain()
    cap_s = time.perf_counter() - t0
    capacity = len(burst) / cap_s
    burst_stats = srv.stats()
    srv.reset_stats()
    # open loop, one trace per load factor
    base = min(a.serve_rate, capacity)
    traces = []
    for f in [float(x) for x in a.serve_loads.split(",") if x]:
        tr = poisson_trace(srv, templates, f * base, a.serve_seconds, g)
        tr["load_factor"] = f
        traces.append(tr)
    srv.close()
    return {"workload": "open-loop Poisson trace of KKLSS mult+relin requests: CKKS/BFV 50/50, "
                        "logN uniform over {14,15,16} (S14/S15/S16 sets), k uniform over {2..16} "
                        "from a per-ring party pool, level uniform (CKKS)",
            "requested_rate_req_s": a.serve_rate, "slots": slots,
            "scratch_pool_gb": pool / 1e9, "key_pool_gb": key_bytes / 1e9,
            "hbm_budget_gb": a.serve_hbm_gb,
            "party_pool": {"logN14": 64, "logN15": 64, "logN16": a.serve_parties16},
            "capacity_req_s": capacity,
            "capacity_burst": {"requests": len(burst), "p50_ms": burst_stats["p50_ms"],
                               "p99_ms": burst_stats["p99_ms"]},
            "traces": traces,
            "latency": "submit -> result complete on the device (host callback)"}


def ctypes_stream(s):
    return ctypes.c_void_p(s.cuda_stream)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_gpu(a)


if __name__ == "__main__":
    main()
