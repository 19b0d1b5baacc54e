"""Batch plans (mkf_batch_create / mkf_batch_launch, mkf_mulrelin_batch):
every job of a mixed batch (party counts, levels, MKF and KKLSS, two ring
degrees) must equal the single-call result bit for bit, eagerly and when
replayed from the captured CUDA graph, including after the operands change."""
import numpy as np
import pytest

from mkf_b200 import capi, params
from mkf_b200 import evaluator as ev
from tests.test_gpu_parity import gpu

pytestmark = pytest.mark.gpu


def _limbs(g, moduli, n, lead=()):
    out = np.empty(tuple(lead) + (len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = g.integers(0, q, size=tuple(lead) + (n,), dtype=np.uint64)
    return out


class _Ring:
    """Random keys for one ring: MKF key bundles per k and a KKLSS key set."""

    def __init__(self, lit, seed, ks):
        self.lit, self.P = lit, gpu(lit, "ckks")
        self.g = np.random.default_rng(seed)
        nQ, nP, N = len(lit.q), len(lit.p), lit.n
        qp = list(lit.q) + list(lit.p)
        beta1 = (nQ - 1 + nP) // nP

        def swk():
            return np.ascontiguousarray(_limbs(self.g, qp, N, (beta1, 2)))
        self.mkf = {k: ev.MKFEvaluator(self.P, ev.MKFKeySet(self.P, [swk() for _ in range(k)], swk()))
                    for k in ks}
        beta2 = (nQ - 1 + nP // 2) // (nP // 2)
        self.rlk = ev.RelinearizationKeySet(self.P, _limbs(self.g, qp, N, (beta2,)))
        for pid in range(6):
            self.rlk.AddRelinearizationKey(pid, np.ascontiguousarray(_limbs(self.g, qp, N, (3, beta2))))
        self.E = ev.Evaluator(self.P)

    def ct(self, ncomp, level, ntt, ids=None):
        a = _limbs(self.g, self.lit.q[: level + 1], self.lit.n, (ncomp,))
        return ev.Ciphertext.from_array(self.P, a, ntt, ids=ids, scale=self.lit.scale)


def _make_jobs(r14, r13):
    jobs, singles = [], []
    for ring, k, level in [(r14, 2, 7), (r14, 3, 4), (r14, 1, 2), (r13, 2, 5), (r13, 3, 3), (r14, 2, 1)]:
        E = ring.mkf[k]
        left, right = ring.ct(k + 1, level, True), ring.ct(k + 1, level, True)
        materialize = level % 2 == 1
        lvl = E.output_level(left, right, True)
        out = ev.Ciphertext(ring.P, k + 1 if materialize else 2, lvl, True)
        jobs.append(("mkf", E, left, right, out, True, materialize))
        singles.append(lambda E=E, l=left, r=right, m=materialize: E.MulRelinNew(l, r, True, m).download())
    # KKLSS: one aligned pair and one pair needing the union alignment
    for ring, ids0, ids1, level in [(r13, [0, 1], [0, 1], 4), (r14, [0, 2], [1, 2, 3], 5)]:
        op0 = ring.ct(len(ids0) + 1, level, False, ids0)
        op1 = ring.ct(len(ids1) + 1, level, False, ids1)
        ref = ring.E.MulRelinNew(op0, op1, ring.rlk)
        out = ev.Ciphertext(ring.P, ref.n_comp, ref.Level(), False)
        jobs.append(("kklss", ring.rlk, op0, op1, out))
        singles.append(lambda ring=ring, a=op0, b=op1: ring.E.MulRelinNew(a, b, ring.rlk).download())
    return jobs, singles


@pytest.fixture(scope="module")
def rings():
    r14 = _Ring(params.small("ckks", log_n=14, n_q=8, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                             scale_bits=45), 11, (1, 2, 3))
    r13 = _Ring(params.small("ckks", log_n=13, n_q=6, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                             scale_bits=45), 12, (2, 3))
    return r14, r13


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_single_calls(rings, graph):
    jobs, singles = _make_jobs(*rings)
    want = [f() for f in singles]
    b = ev.Batch(rings[0].P, jobs, lanes=3, graph=graph)
    assert b.statuses() == [0] * len(jobs)
    for rep in range(2):
        b.launch()
        ev.capi.lib()  # keep the binding loaded
        import torch
        torch.cuda.synchronize()
        for i, j in enumerate(jobs):
            got = j[4].download()
            assert np.array_equal(got, want[i]), f"job {i} differs (graph={graph}, launch {rep})"
    assert b.kernels > 0
    # new operand contents, same handles: the plan recomputes
    g = np.random.default_rng(99)
    for j in jobs:
        for op in (j[2], j[3]):
            lit = rings[0].lit if op.params is rings[0].P else rings[1].lit
            op.upload(_limbs(g, lit.q[: op.Level() + 1], lit.n, (op.n_comp,)))
    want2 = [f() for f in singles]
    b.launch()
    import torch
    torch.cuda.synchronize()
    for i, j in enumerate(jobs):
        assert np.array_equal(j[4].download(), want2[i]), f"job {i} differs after new operands"
    b.close()


def test_batch_rejects_invalid_job(rings):
    r14 = rings[0]
    E = r14.mkf[2]
    left, right = r14.ct(3, 5, True), r14.ct(3, 5, True)
    bad_out = ev.Ciphertext(r14.P, 2, 5, True)  # wrong level: rescale lowers it
    with pytest.raises(capi.MKFError, match="output must have"):
        ev.Batch(r14.P, [("mkf", E, left, right, bad_out, True, False)], lanes=2, graph=True)


def test_one_shot_batch(rings):
    jobs, singles = _make_jobs(*rings)
    want = [f() for f in singles]
    arr = (capi.Job * len(jobs))()
    for i, j in enumerate(jobs):
        if j[0] == "mkf":
            arr[i].kind, arr[i].mkf_keys = capi.JOB_MKF, j[1].keys.handle
            arr[i].flags = capi.FLAG_RESCALE | (capi.FLAG_MATERIALIZE if j[6] else 0)
        else:
            arr[i].kind, arr[i].kklss_keys = capi.JOB_KKLSS, j[1].handle
        arr[i].a, arr[i].b, arr[i].out = j[2].handle, j[3].handle, j[4].handle
    P = rings[0].P
    capi.check(P.handle, capi.lib().mkf_mulrelin_batch(P.handle, arr, len(jobs), None))
    for i, j in enumerate(jobs):
        assert np.array_equal(j[4].download(), want[i]), f"job {i} differs"


def _fused_jobs(ring, E, k, level, count, materialize):
    jobs, singles = [], []
    for _ in range(count):
        left, right = ring.ct(k + 1, level, True), ring.ct(k + 1, level, True)
        out = ev.Ciphertext(ring.P, k + 1 if materialize else 2, E.output_level(left, right, True),
                            True)
        jobs.append(("mkf", E, left, right, out, True, materialize))
        singles.append(lambda E=E, l=left, r=right, m=materialize: E.MulRelinNew(l, r, True, m).download())
    return jobs, singles


@pytest.mark.parametrize("fuse_ip", [0, 1])
@pytest.mark.parametrize("graph", [False, True])
def test_key_fused_batch_matches_single_calls(rings, graph, fuse_ip):
    """MKF_BATCH_FUSE_KEYS: products sharing a key bundle (two bundles, two
    levels, compact and materialized outputs) run as fused calls of several
    products, next to jobs that cannot fuse (KKLSS, another ring); every
    output equals its single call, on both inner-product forms."""
    from mkf_b200 import autotune
    r14, r13 = rings
    for r in rings:
        autotune.set_tuning(r.P, fuse_ip=fuse_ip)
    jobs, singles = [], []
    for E, k, level, count, mat in [(r14.mkf[2], 2, 7, 7, True), (r14.mkf[3], 3, 5, 5, False),
                                    (r14.mkf[2], 2, 4, 3, False), (r13.mkf[2], 2, 5, 4, True)]:
        ring = r14 if E.params is r14.P else r13
        j, s = _fused_jobs(ring, E, k, level, count, mat)
        jobs += j
        singles += s
    extra, extra_singles = _make_jobs(r14, r13)
    jobs += extra[-2:]  # the KKLSS jobs
    singles += extra_singles[-2:]
    want = [f() for f in singles]
    b = ev.Batch(r14.P, jobs, lanes=2, graph=graph, fuse_keys=True)
    assert b.statuses() == [0] * len(jobs)
    import torch
    for rep in range(2):
        b.launch()
        torch.cuda.synchronize()
        for i, j in enumerate(jobs):
            assert np.array_equal(j[4].download(), want[i]), \
                f"job {i} differs (graph={graph}, fuse_ip={fuse_ip}, launch {rep})"
    # fused calls issue far fewer kernels than one call per product
    plain = ev.Batch(r14.P, jobs, lanes=2, graph=False)
    plain.launch()
    torch.cuda.synchronize()
    if not graph:
        assert b.kernels < plain.kernels
    plain.close()
    b.close()
    for r in rings:
        autotune.set_tuning(r.P, fuse_ip=0)


def _mkf_jobs(r14, r13):
    """MKF-CKKS jobs of both rings (party counts, levels, compact and
    materialized outputs) and their single calls."""
    jobs, singles = _make_jobs(r14, r13)
    keep = [i for i, j in enumerate(jobs) if j[0] == "mkf"]
    return [jobs[i] for i in keep], [singles[i] for i in keep]


@pytest.mark.parametrize("fuse_ip", [0, 1])
@pytest.mark.parametrize("fuse_keys", [False, True])
@pytest.mark.parametrize("graph", [False, True])
def test_persistent_batch_matches_single_calls(rings, graph, fuse_keys, fuse_ip):
    """MKF_BATCH_PERSISTENT: the whole plan is one launch of the persistent
    executor; every output equals its single call bit for bit, on repeated
    launches and after the operands change, on both inner-product forms."""
    from mkf_b200 import autotune
    r14, r13 = rings
    orig = [autotune.get_tuning(r.P)["fuse_ip"] for r in rings]
    for r in rings:
        autotune.set_tuning(r.P, fuse_ip=fuse_ip)
    jobs, singles = _mkf_jobs(r14, r13)
    if fuse_keys:
        for E, k, level, count, mat in [(r14.mkf[2], 2, 7, 5, True), (r13.mkf[3], 3, 4, 3, False)]:
            ring = r14 if E.params is r14.P else r13
            j, s = _fused_jobs(ring, E, k, level, count, mat)
            jobs += j
            singles += s
    want = [f() for f in singles]
    b = ev.Batch(r14.P, jobs, lanes=3, graph=graph, fuse_keys=fuse_keys, persistent=True)
    assert b.statuses() == [0] * len(jobs)
    assert b.kernels == 1
    for rep in range(2):
        b.launch()
        b.check()
        for i, j in enumerate(jobs):
            assert np.array_equal(j[4].download(), want[i]), \
                f"job {i} differs (graph={graph}, fuse_keys={fuse_keys}, fuse_ip={fuse_ip}, launch {rep})"
    g = np.random.default_rng(7)
    for j in jobs:
        for op in (j[2], j[3]):
            lit = r14.lit if op.params is r14.P else r13.lit
            op.upload(_limbs(g, lit.q[: op.Level() + 1], lit.n, (op.n_comp,)))
    want2 = [f() for f in singles]
    b.launch()
    b.check()
    for i, j in enumerate(jobs):
        assert np.array_equal(j[4].download(), want2[i]), f"job {i} differs after new operands"
    b.close()
    for r, f in zip(rings, orig):
        autotune.set_tuning(r.P, fuse_ip=f)


def test_persistent_batch_refuses_jobs_it_cannot_run(rings):
    """KKLSS jobs launch kernels the executor has no body for: the plan is
    refused, not run some other way."""
    jobs, _ = _make_jobs(*rings)
    kk = [j for j in jobs if j[0] == "kklss"]
    with pytest.raises(capi.MKFError, match="persistent plan"):
        ev.Batch(rings[0].P, kk, lanes=2, graph=False, persistent=True)


def test_persistent_wait_bound_reports_timeout(rings):
    """A wait that nothing completes (the test hook raises the last launch's
    count by one) runs out after its bound: the launch ends, check() reports
    MKF_ERR_TIMEOUT, and the context still runs a plan correctly after."""
    r14, r13 = rings
    jobs, singles = _mkf_jobs(r14, r13)
    jobs, singles = jobs[:2], singles[:2]
    want = [f() for f in singles]
    bad = ev.Batch(r14.P, jobs, lanes=2, graph=False, persistent=True,
                   extra_flags=capi.BATCH_TEST_STALL)
    bad.launch()
    with pytest.raises(capi.MKFError, match="MKF_ERR_TIMEOUT"):
        bad.check()
    bad.close()
    good = ev.Batch(r14.P, jobs, lanes=2, graph=False, persistent=True)
    good.launch()
    good.check()
    for i, j in enumerate(jobs):
        assert np.array_equal(j[4].download(), want[i])
    good.close()


@pytest.mark.parametrize("persistent", [False, True])
def test_plan_keeps_its_scratch_when_a_later_plan_grows_the_lanes(rings, persistent):
    """A graph (or persistent) plan records addresses in its lanes' scratch;
    a later plan on the same lanes that needs more scratch must not free it:
    the first plan, launched again after the second was made, still gives
    the single-call results."""
    r14, r13 = rings
    small, small_want = _mkf_jobs(r14, r13)
    small, small_want = small[:3], [f() for f in small_want[:3]]
    a = ev.Batch(r14.P, small, lanes=2, graph=True, persistent=persistent)
    # a wider fused group than any plan before it made on these lanes
    big, big_singles = _fused_jobs(r14, r14.mkf[3], 3, 7, 10 if persistent else 8, True)
    big_want = [f() for f in big_singles]
    b = ev.Batch(r14.P, big, lanes=2, graph=True, fuse_keys=True, persistent=persistent)
    for plan, jobs, want in [(a, small, small_want), (b, big, big_want), (a, small, small_want)]:
        for j in jobs:
            j[4].upload(np.zeros_like(j[4].download()))
        plan.launch()
        plan.check()
        for i, j in enumerate(jobs):
            assert np.array_equal(j[4].download(), want[i]), f"job {i} differs"
    a.close()
    b.close()


@pytest.mark.parametrize("log_n,row_log", [(15, 0), (15, 7), (16, 0), (14, 8)])
def test_persistent_batch_on_larger_rings_and_splits(log_n, row_log):
    """The executor's bodies for every phase shape: rings of logN 14-16 with
    their default and other NTT split, a few products of uneven party count
    and level, one persistent launch, each output equal to its single call."""
    lit = params.small("ckks", log_n=log_n, n_q=5, n_p=2, q_bits=45, first_bits=55, p_bits=55,
                       scale_bits=45)
    P = ev.Parameters(lit, "ckks", ntt_row_log=row_log)
    g = np.random.default_rng(log_n * 10 + row_log)
    qp = list(lit.q) + list(lit.p)
    beta = (len(lit.q) - 1 + len(lit.p)) // len(lit.p)
    jobs, singles = [], []
    for k, level, mat in [(2, lit.max_level, True), (3, 2, False)]:
        keys = ev.MKFKeySet(P, [np.ascontiguousarray(_limbs(g, qp, lit.n, (beta, 2))) for _ in range(k)],
                            np.ascontiguousarray(_limbs(g, qp, lit.n, (beta, 2))))
        E = ev.MKFEvaluator(P, keys)
        left, right = (ev.Ciphertext.from_array(P, _limbs(g, lit.q[: level + 1], lit.n, (k + 1,)), True,
                                                scale=lit.scale) for _ in range(2))
        out = ev.Ciphertext(P, k + 1 if mat else 2, E.output_level(left, right, True), True)
        jobs.append(("mkf", E, left, right, out, True, mat))
        singles.append(lambda E=E, l=left, r=right, m=mat: E.MulRelinNew(l, r, True, m).download())
    want = [f() for f in singles]
    b = ev.Batch(P, jobs, lanes=2, graph=True, persistent=True)
    b.launch()
    b.check()
    for i, j in enumerate(jobs):
        assert np.array_equal(j[4].download(), want[i]), f"job {i} differs (logN {log_n}, row_log {row_log})"
    b.close()
