"""Serving loop (mkf_server_*): results of requests served concurrently with
others equal the same products run alone, bit for bit; admission follows the
scratch pool; a full queue refuses (BUSY); waits are bounded (TIMEOUT)."""
import numpy as np
import pytest

from mkf_b200 import capi
from mkf_b200 import evaluator as ev
from tests.test_gpu_batch import _make_jobs, rings  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _fresh_out(job):
    out = job[4]
    new = ev.Ciphertext(out.params, out.n_comp, out.Level(), job[0] == "mkf")
    return job[:4] + (new,) + job[5:]


def test_server_results_equal_alone(rings):  # noqa: F811
    jobs, singles = _make_jobs(*rings)
    want = [f() for f in singles]
    srv = ev.Server(scratch_bytes=6 << 30, slots=4, queue_cap=1024)
    # three rounds of the whole mix, interleaved, each with its own outputs
    subs = []
    for rnd in range(3):
        for i, j in enumerate(jobs):
            jj = _fresh_out(j)
            subs.append((i, jj, srv.submit(jj)))
    for i, jj, t in subs:
        st, lat = srv.wait(t, timeout_s=60)
        assert st == capi.OK
        assert lat > 0
        assert np.array_equal(jj[4].download(), want[i]), f"job {i} differs in the mix"
    s = srv.stats()
    assert s["completed"] == len(subs) and s["failed"] == 0
    assert s["inflight_peak"] >= 2  # requests overlapped on the device
    assert 0 < s["p50_ms"] <= s["p99_ms"] <= s["max_ms"]
    srv.close()


def test_server_admission_follows_scratch_pool(rings):  # noqa: F811
    jobs, _ = _make_jobs(*rings)
    need = [ev.job_scratch_bytes(j) for j in jobs]
    big = max(need)
    # room for one largest request only: never two of them at once
    srv = ev.Server(scratch_bytes=int(big * 1.5), slots=8, queue_cap=64)
    i_big = need.index(big)
    tickets = [srv.submit(_fresh_out(jobs[i_big])) for _ in range(4)]
    for t in tickets:
        assert srv.wait(t, 60)[0] == capi.OK
    assert srv.stats()["inflight_peak"] == 1
    assert srv.stats()["scratch_peak_bytes"] <= int(big * 1.5)
    srv.close()
    tiny = ev.Server(scratch_bytes=big // 2, slots=2, queue_cap=4)
    with pytest.raises(capi.MKFError, match="MKF_ERR_OOM"):
        tiny.submit(_fresh_out(jobs[i_big]))
    tiny.close()


def test_server_busy_timeout_and_resume(rings):  # noqa: F811
    jobs, singles = _make_jobs(*rings)
    srv = ev.Server(scratch_bytes=4 << 30, slots=2, queue_cap=3)
    srv.pause(True)
    subs = [_fresh_out(jobs[0]) for _ in range(3)]
    tickets = [srv.submit(j) for j in subs]
    with pytest.raises(capi.MKFError, match="MKF_ERR_BUSY"):
        srv.submit(_fresh_out(jobs[0]))
    with pytest.raises(capi.MKFError, match="MKF_ERR_TIMEOUT"):
        srv.wait(tickets[0], timeout_s=0.05)
    srv.pause(False)
    want = singles[0]()
    for j, t in zip(subs, tickets):
        assert srv.wait(t, 60)[0] == capi.OK
        assert np.array_equal(j[4].download(), want)
    s = srv.stats()
    assert s["rejected"] == 1 and s["completed"] == 3
    srv.close()


def test_server_rejects_invalid_job(rings):  # noqa: F811
    r14 = rings[0]
    E = r14.mkf[2]
    left, right = r14.ct(3, 5, True), r14.ct(3, 5, True)
    bad = ("mkf", E, left, right, ev.Ciphertext(r14.P, 2, 5, True), True, False)
    srv = ev.Server(scratch_bytes=1 << 30, slots=2, queue_cap=4)
    with pytest.raises(capi.MKFError, match="output must have"):
        srv.submit(bad)
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_server_cancels_queued_requests_on_close(rings):  # noqa: F811
    jobs, _ = _make_jobs(*rings)
    srv = ev.Server(scratch_bytes=1 << 30, slots=1, queue_cap=8)
    srv.pause(True)
    for _ in range(3):
        srv.submit(_fresh_out(jobs[0]))
    srv.close()  # must return: queued requests are cancelled, nothing in flight


def test_server_fuses_requests_sharing_a_key_bundle(rings):  # noqa: F811
    """fuse_max: queued MKF-CKKS requests of one key bundle are served as fused
    calls; each result equals the product run alone, and the fused groups
    keep requests of other bundles (and KKLSS requests) apart."""
    from tests.test_gpu_batch import _fused_jobs
    r14, r13 = rings
    jobs, singles = [], []
    for E, ring, k, level, count, mat in [(r14.mkf[2], r14, 2, 7, 6, True),
                                          (r14.mkf[3], r14, 3, 5, 3, False),
                                          (r13.mkf[2], r13, 2, 5, 4, True)]:
        j, s = _fused_jobs(ring, E, k, level, count, mat)
        jobs += j
        singles += s
    extra, extra_singles = _make_jobs(r14, r13)
    jobs += extra[-2:]
    singles += extra_singles[-2:]
    want = [f() for f in singles]
    srv = ev.Server(scratch_bytes=6 << 30, slots=2, queue_cap=256, fuse_max=4)
    srv.pause(True)  # queue everything first, so that groups form
    tickets = [srv.submit(j) for j in jobs]
    srv.pause(False)
    for i, t in enumerate(tickets):
        st, _ = srv.wait(t, timeout_s=60)
        assert st == capi.OK
        assert np.array_equal(jobs[i][4].download(), want[i]), f"request {i} differs when fused"
    s = srv.stats()
    assert s["completed"] == len(jobs) and s["failed"] == 0
    assert s["inflight_peak"] > 2  # more requests in flight than slots: groups ran
    srv.close()
