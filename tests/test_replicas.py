"""The replica plumbing of multi-GPU runs on CPU: two gloo ranks agree on the
maximum over ranks and on the whole-job throughput; a rank that fails before
the barrier makes the other one fail within the process-group timeout
instead of hanging."""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK=str(rank), LOCAL_RANK=str(rank))


def _put(q, item):
    q.put(item)
    q.close()
    q.join_thread()  # flushed before the process leaves


def _agree(rank, port, q):
    _env(rank, port)
    from mkf_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=30)
    r.barrier()
    m = r.max_over_ranks(1.0 + rank)        # rank 1 is the slower one
    thr = r.throughput(10, 1.0 + rank)      # 2 ranks x 10 units over 2 s
    q.put((rank, r.world, m, thr))
    r.close()


def _fail_one(rank, port, q):
    _env(rank, port)
    from mkf_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=3)
    if rank == 1:
        _put(q, (rank, "left"))
        os._exit(0)                         # leaves between steps, without the barrier
    t0 = time.time()
    try:
        r.barrier()
        msg = "no error"
    except Exception as e:  # noqa: BLE001
        msg = f"error after {time.time() - t0:.1f}s: {type(e).__name__}"
    _put(q, (rank, msg))
    os._exit(0)


def _run(fn):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=fn, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=60) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda x: x[0])


def test_two_ranks_agree():
    out = _run(_agree)
    for rank, world, m, thr in out:
        assert world == 2 and m == 2.0 and thr == pytest.approx(10.0)


def test_a_departed_rank_ends_the_other_ranks_barrier():
    out = _run(_fail_one)
    assert out[1][1] == "left"
    assert out[0][1].startswith("error"), out
