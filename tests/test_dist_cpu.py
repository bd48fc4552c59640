"""The multi-rank host path of the benchmark on CPU: two gloo ranks on
127.0.0.1, each with its own ray batch seed, a barrier and the max-over-ranks
time, and the whole-job (weak scaling) rate computed from it."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from nrt import dist

    r, w, local = dist.init("gloo", timeout_s=60)
    seed = dist.rank_seed(1, r)
    dist.barrier()
    ms = 10.0 + 5.0 * r  # rank 1 is the slower one
    mx = dist.max_over_ranks(ms)
    rate = dist.weak_scaling_rate(1000, w, mx * 1e-3)
    q.put((r, w, local, seed, mx, rate))
    dist.barrier()
    dist.finalize()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    assert got[0][3] != got[1][3]                    # each rank its own ray batch
    assert all(g[4] == pytest.approx(15.0) for g in got)  # max over ranks, seen by every rank
    assert all(g[5] == pytest.approx(2 * 1000 / 0.015) for g in got)
