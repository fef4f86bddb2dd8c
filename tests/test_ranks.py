"""The multi-rank path (independent replicas) with two gloo ranks on CPU: distinct
per-rank systems, max-over-ranks timing, whole-job throughput."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from conductorrigid_b200 import ranks, systems

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, _, w = ranks.rank_info()
        s = systems.workload("plain_small", seed=ranks.replica_seed(1, r), scale=0.2).system
        ms = 100.0 + 50.0 * r  # this rank's step time
        ranks.barrier(w)
        worst = ranks.max_over_ranks(ms, w)
        out.put((r, w, float(s.body_pos.sum()), worst, ranks.job_throughput(1.0, worst, w)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_distinct_replicas_and_agree_on_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert res[0][2] != res[1][2]  # different replicas
    assert all(r[3] == 150.0 for r in res)  # the slowest rank's time on every rank
    assert all(abs(r[4] - 2 * 1e3 / 150.0) < 1e-12 for r in res)


def test_single_process_defaults(monkeypatch):
    from conductorrigid_b200 import ranks

    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    assert ranks.rank_info() == (0, 0, 1)
    assert ranks.max_over_ranks(3.5, 1) == 3.5
    assert ranks.job_throughput(2.0, 500.0, 1) == pytest.approx(4.0)
    assert np.isclose(ranks.job_throughput(1.0, 250.0, 4), 16.0)
