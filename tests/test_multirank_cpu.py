"""The bench's multi-rank plumbing (cuda_pf_localization_b200/multi.py) on
CPU: two gloo ranks rendezvous at 127.0.0.1, meet at the barrier, and agree
on the max over ranks of their timings; the whole-job rate is world x the
units of one rank over that max."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from cuda_pf_localization_b200 import multi
    dist = multi.init("gloo", timeout_s=30)
    try:
        assert multi.world_info() == (world, rank, rank)
        multi.sync_all(dist, None)
        m = multi.max_over_ranks([1.0 + rank, 10.0 - rank, 0.25 * rank], dist, None)
        out[rank] = m
    finally:
        multi.finish(dist)


def test_two_gloo_ranks_agree_on_max():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == [2.0, 10.0, 0.25]


def test_single_process_passthrough_and_rate():
    from cuda_pf_localization_b200 import multi
    assert multi.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]
    assert multi.weak_scaling_rate(4, 1e6 * 100, 2.0) == pytest.approx(2e8)
