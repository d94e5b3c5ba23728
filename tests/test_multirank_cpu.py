"""The multi-rank plumbing (cuda_pf_localization_b200/multi.py) on CPU: two
gloo ranks rendezvous at 127.0.0.1, meet at the barrier, and agree on the max
over ranks of their timings (the whole-job rate is world x the units of one
rank over that max); a benchmark asked for N GPUs outside torchrun spawns N
ranks; the bottom-k of a global-localization query sharded by hypotheses,
merged with one all-gather, equals the bottom-k of the whole set; and the
sharded filter's exchange gives every rank every rank's slice."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


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


def test_launch_plan():
    from cuda_pf_localization_b200 import multi
    assert multi.launch_plan(1, {}) == ("run", 1)
    assert multi.launch_plan(4, {}) == ("spawn", 4)
    assert multi.launch_plan(2, {"WORLD_SIZE": "2"}) == ("run", 2)
    assert multi.launch_plan(1, {"WORLD_SIZE": "1"}) == ("run", 1)
    with pytest.raises(ValueError):
        multi.launch_plan(8, {"WORLD_SIZE": "2"})
    with pytest.raises(ValueError):
        multi.launch_plan(0, {})
    cmd = multi.spawn_command("bench.py", ["--gpus", "2"], 2, 29555)
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=2" in cmd and "--master-addr=127.0.0.1" in cmd
    assert cmd[-3:] == ["bench.py", "--gpus", "2"]


_RANK_SCRIPT = """
import os, sys
sys.path.insert(0, {root!r})
from cuda_pf_localization_b200 import multi
dist = multi.init("gloo", timeout_s=30)
m = multi.max_over_ranks([float(os.environ["RANK"])], dist, None)
sys.stdout.write("rank %s of %s max %s\\n" % (os.environ["RANK"], os.environ["WORLD_SIZE"], m[0]))
sys.stdout.flush()
multi.finish(dist)
"""  # one write per line: the ranks' output is unbuffered and shares one pipe


def test_spawn_ranks_runs_one_process_per_rank(tmp_path):
    from cuda_pf_localization_b200 import multi
    script = tmp_path / "ranks.py"
    script.write_text(_RANK_SCRIPT.format(root=str(ROOT)))
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    out = subprocess.run(multi.spawn_command(str(script), [], 2, _free_port()), env=env,
                         capture_output=True, text=True, timeout=180)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = sorted(l for l in out.stdout.splitlines() if l.startswith("rank "))
    assert lines == ["rank 0 of 2 max 1.0", "rank 1 of 2 max 1.0"]


def _scores(n_pos, n_yaw, seed):
    """Stand-in CAERs of a global hypothesis set (ties and infinities
    included), indexed like the library's dispersion: pos * n_yaw + yaw."""
    rng = np.random.default_rng(seed)
    c = rng.integers(0, 50, size=n_pos * n_yaw).astype(np.float32) * 0.5
    c[rng.integers(0, len(c), size=5)] = np.inf
    return c


def _merge_worker(rank, world, port, n_pos, n_yaw, k, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from cuda_pf_localization_b200 import multi
    dist = multi.init("gloo", timeout_s=30)
    try:
        c = _scores(n_pos, n_yaw, 3)
        p0, p1 = multi.shard_range(n_pos, world, rank)
        gidx = np.arange(p0 * n_yaw, p1 * n_yaw)
        keys = multi.composite_keys(c[gidx], gidx)
        poses = np.stack([gidx, gidx + 0.5, -gidx], 1).astype(np.float32)
        kk, pp = multi.merge_bottom_k(keys, poses, k, dist)
        out[rank] = (kk.tolist(), pp.tolist())
    finally:
        multi.finish(dist)


@pytest.mark.parametrize("n_pos,k", [(1000, 64), (3, 64), (1, 8)])
def test_sharded_bottom_k_equals_whole_set(n_pos, k):
    from cuda_pf_localization_b200 import multi
    world, n_yaw = 2, 16
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_merge_worker, args=(r, world, port, n_pos, n_yaw, k, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    c = _scores(n_pos, n_yaw, 3)
    order = np.argsort(c, kind="stable")[:k]       # stable: ties to the lower index
    for rank in range(world):
        kk, pp = np.array(res[rank][0], np.uint64), np.array(res[rank][1], np.float32)
        np.testing.assert_array_equal((kk & np.uint64(0xFFFFFFFF)).astype(np.int64), order)
        np.testing.assert_array_equal(multi.key_caer(kk), c[order])
        np.testing.assert_array_equal(pp[:, 0], order.astype(np.float32))


def test_emulated_shards_merge_in_one_process():
    from cuda_pf_localization_b200 import multi
    n_pos, n_yaw, k = 777, 16, 64
    c = _scores(n_pos, n_yaw, 9)
    keys, poses = [], []
    for rank in range(5):
        p0, p1 = multi.shard_range(n_pos, 5, rank)
        gidx = np.arange(p0 * n_yaw, p1 * n_yaw)
        part = np.argsort(c[gidx], kind="stable")[:k]
        keys.append(multi.composite_keys(c[gidx][part], gidx[part]))
        poses.append(np.zeros((len(part), 3), np.float32))
    kk, _ = multi.merge_bottom_k(np.concatenate(keys), np.concatenate(poses), k, None)
    np.testing.assert_array_equal((kk & np.uint64(0xFFFFFFFF)).astype(np.int64),
                                  np.argsort(c, kind="stable")[:k])


def _chunks(world, c, rank, seed):
    """Rank `rank`'s view list for the shard exchange: two arrays of world
    chunks, its own chunk filled with values that name the rank, the others
    with a fill the exchange must overwrite."""
    import torch
    g = torch.Generator().manual_seed(seed + rank)
    a = torch.full((world * c,), -1.0)
    b = torch.full((world * (c // 4),), -2.0)
    a[rank * c:(rank + 1) * c] = rank + torch.rand(c, generator=g)
    b[rank * (c // 4):(rank + 1) * (c // 4)] = 100 * rank + torch.rand(c // 4, generator=g)
    return [(a, c), (b, c // 4)]


def _exchange_worker(rank, world, port, c, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from cuda_pf_localization_b200 import multi
    dist = multi.init("gloo", timeout_s=30)
    try:
        views = _chunks(world, c, rank, 5)
        multi.exchange_views(views, rank, dist)
        out[rank] = [v.tolist() for v, _ in views]
    finally:
        multi.finish(dist)


def test_shard_exchange_over_gloo_ranks():
    """The sharded filter's all-gather (exchange_views): every rank ends with
    every rank's chunk of every array, in rank order."""
    world, c = 2, 64
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, c, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    want = [_chunks(world, c, r, 5) for r in range(world)]
    for rank in range(world):
        for a in range(2):
            got = np.array(res[rank][a], np.float32)
            cc = want[0][a][1]
            for r in range(world):
                np.testing.assert_array_equal(got[r * cc:(r + 1) * cc],
                                              want[r][a][0][r * cc:(r + 1) * cc].numpy())


def test_shard_exchange_in_process():
    """The one-process form used by the single-GPU tests (three shards)."""
    from cuda_pf_localization_b200 import multi
    world, c = 3, 32
    views = [_chunks(world, c, r, 11) for r in range(world)]
    own = [[v[r * cc:(r + 1) * cc].clone() for v, cc in views[r]] for r in range(world)]
    multi.exchange_in_process(views)
    for q in range(world):
        for a, (v, cc) in enumerate(views[q]):
            for r in range(world):
                assert (v[r * cc:(r + 1) * cc] == own[r][a]).all()
