"""Host-side plumbing for one process per GPU (torch.distributed).

Three multi-GPU modes live here:
  * replicas: N GPUs run N independent filters (weak scaling); the
    cross-rank steps are the barrier around a timed region and the max over
    ranks of the measured times;
  * a sharded filter: one filter over N ranks (ShardedFilter).  Every rank
    predicts and weights its slice of the particles, an all-gather of the
    slices (poses, log-likelihoods, softmax block partials) gives every rank
    the whole weighted cloud, and every rank finishes the cycle on it, so
    the result equals the one-GPU filter's bit for bit;
  * a sharded global-localization query: every rank scores a contiguous
    slice of one global hypothesis set, keeps its k best (CAER, global
    index) keys, and one all-gather of k keys and poses per rank gives the
    global bottom-k (sharded_localize).
This module keeps those steps in one place so that the CPU tests can
exercise them with the gloo backend.
"""
from __future__ import annotations

import datetime
import os
import socket
import subprocess
import sys

import numpy as np


def world_info() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    """Initialise the default process group from the environment (rendezvous
    at MASTER_ADDR / MASTER_PORT); returns torch.distributed, or None for a
    single process."""
    world, _, _ = world_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def sync_all(dist, device=None):
    """Barrier across ranks with the local device drained on both sides."""
    import torch
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(values, dist, device=None):
    """Element-wise max of a list of floats over all ranks."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    dev = device if (device is not None and device.type == "cuda") else torch.device("cpu")
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def weak_scaling_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank in at most
    `seconds` (the max over ranks)."""
    return world * units_per_rank / seconds


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ rank launch

def launch_plan(gpus: int, env=None) -> tuple[str, int]:
    """What a benchmark process asked for ``gpus`` GPUs should do:
    ("run", world) when it is already one rank of a torchrun world of that
    size (or a single process for gpus == 1), ("spawn", gpus) when gpus > 1
    and no torchrun environment is present.  A torchrun world of another size
    is an error."""
    env = os.environ if env is None else env
    if gpus < 1:
        raise ValueError(f"--gpus must be >= 1, got {gpus}")
    ws = env.get("WORLD_SIZE")
    if ws is None:
        return ("spawn", gpus) if gpus > 1 else ("run", 1)
    if int(ws) != gpus:
        raise ValueError(f"WORLD_SIZE={ws} but --gpus {gpus}")
    return ("run", int(ws))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn_command(script: str, argv: list[str], gpus: int, port: int) -> list[str]:
    """torchrun command that runs ``script argv`` as ``gpus`` local ranks with
    the rendezvous on 127.0.0.1."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1",
            f"--master-port={port}", script, *argv]


def spawn_ranks(script: str, argv: list[str], gpus: int) -> int:
    """Run ``script`` as ``gpus`` ranks (one process per GPU); returns the
    launcher's exit code."""
    return subprocess.call(spawn_command(script, argv, gpus, free_port()))


# ------------------------------------------------- sharded global localization

def shard_range(n_units: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [a, b) of n_units for this rank (sizes differ by at
    most one)."""
    q, r = divmod(int(n_units), int(world))
    a = rank * q + min(rank, r)
    return a, a + q + (1 if rank < r else 0)


def ordered_u32(caer: np.ndarray) -> np.ndarray:
    """Unsigned image of a float whose integer order is the float order (the
    reference's float_as_ordered, src/cuda/pf_kernels.cu:151-155, with the
    sign bit flipped), as the library's composite keys carry it."""
    i = np.ascontiguousarray(caer, np.float32).view(np.int32)
    o = np.where(i >= 0, i, i ^ np.int32(0x7FFFFFFF)).astype(np.int32)
    return o.view(np.uint32) ^ np.uint32(0x80000000)


def composite_keys(caer: np.ndarray, global_idx: np.ndarray) -> np.ndarray:
    """(ordered CAER << 32) | global hypothesis index: ascending order is a
    stable sort by CAER, ties to the lower index."""
    return (ordered_u32(caer).astype(np.uint64) << np.uint64(32)) | \
        np.asarray(global_idx, np.uint64)


_NO_KEY = np.uint64(0xFFFFFFFFFFFFFFFF)


def merge_bottom_k(keys: np.ndarray, poses: np.ndarray, k: int, dist, device=None):
    """Global bottom-k from every rank's local candidates: the k smallest local
    keys of each rank go through one all-gather of k (key, pose) slots per
    rank (empty slots carry the all-ones key), then the k smallest keys of
    the union are kept.  Keys are unique (they hold the global index), so the
    result is the bottom-k of the union exactly.  With dist None the local
    candidates are the union (one rank, or ranks emulated in one process).
    Returns (keys, poses) ascending."""
    keys = np.asarray(keys, np.uint64)
    poses = np.asarray(poses, np.float32).reshape(-1, 3)
    first = np.argsort(keys, kind="stable")[:k]
    kk = np.full(k, _NO_KEY, np.uint64)
    pp = np.zeros((k, 3), np.float32)
    kk[:len(first)] = keys[first]
    pp[:len(first)] = poses[first]
    if dist is not None:
        import torch
        dev = device if device is not None else torch.device("cpu")
        world = dist.get_world_size()
        tk = torch.from_numpy(kk.view(np.int64).copy()).to(dev)
        tp = torch.from_numpy(pp.copy()).to(dev)
        gk = [torch.empty_like(tk) for _ in range(world)]
        gp = [torch.empty_like(tp) for _ in range(world)]
        dist.all_gather(gk, tk)
        dist.all_gather(gp, tp)
        kk = np.concatenate([g.cpu().numpy() for g in gk]).view(np.uint64)
        pp = np.concatenate([g.cpu().numpy() for g in gp])
    order = np.argsort(kk, kind="stable")[:k]
    order = order[kk[order] != _NO_KEY]
    return kk[order], pp[order]


def key_caer(keys: np.ndarray) -> np.ndarray:
    """CAER of composite keys (inverse of ordered_u32)."""
    hi = (np.asarray(keys, np.uint64) >> np.uint64(32)).astype(np.uint32) ^ \
        np.uint32(0x80000000)
    o = hi.view(np.int32)
    return np.where(o >= 0, o, o ^ np.int32(0x7FFFFFFF)).astype(np.int32).view(np.float32)


def local_bottom_k(gl_handle, scan: np.ndarray, n_pos: int, n_yaw: int, seed: int,
                   k: int, world: int, rank: int, rmax: float = 10.0,
                   span: float = 2 * np.pi):
    """This rank's part of a sharded CBGL query: positions shard_range(n_pos,
    world, rank) of the dispersion pfgl_generate_yaws(n_pos, n_yaw, seed),
    scored by the pruned localizer of this rank's GPU; returns its k best
    (composite keys with global indices, poses)."""
    from . import fptr, iptr, kernels, last_error
    lib = kernels()
    p0, p1 = shard_range(n_pos, world, rank)
    if p1 <= p0:
        return np.zeros(0, np.uint64), np.zeros((0, 3), np.float32)
    if lib.pfgl_generate_yaws_range(gl_handle, p0, p1 - p0, n_yaw, seed) != 0:
        raise RuntimeError("pfgl_generate_yaws_range failed: " + last_error())
    kl = min(k, (p1 - p0) * n_yaw)
    out = np.zeros(3 * kl, np.float32)
    cs = np.zeros(kl, np.float32)
    ids = np.zeros(kl, np.int32)
    scan = np.ascontiguousarray(scan, np.float32)
    r = lib.pfgl_localize(gl_handle, fptr(scan), len(scan), rmax, span, kl, fptr(out),
                          fptr(cs), iptr(ids))
    if r < 0:
        raise RuntimeError("pfgl_localize failed: " + last_error())
    keys = composite_keys(cs[:r], ids[:r].astype(np.int64) + p0 * n_yaw)
    return keys, out[:3 * r].reshape(r, 3)


def sharded_localize(gl_handle, scan: np.ndarray, n_pos: int, n_yaw: int, seed: int,
                     k: int, dist, device=None, rmax: float = 10.0,
                     span: float = 2 * np.pi):
    """One CBGL query over n_pos positions x n_yaw yaws, its positions split
    across the ranks of ``dist`` (None: one rank): local_bottom_k on every
    rank, then merge_bottom_k.  Returns (keys, poses, caer, global indices)
    of the global bottom-k, ascending: identical to localizing the whole set
    on one GPU."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    keys, poses = local_bottom_k(gl_handle, scan, n_pos, n_yaw, seed, k, world, rank,
                                 rmax, span)
    kk, pp = merge_bottom_k(keys, poses, k, dist, device)
    return kk, pp, key_caer(kk), (kk & np.uint64(0xFFFFFFFF)).astype(np.int64)


# ------------------------------------------------------------ sharded filter

class DeviceArray:
    """A 1-D view of library-owned device memory that torch can wrap without
    a copy (``torch.as_tensor(DeviceArray(...), device=...)``, through the
    CUDA array interface).  The memory belongs to the library handle, which
    must outlive the tensor."""

    def __init__(self, ptr: int, length: int, typestr: str = "<f4"):
        self.__cuda_array_interface__ = {
            "shape": (int(length),), "typestr": typestr, "data": (int(ptr), False),
            "strides": None, "version": 3}


def exchange_views(views, rank: int, dist) -> None:
    """All-gather of one rank's chunks: views is a list of (tensor of
    world * c elements, c); every rank contributes elements
    [rank * c, (rank + 1) * c) of each tensor and receives the others' in
    place.  NCCL gathers straight into the tensor; other backends (gloo on
    CPU tensors) gather into its chunk views."""
    for full, c in views:
        mine = full[rank * c:(rank + 1) * c].clone()
        if dist.get_backend() == "nccl":
            dist.all_gather_into_tensor(full, mine)
        else:
            dist.all_gather(list(full.split(c)), mine)


def exchange_in_process(shard_views) -> None:
    """The same exchange between the shards of one process (one GPU, or CPU
    tensors): shard_views[r] is rank r's view list; chunk r of every tensor
    is copied from rank r to every other rank."""
    world = len(shard_views)
    for a in range(len(shard_views[0])):
        for r in range(world):
            full, c = shard_views[r][a]
            src = full[r * c:(r + 1) * c]
            for q in range(world):
                if q != r:
                    shard_views[q][a][0][r * c:(r + 1) * c].copy_(src)


class ShardedFilter:
    """One rank's handle of a particle filter sharded over ``world`` ranks
    (pfc_shard_*): it holds the whole cloud, predicts and weights particles
    [rank * chunk, min((rank + 1) * chunk, n)), and finishes every cycle on
    the whole cloud after the exchange.  Give every rank the same n, seed,
    landmarks, prior and cycle inputs."""

    def __init__(self, n: int, world: int, rank: int, seed: int = 42, cap_obs: int = 256,
                 device=None):
        import ctypes as C

        import torch

        from . import kernels, last_error
        self.lib = kernels()
        self.h = self.lib.pfc_create(cap_obs)
        if not self.h:
            raise RuntimeError("pfc_create failed: " + last_error())
        if self.lib.pfc_shard_init(self.h, n, world, rank, seed) != 0:
            err = last_error()
            self.lib.pfc_destroy(self.h)
            self.h = None
            raise RuntimeError("pfc_shard_init failed: " + err)
        chunk, n_pad = C.c_int(), C.c_int()
        self.lib.pfc_shard_layout(self.h, C.byref(chunk), C.byref(n_pad))
        self.n, self.world, self.rank = n, world, rank
        self.chunk = chunk.value
        self.device = device if device is not None else torch.device(
            "cuda", torch.cuda.current_device())

    def weigh(self, odom, obs_rows, prm) -> None:
        """Predict and weight this rank's slice (asynchronous)."""
        import ctypes as C

        from . import last_error, make_cobs
        arr = make_cobs(obs_rows) if len(obs_rows) else None
        ptr = C.cast(arr, C.c_void_p) if arr is not None else None
        if self.lib.pfc_shard_weight(self.h, C.byref(odom), ptr, len(obs_rows),
                                     C.byref(prm)) != 0:
            raise RuntimeError("pfc_shard_weight failed: " + last_error())

    def views(self):
        """(tensor, chunk) for the seven live planes, the log-likelihoods and
        the f32 softmax block partials (two floats per 256 particles), each
        covering world chunks; after the slice's kernels completed."""
        import ctypes as C

        import torch

        from . import last_error
        p7 = (C.c_void_p * 7)()
        ll, part = C.c_void_p(), C.c_void_p()
        if self.lib.pfc_shard_views(self.h, p7, C.byref(ll), C.byref(part)) != 0:
            raise RuntimeError("pfc_shard_views failed: " + last_error())
        full, c = self.world * self.chunk, self.chunk
        out = [(torch.as_tensor(DeviceArray(p7[k], full), device=self.device), c)
               for k in range(7)]
        out.append((torch.as_tensor(DeviceArray(ll.value, full), device=self.device), c))
        out.append((torch.as_tensor(DeviceArray(part.value, full // 128), device=self.device),
                    c // 128))
        return out

    def finish(self, prm) -> np.ndarray:
        """The rest of the cycle on the whole cloud; the 24-value record of
        pfc_cycle."""
        import ctypes as C

        from . import PFC_EST_LEN, dptr, last_error
        est = np.zeros(PFC_EST_LEN)
        if self.lib.pfc_shard_finish(self.h, C.byref(prm), dptr(est)) != 0:
            raise RuntimeError("pfc_shard_finish failed: " + last_error())
        return est

    def update(self, odom, obs_rows, prm, dist) -> np.ndarray:
        """One cycle with the exchange over ``dist`` (every rank calls it)."""
        import torch
        self.weigh(odom, obs_rows, prm)
        views = self.views()
        if dist is not None and self.world > 1:
            exchange_views(views, self.rank, dist)
            torch.cuda.synchronize(self.device)
        return self.finish(prm)

    def close(self) -> None:
        if self.h:
            self.lib.pfc_destroy(self.h)
            self.h = None


def update_in_process(shards, odom, obs_rows, prm):
    """One cycle of the shards of one filter held by one process (tests on
    one GPU): every slice weighted, the in-process exchange, every shard
    finished.  Returns each shard's record."""
    import torch
    for s in shards:
        s.weigh(odom, obs_rows, prm)
    exchange_in_process([s.views() for s in shards])
    torch.cuda.synchronize(shards[0].device)
    return [s.finish(prm) for s in shards]
