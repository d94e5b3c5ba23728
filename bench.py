#!/usr/bin/env python
"""Benchmark: particle-filter cycle throughput at N = 1M particles on the
at-scale workload (64 landmarks in a 50 x 50 x 10 m box, 256 observations per
cycle of which 10 % are outliers, random_inject_ratio 0.01, helix trajectory),
plus the other workloads of the hot path: the tracking workload (10k
particles, 12 landmarks, 100 cycles), range-bearing observations at scale,
batched filters, and global localization (uniform CBGL and the learned
proposal at iso-success on the same maps and poses).

One step = one full ParticleFilter::update cycle (predict, gated weighting,
softmax, estimate, resample when ESS < N/2 with injection, estimate) over all
N particles.  Metric: particle-updates/s = N * steps / time.

  value  device-resident inputs (all cycles' observations in HBM), the fused
         cycle entry point, CUDA events on the library's stream around each
         step, L2 flushed (256 MiB write) between steps outside the events.
  e2e    the drop-in path: the C++ mirror of pf_core's ParticleFilter::update
         calling the pfc_* C-ABI with host observation arrays (host->device
         copy and device->host estimate read inside every timed step), wall
         clock per step with L2 flushed between steps.

--impl reference times the reference's CPU implementation of the same cycle
(the CPU oracle port of crates/pf_core/src/cpu.rs, all host threads) on the
same workload: --warmup untimed and --steps timed cycles, each over a bounded
sample of the particles so the run ends within minutes.

Multi-GPU: --gpus N outside torchrun launches N ranks (torch.distributed.run,
one process per GPU); every rank runs an independent filter of N particles
(replicas, weak scaling); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PF particle-updates/s @1M"
UNIT = "particle-updates/s"
L2_FLUSH_BYTES = 256 << 20
CPU_RUN_SECONDS = 90.0  # budget of the reference arm's timed cycles


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--batch-filters", type=int, default=512)
    ap.add_argument("--batch-cycles", type=int, default=200)
    ap.add_argument("--batch-seq-cycles", type=int, default=20)
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the batched-filter leg and print its JSON")
    ap.add_argument("--gl-only", action="store_true",
                    help="run only the global-localization legs and print their JSON")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the GL, batched, other-workload and CPU-baseline legs")
    ap.add_argument("--gl-hyps", type=int, default=1_000_000)
    ap.add_argument("--gl-trials", type=int, default=20)
    ap.add_argument("--gl-maps", type=int, default=16)
    ap.add_argument("--gl-queries", type=int, default=1000)
    ap.add_argument("--gl-pairs", type=int, default=2_000_000)
    ap.add_argument("--gl-train-steps", type=int, default=1200)
    ap.add_argument("--gl-batch", type=int, default=8192)
    ap.add_argument("--gl-lr", type=float, default=2e-3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    return ap.parse_args()


# ----------------------------------------------------------------- helpers

class ClockSampler:
    """nvidia-smi clock/throttle sampling during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_id_for(local_rank: int) -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


def peaks():
    """HBM copy bandwidth (GB/s) and where it comes from."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "hbm_gbs" in d:
            return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def scenario(args, cycles):
    from cuda_pf_localization_b200 import sim
    return sim.helix_scenario(cycles, 64, (50.0, 50.0, 10.0), 256, 0.10, args.seed)


def obs_array(rows):
    import cuda_pf_localization_b200 as pkg
    a = np.zeros(len(rows), dtype=[("id", "<i4"), ("mode", "<i4"), ("dx", "<f4"),
                                   ("dy", "<f4"), ("dz", "<f4"), ("range", "<f4")])
    a["id"] = rows[:, 0].astype(np.int32)
    a["mode"] = rows[:, 1].astype(np.int32)
    a["dx"], a["dy"], a["dz"], a["range"] = rows[:, 2], rows[:, 3], rows[:, 4], rows[:, 5]
    assert a.itemsize == C.sizeof(pkg.CObservation)
    return a


FILTER = dict(range_noise=0.05, bearing_noise=0.02, gate_sigma=3.0, resample_ess_ratio=0.5,
              random_inject_ratio=0.01)


def workload_config(args, world: int) -> dict:
    """The workload both arms measure (identical dict in both JSON lines)."""
    return {
        "workload": "at-scale PF cycle: N=1M f32 particles, 64 landmarks in 50x50x10 m, "
                    "256 obs/cycle (10% uniform outliers), gate 3 sigma, ESS<N/2 resample, "
                    "random_inject_ratio 0.01, helix trajectory",
        "particles": args.particles, "obs_per_cycle": 256,
        "parallelism": f"replicas x{world}",
        "l2": "flushed (256 MiB write) between timed GPU steps, outside the timed region",
    }


# ------------------------------------------------------- reference (CPU) arm

def run_cpu_cycles(sc, n, seconds, max_cycles, warm=1, filt=FILTER):
    """The CPU oracle's ParticleFilter::update (cpu.rs restated, OpenMP over the
    par_iter regions) for a bounded number of cycles; returns (cycles, s)."""
    import oracle
    pf = oracle.OraclePF(n, seed=42, range_noise=filt["range_noise"],
                         bearing_noise=filt["bearing_noise"], gate=filt["gate_sigma"],
                         ess_ratio=filt["resample_ess_ratio"],
                         inject=filt["random_inject_ratio"])
    pf.reinit(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
    tn, rn = sc.trans_noise, sc.rot_noise
    steps = sc.steps
    for k in range(warm):
        st = steps[k % len(steps)]
        pf.update(st.odom_t, st.odom_q, tn, rn, sc.landmarks, st.obs)
    done, t0 = 0, time.perf_counter()
    while done < max_cycles:
        st = steps[(warm + done) % len(steps)]
        pf.update(st.odom_t, st.odom_q, tn, rn, sc.landmarks, st.obs)
        done += 1
        if time.perf_counter() - t0 > seconds:
            break
    return done, time.perf_counter() - t0


def reference_sample(args, sc) -> int:
    """Particles per timed reference step: the workload's N, or fewer so that
    warmup + steps cycles fit CPU_RUN_SECONDS (the CPU cost of a cycle is
    linear in N; one probe cycle at 100k measures it)."""
    n = args.particles
    probe = min(n, 100_000)
    _, secs = run_cpu_cycles(sc, probe, 1e9, 1, warm=0)
    per_particle = secs / probe
    budget = CPU_RUN_SECONDS / max(1, args.steps + args.warmup)
    return int(max(10_000, min(n, budget / per_particle)))


def reference_arm(args, world):
    import oracle
    sc = scenario(args, max(8, min(args.steps + args.warmup, 200)))
    threads = oracle.lib().orc_threads()
    ns = reference_sample(args, sc)
    done, secs = run_cpu_cycles(sc, ns, 1e9, args.steps, warm=args.warmup)
    v = ns * done / secs
    sample = (f"{args.warmup} untimed + {done} timed cycles of the workload over {ns} "
              f"particles each (of N={args.particles}; the CPU cost is linear in N)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * secs / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ our GPU arm

FP32_OPS_PER_PAIR = 29  # gated Cartesian term with the reference's roundings
# DRAM bytes (read + write) of one k_weight launch at N = 1M, 256 observations,
# from ncu (dram__bytes_read.sum + dram__bytes_write.sum; the capture command
# is in profiles/pf_cycle_1M_scale.md): the poses are read from HBM, the
# predicted poses and log-likelihoods it writes stay in L2.
KWEIGHT_DRAM_BYTES_1M = 28.06e6
# Algorithmic bytes per particle of each kernel of a resampling cycle, by the
# library's kernel kinds: weight (fused predict + weighting: pose R 28 + W 28,
# ll W 4), est (weight pass: ll R 4, w W 4), scan (run starts: w R 4), gather
# (ancestors R 28, new cloud W 28), covs (pose R 28; uniform weights).
STAGE_BYTES = {"weight": 60, "est": 8, "scan": 4, "gather": 56, "covs": 28}
KINDS = ("reinit", "predict", "weight", "est", "covs", "scan", "gather", "inject",
         "commit", "misc")


def run_value(args, sc, torch, dev, dist=None, n=None, steps=None, warmup=None,
              filt=FILTER, profile=True):
    """Fused cycles with observations resident in HBM; per-step CUDA events."""
    import cuda_pf_localization_b200 as pkg
    lib = pkg.kernels()
    n = n or args.particles
    K = steps if steps is not None else args.steps
    W = warmup if warmup is not None else args.warmup
    nobs = len(sc.steps[0].obs)
    h = lib.pfc_create(max(256, nobs))
    assert h
    try:
        assert lib.pfc_init(h, n, 42) == 0
        lm = np.ascontiguousarray(sc.landmarks, np.float32).reshape(-1)
        assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), len(sc.landmarks)) == 0
        pri = np.r_[sc.prior_p, sc.prior_q].astype(np.float32)
        ps = np.full(3, 0.5, np.float32)
        rs = np.full(3, 0.2, np.float32)
        assert lib.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs)) == 0
        allobs = np.concatenate([obs_array(st.obs) for st in sc.steps])
        d_obs = torch.from_numpy(allobs.view(np.uint8).copy()).to(dev)
        base = d_obs.data_ptr()
        rec = 24 * nobs
        odoms = []
        for st in sc.steps:
            o = pkg.PfcOdom()
            o.t[:] = list(map(float, st.odom_t))
            o.q[:] = list(map(float, st.odom_q))
            o.tstd[:] = list(sc.trans_noise)
            o.rstd[:] = list(sc.rot_noise)
            odoms.append(o)
        prm = pkg.PfcCycleParams(filt["range_noise"], filt["bearing_noise"],
                                 filt["gate_sigma"], filt["resample_ess_ratio"],
                                 filt["random_inject_ratio"], 0)
        est = np.zeros(pkg.PFC_EST_LEN)
        stream = torch.cuda.ExternalStream(lib.pfc_stream(h), device=dev)
        flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
        for k in range(W):
            assert lib.pfc_cycle_device(h, C.byref(odoms[k]), C.c_void_p(base + k * rec), nobs,
                                        C.byref(prm), pkg.dptr(est)) == 0
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(K)]
        lib.pfc_reset_stats(h)
        from cuda_pf_localization_b200 import multi
        multi.sync_all(dist, dev)
        with ClockSampler(gpu_id_for(dev.index)) as clk:
            t_wall = time.perf_counter()
            with torch.cuda.stream(stream):
                for k in range(K):
                    flush.fill_(k & 0xFF)
                    evs[k][0].record(stream)
                    rc = lib.pfc_cycle_device(h, C.byref(odoms[W + k]),
                                              C.c_void_p(base + (W + k) * rec), nobs,
                                              C.byref(prm), None)
                    evs[k][1].record(stream)
                    if rc != 0:
                        raise RuntimeError(pkg.last_error())
            stream.synchronize()
            t_wall = time.perf_counter() - t_wall
            multi.sync_all(dist, dev)
        stats = pkg.PfcStats()
        lib.pfc_get_stats(h, C.byref(stats))
        step_ms = np.array([a.elapsed_time(b) for a, b in evs])
        assert lib.pfc_cycle_result(h, pkg.dptr(est)) == 0
        out = dict(step_ms=step_ms, wall=t_wall, launches=int(stats.launches),
                   clocks=clk.summary(), resampled_last=bool(est[pkg.PFC_EST_RESAMPLED]))
        if profile:
            # Per-kernel CUDA-event times: the timed cycles above are graph
            # replays (no per-kernel events), so the next cycles of the same
            # trajectory run with the library's per-kernel events (direct
            # launches).
            P = min(K, 100)
            lib.pfc_profile(h, 1)
            with torch.cuda.stream(stream):
                for k in range(P):
                    flush.fill_(k & 0xFF)
                    assert lib.pfc_cycle_device(h, C.byref(odoms[W + K + k]),
                                                C.c_void_p(base + (W + K + k) * rec), nobs,
                                                C.byref(prm), None) == 0
            stream.synchronize()
            ms = np.zeros(10)
            cnt = np.zeros(10, dtype=np.int64)
            lib.pfc_profile_read(h, pkg.dptr(ms), cnt.ctypes.data_as(C.POINTER(C.c_longlong)))
            lib.pfc_profile(h, 0)
            out.update(kernel_ms=ms, kernel_count=cnt, profiled_steps=P)
        return out
    finally:
        lib.pfc_destroy(h)


def run_e2e(args, sc, torch, dev, dist=None, n=None, steps=None, warmup=None, filt=FILTER,
            truth_offset=0):
    """ParticleFilter::update through the drop-in C-ABI with host buffers."""
    import cuda_pf_localization_b200 as pkg
    lib = pkg.kernels()
    n = n or args.particles
    K = steps if steps is not None else args.steps
    W = warmup if warmup is not None else args.warmup
    pf = pkg.ParticleFilter(n, seed=42, trans_noise=sc.trans_noise, rot_noise=sc.rot_noise,
                            **filt)
    try:
        pf.set_map(sc.landmark_dict())
        pf.reinitialize(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
        odoms = [pkg.make_core_odom(st.odom_t, st.odom_q, sc.trans_noise, sc.rot_noise)
                 for st in sc.steps]
        obs = [pkg.make_core_obs(st.obs) for st in sc.steps]
        nob = [len(st.obs) for st in sc.steps]
        core = pkg.core()
        est = pkg.PfcoreEstimate()
        for k in range(W):
            assert core.pfcore_filter_update(pf._h, C.byref(odoms[k]), obs[k], nob[k],
                                             C.byref(est)) == 0
        flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
        h = pf.handle
        lib.pfc_reset_stats(h)
        from cuda_pf_localization_b200 import multi
        multi.sync_all(dist, dev)
        times, errs, resampled = [], [], 0
        for k in range(K):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            rc = core.pfcore_filter_update(pf._h, C.byref(odoms[W + k]), obs[W + k], nob[W + k],
                                           C.byref(est))
            t1 = time.perf_counter()
            if rc != 0:
                raise RuntimeError(core.pfcore_last_error().decode())
            times.append(t1 - t0)
            errs.append(float(np.linalg.norm(np.array(est.position[:]) - sc.steps[W + k].truth_p)))
            resampled += int(est.resampled)
        multi.sync_all(dist, dev)
        stats = pkg.PfcStats()
        lib.pfc_get_stats(h, C.byref(stats))
        return dict(times=np.array(times), errs=np.array(errs), resampled=resampled,
                    h2d=stats.h2d_bytes / K, d2h=stats.d2h_bytes / K,
                    launches=int(stats.launches), syncs=stats.host_syncs / K)
    finally:
        pf.close()


def run_tracking(args, torch, dev):
    """The tracking workload (N=10k, 12 landmarks in 20x20x5 m, every landmark
    observed, 3-sigma gate, 100 cycles of the helix): the fused device path,
    the drop-in path with host arrays, and the CPU port, each over the 100
    cycles after a warm-up run of the same trajectory."""
    from cuda_pf_localization_b200 import sim
    sc = sim.tracking_config(cycles=200, seed=7)
    filt = dict(FILTER, random_inject_ratio=0.0)
    n, K, W = 10_000, 100, 100
    v = run_value(args, sc, torch, dev, n=n, steps=K, warmup=W, filt=filt, profile=False)
    e = run_e2e(args, sc, torch, dev, n=n, steps=K, warmup=W, filt=filt)
    done, secs = run_cpu_cycles(sc, n, args.cpu_seconds, K, warm=3, filt=filt)
    import oracle
    t_v = float(v["step_ms"].sum()) / 1e3
    return {"workload": "tracking: N=10k, 12 landmarks in 20x20x5 m, all observed, "
                        "gate 3 sigma, helix, 100 cycles",
            "value": n * K / t_v, "unit": UNIT, "ms_per_step": 1e3 * t_v / K,
            "e2e": {"value": n * K / float(e["times"].sum()),
                    "ms_per_step": 1e3 * float(e["times"].mean()),
                    "host_syncs_per_step": float(e["syncs"])},
            "cpu_baseline": {"value": n * done / secs, "unit": UNIT,
                             "cores": int(oracle.lib().orc_threads()), "kind": "port",
                             "sample": f"{done} cycles at N={n}"},
            "mean_track_err_m": float(e["errs"].mean())}


def run_range_bearing(args, sc, torch, dev):
    """The at-scale workload with every observation range-bearing (mode 1:
    range and unit direction, the gated acos bearing term)."""
    from cuda_pf_localization_b200 import sim
    rb = sim.as_range_bearing(sc)
    K = min(args.steps, 200)
    v = run_value(args, rb, torch, dev, steps=K, warmup=args.warmup, profile=True)
    t = float(v["step_ms"].sum()) / 1e3
    w_ms = v["kernel_ms"][KINDS.index("weight")] / max(1, v["kernel_count"][KINDS.index("weight")])
    return {"workload": "at-scale PF cycle with all 256 observations range-bearing",
            "value": args.particles * K / t, "unit": UNIT, "ms_per_step": 1e3 * t / K,
            "steps": K, "k_weight_ms": float(w_ms),
            "pairs_per_s": args.particles * 256 / (w_ms * 1e-3)}


# Tensor-core work of one training sample: forward (2 * sum in*out) + weight
# gradients (the same) + input gradients of layers 1..4.
LP_FLOPS_PER_SAMPLE = 2 * (2 * (384 * 1024 + 3 * 1024 * 1024 + 1024 * 384)
                           + 3 * 1024 * 1024 + 1024 * 384)


def _pose_err(top, truth):
    dp = math.hypot(top[0] - truth[0], top[1] - truth[1])
    dth = abs((top[2] - truth[2] + math.pi) % (2 * math.pi) - math.pi)
    return dp, dth


def _success(top, poses):
    top, poses = np.asarray(top, np.float64), np.asarray(poses, np.float64)
    dp = np.hypot(top[:, 0] - poses[:, 0], top[:, 1] - poses[:, 1])
    dth = np.abs((top[:, 2] - poses[:, 2] + np.pi) % (2 * np.pi) - np.pi)
    return (dp <= 0.5) & (dth <= 0.1)


# uniform hypothesis counts of the iso-success sweep (positions x 16 yaws), the
# learned configurations (samples per query, calibration quantile), the one
# quoted in the headline ratio
UNIFORM_SWEEP = (50_000, 56_000, 64_000, 100_000, 200_000)
LEARNED_SWEEP = ((100, 0.995), (250, 0.995), (250, 0.999), (1000, 0.995), (20_000, 0.98))
UNIFORM_1M_POSES = 20   # poses per map of the 1M-hypothesis uniform leg


def iso_headline(iso: dict, min_queries: int, bar: float = 0.95) -> None:
    """The C5 comparison at iso-success, one rule for both sides: the cheapest
    uniform hypothesis count whose success within 0.5 m / 0.1 rad reaches
    `bar` (in its faster mode, one query at a time or batched) and the
    fastest learned configuration that reaches it, both over at least
    min_queries queries.  Adds iso["comparator"], iso["learned_headline"] and
    iso["learned_vs_uniform_solves_ratio"] when both sides have one."""
    cands = sorted((u, d) for u, d in ((int(k2), d2) for k2, d2 in iso["uniform"].items())
                   if d["success_pos_yaw"] >= bar and d["queries"] >= min_queries)
    learned_ok = [d for d in iso["learned"].values()
                  if d["success_pos_yaw"] >= bar and d["queries"] >= min_queries]
    if not cands or not learned_ok:
        return
    head = max(learned_ok, key=lambda d: d["solves_per_s"])
    u, d = cands[0]
    best_uni = max(d["solves_per_s"],
                   iso.get("uniform_batched", {}).get(str(u), {}).get("solves_per_s", 0.0))
    iso["comparator"] = dict(hyps=u, success_pos_yaw=d["success_pos_yaw"],
                             solves_per_s=best_uni,
                             rule="cheapest uniform count of the sweep with success "
                                  "within 0.5 m / 0.1 rad >= 0.95 on the same poses; "
                                  "its faster mode")
    iso["learned_headline"] = dict(head, rule="fastest learned configuration of the "
                                              "sweep with success within 0.5 m / 0.1 rad "
                                              ">= 0.95 on the same poses")
    iso["learned_vs_uniform_solves_ratio"] = head["solves_per_s"] / best_uni


def run_gl(args):
    """CBGL on 10 x 10 m rooms with 30 boxes (200 x 200 at 0.05 m), 360-ray
    scans (rmax 10 m, N(0, 0.01 m) noise) rendered by the library's raycaster.

    c3:       uniform CBGL on one room, 20 trials at 50k / 200k / 1M
              hypotheses (positions x 16 yaws), k = 64: the fused pruned
              localizer and the reference's call pattern (pfgl_score +
              pfgl_topk).
    iso:      16 maps x 1000 unseen poses.  Uniform CBGL (pruned localizer,
              one query at a time) at every count of UNIFORM_SWEEP, and the
              same queries batched; the learned proposal (per map: 2M
              (scan, pose) pairs generated on the device, the MLP trained by
              the library's tcgen05 kernels, the fallback threshold calibrated
              on 1000 held-out poses) localizing the same poses in batches at
              each of LEARNED_SWEEP's sample counts with a 200k uniform
              fallback.  The headline ratio applies one rule to both sides:
              the fastest learned configuration of the sweep and the
              cheapest uniform count (in its faster mode) whose success
              within 0.5 m and 0.1 rad is at least 95 % on the same poses."""
    import cuda_pf_localization_b200 as pkg
    from cuda_pf_localization_b200 import sim
    lib = pkg.kernels()
    span, rmax, k = 2 * math.pi, 10.0, 64
    res = {"c3": {}, "iso": {}}
    out = np.zeros(3 * k, np.float32)

    def trials_for(g, rng, n, h):
        poses = np.array([sim.free_pose(g, rng) for _ in range(n)], np.float32)
        return poses, pkg.render_scans(h, poses, noise=0.01, seed=int(rng.integers(1 << 31)))

    # ---- config 3: uniform CBGL, the reference method, 20 trials per size
    g = np.ascontiguousarray(sim.rooms_grid(args.seed))
    h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), max(args.gl_hyps, 200_000))
    try:
        poses, scans = trials_for(g, np.random.default_rng(args.seed + 1), args.gl_trials, h)
        for nh in sorted({50_000, 200_000, args.gl_hyps}):
            for mode in ("pruned", "abi"):
                lib.pfgl_generate_yaws(h, nh // 16, 16, 1)
                lib.pfgl_localize(h, pkg.fptr(scans[0]), 360, rmax, span, k, pkg.fptr(out),
                                  None, None)  # warm-up
                ok_p = ok_pt = 0
                t0 = time.perf_counter()
                for t in range(len(poses)):
                    assert lib.pfgl_generate_yaws(h, nh // 16, 16, 1000 + t) == 0
                    if mode == "pruned":
                        r = lib.pfgl_localize(h, pkg.fptr(scans[t]), 360, rmax, span, k,
                                              pkg.fptr(out), None, None)
                    else:
                        assert lib.pfgl_score(h, pkg.fptr(scans[t]), 360, rmax, span) == 0
                        r = lib.pfgl_topk(h, k, pkg.fptr(out))
                    assert r == k
                    dp, dth = _pose_err(out[:3], poses[t])
                    ok_p += dp <= 0.5
                    ok_pt += dp <= 0.5 and dth <= 0.1
                dt = time.perf_counter() - t0
                # algorithmic work: DDA cell visits of exhaustive scoring of the
                # last trial's hypotheses (counted by an untimed replay kernel)
                visits = lib.pfgl_count_visits(h, 360, span)
                sps = len(poses) / dt
                res["c3"][f"{nh}_{mode}"] = dict(
                    solves_per_s=sps, success_pos=ok_p / len(poses),
                    success_pos_yaw=ok_pt / len(poses), trials=len(poses),
                    hyps_per_s=nh * sps, dda_visits_per_solve=int(visits),
                    dda_visits_per_s=visits * sps,
                    visits_note="exhaustive-scoring visits x solves/s" +
                                ("" if mode == "abi" else
                                 " (the pruned scorer visits fewer cells)"))
    finally:
        lib.pfgl_destroy(h)

    # ---- iso-success: learned vs uniform on the same maps and poses
    uni = {u: dict(ok=0, n=0, t=0.0) for u in UNIFORM_SWEEP + (args.gl_hyps,)}
    uni_b = {u: dict(ok=0, n=0, t=0.0) for u in UNIFORM_SWEEP[:3]}
    lrn = {c: dict(ok=0, n=0, t=0.0, fb=0, tau=[], held=[]) for c in LEARNED_SWEEP}
    t_train = t_steps = 0.0
    losses = []
    for m in range(args.gl_maps):
        gseed = 1000 + 17 * m
        g = np.ascontiguousarray(sim.rooms_grid(gseed))
        h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), max(args.gl_hyps, 200_000))
        lp = None
        try:
            lp = pkg.LearnedProposal(h, batch=args.gl_batch, seed=gseed)
            t0 = time.perf_counter()
            lp.make_data(args.gl_pairs, seed=gseed + 1)
            t1 = time.perf_counter()
            loss = lp.train(args.gl_train_steps, lr=args.gl_lr)
            t2 = time.perf_counter()
            t_train += t2 - t0
            t_steps += t2 - t1
            losses.append(float(loss[-50:].mean()))
            poses, scans = trials_for(g, np.random.default_rng(gseed + 3), args.gl_queries, h)
            for (S, ql), a in lrn.items():
                tau, held = lp.calibrate(n_queries=1000, n_samples=S, quantile=ql,
                                         seed=gseed + 2)
                a["tau"].append(tau)
                a["held"].append(held)
                lp.localize_batch(scans[:4], n_samples=S, n_fallback=200_000, k=k)  # warm-up
                t0 = time.perf_counter()
                top, _, _, info = lp.localize_batch(scans, n_samples=S, n_fallback=200_000, k=k)
                a["t"] += time.perf_counter() - t0
                a["ok"] += int(_success(top[:, 0], poses).sum())
                a["n"] += len(poses)
                a["fb"] += int((info > 0).sum())
            for u, a in uni.items():
                nq = len(poses) if u in UNIFORM_SWEEP else min(UNIFORM_1M_POSES, len(poses))
                lib.pfgl_generate_yaws(h, u // 16, 16, 1)
                lib.pfgl_localize(h, pkg.fptr(scans[0]), 360, rmax, span, k, pkg.fptr(out),
                                  None, None)  # warm-up
                tops = np.zeros((nq, 3), np.float32)
                t0 = time.perf_counter()
                for q in range(nq):
                    lib.pfgl_generate_yaws(h, u // 16, 16, 7000 + q)
                    lib.pfgl_localize(h, pkg.fptr(scans[q]), 360, rmax, span, k, pkg.fptr(out),
                                      None, None)
                    tops[q] = out[:3]
                a["t"] += time.perf_counter() - t0
                a["ok"] += int(_success(tops, poses[:nq]).sum())
                a["n"] += nq
            for u, a in uni_b.items():
                seeds = np.arange(7000, 7000 + len(poses), dtype=np.uint64)
                pkg.localize_batch(h, scans[:2], u // 16, 16, seeds[:2], k)  # warm-up
                t0 = time.perf_counter()
                bp, _, _ = pkg.localize_batch(h, scans, u // 16, 16, seeds, k)
                a["t"] += time.perf_counter() - t0
                a["ok"] += int(_success(bp[:, 0], poses).sum())
                a["n"] += len(poses)
        finally:
            if lp is not None:
                lp.close()
            lib.pfgl_destroy(h)
    if args.gl_maps <= 0:
        return res
    iso = res["iso"]
    iso["uniform"] = {str(u): dict(hyps=u, queries=a["n"], success_pos_yaw=a["ok"] / a["n"],
                                   solves_per_s=a["n"] / a["t"],
                                   mode="pruned localizer, one query at a time")
                      for u, a in uni.items() if a["n"]}
    iso["uniform_batched"] = {str(u): dict(hyps=u, queries=a["n"],
                                           success_pos_yaw=a["ok"] / a["n"],
                                           solves_per_s=a["n"] / a["t"],
                                           mode="pfgl_localize_batch (exhaustive)")
                              for u, a in uni_b.items() if a["n"]}
    iso["learned"] = {f"{S}_q{ql}": dict(samples_per_query=S, calibration_quantile=ql,
                                         queries=a["n"], success_pos_yaw=a["ok"] / a["n"],
                                         solves_per_s=a["n"] / a["t"],
                                         fallback_rate=a["fb"] / a["n"],
                                         fallback_hyps=200_000, tau_mean=float(np.mean(a["tau"])),
                                         held_out_success=float(np.mean(a["held"])),
                                         mode="pfgl_learned_localize_batch")
                      for (S, ql), a in lrn.items()}
    iso["training"] = dict(pairs_per_map=args.gl_pairs, steps_per_map=args.gl_train_steps,
                           batch=args.gl_batch, seconds_per_map=t_train / args.gl_maps,
                           step_ms=1e3 * t_steps / (args.gl_maps * args.gl_train_steps),
                           tflops=LP_FLOPS_PER_SAMPLE * args.gl_batch * args.gl_train_steps
                           * args.gl_maps / t_steps / 1e12,
                           final_loss_mean=float(np.mean(losses)))
    iso_headline(iso, args.gl_queries)
    return res


def run_batched(args, torch, dev):
    """Batched filters: sizes log-uniform in [1k, 200k], own landmarks, helix
    and 4-64 observations per cycle; every cycle of all filters is one graph
    launch with device-resident inputs (CUDA events per cycle on the batch
    stream), against the same filters run one after another through the
    single-filter fused cycle."""
    import cuda_pf_localization_b200 as pkg
    from cuda_pf_localization_b200 import sim
    lib = pkg.kernels()
    F, cycles = args.batch_filters, args.batch_cycles
    sizes, scen, counts = sim.batched_config(F, cycles + args.warmup, args.seed + 5)
    seeds = [1000 + f for f in range(F)]
    prm = dict(sigma_r=0.05, sigma_b=0.02, gate=3.0, ess_ratio=0.5, inject=0.0)

    def odom(sc, st):
        o = pkg.PfcOdom()
        o.t[:] = list(map(float, st.odom_t))
        o.q[:] = list(map(float, st.odom_q))
        o.tstd[:] = list(sc.trans_noise)
        o.rstd[:] = list(sc.rot_noise)
        return o

    total_cycles = cycles + args.warmup
    # device-resident inputs of every cycle
    rec = np.zeros((total_cycles, F), np.dtype((np.void, C.sizeof(pkg.PfcBatchCycle))))
    obs_blocks, n_obs = [], []
    for k in range(total_cycles):
        recs = (pkg.PfcBatchCycle * F)()
        off = 0
        rows = []
        for f in range(F):
            st = scen[f].steps[k]
            recs[f].odom = odom(scen[f], st)
            recs[f].obs_off = off
            recs[f].nobs = len(st.obs)
            off += len(st.obs)
            rows.append(st.obs)
        rec[k] = np.frombuffer(bytes(recs), dtype=rec.dtype)
        obs_blocks.append(pkg.cobs_records(np.concatenate(rows)))
        n_obs.append(off)
    max_obs = max(n_obs)
    obs_all = np.zeros((total_cycles, max_obs), pkg.COBS_DTYPE)
    for k in range(total_cycles):
        obs_all[k, :n_obs[k]] = obs_blocks[k]
    d_rec = torch.from_numpy(rec.view(np.uint8).reshape(total_cycles, -1).copy()).to(dev)
    d_obs = torch.from_numpy(obs_all.view(np.uint8).reshape(total_cycles, -1).copy()).to(dev)
    rec_bytes, obs_bytes = d_rec.shape[1], d_obs.shape[1]
    pose7 = np.array([np.r_[sc.prior_p, sc.prior_q] for sc in scen], np.float32)
    b = pkg.BatchPF(sizes, seeds=seeds, obs_cap=max_obs)
    try:
        b.set_params(**prm)
        b.set_landmarks([sc.landmarks for sc in scen])
        b.reinit(pose7, np.full((F, 3), 0.5), np.full((F, 3), 0.2))
        est = np.zeros((F, pkg.PFC_EST_LEN))
        for k in range(args.warmup):
            assert lib.pfc_batch_cycle_device(
                b.handle, C.c_void_p(d_rec.data_ptr() + k * rec_bytes),
                C.c_void_p(d_obs.data_ptr() + k * obs_bytes), n_obs[k], pkg.dptr(est)) == 0
        tiles, packed = b.autotune(reps=3)
        stream = torch.cuda.ExternalStream(lib.pfc_batch_stream(b.handle), device=dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(cycles)]
        l0 = lib.pfc_batch_launches(b.handle)
        torch.cuda.synchronize(dev)
        for i in range(cycles):
            k = args.warmup + i
            evs[i][0].record(stream)
            assert lib.pfc_batch_cycle_device(
                b.handle, C.c_void_p(d_rec.data_ptr() + k * rec_bytes),
                C.c_void_p(d_obs.data_ptr() + k * obs_bytes), n_obs[k], None) == 0
            evs[i][1].record(stream)
        assert lib.pfc_batch_result(b.handle, pkg.dptr(est)) == 0
        torch.cuda.synchronize(dev)
        launches = lib.pfc_batch_launches(b.handle) - l0
        ms = np.array([a.elapsed_time(c) for a, c in evs])
        resampled = int(est[:, pkg.PFC_EST_RESAMPLED].sum())
        errs = [float(np.linalg.norm(est[f, :3] - scen[f].steps[total_cycles - 1].truth_p))
                for f in range(F)]
    finally:
        b.close()
    # sequential single-filter cycles (the same filters, host inputs)
    seq_cycles = min(args.batch_seq_cycles, cycles)
    hs = []
    seq_ms = float("nan")
    try:
        if seq_cycles <= 0:
            raise StopIteration
        pc = pkg.PfcCycleParams(prm["sigma_r"], prm["sigma_b"], prm["gate"], prm["ess_ratio"],
                                prm["inject"], 0)
        for f in range(F):
            h = lib.pfc_create(64)
            hs.append(h)
            assert lib.pfc_init(h, int(sizes[f]), seeds[f]) == 0
            lm = np.ascontiguousarray(scen[f].landmarks, np.float32).reshape(-1)
            assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), len(scen[f].landmarks)) == 0
            pri = pose7[f]
            ps, rs = np.full(3, 0.5, np.float32), np.full(3, 0.2, np.float32)
            assert lib.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs)) == 0
        cobs = [[pkg.make_cobs(scen[f].steps[k].obs) for f in range(F)]
                for k in range(args.warmup + seq_cycles)]
        odoms = [[odom(scen[f], scen[f].steps[k]) for f in range(F)]
                 for k in range(args.warmup + seq_cycles)]
        e1 = np.zeros(pkg.PFC_EST_LEN)
        for k in range(args.warmup):
            for f in range(F):
                assert lib.pfc_cycle(hs[f], C.byref(odoms[k][f]), cobs[k][f],
                                     len(scen[f].steps[k].obs), C.byref(pc), pkg.dptr(e1)) == 0
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for i in range(seq_cycles):
            k = args.warmup + i
            for f in range(F):
                assert lib.pfc_cycle(hs[f], C.byref(odoms[k][f]), cobs[k][f],
                                     len(scen[f].steps[k].obs), C.byref(pc), pkg.dptr(e1)) == 0
        seq_ms = 1e3 * (time.perf_counter() - t0) / seq_cycles
    except StopIteration:
        pass
    finally:
        for h in hs:
            lib.pfc_destroy(h)
    total = int(sizes.sum())
    return dict(
        filters=F, particles_total=total, cycles=cycles, ms_per_cycle=float(ms.mean()),
        particle_updates_per_s=total * cycles / (ms.sum() * 1e-3),
        sequential_ms_per_cycle=seq_ms, sequential_cycles_timed=seq_cycles,
        speedup_vs_sequential=seq_ms / float(ms.mean()),
        kernels_per_cycle=launches / cycles, graph_launches_per_cycle=1,
        est_tiles_per_bucket=[int(t) for t in tiles],
        resampled_filters_last_cycle=resampled,
        mean_track_err_m=float(np.mean(errs)), n_min=int(sizes.min()), n_max=int(sizes.max()))


def rooflines(val, n, nobs, t_cycle_s, hbm, peak_kind):
    """The dominant kernel's roofline (k_weight: FP32 issue bound) and the
    cycle's per-stage roofline sum_s max(B_s / BW, I_s / issue) / t_cycle."""
    ms, cnt = val["kernel_ms"], val["kernel_count"]
    per = {k: (ms[i] / cnt[i] if cnt[i] else 0.0) for i, k in enumerate(KINDS)}
    sm_mhz = val["clocks"]["sm_mhz"] or 1965.0
    issue_peak = 148 * 128 * sm_mhz * 1e6  # FP32 lane operations / s
    w_ms = per["weight"]
    pair_rate = n * nobs / (w_ms * 1e-3)
    achieved_ops = FP32_OPS_PER_PAIR * pair_rate
    hbm_bytes = STAGE_BYTES["weight"] * n
    roof = {"bound": "fp32 issue", "kernel": "k_weight (fused predict + gated weighting)",
            "achieved": achieved_ops / 1e12, "peak": issue_peak / 1e12,
            "unit": "T FP32 lane-ops/s", "frac": achieved_ops / issue_peak,
            "traffic": (KWEIGHT_DRAM_BYTES_1M if (n, nobs) == (1_000_000, 256) else None),
            "traffic_source": "ncu capture of one k_weight launch at this workload "
                              "(dram__bytes_read.sum + dram__bytes_write.sum)",
            "ops_per_launch": FP32_OPS_PER_PAIR * n * nobs,
            "ops_note": f"{FP32_OPS_PER_PAIR} rounded FP32 operations per particle-observation "
                        "pair are required for the reference's bits (an FMA counts once); "
                        "peak = 148 SM x 128 lanes x sampled SM clock",
            "avg_launch_ms": w_ms, "sm_mhz": sm_mhz,
            "hbm": {"achieved": hbm_bytes / (w_ms * 1e-3) / 1e9, "peak": hbm,
                    "unit": "GB/s", "frac": hbm_bytes / (w_ms * 1e-3) / 1e9 / hbm,
                    "alg_bytes_per_launch": hbm_bytes, "peak_source": peak_kind},
            "timing": f"CUDA events around each k_weight launch on the library stream over "
                      f"the {val['profiled_steps']} cycles that continue the timed "
                      f"(graph-launched) cycles' trajectory (direct launches)"}
    stages = {}
    t_roof = 0.0
    for name, b in STAGE_BYTES.items():
        t_b = b * n / (hbm * 1e9)
        t_i = (FP32_OPS_PER_PAIR * n * nobs / issue_peak) if name == "weight" else 0.0
        t_s = max(t_b, t_i)
        t_roof += t_s
        stages[name] = {"alg_bytes_per_particle": b, "roof_us": 1e6 * t_s,
                        "measured_us": 1e3 * per[name],
                        "bound": "fp32 issue" if t_i > t_b else "hbm"}
    cycle = {"frac": t_roof / t_cycle_s, "roof_us": 1e6 * t_roof,
             "measured_cycle_us": 1e6 * t_cycle_s, "stages": stages,
             "rule": "sum over the cycle's kernels of max(alg bytes / measured HBM copy "
                     "bandwidth, FP32 ops / FP32 issue peak), divided by the measured "
                     "(graph-replayed) cycle time; a resampling cycle"}
    return roof, cycle


def main():
    args = parse()
    from cuda_pf_localization_b200 import multi
    try:
        plan, world = multi.launch_plan(args.gpus)
    except ValueError as e:
        sys.exit(f"bench.py: {e}")
    if plan == "spawn":
        sys.exit(multi.spawn_ranks(str(Path(__file__).resolve()), sys.argv[1:], world))
    _, rank, local = multi.world_info()
    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, world)
        return

    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.gl_only:
        if rank == 0:
            print(json.dumps({"gl": run_gl(args)}), flush=True)
        return
    if args.batch_only:
        if rank == 0:
            print(json.dumps({"batched": run_batched(args, torch, dev)}), flush=True)
        return
    dist = multi.init("nccl") if world > 1 else None

    # the profiled pass after the timed cycles continues the same trajectory
    sc = scenario(args, args.warmup + args.steps + min(args.steps, 100) + 1)
    n = args.particles
    val = run_value(args, sc, torch, dev, dist)
    e2e = run_e2e(args, sc, torch, dev, dist)
    t_value, t_e2e = multi.max_over_ranks(
        [float(val["step_ms"].sum()) / 1e3, float(e2e["times"].sum())], dist, dev)

    K = args.steps
    value = multi.weak_scaling_rate(world, n * K, t_value)
    e2e_value = multi.weak_scaling_rate(world, n * K, t_e2e)
    nobs = 256
    hbm, peak_kind = peaks()
    roof, cycle_roof = rooflines(val, n, nobs, t_value / K, hbm, peak_kind)
    kernel_share = {name: float(val["kernel_ms"][i]) for i, name in enumerate(KINDS)}
    tot_k = sum(kernel_share.values())

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_value / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, world),
        "launch": "each cycle replayed from a CUDA graph (pfc_cycle_device)",
        "accuracy": {"mean_track_err_m": float(e2e["errs"].mean()),
                     "resamples_in_e2e": int(e2e["resampled"])},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": float(e2e["h2d"]),
                "d2h_bytes_per_step": float(e2e["d2h"]),
                "ms_per_step": 1e3 * t_e2e / K, "host_syncs_per_step": float(e2e["syncs"]),
                "path": "pf_core ParticleFilter::update mirror -> pfc_* C-ABI"},
        "gpu_launches": val["launches"],
        "roofline": roof,
        "cycle_roofline": cycle_roof,
        "kernel_ms_share": {k2: v / tot_k for k2, v in kernel_share.items() if tot_k > 0},
        "clocks": val["clocks"],
    }

    if rank == 0 and world == 1 and not args.no_extras:
        import oracle
        sc_cpu = scenario(args, 8)
        done, secs = run_cpu_cycles(sc_cpu, n, args.cpu_seconds, 50)
        line["cpu_baseline"] = {"value": n * done / secs, "unit": UNIT,
                                "cores": int(oracle.lib().orc_threads()), "kind": "port",
                                "sample": f"{done} cycles at N={n} (time-bounded)"}
        # the same workload at the other particle counts of the at-scale config,
        # the tracking workload, and range-bearing observations at scale
        sizes = {}
        for n_other in (100_000, 4_000_000):
            a2 = argparse.Namespace(**vars(args))
            a2.particles, a2.steps = n_other, min(args.steps, 200)
            v2 = run_value(a2, sc, torch, dev, profile=False)
            t2 = float(v2["step_ms"].sum()) / 1e3
            sizes[str(n_other)] = {"value": n_other * a2.steps / t2, "unit": UNIT,
                                   "ms_per_step": 1e3 * t2 / a2.steps, "steps": a2.steps}
        sizes["10000_tracking"] = run_tracking(args, torch, dev)
        sizes["1000000_range_bearing"] = run_range_bearing(args, sc, torch, dev)
        line["other_sizes"] = sizes
        line["batched"] = run_batched(args, torch, dev)
        line["batched"]["config"] = ("512 filters, N log-uniform in [1k, 200k], 8-64 landmarks "
                                     "in 20x20x5 m each, own helix, 4-64 obs per cycle, "
                                     "gate 3 sigma, ESS<N/2 resample; one graph launch per "
                                     "cycle vs the same filters through pfc_cycle one after "
                                     "another")
        line["gl"] = run_gl(args)
        line["gl"]["config"] = ("10x10 m rooms at 0.05 m (200x200), 30 boxes 0.2-1.0 m, 360 rays, "
                                "rmax 10, scan noise N(0, 0.01 m); c3: positions x 16 yaws, k=64, "
                                f"{args.gl_trials} trials per size on one room; iso: "
                                f"{args.gl_maps} maps x {args.gl_queries} unseen poses, success "
                                "within 0.5 m and 0.1 rad, learned and uniform on the same poses")
    if rank == 0:
        print(json.dumps(line), flush=True)
    multi.finish(dist)


if __name__ == "__main__":
    main()
