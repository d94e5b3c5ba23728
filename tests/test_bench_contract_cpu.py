"""bench.py's reference arm runs on the host cores (the oracle's restatement of
the reference CPU path) and prints the one JSON line the benchmark contract
asks for: the metric, unit and direction of the GPU arm, `impl: reference`,
a `cpu_baseline` describing the run and an `e2e` with no host<->device bytes.
Run here at 20k particles so it takes about a second.  Also the rule that
picks the C5 iso-success comparison from the global-localization sweeps."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "3",
                        "--warmup", "3", "--particles", "20000"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "PF particle-updates/s @1M"
    assert d["unit"] == "particle-updates/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def _ref_run(extra_env, *args):
    env = dict(os.environ, **extra_env)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2",
                           "--warmup", "1", "--particles", "20000", *args],
                          cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)


def test_reference_arm_config_is_the_gpu_arms():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    r = _ref_run({})
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    ns = argparse.Namespace(particles=20000)
    assert d["config"] == bench.workload_config(ns, 1)
    assert d["steps"] == 2 and d["warmup"] == 1


def test_reference_arm_ranks_of_a_two_rank_world():
    base = {"WORLD_SIZE": "2", "LOCAL_RANK": "0", "MASTER_ADDR": "127.0.0.1",
            "MASTER_PORT": "29500"}
    r0 = _ref_run(dict(base, RANK="0"), "--gpus", "2")
    assert r0.returncode == 0, r0.stderr[-2000:]
    lines = [l for l in r0.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and json.loads(lines[0])["n_gpus"] == 2
    r1 = _ref_run(dict(base, RANK="1", LOCAL_RANK="1"), "--gpus", "2")
    assert r1.returncode == 0 and not r1.stdout.strip()
    # a torchrun world of another size is refused
    bad = _ref_run(dict(base, RANK="0"), "--gpus", "4")
    assert bad.returncode != 0


def test_iso_success_rule_is_the_same_for_both_sides():
    """C5's headline: the cheapest uniform count and the fastest learned
    configuration that reach 95 % on at least the required queries; slower
    or failing configurations and short sweeps are not chosen."""
    sys.path.insert(0, ROOT)
    import bench

    def u(succ, rate, q=1000):
        return {"success_pos_yaw": succ, "solves_per_s": rate, "queries": q}
    iso = {"uniform": {"50000": u(0.94, 1300.0), "56000": u(0.956, 1200.0),
                       "64000": u(0.97, 1100.0), "1000000": u(1.0, 120.0, q=20)},
           "uniform_batched": {"56000": u(0.956, 1250.0)},
           "learned": {"100_q0.995": u(0.93, 90000.0), "250_q0.995": u(0.99, 40000.0),
                       "250_q0.999": u(0.97, 60000.0), "20000_q0.98": u(1.0, 3000.0)}}
    bench.iso_headline(iso, 1000)
    assert iso["comparator"]["hyps"] == 56000
    assert iso["comparator"]["solves_per_s"] == 1250.0      # its faster mode
    assert iso["learned_headline"]["solves_per_s"] == 60000.0  # 100 samples fail the bar
    assert iso["learned_vs_uniform_solves_ratio"] == 60000.0 / 1250.0
    none = {"uniform": {"50000": u(0.9, 1.0)}, "learned": {"x": u(0.99, 2.0)}}
    bench.iso_headline(none, 1000)
    assert "learned_vs_uniform_solves_ratio" not in none
