"""Build the test-only checkers under oracle/ (TEST INFRASTRUCTURE ONLY).

    python oracle/build.py                       # liboracle.so
    PF_REFERENCE=<reference checkout> python oracle/build.py   # + _ref/

* oracle/liboracle.so — the C++ restatement of the reference's CPU path
  (pf_oracle.cpp), built with g++ and OpenMP.
* oracle/_ref/libpf_kernels_ref.so — the reference's own CUDA library,
  compiled for sm_100a from its source file where it lies (read-only, never
  copied) together with ref_shim.cu's test accessors.  Built only when a
  reference checkout is named (the `reference` argument or the PF_REFERENCE
  environment variable) and holds that file; otherwise an already built
  library is used as it is.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd):
    print(" ".join(map(str, cmd)), flush=True)
    subprocess.run(list(map(str, cmd)), check=True)


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).exists() and Path(d).stat().st_mtime > t for d in deps)


def build_oracle(force: bool = False) -> Path:
    out = HERE / "liboracle.so"
    src = HERE / "pf_oracle.cpp"
    if force or _stale(out, [src]):
        # -ffp-contract=off: the f32 mirrors must round every operation.
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
              "-ffp-contract=off", src, "-o", out])
    return out


def build_ref(force: bool = False, reference: str | Path | None = None) -> Path | None:
    out = HERE / "_ref" / "libpf_kernels_ref.so"
    root = reference or os.environ.get("PF_REFERENCE")
    src = Path(root) / "src" / "cuda" / "pf_kernels.cu" if root else None
    if src is None or not src.exists():
        return out if out.exists() else None
    if force or _stale(out, [src, HERE / "ref_shim.cu"]):
        out.parent.mkdir(exist_ok=True)
        _run([NVCC, "-O3", "-std=c++17", "-gencode",
              "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler",
              "-fPIC", "-Xlinker", "-Bsymbolic",
              f'-DPF_REF_SOURCE="{src}"', HERE / "ref_shim.cu", "-o", out])
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_oracle(force)
    build_ref(force)
