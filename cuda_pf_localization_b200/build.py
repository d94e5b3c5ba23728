"""Build recipe for the in-tree shared libraries.

    python -m cuda_pf_localization_b200.build          # kernels + host mirror

Produces, next to this file:
  libpf_kernels.so  the drop-in C-ABI (pfc_* / pfgl_*) compiled for sm_100a
  libpf_core.so     the C++ host mirror of pf_core (ParticleFilter,
                    CudaBackend, CudaGlobalLoc, loaders), linked to the above
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

KERNEL_SOURCES = ["pf_update.cu", "pf_estimate.cu", "pf_resample.cu",
                  "pf_abi.cu", "pf_batch.cu", "gl.cu", "gl_learned.cu"]
HOST_SOURCES = ["host/pf_core.cpp"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_kernels(force: bool = False) -> Path:
    out = PKG / "libpf_kernels.so"
    deps = [CSRC / s for s in KERNEL_SOURCES] + list(CSRC.glob("*.h")) + \
        list(CSRC.glob("*.cuh")) + [ROOT / "include" / "pfc_abi.h"]
    if not force and not _stale(out, deps):
        return out
    objdir = ROOT / "_build" / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in KERNEL_SOURCES:
        o = objdir / (Path(s).stem + ".o")
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-c", str(CSRC / s), "-o", str(o)])
        objs.append(str(o))
    _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC",
          "-Xlinker", "-Bsymbolic", "-o", str(out), *objs])
    return out


def build_host(force: bool = False) -> Path:
    out = PKG / "libpf_core.so"
    srcs = [CSRC / s for s in HOST_SOURCES]
    deps = srcs + list((CSRC / "host").glob("*.h")) + [CSRC / "markley.h",
                                                       ROOT / "include" / "pfc_abi.h",
                                                       PKG / "libpf_kernels.so"]
    if not force and not _stale(out, deps):
        return out
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared",
          "-I", str(ROOT / "include"), "-I", str(CSRC),
          *map(str, srcs), "-o", str(out),
          "-L", str(PKG), "-lpf_kernels", "-Wl,-rpath,$ORIGIN"])
    return out


def build_all(force: bool = False) -> None:
    build_kernels(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
