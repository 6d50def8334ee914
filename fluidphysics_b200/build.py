"""Build the CUDA library of the unified-particle step in-tree.

Outputs (next to this file):
  libupbd.so         the product: sm_100a, -O3, fused multiply-add allowed
  libupbd_parity.so  the same sources with --fmad=false, so every FP32
                     operation rounds exactly as the CPU oracle's does
                     (per-pass bit-exact parity checks)
  libupbd_checked.so test-only: the product sources with device-side index
                     guards (UPBD_CHECKED_BUILD): an out-of-range index sets a
                     health bit and its access is skipped
  libupbd_fp64.so    test-only: the single-scene library with the pass
                     bodies instantiated on double (UPBD_FP64_BUILD), the
                     reference trajectory of the 600-frame drift test

Both are cross-compiled with nvcc; no GPU is needed to build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
          "-I", str(INCLUDE), "-Xptxas", "-warn-spills"]

SOURCES = ["upbd.cu", "upbd_scene.cu", "upbd_batch.cu", "upbd_server.cu"]
TARGETS = {
    "libupbd.so": SOURCES,
    "libupbd_parity.so": SOURCES,
    "libupbd_fp64.so": ["upbd.cu", "upbd_scene.cu"],
    "libupbd_checked.so": SOURCES,
}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(out: Path) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(src.stat().st_mtime > t for src in _sources())


def build(force: bool = False, verbose: bool = False) -> list[Path]:
    """Compile every library target that is missing or older than its sources."""
    nvcc = _nvcc()
    built = []
    for name, srcs in TARGETS.items():
        out = HERE / name
        if not force and not _stale(out):
            built.append(out)
            continue
        flags = list(COMMON)
        if name == "libupbd_parity.so":
            flags += ["--fmad=false", "-DUPBD_PARITY_BUILD=1"]
        if name == "libupbd_fp64.so":
            flags += ["-DUPBD_FP64_BUILD=1"]
        if name == "libupbd_checked.so":
            flags += ["-DUPBD_CHECKED_BUILD=1"]
        cmd = [nvcc, *ARCH, *flags, "-o", str(out) + ".tmp", *[str(CSRC / s) for s in srcs]]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{res.stdout}\n{res.stderr}")
        if verbose and res.stderr.strip():
            print(res.stderr, file=sys.stderr)
        os.replace(str(out) + ".tmp", out)
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose=True):
        print(p)
