"""Build recipe of the B200 library: compiles the CUDA kernels, the C ABI and
the host-side problem setup into ``gamera-op_b200/libgamera_op.so`` for
sm_100a with nvcc (no JIT, no torch extension cache: the .so lives in the
tree next to its sources)."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libgamera_op.so"
SOURCES = [
    PKG / "csrc" / "gop_api.cu",
    PKG / "csrc" / "gop_kernels.cu",
    PKG / "csrc" / "gop_sweep.cu",
    PKG / "csrc" / "gop_noalloc.cu",
    PKG / "csrc" / "gop_init.cu",
    PKG / "csrc" / "gop_bgdev.cu",
    PKG / "csrc" / "gop_peak.cu",
    PKG / "csrc" / "gop_ring.cu",
    PKG / "host" / "gop_problems.c",
    PKG / "host" / "gop_background.c",
]
HEADERS = [ROOT / "include" / "gamera_op.h", PKG / "csrc" / "gop_device.cuh",
           PKG / "csrc" / "gop_kernels.h", PKG / "csrc" / "gop_internal.h",
           PKG / "csrc" / "gop_stage.cuh", PKG / "csrc" / "gop_tma.cuh",
           PKG / "csrc" / "gop_fields.h", PKG / "csrc" / "gop_bgfield.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xptxas", "-O3",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


# per-source extra nvcc flags: the background field's quadratures and
# stress differences keep the host port's operation order (no contraction
# into fused multiply-adds), so they differ from it only by the device's
# pow, sin and cos
EXTRA = {"gop_bgdev.cu": ["-fmad=false"]}


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = objdir / (src.stem + ".o")
        if src.suffix == ".cu":
            cmd = [nvcc(), *NVCC_FLAGS, *EXTRA.get(src.name, []), "-I", str(ROOT / "include"), "-c",
                   str(src), "-o", str(obj)]
        else:
            cmd = ["gcc", "-std=gnu99", "-O2", "-fPIC", "-I", str(ROOT / "include"),
                   "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs,
           "-o", str(tmp), "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
