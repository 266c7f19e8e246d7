"""Runs GAMERA-OP's own solver (compiled by oracle/Makefile into
oracle/_ref/) on one workload and reads its per-step output back.

Test infrastructure only: tests/, bench.py's reference arm and the golden
fixture script use it as the checker or as the timed CPU baseline; the
product never imports it.

The binary is the reference's unmodified ``run_mhd`` (src/main.c:14-99) with
the single-rank MPI / flat-file HDF5 stand-ins from oracle/shim and the
problem hooks in oracle/problems/problem_gop.c.  Each run happens in a fresh
temporary directory (the reference restarts from any ``mhd_*.h5`` it finds in
its working directory, src/solver_init.c:394-448).
"""
from __future__ import annotations

import os
import re
import shutil
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

# field slots of the reference's state arrays (src/config.h:255-499)
GAS_PRIM = ["rho", "v1", "v2", "v3", "p", "pS"]
GEM_FACE = ["bi", "bj", "bk"]


def read_raw(path: str | os.PathLike) -> dict:
    """Reads one GOPRAW01 file written by oracle/shim/hdf5_shim.c."""
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"GOPRAW01":
            raise ValueError(f"{path}: not a GOPRAW01 file")
        (n,) = struct.unpack("<I", f.read(4))
        for _ in range(n):
            (ln,) = struct.unpack("<I", f.read(4))
            name = f.read(ln).decode()
            typ, nd = struct.unpack("<ii", f.read(8))
            dims = struct.unpack("<" + "Q" * nd, f.read(8 * nd))
            (nbytes,) = struct.unpack("<Q", f.read(8))
            dt = np.float64 if typ == 0 else np.int32
            arr = np.frombuffer(f.read(nbytes), dtype=dt).reshape(dims)
            out[name] = arr.copy()
    return out


def binary(coord: str = "cart", flavor: str = "strict") -> Path:
    """Path of a reference build; ``flavor`` 'release' picks the AVX-512 build
    when the host supports it."""
    if flavor == "release":
        v = "v3"
        if coord == "cart":
            try:
                flags = Path("/proc/cpuinfo").read_text()
                if " avx512f" in flags and " avx512bw" in flags:
                    v = "v4"
            except OSError:
                pass
        name = f"ref_{coord}_release_{v}"
    else:
        name = f"ref_{coord}_strict"
    return REF_DIR / name


def available(coord: str = "cart", flavor: str = "strict") -> bool:
    return binary(coord, flavor).exists()


@dataclass
class RefRun:
    """Outputs of one reference run."""

    dumps: list  # per output file: dict of datasets
    stderr: str
    wall_steps: int = 0
    wall_seconds: float = 0.0
    files: list = field(default_factory=list)
    step_starts: list = field(default_factory=list)

    def state(self, idx: int = -1) -> dict:
        """Primitive state and face B (ghost-extended, reference layout
        [i][j][k], k fastest) of dump ``idx``."""
        d = self.dumps[idx]
        gas = d["gas"][0]
        gem = d["gem"]
        st = {n: gas[m] for m, n in enumerate(GAS_PRIM)}
        st.update({f"{n}_h": gas[6 + m] for m, n in enumerate(GAS_PRIM)})
        st.update({f"{n}_p": gas[12 + m] for m, n in enumerate(GAS_PRIM)})
        st.update({n: gem[m] for m, n in enumerate(GEM_FACE)})
        st.update({f"mags{m + 1}": gem[3 + m] for m in range(3)})
        st.update({f"{n}_h": gem[6 + m] for m, n in enumerate(GEM_FACE)})
        st.update({f"{n}_p": gem[9 + m] for m, n in enumerate(GEM_FACE)})
        st["time"] = float(d["time_sim"][0])
        st["dt0"] = float(d["dt0"][0])
        return st


def run(
    n: tuple,
    steps: int,
    problem: str = "blast",
    coord: str = "cart",
    flavor: str = "strict",
    env: dict | None = None,
    threads: int = 1,
    keep_output: bool = True,
    time_stop: float = 1e30,
    timeout: float | None = None,
    exe: str | os.PathLike | None = None,
    output_interval: float = 1e30,
) -> RefRun:
    """Runs ``steps`` steps of the reference on an ``n=(ni,nj,nk)`` grid.

    With ``keep_output`` the step-0 dump and the final dump are read back;
    otherwise writes are discarded (used for timing) and the shim reports the
    wall time of the step loop.
    """
    exe = Path(exe) if exe else binary(coord, flavor)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is not built (make -C oracle reference)")
    ni, nj, nk = n
    tmp = tempfile.mkdtemp(prefix="gop_ref_")
    try:
        cfg = (
            f"ni_global: {ni}\nnj_global: {nj}\nnk_global: {nk}\n"
            "proc_dims_i: 1\nproc_dims_j: 1\nproc_dims_k: 1\n"
            f"Nt: {steps}\ntime_stop: {time_stop!r}\n"
            f"output_interval: {output_interval!r}\n"
            "x_Norm: 1.0\nu_Norm: 1.0\nrho_Norm: 1.0\n"
        )
        Path(tmp, "config.yaml").write_text(cfg)
        e = dict(os.environ)
        e.update({"OMP_NUM_THREADS": str(threads), "GOP_PROBLEM": problem,
                  "GOP_SHIM_TIMING": "1"})
        if not keep_output:
            e["GOP_H5_DISCARD"] = "1"
        e.update(env or {})
        p = subprocess.run([str(exe), "config.yaml"], cwd=tmp, env=e,
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference run failed ({p.returncode}): {p.stderr[-2000:]}")
        files = sorted(f for f in os.listdir(tmp) if f.startswith("mhd_") and f.endswith(".h5"))
        dumps = [read_raw(Path(tmp, f)) for f in files] if keep_output else []
        rr = RefRun(dumps=dumps, stderr=p.stderr, files=files)
        m = re.search(r"GOP_SHIM_TIMING calls=(\d+) t1=([\d.]+) tlast=([\d.]+)", p.stderr)
        if m:
            calls = int(m.group(1))
            rr.wall_steps = calls - 2
            rr.wall_seconds = float(m.group(3)) - float(m.group(2))
        m = re.search(r"GOP_SHIM_TIMES ([\d. ]+)", p.stderr)
        if m:
            # call 0 = initial dt, call n = start of step n
            rr.step_starts = [float(v) for v in m.group(1).split()][1:]
        return rr
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
