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
    log: str = ""  # the run's log files (rank order), where log_info writes

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


def _coords(dims):
    from itertools import product
    return list(product(*(range(d) for d in dims)))


def stitch(parts: list, dims: tuple, n: tuple) -> dict:
    """One dump of a run on a ``dims`` process grid, from the per-rank dumps
    ``parts`` (in rank order, the last axis fastest): every rank's active
    cells and its lower faces, the upper boundary faces from the last rank
    along each axis.  Ghost layers of the whole grid are left zero (a GPU
    instance fills them from its own boundary kinds)."""
    from itertools import product
    nl = tuple(n[a] // dims[a] for a in range(3))
    N = tuple(v + 2 * NG + 1 for v in n)
    out = {k: v for k, v in parts[0].items() if k not in ("gas", "gem")}
    for key in ("gas", "gem"):
        if key not in parts[0]:
            continue
        lead = parts[0][key].shape[:-3]
        arr = np.zeros(lead + N)
        for r, c in enumerate(product(*(range(d) for d in dims))):
            src = parts[r][key]
            sl_g, sl_l = [], []
            for a in range(3):
                top = 1 if c[a] == dims[a] - 1 else 0  # the upper boundary face
                sl_g.append(slice(NG + c[a] * nl[a], NG + (c[a] + 1) * nl[a] + top))
                sl_l.append(slice(NG, NG + nl[a] + top))
            arr[(Ellipsis,) + tuple(sl_g)] = src[(Ellipsis,) + tuple(sl_l)]
        out[key] = arr
    return out


NG = 4


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
    dims: tuple = (1, 1, 1),
) -> RefRun:
    """Runs ``steps`` steps of the reference on an ``n=(ni,nj,nk)`` grid.

    With ``keep_output`` the step-0 dump and the final dump are read back;
    otherwise writes are discarded (used for timing) and the shim reports the
    wall time of the step loop.  ``dims`` > (1, 1, 1) runs the reference as
    that many ranks (the MPI stand-in forks them, one process per rank) on a
    ``dims`` process grid; the per-rank dumps are stitched back into one.
    """
    exe = Path(exe) if exe else binary(coord, flavor)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is not built (make -C oracle reference)")
    ni, nj, nk = n
    nranks = dims[0] * dims[1] * dims[2]
    tmp = tempfile.mkdtemp(prefix="gop_ref_")
    try:
        cfg = (
            f"ni_global: {ni}\nnj_global: {nj}\nnk_global: {nk}\n"
            f"proc_dims_i: {dims[0]}\nproc_dims_j: {dims[1]}\nproc_dims_k: {dims[2]}\n"
            f"Nt: {steps}\ntime_stop: {time_stop!r}\n"
            f"output_interval: {output_interval!r}\n"
            "x_Norm: 1.0\nu_Norm: 1.0\nrho_Norm: 1.0\n"
        )
        Path(tmp, "config.yaml").write_text(cfg)
        e = dict(os.environ)
        e.update({"OMP_NUM_THREADS": str(threads), "GOP_PROBLEM": problem,
                  "GOP_SHIM_TIMING": "1", "GOP_SHIM_RANKS": str(nranks)})
        if not keep_output:
            e["GOP_H5_DISCARD"] = "1"
        e.update(env or {})
        # its own session, so a timeout takes down every rank
        proc = subprocess.Popen([str(exe), "config.yaml"], cwd=tmp, env=e, text=True,
                                stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                start_new_session=True)
        try:
            _, err = proc.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            os.killpg(proc.pid, 9)
            proc.communicate()
            raise
        if proc.returncode != 0:
            raise RuntimeError(f"reference run failed ({proc.returncode}): {err[-2000:]}")
        files = sorted(f for f in os.listdir(tmp) if f.startswith("mhd_") and f.endswith(".h5"))
        dumps = []
        if keep_output:
            if nranks == 1:
                dumps = [read_raw(Path(tmp, f)) for f in files]
            else:
                # mhd_II-JJ-KK_SEQ.h5: group the ranks' files by output number
                seqs = sorted({f.rsplit("_", 1)[1] for f in files})
                for q in seqs:
                    parts = [read_raw(Path(tmp, f"mhd_{c[0]:02d}-{c[1]:02d}-{c[2]:02d}_{q}"))
                             for c in _coords(dims)]
                    dumps.append(stitch(parts, dims, n))
        logs = sorted(f for f in os.listdir(tmp) if f.endswith(".log"))
        rr = RefRun(dumps=dumps, stderr=err, files=files,
                    log="".join(Path(tmp, f).read_text(errors="replace") for f in logs))
        m = re.search(r"GOP_SHIM_TIMING calls=(\d+) t1=([\d.]+) tlast=([\d.]+)", err)
        if m:
            calls = int(m.group(1))
            rr.wall_steps = calls - 2
            rr.wall_seconds = float(m.group(3)) - float(m.group(2))
        m = re.search(r"GOP_SHIM_TIMES ([\d. ]+)", err)
        if m:
            # call 0 = initial dt, call n = start of step n
            rr.step_starts = [float(v) for v in m.group(1).split()][1:]
        return rr
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
