"""Generates the golden fixtures in this directory by running GAMERA-OP's own
solver (built from the reference sources by ``make -C oracle reference``).

Each fixture holds, for one small workload: the grid coordinates, the
ghost-filled initial state the reference dumps before its first step
(src/solver_solve.c:45-53), the reference's state after ``steps`` steps
(active cells and every evolved face), and the simulated time / dt0.

Usage (needs the reference tree; the fixtures are committed):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import ref_run  # noqa: E402

# name: (n, steps, problem, coord, bc, extra env)
CASES = {
    "ot_16x16x4": ((16, 16, 4), 20, "ot", "cart", "pppppp",
                   {"GOP_DOMAIN": "0,1,0,1,0,0.015625"}),
    "blast_12": ((12, 12, 12), 10, "blast", "cart", "pppppp", {}),
    "blast_bcmix": ((12, 10, 8), 10, "blast", "cart", "ssrrfe",
                    {"GOP_CENTER": "0.1,-0.05,0.0", "GOP_B": "0.3,0.5,0.2"}),
    "loop_sph": ((12, 10, 8), 10, "loop_sph", "sph", "eeeeee",
                 {"GOP_LOOP": "1.5,0,0.3,1e-3"}),
}


def make(name, n, steps, problem, coord, bc, env):
    e = {"GOP_BC": bc}
    e.update(env)
    r = ref_run.run(n, steps, problem=problem, coord=coord, env=e)
    s0, s1 = r.state(0), r.state(-1)
    d0 = r.dumps[0]
    W0 = np.stack([s0[k] for k in ref_run.GAS_PRIM])
    B0 = np.stack([s0[k] for k in ref_run.GEM_FACE])
    W1 = np.stack([s1[k] for k in ref_run.GAS_PRIM])
    B1 = np.stack([s1[k] for k in ref_run.GEM_FACE])
    G = 4
    act = tuple(slice(G, G + m + 1) for m in n)  # active cells plus the upper face
    np.savez_compressed(
        Path(__file__).with_name(f"{name}.npz"),
        n=np.array(n), steps=steps, problem=problem, coord=coord, bc=bc,
        env=repr(env),
        x1=d0["x1"][:, 0, 0], x2=d0["x2"][0, :, 0], x3=d0["x3"][0, 0, :],
        W0=W0, B0=B0,
        W1=W1[(slice(None),) + act], B1=B1[(slice(None),) + act],
        time=s1["time"], dt0=s1["dt0"],
    )


if __name__ == "__main__":
    for name, spec in CASES.items():
        make(name, *spec)
        p = Path(__file__).with_name(f"{name}.npz")
        print(f"{p.name}: {p.stat().st_size / 1024:.0f} KiB")
