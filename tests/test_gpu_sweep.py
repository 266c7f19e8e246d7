"""The tile-staged flux and edge-EMF sweeps (gop_sweep.cu) against the
per-face and per-edge kernels they replace.

Both compute every face with the same arithmetic in the same order, so the
same state stepped with either must come out the same: the tests allow
1e-13 relative L1 per variable (round-off from a different contraction of
a multiply-add by the compiler) and report the largest difference.  The
cases cover what changes the sweeps' tiles: partial tiles on every axis
(ragged sizes), i rows whose upper boundary face is computed by the last
tile's row-end pass (ni a multiple of 32), thin axes (4 cells), a
spherical grid with its per-face weight tables, boundary fills, a
background field and the FP32 stages of the mixed path.  Parity of the
default path with the reference itself is in test_gpu_parity.py, which
runs the sweeps.
"""
import math

import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


def _grid(gop, n, dom):
    return [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]


def _run(gop, n, xs, coord, bc, W0, B0, steps, sweep, precision=0, bg=None):
    inst = gop.Instance(n, *xs, coord=coord, bc=bc, precision=precision)
    if bg is not None:
        inst.set_background(bg)
    inst.set_sweep(sweep)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(steps)
    d = inst.download(("gas", "face_b"))
    st = inst.stats()
    inst.close()
    return d, st


def _diff(n, a, b):
    act = tuple(slice(NG, NG + m) for m in n)
    errs = {f"W{m}": rel_l1(a["gas"][m][act], b["gas"][m][act]) for m in range(5)}
    for c in range(3):
        s = list(act)
        s[c] = slice(NG, NG + n[c] + 1)
        errs[f"B{c}"] = rel_l1(a["face_b"][c][tuple(s)], b["face_b"][c][tuple(s)])
    return errs


CASES = [
    dict(id="blast_32_fp64", n=(32, 32, 32), dom=(-0.5, 0.5) * 3, coord=0, bc="pppppp",
         kind="blast", prec=0, steps=20),
    dict(id="blast_ragged_77x45x21_bcmix", n=(77, 45, 21), dom=(-0.5, 0.5) * 3, coord=0,
         bc="srfepp", kind="blast", prec=0, steps=12),
    dict(id="ot_thin_64x64x4", n=(64, 64, 4), dom=(0, 1, 0, 1, 0, 1 / 64), coord=0, bc="pppppp",
         kind="ot", prec=0, steps=30),
    dict(id="sphere_67x35x19", n=(67, 35, 19),
         dom=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         coord=2, bc="eeeeee", kind="loop_sph", prec=0, steps=12),
    dict(id="blast_ragged_mixed", n=(77, 45, 21), dom=(-0.5, 0.5) * 3, coord=0, bc="pppppp",
         kind="blast", prec=1, steps=12),
    dict(id="sphere_mixed", n=(67, 35, 19),
         dom=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         coord=2, bc="eeeeee", kind="loop_sph", prec=1, steps=12),
    # ni a multiple of 32: the i rows' upper boundary faces come with the
    # last tile of each row (the row-end pass of the EMF sweeps on i faces)
    dict(id="blast_64x48x40_mixed", n=(64, 48, 40), dom=(-0.5, 0.5) * 3, coord=0, bc="pppppp",
         kind="blast", prec=1, steps=12),
    dict(id="sphere_96x35x19", n=(96, 35, 19),
         dom=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         coord=2, bc="eeeeee", kind="loop_sph", prec=0, steps=12),
]


@pytest.mark.parametrize("c", CASES, ids=[c["id"] for c in CASES])
def test_sweep_equals_per_face_kernels(gop, c):
    n = c["n"]
    xs = _grid(gop, n, c["dom"])
    probe = gop.Instance(n, *xs, coord=c["coord"], bc=c["bc"])
    kind = {"blast": gop.PROBLEM_BLAST, "ot": gop.PROBLEM_OT, "loop_sph": gop.PROBLEM_LOOP_SPH}[c["kind"]]
    over = {"b": (0.4, 0.5, 0.3), "center": (0.03, -0.02, 0.01)} if c["kind"] == "blast" else {}
    W0, B0 = probe.init_problem(kind, **over)
    probe.close()
    a, sa = _run(gop, n, xs, c["coord"], c["bc"], W0, B0, c["steps"], True, c["prec"])
    b, sb = _run(gop, n, xs, c["coord"], c["bc"], W0, B0, c["steps"], False, c["prec"])
    errs = _diff(n, a, b)
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, f"{c['id']}: {bad} (all {errs})"
    assert math.isclose(sa["time"], sb["time"], rel_tol=1e-13)
    assert sa["steps"] == sb["steps"] == c["steps"]


def test_sweep_with_background_field(gop):
    n = (24, 20, 16)
    dom = (1.0, 2.0, -0.5, 0.5, -0.5, 0.5)
    xs = _grid(gop, n, dom)
    probe = gop.Instance(n, *xs, bc="eeeeee")
    W0, B0 = probe.init_problem(gop.PROBLEM_BLAST, center=(1.5, 0.0, 0.0), b=(0.0, 0.0, 0.0))
    bg = probe.background_fields(gop.BG_DIPOLE)
    probe.close()
    a, _ = _run(gop, n, xs, 0, "eeeeee", W0, B0, 10, True, bg=bg)
    b, _ = _run(gop, n, xs, 0, "eeeeee", W0, B0, 10, False, bg=bg)
    errs = _diff(n, a, b)
    assert all(v <= TOL for v in errs.values()), errs


def test_autotune_may_pick_the_sweep(gop):
    """The autotuner times the sweep kernel as one more candidate of each
    flux launch (index GOP_TUNE_SWEEP) and keeps what is fastest."""
    n = (64, 64, 64)
    xs = _grid(gop, n, (-0.5, 0.5) * 3)
    inst = gop.Instance(n, *xs)
    W0, B0 = inst.init_problem(gop.PROBLEM_BLAST)
    inst.upload(W0, B0)
    inst.prepare()
    picks = inst.autotune(reps=1)
    for s in ("flux_i", "flux_j", "flux_k"):
        assert 0 <= picks[s] <= 14
    inst.step(3)
    assert inst.stats()["flags"] == 0
    inst.close()


def test_autotuned_launch_order_changes_no_result(gop):
    """The autotuner also picks the order of the three flux launches and of
    the three EMF launches (rotations of the axes) by timing whole steps, and
    restores the state after each trial: a tuned instance steps to the same
    state as an untuned one."""
    n = (48, 40, 32)
    xs = _grid(gop, n, (-0.5, 0.5) * 3)
    probe = gop.Instance(n, *xs)
    W0, B0 = probe.init_problem(gop.PROBLEM_BLAST, b=(0.4, 0.5, 0.3))
    probe.close()
    out = []
    for tune in (True, False):
        inst = gop.Instance(n, *xs)
        inst.upload(W0, B0)
        inst.prepare()
        if tune:
            inst.autotune(reps=1)
            order = inst.launch_order()
            rot = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]
            assert order["flux"] in rot and order["emf"] in rot, order
        else:
            assert inst.launch_order() == {"flux": [0, 1, 2], "emf": [0, 1, 2]}
        inst.step(8)
        out.append((inst.download(("gas", "face_b")), inst.stats()))
        inst.close()
    (a, sa), (b, sb) = out
    errs = _diff(n, a, b)
    assert all(v <= TOL for v in errs.values()), errs
    assert sa["steps"] == sb["steps"] == 8
    assert math.isclose(sa["time"], sb["time"], rel_tol=1e-13)
