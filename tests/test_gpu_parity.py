"""Parity of the CUDA path (through the C ABI) with the reference.

Small cases compare against the golden vectors of GAMERA-OP's own solver and
against the C restatement in oracle/ on the same inputs; the plain FP64 path
must agree to relative L1 <= 1e-10 per variable (the parity bar of this
path, after 100 steps on the Orszag-Tang case).  Size-independent properties (div B
at round-off, exact mass conservation in periodic boxes, determinism,
restart equivalence) cover larger grids.
"""
import math

import numpy as np
import pytest

from conftest import NG, load_golden, rel_l1

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10   # relative L1 per variable, plain path vs oracle/reference
TOL_MIXED = 1e-5   # relative L1 per variable, mixed path vs FP64 oracle


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


def coord_of(g):
    return 0 if str(g["coord"]) == "cart" else 2


def device_from_arrays(gop, n, x, coord, bc, W0, B0, precision=0):
    inst = gop.Instance(n, *x, coord=coord, bc=bc, precision=precision)
    inst.upload(W0, B0)
    inst.prepare()
    return inst


def compare(n, Wd, Bd, Wr, Br, tol, what=""):
    """Per-variable relative L1 over active cells and every evolved face."""
    sl = tuple(slice(NG, NG + m) for m in n)
    errs = {}
    for m in range(5):  # rho v1 v2 v3 p (p_S stays identically 0)
        errs[f"W{m}"] = rel_l1(Wd[m][sl], Wr[m][sl])
    for a in range(3):
        s = list(sl)
        s[a] = slice(NG, NG + n[a] + 1)
        errs[f"B{a}"] = rel_l1(Bd[a][tuple(s)], Br[a][tuple(s)])
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"{what}: {bad} (all: {errs})"
    return errs


def run_oracle(oracle_mod, n, x, coord, bc, W0, B0, steps, **params):
    o = oracle_mod.Oracle(n, *x, coord=coord, bc=bc, **params)
    o.set_state(W0, B0)
    o.prepare()
    o.run(steps)
    return o.state()


@pytest.mark.parametrize("name", ["ot_16x16x4", "blast_12", "blast_bcmix", "loop_sph"])
def test_golden_vectors(gop, name):
    g = load_golden(name)
    n = tuple(int(v) for v in g["n"])
    x = (g["x1"], g["x2"], g["x3"])
    inst = device_from_arrays(gop, n, x, coord_of(g), str(g["bc"]), g["W0"], g["B0"])
    t = inst.step(int(g["steps"]))
    out = inst.download(("gas", "face_b"))
    act = tuple(slice(NG, NG + m + 1) for m in n)
    Wd = out["gas"][(slice(None),) + act]
    Bd = out["face_b"][(slice(None),) + act]
    # golden arrays hold the active block plus one upper layer (faces)
    nn = tuple(m for m in n)
    pad = lambda a: np.pad(a, [(0, 0)] + [(NG, NG)] * 3)
    compare(nn, pad(Wd), pad(Bd), pad(g["W1"]), pad(g["B1"]), TOL_FP64, name)
    assert math.isclose(t, float(g["time"]), rel_tol=1e-12)


def _ot_case(gop, n=(64, 64, 4)):
    x = [gop.grid_uniform(n[0], 0.0, 1.0), gop.grid_uniform(n[1], 0.0, 1.0),
         gop.grid_uniform(n[2], 0.0, 1.0 / 64)]
    inst = gop.Instance(n, *x)
    W0, B0 = inst.init_problem(gop.PROBLEM_OT)
    return inst, x, W0, B0


def test_orszag_tang_100_steps_matches_oracle(gop, oracle_mod):
    n = (64, 64, 4)
    inst, x, W0, B0 = _ot_case(gop, n)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(100)
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, 0, "pppppp", W0, B0, 100)
    compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_FP64, "OT 64x64x4 x100")
    st = inst.stats()
    assert math.isclose(st["time"], ref["time"], rel_tol=1e-12)
    assert st["steps"] == 100


def test_orszag_tang_256x256x4_100_steps_matches_reference_binary(gop):
    """The parity bar at the full Orszag-Tang size: GAMERA-OP's own FP64
    solver (built from its sources, strict flags, one thread) and the CUDA
    path start from the reference's step-0 state and must agree to relative
    L1 <= 1e-10 per variable after 100 steps, with div B at round-off."""
    ref_run = pytest.importorskip("ref_run")
    if not ref_run.available("cart", "strict"):
        pytest.skip("oracle/_ref/ref_cart_strict not built")
    n = (256, 256, 4)
    ref = ref_run.run(n, 100, problem="ot", coord="cart",
                      env={"GOP_BC": "pppppp", "GOP_DOMAIN": "0,1,0,1,0,0.015625"}, timeout=1500)
    s0, s1 = ref.state(0), ref.state(-1)
    x = [gop.grid_uniform(n[0], 0.0, 1.0), gop.grid_uniform(n[1], 0.0, 1.0),
         gop.grid_uniform(n[2], 0.0, 1.0 / 64)]
    inst = gop.Instance(n, *x)
    W0 = np.stack([s0[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    B0 = np.stack([s0[k] for k in ("bi", "bj", "bk")])
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(100)
    d = inst.download(("gas", "face_b"))
    Wr = np.stack([s1[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    Br = np.stack([s1[k] for k in ("bi", "bj", "bk")])
    compare(n, d["gas"], d["face_b"], Wr, Br, TOL_FP64, "OT 256x256x4 x100 vs reference")
    st = inst.stats()
    assert math.isclose(st["time"], s1["time"], rel_tol=1e-12)
    assert st["divb_max"] < 1e-10


def test_blast_c2_length_64cube_200_steps_matches_reference_binary(gop):
    """The C2 blast (p = 10 inside r < 0.1 of the centre, 0.1 outside,
    B = (1/sqrt2, 1/sqrt2, 0), periodic) for C2's full 200 steps, at 64^3:
    the largest cube GAMERA-OP's strict FP64 build (one thread) finishes in a
    few minutes.  Both start from the reference's step-0 state; relative L1
    <= 1e-10 per variable, equal simulated time, div B at round-off."""
    ref_run = pytest.importorskip("ref_run")
    if not ref_run.available("cart", "strict"):
        pytest.skip("oracle/_ref/ref_cart_strict not built")
    n = (64, 64, 64)
    ref = ref_run.run(n, 200, problem="blast",
                      env={"GOP_BC": "pppppp", "GOP_DOMAIN": "-0.5,0.5,-0.5,0.5,-0.5,0.5"},
                      timeout=3000)
    s0, s1 = ref.state(0), ref.state(-1)
    x = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
    inst = gop.Instance(n, *x)
    W0 = np.stack([s0[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    B0 = np.stack([s0[k] for k in ("bi", "bj", "bk")])
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(200)
    d = inst.download(("gas", "face_b"))
    Wr = np.stack([s1[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    Br = np.stack([s1[k] for k in ("bi", "bj", "bk")])
    compare(n, d["gas"], d["face_b"], Wr, Br, TOL_FP64, "blast 64^3 x200 vs reference")
    st = inst.stats()
    assert math.isclose(st["time"], s1["time"], rel_tol=1e-12)
    assert st["divb_max"] < 1e-10


def test_blast_3d_matches_oracle(gop, oracle_mod):
    n = (32, 32, 32)
    x = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
    inst = gop.Instance(n, *x)
    W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, b=(0.4, 0.5, 0.3), center=(0.03, -0.02, 0.01))
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(40)
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, 0, "pppppp", W0, B0, 40)
    compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_FP64, "blast 32^3 x40")


@pytest.mark.parametrize("bc", ["eeeeee", "ssrrff", "rrsspp", "ffeess", "ppnnee"])
def test_boundary_kinds_match_oracle(gop, oracle_mod, bc):
    n = (16, 12, 8)
    x = [gop.grid_uniform(16, -0.5, 0.5), gop.grid_uniform(12, -0.5, 0.5),
         gop.grid_uniform(8, -0.5, 0.5)]
    inst = gop.Instance(n, *x, bc=bc)
    W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, b=(0.3, 0.5, 0.2), center=(0.1, -0.05, 0.0))
    if "n" in bc:  # 'none' keeps whatever the ghosts hold: give them a state
        W0[0][W0[0] == 0] = 1.0
        W0[4][W0[4] == 0] = 0.1
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(20)
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, 0, bc, W0, B0, 20)
    compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_FP64, f"bc {bc}")


def test_spherical_shell_matches_oracle(gop, oracle_mod):
    n = (24, 16, 16)
    x = [gop.grid_uniform(24, 1.0, 2.0), gop.grid_uniform(16, 0.25 * math.pi, 0.75 * math.pi),
         gop.grid_uniform(16, -0.25 * math.pi, 0.25 * math.pi)]
    inst = gop.Instance(n, *x, coord=gop.COORD_SPHERICAL, bc="eeeeee")
    W0, B0 = inst.init_problem(gop.PROBLEM_LOOP_SPH, loop=(1.5, 0.0, 0.3, 1e-3))
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(30)
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, 2, "eeeeee", W0, B0, 30)
    compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_FP64, "spherical shell")


@pytest.mark.parametrize("case", [
    dict(coord=0, n=(77, 45, 21), bc="sfrepp", steps=6),
    dict(coord=2, n=(67, 35, 19), bc="eeeeee", steps=5),
], ids=["blast_77x45x21", "sphere_67x35x19"])
def test_ragged_sizes_match_oracle(gop, oracle_mod, case):
    """Grid sizes that fill no launch block evenly in any direction (the
    last blocks along every axis are partial; the spherical case also runs
    the separate constrained-transport launch), against the C restatement."""
    n, coord = case["n"], case["coord"]
    if coord == 0:
        x = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
        inst = gop.Instance(n, *x, bc=case["bc"])
        W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, b=(0.4, 0.5, 0.3), center=(0.05, -0.1, 0.02))
    else:
        dom = (1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi)
        x = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
        inst = gop.Instance(n, *x, coord=gop.COORD_SPHERICAL, bc=case["bc"])
        W0, B0 = inst.init_problem(gop.PROBLEM_LOOP_SPH, loop=(1.4, 0.1, 0.3, 1e-3))
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(case["steps"])
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, coord, case["bc"], W0, B0, case["steps"])
    compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_FP64, str(n))
    assert math.isclose(inst.stats()["time"], ref["time"], rel_tol=1e-12)
    inst.close()


def test_div_b_stays_at_roundoff_and_mass_is_conserved(gop):
    n = (48, 48, 48)
    inst = gop.make(gop.PROBLEM_BLAST, n, b=(0.5, 0.4, 0.3))
    inst.prepare()
    x = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
    vol = np.einsum("i,j,k->ijk", np.diff(x[0])[NG:NG + n[0]], np.diff(x[1])[NG:NG + n[1]],
                    np.diff(x[2])[NG:NG + n[2]])
    sl = tuple(slice(NG, NG + m) for m in n)
    m0 = (inst.download(("gas",))["gas"][0][sl] * vol).sum()
    inst.step(60)
    st = inst.stats()
    assert st["divb_max"] < 1e-10, st
    m1 = (inst.download(("gas",))["gas"][0][sl] * vol).sum()
    assert abs(m1 - m0) / m0 < 1e-13


@pytest.mark.parametrize("prec,first", [(0, 10), (1, 11)], ids=["fp64", "mixed_odd_parity"])
def test_restart_continues_bit_identically(gop, prec, first):
    """Download the state and its AB2 history mid-run, upload both into a
    fresh instance and prepare it for a restart: the next steps are
    bit-identical to the uninterrupted run.  gop_prepare takes the first dt
    in the form and arithmetic of the step's own estimate (FP32 on the mixed
    path), so the restarted run takes the same step."""
    n = (24, 24, 24)
    a = gop.make(gop.PROBLEM_BLAST, n, b=(0.5, 0.4, 0.3), precision=prec)
    a.prepare()
    a.step(first)
    mid = a.download(("gas", "face_b", "gas_p", "face_b_p"))
    sa = a.stats()
    a.step(10)
    full = a.download(("gas", "face_b"))
    x = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
    b = gop.Instance(n, *x, precision=prec)
    b.upload(mid["gas"], mid["face_b"], mid["gas_p"], mid["face_b_p"], time=sa["time"], dt0=sa["dt0"])
    b.prepare(restart=True)
    b.step(10)
    rest = b.download(("gas", "face_b"))
    assert np.array_equal(rest["gas"], full["gas"])
    assert np.array_equal(rest["face_b"], full["face_b"])


def test_time_stop_ends_the_loop(gop):
    inst = gop.make(gop.PROBLEM_BLAST, (16, 16, 16))
    inst.prepare()
    inst.step(3)
    t3 = inst.stats()["time"]
    t = inst.step(100, time_stop=t3 * 1.5)
    st = inst.stats()
    # the reference stops after the first step that passes time_stop
    assert t > t3 * 1.5
    assert st["steps"] < 103
    assert st["time"] - st["dt"] <= t3 * 1.5


def test_mixed_precision_against_fp64_oracle(gop, oracle_mod):
    n = (64, 64, 4)
    inst0, x, W0, B0 = _ot_case(gop, n)
    inst = gop.Instance(n, *x, precision=gop.PREC_MIXED)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(100)
    d = inst.download(("gas", "face_b"))
    ref = run_oracle(oracle_mod, n, x, 0, "pppppp", W0, B0, 100)
    errs = compare(n, d["gas"], d["face_b"], ref["W"], ref["B"], TOL_MIXED, "mixed OT")
    assert inst.stats()["divb_max"] < 1e-9


def test_batch_results_equal_single_runs(gop):
    specs = [((16, 16, 16), {}), ((24, 16, 8), {"b": (0.2, 0.6, 0.1)}), ((32, 32, 4), {})]
    alone, members = [], []
    for n, over in specs:
        a = gop.make(gop.PROBLEM_BLAST, n, **over)
        a.prepare()
        a.step(7)
        alone.append(a.download(("gas", "face_b")))
        m = gop.make(gop.PROBLEM_BLAST, n, **over)
        m.prepare()
        members.append(m)
    b = gop.Batch(members)
    b.step([3, 3, 3])
    b.step([4, 4, 4])
    for a, m in zip(alone, members):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], a["gas"])
        assert np.array_equal(d["face_b"], a["face_b"])


def test_heterogeneous_batch_equals_members_run_alone(gop):
    """Cartesian and spherical grids, FP64 and mixed precision, periodic and
    outflow/reflective/fixed boundaries, uneven step budgets (0 included) in
    one batch: every member ends bit-identical to gop_step on it alone."""
    specs = [
        dict(kind=gop.PROBLEM_BLAST, n=(20, 12, 8), bc="ssrrfe", b=(0.3, 0.5, 0.2), steps=6),
        dict(kind=gop.PROBLEM_LOOP_SPH, n=(12, 10, 8), bc="eeeeee", steps=4),
        dict(kind=gop.PROBLEM_OT, n=(24, 24, 4), bc="pppppp", domain=(0, 1, 0, 1, 0, 1 / 6),
             precision=gop.PREC_MIXED, steps=9),
        dict(kind=gop.PROBLEM_BLAST, n=(8, 8, 8), bc="pppppp", steps=0),
        dict(kind=gop.PROBLEM_LOOP_CART, n=(16, 16, 16), bc="eeeeee", precision=gop.PREC_MIXED,
             steps=5),
    ]

    def build(sp):
        kw = {k: v for k, v in sp.items() if k not in ("kind", "n", "steps")}
        m = gop.make(sp["kind"], sp["n"], **kw)
        m.prepare()
        return m

    alone = []
    for sp in specs:
        a = build(sp)
        a.step(sp["steps"])
        alone.append((a.download(("gas", "face_b")), a.stats()))
    members = [build(sp) for sp in specs]
    b = gop.Batch(members)
    b.step([sp["steps"] for sp in specs])
    for (ref, st), m, sp in zip(alone, members, specs):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], ref["gas"]), sp
        assert np.array_equal(d["face_b"], ref["face_b"]), sp
        assert m.stats()["steps"] == sp["steps"]
        assert m.stats()["time"] == st["time"]


def test_uneven_steps_in_one_batch(gop):
    ms = [gop.make(gop.PROBLEM_BLAST, (16, 16, 16)) for _ in range(3)]
    for m in ms:
        m.prepare()
    b = gop.Batch(ms)
    b.step([1, 5, 0])
    assert [m.stats()["steps"] for m in ms] == [1, 5, 0]


def test_autotune_keeps_the_state_and_the_result(gop):
    a = gop.make(gop.PROBLEM_BLAST, (24, 20, 16), b=(0.5, 0.4, 0.3))
    b = gop.make(gop.PROBLEM_BLAST, (24, 20, 16), b=(0.5, 0.4, 0.3))
    for m in (a, b):
        m.prepare()
        m.step(3)
    chosen = b.autotune(reps=1)
    assert len(chosen) == 11
    a.step(5)
    b.step(5)
    da, db = a.download(("gas", "face_b")), b.download(("gas", "face_b"))
    # block shapes change nothing in the arithmetic of a cell
    assert np.array_equal(da["gas"], db["gas"])
    assert np.array_equal(da["face_b"], db["face_b"])
    assert a.stats()["time"] == b.stats()["time"]


def test_kernels_are_launched(gop):
    before = gop.kernel_launches()
    inst = gop.make(gop.PROBLEM_OT, (32, 32, 4), domain=(0, 1, 0, 1, 0, 1 / 64))
    inst.prepare()
    inst.step(2)
    assert gop.kernel_launches() - before > 20
