"""Background magnetic field B0 on the CUDA path.

The reference adds a fixed background field (its B10/B20/B30 hooks,
integrated once by set_background_field, src/solver_func.c:1851-2077) to
the fluxes, the stress, the edge EMFs, the Alfven correction and the CFL
dt.  Here the background comes from gop_background_init (the host port of
set_background_field, checked bit for bit against the reference's dumps in
tests/test_background_host.py), goes to the device with
gop_set_background, and the steps are compared with GAMERA-OP's own FP64
solver run with the same hooks (GOP_B0 in the oracle's problem file).
"""
import math

import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10   # relative L1 per variable against the reference
TOL_MIXED = 1e-5   # mixed path against the FP64 path
ref_run = pytest.importorskip("ref_run")


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


def _state(s):
    W = np.stack([s[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    B = np.stack([s[k] for k in ("bi", "bj", "bk")])
    return W, B


def _errors(n, d, W, B):
    act = tuple(slice(NG, NG + m) for m in n)
    errs = {f"W{m}": rel_l1(d["gas"][m][act], W[m][act]) for m in range(5)}
    for a in range(3):
        s = list(act)
        s[a] = slice(NG, NG + n[a] + 1)
        errs[f"B{a}"] = rel_l1(d["face_b"][a][tuple(s)], B[a][tuple(s)])
    return errs


CASES = [
    dict(id="cart_uniform", n=(16, 16, 12), coord="cart", bc="pppppp", problem="blast",
         domain=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), bg=1, env={"GOP_B0": "uniform"}),
    dict(id="cart_dipole", n=(16, 16, 12), coord="cart", bc="eeeeee", problem="blast",
         domain=(1.0, 2.0, -0.5, 0.5, -0.5, 0.5), bg=2,
         env={"GOP_B0": "dipole", "GOP_CENTER": "1.5,0.0,0.0", "GOP_B": "0,0,0"}),
    dict(id="sph_dipole", n=(20, 16, 12), coord="sph", bc="eeeeee", problem="loop_sph",
         domain=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         bg=2, env={"GOP_B0": "dipole", "GOP_LOOP": "1.5,0,0.3,1e-3"}),
]


def _instance(gop, c, precision=0, background=True):
    n, dom = c["n"], c["domain"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    coord = gop.COORD_SPHERICAL if c["coord"] == "sph" else gop.COORD_CARTESIAN
    inst = gop.Instance(n, *xs, coord=coord, bc=c["bc"], precision=precision)
    return inst, xs, coord


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_background_steps_match_reference_binary(gop, case):
    if not ref_run.available(case["coord"], "strict"):
        pytest.skip("reference binary not built")
    steps = 20
    env = {"GOP_BC": case["bc"], "GOP_DOMAIN": ",".join(repr(v) for v in case["domain"]),
           **case["env"]}
    ref = ref_run.run(case["n"], steps, problem=case["problem"], coord=case["coord"], env=env,
                      timeout=600)
    inst, xs, coord = _instance(gop, case)
    bgf = gop.background_fields(case["n"], xs, case["bg"], coord=coord,
                                b=(1 / math.sqrt(2),) * 3)
    # the host port gives the reference's own face and cell averages
    d0 = ref.dumps[0]
    assert np.array_equal(bgf["b0"][0], np.asarray(d0["B0_1"]).reshape(bgf["b0"][0].shape))
    assert np.array_equal(bgf["b0_face"][0], np.asarray(d0["B0_i"]).reshape(bgf["b0"][0].shape))
    W0, B0 = _state(ref.state(0))
    inst.upload(W0, B0)
    inst.set_background(bgf)
    inst.prepare()
    inst.step(steps)
    W1, B1 = _state(ref.state(-1))
    errs = _errors(case["n"], inst.download(("gas", "face_b")), W1, B1)
    bad = {k: v for k, v in errs.items() if not v <= TOL_FP64}
    assert not bad, (bad, errs)
    assert math.isclose(inst.stats()["time"], ref.state(-1)["time"], rel_tol=1e-12)
    inst.close()


def test_zero_background_equals_no_background(gop):
    c = CASES[1]
    res = []
    for with_bg in (False, True):
        inst, xs, coord = _instance(gop, c)
        W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, center=(1.5, 0.0, 0.0), b=(0.3, -0.2, 0.4))
        inst.upload(W0, B0)
        if with_bg:
            bgf = gop.background_fields(c["n"], xs, gop.BG_UNIFORM, b=(0.0, 0.0, 0.0))
            inst.set_background(bgf)
        inst.prepare()
        inst.step(15)
        res.append(inst.download(("gas", "face_b")))
        inst.close()
    for key in ("gas", "face_b"):
        a, b = res[0][key], res[1][key]
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max(), key


def test_mixed_precision_with_background(gop):
    c = CASES[1]
    out = []
    for prec in (gop.PREC_FP64, gop.PREC_MIXED):
        inst, xs, coord = _instance(gop, c, precision=prec)
        W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, center=(1.5, 0.0, 0.0), b=(0.0, 0.0, 0.0))
        inst.upload(W0, B0)
        inst.set_background(gop.background_fields(c["n"], xs, gop.BG_DIPOLE))
        inst.prepare()
        inst.step(20)
        out.append(inst.download(("gas", "face_b")))
        inst.close()
    n = c["n"]
    errs = _errors(n, out[1], out[0]["gas"], out[0]["face_b"])
    assert max(errs.values()) <= TOL_MIXED, errs


def test_background_arguments_go_together(gop):
    c = CASES[0]
    inst, xs, coord = _instance(gop, c)
    bgf = gop.background_fields(c["n"], xs, gop.BG_UNIFORM, b=(0.1, 0.2, 0.3))
    import ctypes as C
    with pytest.raises(gop.GopError):
        gop._check(gop.lib().gop_set_background(inst.handle, gop._ptr(bgf["b0"]), None, None, None))
    inst.set_background(bgf)
    inst.set_background(None)  # removing it again is allowed
    inst.close()


DEV_CASES = [
    dict(id="cart_uniform", n=(20, 16, 12), coord="cart", dom=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
         kind=1, b=(0.3, -0.2, 0.7)),
    dict(id="cart_dipole", n=(20, 16, 12), coord="cart", dom=(1.0, 2.0, -0.5, 0.5, -0.5, 0.5),
         kind=2, b=(0.0, 0.0, 0.0)),
    dict(id="sph_dipole", n=(24, 20, 16), coord="sph",
         dom=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         kind=2, b=(0.0, 0.0, 0.0)),
]


@pytest.mark.parametrize("case", DEV_CASES, ids=[c["id"] for c in DEV_CASES])
def test_device_background_matches_host_port(gop, case):
    """set_background_field evaluated on the device (gop_set_background_device)
    against the host port that equals the reference's arrays bit for bit:
    B0 and its face and edge averages agree to 1e-13 of their largest value
    (the device's pow, sin and cos).  The Lorentz force of these fields is
    a near-total cancellation of face stresses of size |B0|^2 / dx, so it is
    held to 1e-12 of that scale."""
    n, dom = case["n"], case["dom"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    coord = gop.COORD_SPHERICAL if case["coord"] == "sph" else gop.COORD_CARTESIAN
    host = gop.background_fields(n, xs, case["kind"], coord=coord, b=case["b"])
    inst = gop.Instance(n, *xs, coord=coord, bc="eeeeee")
    inst.set_background_device(case["kind"], b=case["b"])
    dev = inst.get_background()
    for k in ("b0", "b0_face", "b0_edge"):
        scale = max(np.abs(host[k]).max(), 1e-300)
        err = np.abs(dev[k] - host[k]).max() / scale
        assert err <= 1e-13, (k, err)
    b2 = (host["b0"] ** 2).sum(axis=0).max()
    r_min = dom[0] if coord == gop.COORD_SPHERICAL else 1.0
    dx = min(r_min * (dom[2 * a + 1] - dom[2 * a]) / n[a] if a else (dom[1] - dom[0]) / n[0]
             for a in range(3))
    err = np.abs(dev["lorentz"] - host["lorentz"]).max() / (b2 / dx)
    assert err <= 1e-12, ("lorentz", err)
    inst.close()


def test_device_background_steps_like_host_background(gop):
    n = (24, 20, 16)
    dom = (1.0, 2.0, -0.5, 0.5, -0.5, 0.5)
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    out = []
    for device in (False, True):
        inst = gop.Instance(n, *xs, bc="eeeeee")
        W0, B0 = inst.init_problem(gop.PROBLEM_BLAST, center=(1.5, 0.0, 0.0), b=(0.0, 0.0, 0.0))
        if device:
            inst.set_background_device(gop.BG_DIPOLE)
        else:
            inst.set_background(inst.background_fields(gop.BG_DIPOLE))
        inst.upload(W0, B0)
        inst.prepare()
        inst.step(10)
        out.append(inst.download(("gas", "face_b")))
        inst.close()
    errs = _errors(n, out[1], out[0]["gas"], out[0]["face_b"])
    assert all(v <= 1e-12 for v in errs.values()), errs
