"""Pole ring average on spherical grids that reach a pole (doRingAverage).

GAMERA-OP averages the cells of the rings nearest a pole in phi after every
update, fixes the E and B fields on the pole faces and fills the ghost cells
across the pole half a turn away in phi
(src/spherical/spherical_RingAverage.c, spherical_boundary.c).  The CUDA
path starts from the reference's own step-0 state and must agree with
GAMERA-OP's FP64 solver (built from its sources, GOP_RING=1 in the oracle's
problem file) to relative L1 <= 1e-10 per variable, on a hemisphere (one
pole) and on the full sphere (both poles); the drop-in program runs the same
case through the reference's main.
"""
import math

import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-5
# The loop's field has the same magnitude on many neighbouring faces; the
# FP32 limiter resolves those exact ties differently from FP64 once, in the
# first step (measured on B200: face-field relative L1 ~1e-5 per theta row
# after 1 step, 1.2e-4 in total after 20, the largest share at mid
# latitudes, not in the ring rows), so the mixed face field is held to 1e-3.
TOL_MIXED_RING_B = 1e-3
ref_run = pytest.importorskip("ref_run")


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


CASES = [
    dict(id="hemisphere_nk32", n=(16, 12, 32), bc="eeoepp",
         domain=(1.0, 2.0, 0.0, 0.5 * math.pi, 0.0, 2 * math.pi), loop="1.0,0,0.3,1e-3"),
    dict(id="sphere_nk64", n=(12, 24, 64), bc="eeoopp",
         domain=(1.0, 2.0, 0.0, math.pi, 0.0, 2 * math.pi), loop="0.6,0.2,0.3,1e-3"),
]


def _errors(n, d, W, B):
    act = tuple(slice(NG, NG + m) for m in n)
    errs = {f"W{m}": rel_l1(d["gas"][m][act], W[m][act]) for m in range(5)}
    for a in range(3):
        s = list(act)
        s[a] = slice(NG, NG + n[a] + 1)
        errs[f"B{a}"] = rel_l1(d["face_b"][a][tuple(s)], B[a][tuple(s)])
    return errs


def _state(s):
    W = np.stack([s[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    B = np.stack([s[k] for k in ("bi", "bj", "bk")])
    return W, B


def _env(c):
    return {"GOP_RING": "1", "GOP_BC": c["bc"],
            "GOP_DOMAIN": ",".join(repr(v) for v in c["domain"]), "GOP_LOOP": c["loop"]}


def _instance(gop, c, precision=0):
    n, dom = c["n"], c["domain"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    return gop.Instance(n, *xs, coord=gop.COORD_SPHERICAL, bc=c["bc"], precision=precision,
                        ring_average=True)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_ring_average_matches_reference_binary(gop, case):
    if not ref_run.available("sph", "strict"):
        pytest.skip("reference binary not built")
    steps = 20
    ref = ref_run.run(case["n"], steps, problem="loop_sph", coord="sph", env=_env(case),
                      timeout=600)
    inst = _instance(gop, case)
    W0, B0 = _state(ref.state(0))
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(steps)
    W1, B1 = _state(ref.state(-1))
    errs = _errors(case["n"], inst.download(("gas", "face_b")), W1, B1)
    bad = {k: v for k, v in errs.items() if not v <= TOL_FP64}
    assert not bad, (bad, errs)
    assert math.isclose(inst.stats()["time"], ref.state(-1)["time"], rel_tol=1e-12)
    inst.close()


def test_ring_average_mixed_precision(gop):
    c = CASES[0]
    out = []
    for prec in (gop.PREC_FP64, gop.PREC_MIXED):
        inst = _instance(gop, c, precision=prec)
        W0, B0 = inst.init_problem(gop.PROBLEM_LOOP_SPH, loop=(1.0, 0.0, 0.3, 1e-3))
        inst.upload(W0, B0)
        inst.prepare()
        inst.step(20)
        out.append(inst.download(("gas", "face_b")))
        inst.close()
    errs = _errors(c["n"], out[1], out[0]["gas"], out[0]["face_b"])
    assert max(v for k, v in errs.items() if k[0] == "W") <= TOL_MIXED, errs
    assert max(v for k, v in errs.items() if k[0] == "B") <= TOL_MIXED_RING_B, errs


def test_dropin_with_ring_average_matches_reference_program():
    for nm in ("ref_sph_strict", "ref_sph_gpu"):
        if not (ref_run.REF_DIR / nm).exists():
            pytest.skip(f"oracle/_ref/{nm} not built")
    c = CASES[0]
    kw = dict(problem="loop_sph", coord="sph", env=_env(c), timeout=600)
    ref = ref_run.run(c["n"], 15, **kw)
    gpu = ref_run.run(c["n"], 15, exe=ref_run.REF_DIR / "ref_sph_gpu", **kw)
    assert gpu.files == ref.files
    a, b = gpu.dumps[-1], ref.dumps[-1]
    act = tuple(slice(NG, NG + m) for m in c["n"])
    for slot in range(5):
        assert rel_l1(a["gas"][0][slot][act], b["gas"][0][slot][act]) <= TOL_FP64, slot
    for slot in range(3):
        s = list(act)
        s[slot] = slice(NG, NG + c["n"][slot] + 1)
        assert rel_l1(a["gem"][slot][tuple(s)], b["gem"][slot][tuple(s)]) <= TOL_FP64, slot


def test_ring_average_rejects_unsupported_grids(gop):
    c = CASES[0]
    dom = c["domain"]
    full = CASES[1]["domain"]
    for n, coord, d, bc in (((16, 12, 48), gop.COORD_SPHERICAL, dom, c["bc"]),  # nk 48
                            ((16, 6, 64), gop.COORD_SPHERICAL, full, "eeoopp"),  # bands meet
                            ((16, 12, 32), gop.COORD_CARTESIAN, dom, c["bc"])):
        xs = [gop.grid_uniform(n[a], d[2 * a], d[2 * a + 1]) for a in range(3)]
        with pytest.raises(gop.GopError):
            gop.Instance(n, *xs, coord=coord, bc=bc, ring_average=True)
    # the pole fill only with the ring average, only on theta faces
    n = c["n"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    with pytest.raises(gop.GopError):
        gop.Instance(n, *xs, coord=gop.COORD_SPHERICAL, bc=c["bc"])
    with pytest.raises(gop.GopError):
        gop.Instance(n, *xs, coord=gop.COORD_SPHERICAL, bc="oeeepp", ring_average=True)
