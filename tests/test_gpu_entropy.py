"""The entropy channel p_S (gas_p_S) with nonzero values.

GAMERA-OP carries p_S = S rho^(gamma-1) through the step with its own
Rusanov flux (VF_entropy, src/solver_func.c:940-1033) and the
conservative update of S (src/solver_solve.c:326-377); every supplied
problem leaves it at zero.  gop_prepare checks p_S of the state and its
AB2 history; while it is identically zero (then it stays zero) the step
runs kernel variants that leave the channel out.  These cases, with
p_S = f * p from GOP_PS in the oracle's problem file, check the live
channel against the reference binary and the C restatement, and that a
batch picks up a member whose channel turns live.
"""
import math

import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-5
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
    errs = {f"W{m}": rel_l1(d["gas"][m][act], W[m][act]) for m in range(6)}
    for a in range(3):
        s = list(act)
        s[a] = slice(NG, NG + n[a] + 1)
        errs[f"B{a}"] = rel_l1(d["face_b"][a][tuple(s)], B[a][tuple(s)])
    return errs


CASES = [
    dict(id="blast_periodic", n=(16, 16, 12), coord="cart", bc="pppppp", problem="blast",
         domain=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), env={"GOP_PS": "0.3"}),
    dict(id="blast_mixed_bc", n=(20, 16, 12), coord="cart", bc="ssrrfe", problem="blast",
         domain=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
         env={"GOP_PS": "0.2", "GOP_CENTER": "0.1,-0.05,0.0", "GOP_B": "0.3,0.5,0.2"}),
    dict(id="loop_sph", n=(20, 16, 12), coord="sph", bc="eeeeee", problem="loop_sph",
         domain=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         env={"GOP_PS": "0.5", "GOP_LOOP": "1.5,0,0.3,1e-3"}),
]


def _instance(gop, c, precision=0):
    n, dom = c["n"], c["domain"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    coord = gop.COORD_SPHERICAL if c["coord"] == "sph" else gop.COORD_CARTESIAN
    return gop.Instance(n, *xs, coord=coord, bc=c["bc"], precision=precision)


def _reference(c, steps):
    if not ref_run.available(c["coord"], "strict"):
        pytest.skip("reference binary not built")
    env = {"GOP_BC": c["bc"], "GOP_DOMAIN": ",".join(repr(v) for v in c["domain"]), **c["env"]}
    return ref_run.run(c["n"], steps, problem=c["problem"], coord=c["coord"], env=env,
                       timeout=600)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_entropy_channel_matches_reference_binary(gop, case):
    steps = 20
    ref = _reference(case, steps)
    W0, B0 = _state(ref.state(0))
    act = tuple(slice(NG, NG + m) for m in case["n"])
    assert np.abs(W0[5][act]).min() > 0.0  # the channel is live from the start
    inst = _instance(gop, case)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(steps)
    W1, B1 = _state(ref.state(-1))
    errs = _errors(case["n"], inst.download(("gas", "face_b")), W1, B1)
    bad = {k: v for k, v in errs.items() if not v <= TOL_FP64}
    assert not bad, (bad, errs)
    assert math.isclose(inst.stats()["time"], ref.state(-1)["time"], rel_tol=1e-12)
    inst.close()


def test_entropy_channel_mixed_precision(gop):
    c = CASES[0]
    ref = _reference(c, 1)
    W0, B0 = _state(ref.state(0))
    out = []
    for prec in (gop.PREC_FP64, gop.PREC_MIXED):
        inst = _instance(gop, c, precision=prec)
        inst.upload(W0, B0)
        inst.prepare()
        inst.step(20)
        out.append(inst.download(("gas", "face_b")))
        inst.close()
    errs = _errors(c["n"], out[1], out[0]["gas"], out[0]["face_b"])
    assert max(errs.values()) <= TOL_MIXED, errs


def test_channel_fed_only_by_boundary_ghosts(gop, oracle_mod):
    """p_S zero in every active cell and nonzero only in the ghost layers of
    a fixed boundary (gas_bc_fixed_* leaves p_S untouched,
    src/boundary_conditions.c:247-402): the flag must come up from the ghost
    cells alone and the entropy that flows in must match the C restatement
    of the step."""
    c = CASES[1]
    ref = _reference(c, 1)
    W0, B0 = _state(ref.state(0))
    W0 = W0.copy()
    W0[5] = 0.0
    n = c["n"]
    W0[5][NG + n[0]:, :, :] = 0.05  # i-high ghost layers: the 'f' face keeps them
    dom = c["domain"]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    bc = "sfrrfe"
    inst = gop.Instance(n, *xs, coord=gop.COORD_CARTESIAN, bc=bc)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(15)
    d = inst.download(("gas", "face_b"))
    o = oracle_mod.Oracle(n, *xs, coord=0, bc=bc)
    o.set_state(W0, B0)
    o.prepare()
    o.run(15)
    r = o.state()
    errs = _errors(n, d, r["W"], r["B"])
    bad = {k: v for k, v in errs.items() if not v <= TOL_FP64}
    assert not bad, (bad, errs)
    act = tuple(slice(NG, NG + m) for m in n)
    assert np.abs(d["gas"][5][act]).max() > 1e-4  # entropy entered the grid
    inst.close()


def test_batch_captures_again_when_a_member_turns_live(gop):
    """A batch member prepared again with a live p_S (another flux kernel)
    makes the batch capture its step again: the batch then steps it exactly
    as the instance alone would."""
    c = CASES[0]
    ref = _reference(c, 1)
    W0, B0 = _state(ref.state(0))
    Wz = W0.copy()
    Wz[5] = 0.0
    a = _instance(gop, c)
    a.upload(Wz, B0)
    a.prepare()
    batch = gop.Batch([a])
    batch.step([3])
    a.upload(W0, B0)
    a.prepare()
    batch.step([6])
    b = _instance(gop, c)
    b.upload(W0, B0)
    b.prepare()
    b.step(6)
    da, db = a.download(("gas", "face_b")), b.download(("gas", "face_b"))
    assert np.array_equal(da["gas"], db["gas"]) and np.array_equal(da["face_b"], db["face_b"])
    batch.close()
    a.close()
    b.close()
