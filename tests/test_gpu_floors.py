"""The positivity floors and the device error flag of the CUDA path.

check_positivity (src/solver_func.c:2117-2135) replaces a density below
rho_floor by rho_floor (and then the pressure by p_floor) and a pressure
below p_floor by p_floor after every update; the Alfven/Boris correction
that follows uses the floored density while the velocities divide the
momenta by the unfloored one.  No supplied problem comes near the floors,
so here the blast's inner sphere starts below both (GOP_RHO_IN and GOP_P_IN
of the oracle's problem file), and the steps are compared with GAMERA-OP's
own FP64 solver from its own step-0 state.

A state that turns non-finite sets the device error flag; gop_step (with a
time read-back) and gop_batch_wait report it as GOP_ENUMERIC.
"""
import math

import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
RHO_FLOOR, P_FLOOR = 0.00316227, 0.000316227
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


FLOOR_ENV = {"GOP_BC": "pppppp", "GOP_DOMAIN": "-0.5,0.5,-0.5,0.5,-0.5,0.5",
             "GOP_RHO_IN": "0.001", "GOP_P_IN": "0.0001", "GOP_P_OUT": "0.1",
             "GOP_RADIUS": "0.2", "GOP_B": "0.3,0.2,0.1"}


@pytest.mark.parametrize("steps", [1, 30])
def test_positivity_floors_match_reference_binary(gop, steps):
    if not ref_run.available("cart", "strict"):
        pytest.skip("reference binary not built")
    n = (24, 24, 24)
    ref = ref_run.run(n, steps, problem="blast", env=FLOOR_ENV, timeout=900)
    W0, B0 = _state(ref.state(0))
    act = tuple(slice(NG, NG + m) for m in n)
    assert W0[0][act].min() < RHO_FLOOR and W0[4][act].min() < P_FLOOR
    xs = [gop.grid_uniform(m, -0.5, 0.5) for m in n]
    inst = gop.Instance(n, *xs)
    inst.upload(W0, B0)
    inst.prepare()
    inst.step(steps)
    d = inst.download(("gas", "face_b"))
    W1, B1 = _state(ref.state(-1))
    errs = _errors(n, d, W1, B1)
    assert all(v <= TOL_FP64 for v in errs.values()), errs
    assert math.isclose(inst.stats()["time"], ref.state(-1)["time"], rel_tol=1e-12)
    if steps == 1:
        # the whole inner sphere was floored: density and pressure exactly at
        # the floors, in the same cells as the reference
        fl = d["gas"][0][act] == RHO_FLOOR
        assert fl.sum() > 50
        assert np.array_equal(fl, W1[0][act] == RHO_FLOOR)
        assert np.array_equal(d["gas"][4][act] == P_FLOOR, W1[4][act] == P_FLOOR)
    inst.close()


def _ot(gop, n=(32, 32, 4)):
    xs = [gop.grid_uniform(n[0], 0.0, 1.0), gop.grid_uniform(n[1], 0.0, 1.0),
          gop.grid_uniform(n[2], 0.0, 1.0 / 64)]
    inst = gop.Instance(n, *xs)
    W, B = inst.init_problem(gop.PROBLEM_OT)
    return inst, W, B


def test_non_finite_state_reports_enumeric(gop):
    inst, W, B = _ot(gop)
    W[0][NG + 5, NG + 7, NG + 1] = float("nan")
    inst.upload(W, B)
    inst.prepare()  # the CFL minimum skips the NaN cell
    with pytest.raises(gop.GopError) as e:
        inst.step(2)
    assert e.value.code == -34
    assert inst.stats()["flags"] == 1
    inst.close()


def test_non_finite_member_fails_the_batch(gop):
    good, Wg, Bg = _ot(gop)
    bad, W, B = _ot(gop)
    W[1][NG + 3, NG + 3, NG + 2] = float("nan")
    good.upload(Wg, Bg)
    good.prepare()
    bad.upload(W, B)
    bad.prepare()
    batch = gop.Batch([good, bad])
    with pytest.raises(gop.GopError) as e:
        batch.step([3, 3])
    assert e.value.code == -34
    assert good.stats()["flags"] == 0 and bad.stats()["flags"] == 1
    batch.close()
    good.close()
    bad.close()
