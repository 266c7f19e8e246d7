"""The C restatement of the step (oracle/gop_oracle.c) against golden
vectors produced by GAMERA-OP's own solver (tests/golden/make_golden.py).

The restatement follows the reference's operation order, so the comparison is
bit-for-bit on every case: periodic Orszag-Tang and blast, a mix of
symmetric / reflective / fixed / extrapolated ghost fills, and the spherical
shell with outflow boundaries.
"""
import numpy as np
import pytest

from conftest import NG, load_golden

CASES = ["ot_16x16x4", "blast_12", "blast_bcmix", "loop_sph"]


def run_oracle(oracle_mod, g):
    n = tuple(int(v) for v in g["n"])
    o = oracle_mod.Oracle(n, g["x1"], g["x2"], g["x3"], coord=0 if str(g["coord"]) == "cart" else 2,
                          bc=str(g["bc"]))
    o.set_state(g["W0"], g["B0"])
    o.prepare()
    o.run(int(g["steps"]))
    return n, o.state()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_bitwise(oracle_mod, name):
    g = load_golden(name)
    n, st = run_oracle(oracle_mod, g)
    sl = tuple(slice(NG, NG + m + 1) for m in n)
    W = st["W"][(slice(None),) + sl]
    B = st["B"][(slice(None),) + sl]
    for m in range(6):
        a, b = W[m][:-1, :-1, :-1], g["W1"][m][:-1, :-1, :-1]
        assert np.array_equal(a, b, equal_nan=True), f"gas field {m}"
    for a in range(3):
        # evolved faces of component a: active cells plus the upper boundary face
        cut = [slice(0, -1)] * 3
        cut[a] = slice(None)
        assert np.array_equal(B[a][tuple(cut)], g["B1"][a][tuple(cut)]), f"face field {a}"
    assert st["time"] == float(g["time"])
    assert st["dt0"] == float(g["dt0"])


def test_oracle_prepare_reproduces_ghost_fill(oracle_mod):
    # the reference's step-0 dump is taken after the halo + boundary fill;
    # re-applying the fill to it must be the identity
    g = load_golden("blast_bcmix")
    n = tuple(int(v) for v in g["n"])
    o = oracle_mod.Oracle(n, g["x1"], g["x2"], g["x3"], bc=str(g["bc"]))
    o.set_state(g["W0"], g["B0"])
    o.prepare()
    st = o.state()
    assert np.array_equal(st["W"][:5], g["W0"][:5])
    assert np.array_equal(st["B"], g["B0"])


def test_oracle_detects_planted_error(oracle_mod):
    # a mistake planted in the oracle's input must show up in the comparison
    g = load_golden("ot_16x16x4")
    g = dict(g)
    W0 = g["W0"].copy()
    W0[0, NG + 3, NG + 5, NG + 1] *= 1.0 + 1e-12
    g["W0"] = W0
    n, st = run_oracle(oracle_mod, g)
    sl = tuple(slice(NG, NG + m) for m in n)
    assert not np.array_equal(st["W"][(0,) + sl], g["W1"][0][:-1, :-1, :-1])


@pytest.mark.parametrize("case", [
    dict(n=(12, 10, 8), coord="cart", problem="blast", bc="ssrrfe", steps=8,
         domain=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
         env={"GOP_PS": "0.2", "GOP_CENTER": "0.1,-0.05,0.0", "GOP_B": "0.3,0.5,0.2"}),
    dict(n=(12, 10, 8), coord="sph", problem="loop_sph", bc="eeeeee", steps=6,
         domain=(1.0, 2.0, 0.7853981633974483, 2.356194490192345, -0.7853981633974483,
                 0.7853981633974483),
         env={"GOP_PS": "0.5", "GOP_LOOP": "1.5,0,0.3,1e-3"}),
], ids=["blast_bcmix_entropy", "loop_sph_entropy"])
def test_oracle_entropy_channel_matches_reference(oracle_mod, case):
    """A live entropy channel (p_S = f * p, GOP_PS in the oracle's problem
    file) through the restatement and through GAMERA-OP's own solver, from
    the reference's step-0 state: bit for bit, p_S included.  This pins the
    checker of the GPU tests that feed p_S through boundary ghosts."""
    ref_run = pytest.importorskip("ref_run")
    if not ref_run.available(case["coord"], "strict"):
        pytest.skip("reference binary not built")
    env = {"GOP_BC": case["bc"], "GOP_DOMAIN": ",".join(repr(v) for v in case["domain"]),
           **case["env"]}
    ref = ref_run.run(case["n"], case["steps"], problem=case["problem"], coord=case["coord"],
                      env=env, timeout=300)
    s0, s1 = ref.state(0), ref.state(-1)
    W0 = np.stack([s0[k] for k in ("rho", "v1", "v2", "v3", "p", "pS")])
    B0 = np.stack([s0[k] for k in ("bi", "bj", "bk")])
    n = case["n"]
    d0 = ref.dumps[0]  # the reference's own face coordinates
    xs = [np.asarray(d0["x1"])[:, 0, 0], np.asarray(d0["x2"])[0, :, 0], np.asarray(d0["x3"])[0, 0, :]]
    o = oracle_mod.Oracle(n, *xs, coord=0 if case["coord"] == "cart" else 2, bc=case["bc"])
    o.set_state(W0, B0)
    o.prepare()
    o.run(case["steps"])
    st = o.state()
    act = tuple(slice(NG, NG + m) for m in n)
    assert np.abs(W0[5][act]).min() > 0.0
    for m, k in enumerate(("rho", "v1", "v2", "v3", "p", "pS")):
        assert np.array_equal(st["W"][m][act], s1[k][act]), k
    for a, k in enumerate(("bi", "bj", "bk")):
        s = list(act)
        s[a] = slice(NG, NG + n[a] + 1)
        assert np.array_equal(st["B"][a][tuple(s)], s1[k][tuple(s)]), k
    assert st["time"] == s1["time"]


def test_oracle_keeps_orszag_tang_point_symmetry(oracle_mod):
    """The Orszag-Tang state is symmetric under the point reflection
    (x, y) -> (1 - x, 1 - y) with the vector fields changing sign, and the
    scheme keeps that up to round-off on a uniform periodic grid (one of the
    invariants the reference itself offers in place of tests).  The checker
    keeps it to 1e-12 after 60 steps."""
    import gop
    n = (32, 32, 4)
    x = [gop.grid_uniform(n[0], 0.0, 1.0), gop.grid_uniform(n[1], 0.0, 1.0),
         gop.grid_uniform(n[2], 0.0, 1.0 / 64)]
    W0, B0 = gop.problem_state(n, x, gop.PROBLEM_OT)
    o = oracle_mod.Oracle(n, *x, coord=0, bc="pppppp")
    o.set_state(W0, B0)
    o.prepare()
    o.run(60)
    st = o.state()
    W, B = st["W"], st["B"]
    ci, cj, ck = (slice(NG, NG + m) for m in n)
    for m, sign in ((0, 1), (1, -1), (2, -1), (3, 1), (4, 1)):  # rho, v1, v2, v3, p
        a = W[m][ci, cj, ck]
        mirrored = sign * a[::-1, ::-1, :]
        assert np.abs(a - mirrored).max() <= 1e-12 * max(np.abs(a).max(), 1e-300), m
    bx = B[0][NG:NG + n[0] + 1, cj, ck]  # the faces mirror into faces
    by = B[1][ci, NG:NG + n[1] + 1, ck]
    for b in (bx, by):
        assert np.abs(b + b[::-1, ::-1, :]).max() <= 1e-12 * np.abs(b).max()
