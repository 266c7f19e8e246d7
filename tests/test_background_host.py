"""Host port of the reference's background-field set-up
(gop_background_init, host/gop_background.c) against the arrays GAMERA-OP's
own set_background_field leaves in its step-0 dump (cell-centroid B0_1..3
and the face-normal averages B0_i/j/k), bit for bit: uniform and dipole
hooks, Cartesian and spherical grids.  Needs the reference binary built
from its sources (oracle/_ref); no GPU."""
import math

import numpy as np
import pytest

ref_run = pytest.importorskip("ref_run")


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


CASES = [
    ("cart", "blast", "uniform", (-0.5, 0.5, -0.5, 0.5, -0.5, 0.5)),
    ("cart", "blast", "dipole", (1.0, 2.0, -0.5, 0.5, -0.5, 0.5)),
    ("sph", "loop_sph", "dipole",
     (1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi)),
]


@pytest.mark.parametrize("case", CASES, ids=["cart_uniform", "cart_dipole", "sph_dipole"])
def test_background_arrays_equal_the_references(gop, case):
    coord, problem, bg, dom = case
    if not ref_run.available(coord, "strict"):
        pytest.skip("reference binary not built")
    n = (12, 10, 8)
    env = {"GOP_B0": bg, "GOP_DOMAIN": ",".join(repr(v) for v in dom)}
    ref = ref_run.run(n, 1, problem=problem, coord=coord, env=env, timeout=300)
    d = ref.dumps[0]
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    f = gop.background_fields(n, xs, gop.BG_UNIFORM if bg == "uniform" else gop.BG_DIPOLE,
                              coord=gop.COORD_SPHERICAL if coord == "sph" else gop.COORD_CARTESIAN,
                              b=(1 / math.sqrt(2),) * 3)
    shape = f["b0"][0].shape
    for name, ours in (("B0_1", f["b0"][0]), ("B0_2", f["b0"][1]), ("B0_3", f["b0"][2]),
                       ("B0_i", f["b0_face"][0]), ("B0_j", f["b0_face"][4]),
                       ("B0_k", f["b0_face"][8])):
        assert np.array_equal(np.asarray(d[name]).reshape(shape), ours), name
    assert np.abs(f["b0"]).max() > 0.1  # the field is really there
