"""Device-side initial conditions (gop_problem_init_device) against the host
set-up (gop_problem_init + gop_upload) on the same grids.

The two evaluate the same source (csrc/gop_fields.h); they may differ only
in the last bits of the device's sin/cos/exp/acos/atan2 and of fused
multiply-adds, so the initial states agree to round-off and the device's
face field is divergence-free to round-off.  After steps the Cartesian
cases still agree to round-off.  On the spherical shell the loop's field
has the same magnitude on many neighbouring faces: values the host builds
exactly equal can differ by an ulp on the device, the PDM limiter's sign of
their difference flips between 0 and +-1, and the face field moves by a
truncation-size amount once (relative L1 ~1e-6 after the first step, not
growing afterwards; measured on B200), so that case is held to relative L1
<= 1e-5 per variable after the steps.
"""
import math

import numpy as np
import pytest

from conftest import NG

pytestmark = pytest.mark.gpu

TOL_INIT = 1e-13   # max |device - host| relative to the field's max |value|
TOL_STEP = 1e-11   # the same after 10 steps (Cartesian)
TOL_STEP_SPH = 1e-5  # relative L1 per variable after 10 steps (spherical shell)
TOL_DIVB = 1e-10


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


CASES = [
    dict(kind=1, n=(32, 32, 4), bc="pppppp", domain=(0.0, 1.0, 0.0, 1.0, 0.0, 1 / 8), over={}),
    dict(kind=2, n=(24, 20, 16), bc="pppppp", domain=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
         over=dict(center=(0.1, -0.05, 0.0), radius=0.2, b=(0.3, -0.2, 0.5))),
    dict(kind=3, n=(24, 24, 24), bc="pppppp", domain=(-2.0, 2.0, -2.0, 2.0, -2.0, 2.0), over={}),
    dict(kind=4, n=(20, 16, 16), bc="eeeeee",
         domain=(1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi),
         over=dict(loop=(1.5, 0.0, 0.3, 1e-3))),
]


def pair(gop, c, precision=0):
    n, d = c["n"], c["domain"]
    xs = [gop.grid_uniform(n[a], d[2 * a], d[2 * a + 1]) for a in range(3)]
    coord = gop.COORD_SPHERICAL if c["kind"] == gop.PROBLEM_LOOP_SPH else gop.COORD_CARTESIAN
    host = gop.Instance(n, *xs, coord=coord, bc=c["bc"], precision=precision)
    gas, fb = host.init_problem(c["kind"], **c["over"])
    host.upload(gas, fb)
    host.prepare()
    dev = gop.Instance(n, *xs, coord=coord, bc=c["bc"], precision=precision)
    dev.init_problem_device(c["kind"], **c["over"])
    dev.prepare()
    return host, dev


def max_rel(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def check(host, dev, tol):
    h = host.download(("gas", "face_b"))
    d = dev.download(("gas", "face_b"))
    errs = {}
    for key, nf in (("gas", 6), ("face_b", 3)):
        for f in range(nf):
            if np.abs(h[key][f]).max() == 0.0:
                assert np.abs(d[key][f]).max() == 0.0, (key, f)
                continue
            errs[f"{key}{f}"] = max_rel(d[key][f], h[key][f])
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, (bad, errs)
    return errs


@pytest.mark.parametrize("case", CASES, ids=["ot", "blast", "loop_cart", "loop_sph"])
def test_device_init_matches_host_init(gop, case):
    host, dev = pair(gop, case)
    check(host, dev, TOL_INIT)
    assert dev.stats()["divb_max"] < TOL_DIVB
    host.step(10)
    dev.step(10)
    if case["kind"] == gop.PROBLEM_LOOP_SPH:
        h = host.download(("gas", "face_b"))
        d = dev.download(("gas", "face_b"))
        sl = tuple(slice(NG, NG + m) for m in case["n"])
        for key, nf in (("gas", 5), ("face_b", 3)):
            for f in range(nf):
                x, y = h[key][f][sl], d[key][f][sl]
                assert np.abs(x - y).sum() <= TOL_STEP_SPH * np.abs(x).sum(), (key, f)
    else:
        check(host, dev, TOL_STEP)
    assert dev.stats()["divb_max"] < TOL_DIVB
    host.close()
    dev.close()


def test_device_init_mixed_precision_instance(gop):
    # the work arrays hold the edge integrals as scratch: FP32 work arrays
    # are large enough too
    host, dev = pair(gop, CASES[0], precision=gop.PREC_MIXED)
    check(host, dev, TOL_INIT)
    host.close()
    dev.close()


def test_device_init_rejects_a_problem_of_the_other_geometry(gop):
    c = CASES[3]
    n, d = c["n"], c["domain"]
    xs = [gop.grid_uniform(n[a], d[2 * a], d[2 * a + 1]) for a in range(3)]
    inst = gop.Instance(n, *xs, coord=gop.COORD_SPHERICAL, bc="eeeeee")
    with pytest.raises(gop.GopError):
        inst.init_problem_device(gop.PROBLEM_OT)
    inst.close()
