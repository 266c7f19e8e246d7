"""Host side of the drop-in boundary, without a GPU: the C ABI library
loads and exports every entry point include/gamera_op.h declares, the
host-side problem setup reproduces the reference's initial states (checked
through the oracle's ghost fill against the reference's step-0 dumps), and
argument errors come back as status codes."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADER = ROOT / "include" / "gamera_op.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gop_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import gop
    L = gop.lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_create_rejects_bad_descriptors_without_touching_the_device():
    import gop
    x = gop.grid_uniform(8, 0.0, 1.0)
    bad = gop.Desc(2, 8, 8, 0, x.ctypes.data_as(C.POINTER(C.c_double)),
                   x.ctypes.data_as(C.POINTER(C.c_double)),
                   x.ctypes.data_as(C.POINTER(C.c_double)), b"pppppp", b"", 0, 0, 0, 0, 0, 0)
    h = C.c_void_p()
    assert gop.lib().gop_create(C.byref(bad), C.byref(h)) == -22
    assert b"at least" in gop.lib().gop_last_error()
    bad.ni = 8
    bad.bc = b"pesppp"  # periodic on one face only
    assert gop.lib().gop_create(C.byref(bad), C.byref(h)) == -22
    assert gop.lib().gop_footprint(C.byref(bad)) == 0


def test_grid_matches_reference_coordinates():
    import gop
    g = load_golden("blast_12")
    assert np.array_equal(gop.grid_uniform(12, -0.5, 0.5), g["x1"])
    o = load_golden("ot_16x16x4")
    assert np.array_equal(gop.grid_uniform(4, 0.0, 0.015625), o["x3"])


def _host_init(name, kind, **over):
    import gop
    g = load_golden(name)
    n = tuple(int(v) for v in g["n"])
    coord = 0 if str(g["coord"]) == "cart" else 2
    xs = [np.ascontiguousarray(g[f"x{a + 1}"]) for a in range(3)]
    N = tuple(v + 9 for v in n)
    d = gop.Desc(n[0], n[1], n[2], coord, *(x.ctypes.data_as(C.POINTER(C.c_double)) for x in xs),
                 str(g["bc"]).encode(), b"", 0, 0, 0, 0, 0, 0)
    p = gop.problem(kind, **over)
    gas = np.zeros((6,) + N)
    fb = np.zeros((3,) + N)
    rc = gop.lib().gop_problem_init(C.byref(d), C.byref(p), gop._ptr(gas), gop._ptr(fb))
    assert rc == 0
    return g, n, coord, gas, fb


@pytest.mark.parametrize("name,kind,over", [
    ("ot_16x16x4", 1, {}),
    ("blast_12", 2, {}),
    ("blast_bcmix", 2, {"center": (0.1, -0.05, 0.0), "b": (0.3, 0.5, 0.2)}),
    ("loop_sph", 4, {"loop": (1.5, 0.0, 0.3, 1e-3)}),
])
def test_host_problem_init_matches_reference_initial_state(oracle_mod, name, kind, over):
    g, n, coord, gas, fb = _host_init(name, kind, **over)
    o = oracle_mod.Oracle(n, g["x1"], g["x2"], g["x3"], coord=coord, bc=str(g["bc"]))
    o.set_state(gas, fb)
    o.prepare()
    st = o.state()
    assert np.array_equal(st["W"][:5], g["W0"][:5])
    assert np.array_equal(st["B"], g["B0"])
