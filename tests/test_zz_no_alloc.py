"""gop_cfl_dt_noalloc: the CFL dt and max|div B| of a state the caller keeps
in device memory, for callers that may not allocate device memory -- a
serving loop whose device memory was reserved once at start-up and may not
grow, or a host program that owns all of its device buffers and hands the
library only pointers.  Its only scratch is a static device array inside the
library.

Checked through the C ABI against the instance path (gop_prepare computes the
same two numbers for the state it was given), each time on two different
states in a row, so the second call shows the shared scratch left by the
first does not leak into it: a Cartesian grid, a spherical shell (centroids,
face areas, volumes and CFL lengths of curvilinear cells) and a state with a
background field B0.  Kept in its own file, collected last.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative, the tolerance of the plain-path parity tests


def _bind(gop):
    L = gop.lib()
    L.gop_cfl_dt_noalloc.argtypes = [C.POINTER(gop.Desc)] + [C.c_void_p] * 6
    return L


def _noalloc(gop, torch, desc, gas, fb, bg=None):
    """One call with device copies of the arrays; returns (dt, divb) and the
    device memory the call itself took."""
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_gas, d_fb = dev(gas), dev(fb)
    d_b0 = d_bf = None
    if bg is not None:
        d_b0, d_bf = dev(bg["b0"]), dev(bg["b0_face"])
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    L = _bind(gop)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    rc = L.gop_cfl_dt_noalloc(C.byref(desc), ptr(d_gas), ptr(d_fb), ptr(d_b0), ptr(d_bf),
                              ptr(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.gop_last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return out.cpu().numpy(), free0 - free1


def _instance_numbers(gop, n, xs, gas, fb, coord=0, bc="pppppp", bg=None):
    """dt and div B the instance path reports for this state."""
    inst = gop.Instance(n, *xs, coord=coord, bc=bc)
    if bg is not None:
        inst.set_background(bg)
    inst.upload(gas, fb)
    inst.prepare()
    st = inst.stats()
    inst.close()
    return st["dt0"], st["divb_max"]


def _two_states(gop, n, xs, kind, coord=0, bc="pppppp", bg=None, steps=6, **over):
    """An initial state and the state a few steps later."""
    a = gop.Instance(n, *xs, coord=coord, bc=bc)
    if bg is not None:
        a.set_background(bg)
    gas_a, fb_a = a.init_problem(kind, **over)
    a.upload(gas_a, fb_a)
    a.prepare()
    a.step(steps)
    st = a.download(("gas", "face_b"))
    desc = a.desc
    return a, desc, (gas_a, fb_a), (st["gas"], st["face_b"])


def _check_pair(gop, torch, n, xs, kind, coord=0, bc="pppppp", bg=None, **over):
    a, desc, (gas_a, fb_a), (gas_b, fb_b) = _two_states(gop, n, xs, kind, coord, bc, bg, **over)
    want = [_instance_numbers(gop, n, xs, g, f, coord, bc, bg) for g, f in ((gas_a, fb_a), (gas_b, fb_b))]
    assert want[0][0] != want[1][0]
    got = []
    for g, f in ((gas_a, fb_a), (gas_b, fb_b)):  # two calls in a row
        out, grew = _noalloc(gop, torch, desc, g, f, bg)
        got.append(out)
    for (dt, db), out in zip(want, got):
        assert abs(out[0] - dt) <= TOL * dt, (out, dt)
        assert abs(out[1] - db) <= TOL * max(db, 1.0), (out, db)
    a.close()
    return grew


def test_noalloc_cartesian_matches_instance_path_twice():
    torch = pytest.importorskip("torch")
    import gop

    n = (48, 40, 8)
    xs = [gop.grid_uniform(48, 0.0, 1.0), gop.grid_uniform(40, 0.0, 1.0),
          gop.grid_uniform(8, 0.0, 0.125)]
    grew = _check_pair(gop, torch, n, xs, gop.PROBLEM_OT)
    # the library is loaded by now: the call itself takes no device memory
    assert grew == 0


def test_noalloc_spherical_shell_matches_instance_path_twice():
    torch = pytest.importorskip("torch")
    import gop

    n = (24, 20, 16)
    dom = (1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi, -0.25 * math.pi, 0.25 * math.pi)
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    grew = _check_pair(gop, torch, n, xs, gop.PROBLEM_LOOP_SPH, coord=gop.COORD_SPHERICAL,
                       bc="eeeeee")
    assert grew == 0


def test_noalloc_with_background_field_matches_instance_path_twice():
    torch = pytest.importorskip("torch")
    import gop

    n = (24, 20, 16)
    dom = (1.0, 2.0, -0.5, 0.5, -0.5, 0.5)
    xs = [gop.grid_uniform(n[a], dom[2 * a], dom[2 * a + 1]) for a in range(3)]
    bg = gop.background_fields(n, xs, gop.BG_DIPOLE)
    _check_pair(gop, torch, n, xs, gop.PROBLEM_BLAST, bc="eeeeee", bg=bg,
                center=(1.5, 0.0, 0.0), b=(0.0, 0.0, 0.0))


def _desc(gop, n, ring=0, coord=0, bc=b"pppppp"):
    xs = [np.ascontiguousarray(gop.grid_uniform(m, 0.0, 1.0)) for m in n]
    d = gop.Desc(n[0], n[1], n[2], coord, *(v.ctypes.data_as(C.POINTER(C.c_double)) for v in xs),
                 bc, b"", 0, 0, 0, 0, 0, 0, ring)
    return d, xs


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    import gop

    d, _keep = _desc(gop, (1025, 4, 4))
    L = _bind(gop)
    rc = L.gop_cfl_dt_noalloc(C.byref(d), C.c_void_p(16), C.c_void_p(16), None, None,
                              C.c_void_p(16), None)
    assert rc == -22
    assert b"static scratch limit" in L.gop_last_error()


def test_noalloc_rejects_half_a_background_and_the_ring_average():
    import gop

    d, _keep = _desc(gop, (16, 16, 16))
    L = _bind(gop)
    rc = L.gop_cfl_dt_noalloc(C.byref(d), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None,
                              C.c_void_p(16), None)
    assert rc == -22 and b"go together" in L.gop_last_error()
    n = (8, 32, 32)
    xs = [np.ascontiguousarray(gop.grid_uniform(8, 1.0, 2.0)),
          np.ascontiguousarray(gop.grid_uniform(32, 0.0, math.pi / 2)),
          np.ascontiguousarray(gop.grid_uniform(32, 0.0, 2 * math.pi))]
    d = gop.Desc(n[0], n[1], n[2], gop.COORD_SPHERICAL,
                 *(v.ctypes.data_as(C.POINTER(C.c_double)) for v in xs),
                 b"eeeepp", b"", 0, 0, 0, 0, 0, 0, 1)
    rc = L.gop_cfl_dt_noalloc(C.byref(d), C.c_void_p(16), C.c_void_p(16), None, None,
                              C.c_void_p(16), None)
    assert rc == -22 and b"ring average" in L.gop_last_error()
