"""gop_cfl_dt_noalloc: the CFL dt and max|div B| of a state the caller keeps
in device memory, for callers that may not allocate (code between the
capture calls of a CUDA graph, or a serving loop with a fixed memory
reservation).  Its only scratch is a static device array inside the library.

Checked through the C ABI against the instance path (gop_prepare computes the
same two numbers for the state it was given), on two different states in a
row so the second call proves the shared scratch from the first does not
leak into it.  Kept in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative, the tolerance of the plain-path parity tests


def _noalloc(gop, torch, inst, gas, fb):
    d_gas = torch.from_numpy(np.ascontiguousarray(gas)).cuda()
    d_fb = torch.from_numpy(np.ascontiguousarray(fb)).cuda()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    L = gop.lib()
    L.gop_cfl_dt_noalloc.argtypes = [C.POINTER(gop.Desc), C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    rc = L.gop_cfl_dt_noalloc(C.byref(inst.desc), C.c_void_p(d_gas.data_ptr()),
                              C.c_void_p(d_fb.data_ptr()), C.c_void_p(out.data_ptr()),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.gop_last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return out.cpu().numpy(), free0 - free1


def _reference_numbers(gop, n, xs, gas, fb):
    """dt and div B the existing entry points report for this state."""
    inst = gop.Instance(n, *xs)
    inst.upload(gas, fb)
    inst.prepare()
    st = inst.stats()
    inst.close()
    return st["dt0"], st["divb_max"]


def test_noalloc_cfl_dt_matches_instance_path_twice():
    torch = pytest.importorskip("torch")
    import gop

    n = (48, 40, 8)
    xs = [gop.grid_uniform(48, 0.0, 1.0), gop.grid_uniform(40, 0.0, 1.0),
          gop.grid_uniform(8, 0.0, 0.125)]
    a = gop.Instance(n, *xs)
    gas_a, fb_a = a.init_problem(gop.PROBLEM_OT)
    a.upload(gas_a, fb_a)
    a.prepare()
    dt_a, db_a = a.stats()["dt0"], a.stats()["divb_max"]
    a.step(6)
    st_b = a.download(("gas", "face_b"))
    gas_b, fb_b = st_b["gas"], st_b["face_b"]
    dt_b, db_b = _reference_numbers(gop, n, xs, gas_b, fb_b)
    assert dt_a != dt_b

    # call 1: initial state
    out1, grew1 = _noalloc(gop, torch, a, gas_a, fb_a)
    assert abs(out1[0] - dt_a) <= TOL * dt_a, (out1, dt_a)
    assert abs(out1[1] - db_a) <= TOL, (out1, db_a)
    # call 2, right after: evolved state; the scratch left by call 1 must not matter
    out2, grew2 = _noalloc(gop, torch, a, gas_b, fb_b)
    assert abs(out2[0] - dt_b) <= TOL * dt_b, (out2, dt_b)
    assert abs(out2[1] - db_b) <= TOL, (out2, db_b)
    # after the first call the library is loaded: the call itself takes no memory
    assert grew2 == 0


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    import gop

    n = (1025, 4, 4)
    xs = [gop.grid_uniform(1025, 0.0, 1.0), gop.grid_uniform(4, 0.0, 1.0),
          gop.grid_uniform(4, 0.0, 1.0)]
    x = [np.ascontiguousarray(v) for v in xs]
    d = gop.Desc(n[0], n[1], n[2], 0, *(v.ctypes.data_as(C.POINTER(C.c_double)) for v in x),
                 b"pppppp", b"", 0, 0, 0, 0, 0, 0)
    L = gop.lib()
    L.gop_cfl_dt_noalloc.argtypes = [C.POINTER(gop.Desc), C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    rc = L.gop_cfl_dt_noalloc(C.byref(d), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None)
    assert rc == -22
    assert b"static scratch limit" in L.gop_last_error()
