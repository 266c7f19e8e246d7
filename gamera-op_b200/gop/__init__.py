"""Python front end of the B200 MHD step library (ctypes over the C ABI in
include/gamera_op.h).

The CUDA library ``gamera-op_b200/libgamera_op.so`` must be built
(``python gamera-op_b200/build.py``); there is no CPU fallback, so every
entry point raises if it is missing.  Arrays use the reference layout
([field][i][j][k], k fastest, n + 9 points per axis).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parents[1]
LIB_PATH = PKG / "libgamera_op.so"

COORD_CARTESIAN = 0
COORD_SPHERICAL = 2
PREC_FP64 = 0
PREC_MIXED = 1
PROBLEM_OT, PROBLEM_BLAST, PROBLEM_LOOP_CART, PROBLEM_LOOP_SPH = 1, 2, 3, 4
NG = 4

ERRORS = {-22: "EINVAL", -12: "ENOMEM", -5: "ECUDA", -19: "ENODEV", -71: "ESTATE",
          -34: "ENUMERIC", -16: "EBUSY"}

_dp = C.POINTER(C.c_double)


class GopError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Desc(C.Structure):
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("coord", C.c_int),
        ("x1", _dp), ("x2", _dp), ("x3", _dp),
        ("bc", C.c_char * 6),
        ("gem_bc", C.c_char * 6),
        ("precision", C.c_int),
        ("gamma", C.c_double), ("cfl", C.c_double), ("ca", C.c_double),
        ("rho_floor", C.c_double), ("p_floor", C.c_double),
        ("ring_average", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("dt", C.c_double), ("dt0", C.c_double),
        ("divb_max", C.c_double), ("steps", C.c_int64), ("flags", C.c_int32),
        ("reserved", C.c_int32), ("device_bytes", C.c_size_t),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("rho", C.c_double), ("p_in", C.c_double),
        ("p_out", C.c_double), ("radius", C.c_double), ("center", C.c_double * 3),
        ("b", C.c_double * 3), ("v", C.c_double * 3), ("loop", C.c_double * 4),
    ]


class Background(C.Structure):
    _fields_ = [("kind", C.c_int), ("b", C.c_double * 3), ("moment", C.c_double)]


BG_UNIFORM, BG_DIPOLE = 1, 2

_lib = None


def lib():
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built: run python gamera-op_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.gop_create.argtypes = [C.POINTER(Desc), C.POINTER(vp)]
        L.gop_destroy.argtypes = [vp]
        L.gop_footprint.argtypes = [C.POINTER(Desc)]
        L.gop_footprint.restype = C.c_size_t
        L.gop_set_stream.argtypes = [vp, vp]
        L.gop_upload.argtypes = [vp, _dp, _dp, _dp, _dp, C.c_double, C.c_double]
        L.gop_prepare.argtypes = [vp, C.c_int]
        L.gop_step.argtypes = [vp, C.c_int, C.c_double, _dp]
        L.gop_download.argtypes = [vp] + [_dp] * 9
        L.gop_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.gop_last_error.restype = C.c_char_p
        L.gop_kernel_launches.restype = C.c_int64
        L.gop_grid_uniform.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
        L.gop_problem_defaults.argtypes = [C.c_int, C.POINTER(Problem)]
        L.gop_problem_init.argtypes = [C.POINTER(Desc), C.POINTER(Problem), _dp, _dp]
        L.gop_problem_init_device.argtypes = [vp, C.POINTER(Problem)]
        L.gop_set_background.argtypes = [vp, _dp, _dp, _dp, _dp]
        L.gop_background_init.argtypes = [C.POINTER(Desc), C.POINTER(Background), _dp, _dp, _dp, _dp]
        L.gop_set_background_device.argtypes = [vp, C.POINTER(Background)]
        L.gop_get_background.argtypes = [vp, _dp, _dp, _dp, _dp]
        L.gop_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.gop_set_profiling.argtypes = [vp, C.c_int]
        L.gop_set_sweep.argtypes = [vp, C.c_int]
        L.gop_get_launch_order.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.gop_measure_fp64_peak.argtypes = [_dp, vp]
        L.gop_get_profile.argtypes = [vp, _dp, C.POINTER(C.c_int64)]
        L.gop_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
        L.gop_batch_destroy.argtypes = [vp]
        L.gop_batch_step.argtypes = [vp, C.POINTER(C.c_int)]
        L.gop_batch_launch.argtypes = [vp, C.POINTER(C.c_int)]
        L.gop_batch_wait.argtypes = [vp]
        L.gop_batch_set_stream.argtypes = [vp, vp]
        L.gop_batch_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise GopError(rc, lib().gop_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def fp64_peak_tflops(stream_ptr=None) -> float:
    """The device's measured FP64 peak (timed fused multiply-add loop)."""
    v = C.c_double(0.0)
    _check(lib().gop_measure_fp64_peak(C.byref(v), C.c_void_p(stream_ptr) if stream_ptr else None))
    return v.value


def kernel_launches() -> int:
    return int(lib().gop_kernel_launches())


def grid_uniform(n: int, xmin: float, xmax: float) -> np.ndarray:
    x = np.zeros(n + 2 * NG + 1)
    _check(lib().gop_grid_uniform(n, xmin, xmax, _ptr(x)))
    return x


def footprint(n, coord=COORD_CARTESIAN, precision=PREC_FP64) -> int:
    """Device bytes gop_create would allocate for a grid (host-only)."""
    n = tuple(int(v) for v in n)
    xs = [np.linspace(1.0, 2.0, v + 2 * NG + 1) for v in n]
    d = Desc(n[0], n[1], n[2], coord, _ptr(xs[0]), _ptr(xs[1]), _ptr(xs[2]), b"pppppp", b"",
             precision, 0, 0, 0, 0, 0)
    return int(lib().gop_footprint(C.byref(d)))


def problem(kind: int, **over) -> Problem:
    p = Problem()
    lib().gop_problem_defaults(kind, C.byref(p))
    for k, v in over.items():
        if isinstance(v, (list, tuple, np.ndarray)):
            arr = getattr(p, k)
            for t, val in enumerate(v):
                arr[t] = val
        else:
            setattr(p, k, v)
    return p


def _contig(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != shape:
        a = a.reshape(shape)
    return a


class Instance:
    """One single-domain grid advanced on the GPU."""

    def __init__(self, n, x1, x2, x3, coord=COORD_CARTESIAN, bc="pppppp",
                 precision=PREC_FP64, gamma=0.0, cfl=0.0, ca=0.0, rho_floor=0.0,
                 p_floor=0.0, gem_bc="", ring_average=False):
        self.n = tuple(int(v) for v in n)
        self.N = tuple(v + 2 * NG + 1 for v in self.n)
        self._x = [np.ascontiguousarray(x, dtype=np.float64) for x in (x1, x2, x3)]
        self.coord, self.bc, self.precision = coord, bc, precision
        self.desc = Desc(self.n[0], self.n[1], self.n[2], coord,
                         _ptr(self._x[0]), _ptr(self._x[1]), _ptr(self._x[2]),
                         bc.encode(), gem_bc.encode(), precision, gamma, cfl, ca, rho_floor,
                         p_floor, int(bool(ring_average)))
        h = C.c_void_p()
        _check(lib().gop_create(C.byref(self.desc), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().gop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, nf):
        return (nf,) + self.N

    def footprint(self) -> int:
        return int(lib().gop_footprint(C.byref(self.desc)))

    def set_stream(self, stream_ptr: int):
        _check(lib().gop_set_stream(self._h, C.c_void_p(stream_ptr)))

    def init_problem(self, kind: int, out=None, **over):
        """Builds a problem's initial state on the host (into ``out`` =
        (gas, face_b) arrays when given, zeroed first) and returns it."""
        if out is None:
            gas, fb = np.zeros(self.shape(6)), np.zeros(self.shape(3))
        else:
            gas, fb = out
            if gas.shape != self.shape(6) or fb.shape != self.shape(3):
                raise ValueError("init_problem: wrong output shapes")
            gas.fill(0.0)
            fb.fill(0.0)
        p = problem(kind, **over)
        _check(lib().gop_problem_init(C.byref(self.desc), C.byref(p), _ptr(gas), _ptr(fb)))
        return gas, fb

    def init_problem_device(self, kind: int, **over):
        """Builds a problem's initial state on the device, in place of
        init_problem + upload (gop_problem_init_device); prepare follows."""
        p = problem(kind, **over)
        _check(lib().gop_problem_init_device(self._h, C.byref(p)))

    def background_fields(self, kind: int, b=(0.0, 0.0, 0.0), moment=1.0) -> dict:
        """A built-in background field on this instance's grid (see the
        module function background_fields)."""
        return _background(self.desc, self.N, kind, b, moment)

    def set_background(self, fields):
        """Installs a background field (the arrays of background_fields, or
        None to remove it); prepare must follow."""
        if fields is None:
            _check(lib().gop_set_background(self._h, None, None, None, None))
            return
        arr = [_contig(fields[k], self.shape(nf)) for k, nf in
               (("b0", 3), ("lorentz", 3), ("b0_face", 9), ("b0_edge", 9))]
        _check(lib().gop_set_background(self._h, *[_ptr(a) for a in arr]))

    def set_background_device(self, kind: int, b=(0.0, 0.0, 0.0), moment=1.0):
        """Builds a built-in background field on the device, straight into
        the instance (gop_set_background_device); prepare must follow."""
        bg = Background(kind, (C.c_double * 3)(*b), moment)
        _check(lib().gop_set_background_device(self._h, C.byref(bg)))

    def get_background(self) -> dict:
        """The instance's background field in the layout of background_fields."""
        out = {"b0": np.zeros(self.shape(3)), "lorentz": np.zeros(self.shape(3)),
               "b0_face": np.zeros(self.shape(9)), "b0_edge": np.zeros(self.shape(9))}
        _check(lib().gop_get_background(self._h, _ptr(out["b0"]), _ptr(out["lorentz"]),
                                        _ptr(out["b0_face"]), _ptr(out["b0_edge"])))
        return out

    def upload(self, gas, face_b, gas_p=None, face_b_p=None, time=0.0, dt0=0.0):
        gas = _contig(gas, self.shape(6))
        face_b = _contig(face_b, self.shape(3))
        gas_p = None if gas_p is None else _contig(gas_p, self.shape(6))
        face_b_p = None if face_b_p is None else _contig(face_b_p, self.shape(3))
        _check(lib().gop_upload(self._h, _ptr(gas), _ptr(face_b), _ptr(gas_p), _ptr(face_b_p),
                                time, dt0))

    def prepare(self, restart=False):
        _check(lib().gop_prepare(self._h, int(bool(restart))))

    def step(self, nsteps=1, time_stop=math.inf, sync=True):
        t = C.c_double(0.0)
        ts = time_stop if math.isfinite(time_stop) else 1e300
        _check(lib().gop_step(self._h, int(nsteps), ts, C.byref(t) if sync else None))
        return t.value if sync else None

    def download(self, which=("gas", "face_b"), out=None):
        """Copies fields back; ``out`` may supply destination arrays (e.g.
        pinned host buffers) keyed by field name."""
        names = ["gas", "face_b", "gas_h", "gas_p", "face_b_h", "face_b_p", "mags",
                 "mags_h", "mags_p"]
        nf = {"gas": 6, "gas_h": 6, "gas_p": 6}
        out = dict(out or {})
        args = []
        for nm in names:
            if nm in which:
                shape = self.shape(nf.get(nm, 3))
                if nm not in out:
                    out[nm] = np.zeros(shape)
                if out[nm].shape != shape or not out[nm].flags.c_contiguous or out[nm].dtype != np.float64:
                    raise ValueError(f"{nm}: need a C-contiguous float64 array of shape {shape}")
                args.append(_ptr(out[nm]))
            else:
                args.append(None)
        _check(lib().gop_download(self._h, *args))
        return out

    GROUPS = ("begin", "ab2", "c2c", "emf", "flux", "update", "ghost", "end")
    TUNE_SLOTS = ("ab2", "c2c_i", "c2c_j", "c2c_k", "emf_i", "emf_j", "emf_k", "flux_i",
                  "flux_j", "flux_k", "update")

    def autotune(self, reps=3) -> dict:
        """Times candidate block shapes per launch on the current state and
        keeps the fastest; returns the chosen candidate index per launch."""
        out = (C.c_int * len(self.TUNE_SLOTS))()
        _check(lib().gop_autotune(self._h, int(reps), out))
        return dict(zip(self.TUNE_SLOTS, list(out)))

    def launch_order(self) -> dict:
        """Axis order of the flux and EMF launches (chosen by autotune)."""
        f, e = (C.c_int * 3)(), (C.c_int * 3)()
        _check(lib().gop_get_launch_order(self._h, f, e))
        return {"flux": list(f), "emf": list(e)}

    def set_sweep(self, on: bool):
        """Face fluxes by the tile-staged sweep kernels (default) or the
        per-face kernels."""
        _check(lib().gop_set_sweep(self._h, int(bool(on))))

    def set_profiling(self, on: bool):
        _check(lib().gop_set_profiling(self._h, int(bool(on))))

    def profile(self) -> dict:
        """Summed event-timed milliseconds and occurrence count per kernel group."""
        ms = np.zeros(len(self.GROUPS))
        cnt = (C.c_int64 * len(self.GROUPS))()
        _check(lib().gop_get_profile(self._h, _ptr(ms), cnt))
        return {g: (float(ms[i]), int(cnt[i])) for i, g in enumerate(self.GROUPS)}

    def stats(self) -> dict:
        s = Stats()
        _check(lib().gop_get_stats(self._h, C.byref(s)))
        return dict(time=s.time, dt=s.dt, dt0=s.dt0, divb_max=s.divb_max, steps=s.steps,
                    flags=s.flags, device_bytes=s.device_bytes)


class Batch:
    """Several prepared instances (any sizes, geometries, boundary kinds and
    precisions) advanced together: one step of every member (its own launch
    sequence) is captured in one CUDA graph on up to 16 parallel branches and
    replayed max(steps) times; each member stops after its own step count.
    A member prepared again with other kernels (a live entropy channel, a
    background field, new block shapes) makes the next launch capture the
    graph again."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.handle for m in self.members])
        h = C.c_void_p()
        _check(lib().gop_batch_create(arr, len(self.members), C.byref(h)))
        self._h = h

    def step(self, steps):
        steps = list(steps)
        if len(steps) != len(self.members):
            raise ValueError(f"{len(steps)} step counts for {len(self.members)} members")
        arr = (C.c_int * len(self.members))(*[int(s) for s in steps])
        _check(lib().gop_batch_step(self._h, arr))

    def launch(self, steps):
        """Enqueues the steps and returns at once (see wait)."""
        steps = list(steps)
        if len(steps) != len(self.members):
            raise ValueError(f"{len(steps)} step counts for {len(self.members)} members")
        arr = (C.c_int * len(self.members))(*[int(s) for s in steps])
        _check(lib().gop_batch_launch(self._h, arr))

    def wait(self):
        _check(lib().gop_batch_wait(self._h))

    def set_stream(self, stream_ptr: int):
        _check(lib().gop_batch_set_stream(self._h, C.c_void_p(stream_ptr)))

    def autotune(self, reps=3) -> dict:
        """Chooses block shapes for the batched launches (members must be
        freshly prepared); returns the candidate index per launch."""
        out = (C.c_int * len(Instance.TUNE_SLOTS))()
        _check(lib().gop_batch_autotune(self._h, int(reps), out))
        return dict(zip(Instance.TUNE_SLOTS, list(out)))

    def close(self):
        if getattr(self, "_h", None):
            lib().gop_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def problem_state(n, xs, kind, coord=COORD_CARTESIAN, **over):
    """Host-only: initial (gas, face_b) arrays of a problem on a grid."""
    n = tuple(int(v) for v in n)
    N = tuple(v + 2 * NG + 1 for v in n)
    xs = [np.ascontiguousarray(x, dtype=np.float64) for x in xs]
    d = Desc(n[0], n[1], n[2], coord, _ptr(xs[0]), _ptr(xs[1]), _ptr(xs[2]), b"pppppp",
             b"", 0, 0, 0, 0, 0, 0)
    gas = np.zeros((6,) + N)
    fb = np.zeros((3,) + N)
    p = problem(kind, **over)
    _check(lib().gop_problem_init(C.byref(d), C.byref(p), _ptr(gas), _ptr(fb)))
    return gas, fb


def _background(desc, N, kind, b, moment):
    bg = Background(kind, (C.c_double * 3)(*b), moment)
    out = {"b0": np.zeros((3,) + N), "lorentz": np.zeros((3,) + N),
           "b0_face": np.zeros((9,) + N), "b0_edge": np.zeros((9,) + N)}
    _check(lib().gop_background_init(C.byref(desc), C.byref(bg), _ptr(out["b0"]),
                                     _ptr(out["lorentz"]), _ptr(out["b0_face"]),
                                     _ptr(out["b0_edge"])))
    return out


def background_fields(n, xs, kind, coord=COORD_CARTESIAN, b=(0.0, 0.0, 0.0), moment=1.0):
    """Host-only: a built-in background field B0 (BG_UNIFORM with field b,
    or BG_DIPOLE scaled by moment) integrated over a grid
    (gop_background_init): arrays b0 (3 fields), lorentz (3), b0_face (9),
    b0_edge (9), as Instance.set_background takes them."""
    n = tuple(int(v) for v in n)
    N = tuple(v + 2 * NG + 1 for v in n)
    xs = [np.ascontiguousarray(x, dtype=np.float64) for x in xs]
    d = Desc(n[0], n[1], n[2], coord, _ptr(xs[0]), _ptr(xs[1]), _ptr(xs[2]), b"pppppp",
             b"", 0, 0, 0, 0, 0, 0)
    return _background(d, N, kind, b, moment)


def make(kind, n, domain=None, coord=None, bc="pppppp", precision=PREC_FP64, **over):
    """Creates an instance for one of the reference problems on the default
    uniform grid and uploads its initial state (not yet prepared)."""
    if coord is None:
        coord = COORD_SPHERICAL if kind == PROBLEM_LOOP_SPH else COORD_CARTESIAN
    if domain is None:
        domain = {
            PROBLEM_OT: (0.0, 1.0, 0.0, 1.0, 0.0, 1.0),
            PROBLEM_BLAST: (-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
            PROBLEM_LOOP_CART: (-2.0, 2.0, -2.0, 2.0, -2.0, 2.0),
            PROBLEM_LOOP_SPH: (1.0, 2.0, 0.25 * math.pi, 0.75 * math.pi,
                               -0.25 * math.pi, 0.25 * math.pi),
        }[kind]
    xs = [grid_uniform(n[a], domain[2 * a], domain[2 * a + 1]) for a in range(3)]
    phys = {k: over.pop(k) for k in ("gamma", "cfl", "ca", "rho_floor", "p_floor") if k in over}
    inst = Instance(n, *xs, coord=coord, bc=bc, precision=precision, **phys)
    gas, fb = inst.init_problem(kind, **over)
    inst.upload(gas, fb)
    return inst
