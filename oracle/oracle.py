"""ctypes front end of the C restatement in oracle/gop_oracle.c.

TEST INFRASTRUCTURE ONLY: the checker that tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg use.  Arrays follow the reference layout
([field][i][j][k], k fastest, ghost-extended by 4 + 1 per axis).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgop_oracle.so"

_dp = C.POINTER(C.c_double)


class _Desc(C.Structure):
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("coord", C.c_int),
        ("x1", _dp), ("x2", _dp), ("x3", _dp),
        ("gamma", C.c_double), ("cfl", C.c_double), ("ca", C.c_double),
        ("pdmb", C.c_double), ("rho_floor", C.c_double), ("p_floor", C.c_double),
        ("bc", C.c_char * 6),
    ]


def build() -> Path:
    """Compiles the restatement (no reference tree needed)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "restatement"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.og_create.restype = C.c_void_p
        L.og_create.argtypes = [C.POINTER(_Desc)]
        L.og_destroy.argtypes = [C.c_void_p]
        L.og_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_double, C.c_double]
        L.og_prepare.argtypes = [C.c_void_p, C.c_int]
        L.og_run.argtypes = [C.c_void_p, C.c_int]
        L.og_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.og_get_stage.argtypes = [C.c_void_p, _dp, _dp, _dp]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


# physical constants of the reference (src/config.c:82-90)
REF_PARAMS = dict(gamma=5.0 / 3.0, cfl=0.3, ca=10.0, pdmb=1.0,
                  rho_floor=0.00316227, p_floor=0.000316227)


class Oracle:
    """One single-domain oracle instance."""

    def __init__(self, n, x1, x2, x3, coord=0, bc="pppppp", **params):
        p = dict(REF_PARAMS)
        p.update(params)
        self.n = tuple(int(v) for v in n)
        self.N = tuple(v + 9 for v in self.n)
        self._x = [np.ascontiguousarray(x, dtype=np.float64) for x in (x1, x2, x3)]
        for a in range(3):
            if self._x[a].shape != (self.N[a],):
                raise ValueError(f"x{a + 1} must have {self.N[a]} points")
        d = _Desc(self.n[0], self.n[1], self.n[2], coord,
                  _ptr(self._x[0]), _ptr(self._x[1]), _ptr(self._x[2]),
                  p["gamma"], p["cfl"], p["ca"], p["pdmb"], p["rho_floor"],
                  p["p_floor"], bc.encode())
        self._h = lib().og_create(C.byref(d))
        if not self._h:
            raise ValueError("og_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().og_destroy(h)
            self._h = None

    def _shape(self, nf):
        return (nf,) + self.N

    def set_state(self, W, B, Wp=None, Bp=None, time=0.0, dt0=0.0):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self._shape(6))
        B = np.ascontiguousarray(B, dtype=np.float64).reshape(self._shape(3))
        Wp = None if Wp is None else np.ascontiguousarray(Wp, dtype=np.float64).reshape(self._shape(6))
        Bp = None if Bp is None else np.ascontiguousarray(Bp, dtype=np.float64).reshape(self._shape(3))
        lib().og_set_state(self._h, _ptr(W), _ptr(B), _ptr(Wp), _ptr(Bp), time, dt0)

    def prepare(self, restart=False):
        lib().og_prepare(self._h, int(restart))

    def run(self, nsteps):
        lib().og_run(self._h, int(nsteps))

    def state(self):
        W = np.zeros(self._shape(6))
        B = np.zeros(self._shape(3))
        Wp = np.zeros(self._shape(6))
        Bp = np.zeros(self._shape(3))
        s = np.zeros(5)
        lib().og_get_state(self._h, _ptr(W), _ptr(B), _ptr(Wp), _ptr(Bp), _ptr(s))
        return dict(W=W, B=B, Wp=Wp, Bp=Bp, time=s[0], dt=s[1], dt0=s[2],
                    divb=s[3], steps=int(s[4]))

    def stage(self):
        Wh = np.zeros(self._shape(6))
        Bh = np.zeros(self._shape(3))
        E = np.zeros(self._shape(3))
        lib().og_get_stage(self._h, _ptr(Wh), _ptr(Bh), _ptr(E))
        return dict(Wh=Wh, Bh=Bh, E=E)
