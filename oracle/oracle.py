"""Python handle on the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C restatement of the reference solver's kernel chain
(reference: src/solver.cu), built twice: liborc64.so (FP64) and liborc32.so
(IEEE FP32 without contraction).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this module; the product never imports it.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "fvm-airidynamic-simulator_b200"))
from fvm_b200.abi import SimParams, Ext, Diag, ext_default  # noqa: E402

_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _lib(bits):
    if bits in _LIBS:
        return _LIBS[bits]
    path = os.path.join(HERE, f"liborc{bits}.so")
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    dp = C.POINTER(C.c_double)
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [i, i]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_set_threads.argtypes = [i]
    lib.orc_set_threads.restype = i
    lib.orc_set_params.argtypes = [vp, C.POINTER(SimParams), C.POINTER(Ext)]
    lib.orc_colormap_table.argtypes = [i, C.c_void_p]
    lib.orc_colormap_table.restype = None
    lib.orc_colormap.argtypes = [C.c_void_p, C.c_void_p, C.c_long, i, C.c_float, C.c_float, i, C.c_void_p]
    lib.orc_colormap.restype = None
    lib.orc_reset.argtypes = [vp]
    lib.orc_set_geometry.argtypes = [vp, C.c_void_p, C.c_void_p]
    lib.orc_reinit.argtypes = [vp]
    lib.orc_compute_sdf.argtypes = [vp, C.c_void_p, C.c_void_p]
    lib.orc_update_obstacle.argtypes = [vp]
    lib.orc_step.argtypes = [vp, d]
    lib.orc_compute_dt.argtypes = [vp]
    lib.orc_compute_dt.restype = d
    lib.orc_cfl_maxima.argtypes = [vp, dp, dp]
    for name in ("orc_get_fields", "orc_set_fields"):
        getattr(lib, name).argtypes = [vp] + [C.c_void_p] * 5
    lib.orc_get_primitives.argtypes = [vp] + [C.c_void_p] * 4
    lib.orc_get_mu.argtypes = [vp, C.c_void_p]
    lib.orc_get_geometry.argtypes = [vp, C.c_void_p, C.c_void_p]
    lib.orc_stage1.argtypes = [vp, d, i, C.c_void_p * 5]
    lib.orc_diagnostics.argtypes = [vp, C.POINTER(Diag)]
    lib.orc_shock_standoff.argtypes = [vp]
    lib.orc_shock_standoff.restype = d
    lib.orc_real_size.restype = i
    _LIBS[bits] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    """One solve on the CPU oracle.  `bits` = 64 or 32."""

    def __init__(self, params, ext=None, bits=64, threads=None):
        self.lib = _lib(bits)
        self.bits = bits
        self.nx, self.ny = int(params.nx), int(params.ny)
        self.h = self.lib.orc_create(self.nx, self.ny)
        if not self.h:
            raise ValueError("orc_create failed")
        if threads:
            self.lib.orc_set_threads(int(threads))
        self.params = params
        self.ext = ext if ext is not None else ext_default()
        self.lib.orc_set_params(self.h, C.byref(self.params), C.byref(self.ext))
        self.lib.orc_reset(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.ny, self.nx)

    def set_geometry(self, sdf, ct):
        sdf = np.ascontiguousarray(sdf, dtype=np.float32).reshape(-1)
        ct = np.ascontiguousarray(ct, dtype=np.uint8).reshape(-1)
        self.lib.orc_set_geometry(self.h, _ptr(sdf), _ptr(ct))

    def reinit(self):
        """Freestream + boundary conditions on the current geometry."""
        self.lib.orc_reinit(self.h)

    def compute_sdf(self):
        sdf = np.empty(self.nx * self.ny, np.float32)
        ct = np.empty(self.nx * self.ny, np.uint8)
        self.lib.orc_compute_sdf(self.h, _ptr(sdf), _ptr(ct))
        return sdf.reshape(self.shape), ct.reshape(self.shape)

    def update_obstacle(self, params):
        self.params = params
        self.lib.orc_set_params(self.h, C.byref(self.params), C.byref(self.ext))
        self.lib.orc_update_obstacle(self.h)

    def step(self, dt):
        self.lib.orc_step(self.h, float(dt))

    def compute_dt(self):
        return self.lib.orc_compute_dt(self.h)

    def cfl_maxima(self):
        a, b = C.c_double(), C.c_double()
        self.lib.orc_cfl_maxima(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def fields(self):
        out = [np.empty(self.nx * self.ny, np.float64) for _ in range(5)]
        self.lib.orc_get_fields(self.h, *[_ptr(a) for a in out])
        return np.stack([a.reshape(self.shape) for a in out])

    def set_fields(self, U):
        U = [np.ascontiguousarray(U[k], dtype=np.float64).reshape(-1) for k in range(5)]
        self.lib.orc_set_fields(self.h, *[_ptr(a) for a in U])

    def primitives(self):
        out = [np.empty(self.nx * self.ny, np.float64) for _ in range(4)]
        self.lib.orc_get_primitives(self.h, *[_ptr(a) for a in out])
        return np.stack([a.reshape(self.shape) for a in out])

    def mu(self):
        out = np.empty(self.nx * self.ny, np.float64)
        self.lib.orc_get_mu(self.h, _ptr(out))
        return out.reshape(self.shape)

    def geometry(self):
        sdf = np.empty(self.nx * self.ny, np.float64)
        ct = np.empty(self.nx * self.ny, np.uint8)
        self.lib.orc_get_geometry(self.h, _ptr(sdf), _ptr(ct))
        return sdf.reshape(self.shape), ct.reshape(self.shape)

    def stage1(self, dt, with_ghost=True):
        out = [np.empty(self.nx * self.ny, np.float64) for _ in range(5)]
        arr = (C.c_void_p * 5)(*[a.ctypes.data for a in out])
        self.lib.orc_stage1(self.h, float(dt), 1 if with_ghost else 0, arr)
        return np.stack([a.reshape(self.shape) for a in out])

    def diagnostics(self):
        d = Diag()
        self.lib.orc_diagnostics(self.h, C.byref(d))
        return d

    def shock_standoff(self):
        return self.lib.orc_shock_standoff(self.h)

    def run(self, steps, dt=None, recompute=False):
        """Advance `steps` steps; fixed dt (default: the CFL dt of the start
        state) or, with recompute=True, the CFL dt of each step's start state."""
        if dt is None:
            dt = self.compute_dt()
        for _ in range(steps):
            if recompute:
                dt = self.compute_dt()
            self.step(dt)
        return dt


def colormap_table(cmap):
    """(256, 3) float32 colour table of the renderer's colormap `cmap`."""
    out = np.empty((256, 3), np.float32)
    _lib(32).orc_colormap_table(int(cmap), out.ctypes.data)
    return out


def colormap(field, ct, cmap, lo, hi, fmt=0):
    """Field fragment shader on the CPU: field (float32) and ct (uint8) of the
    same shape -> (..., 4) float32 (fmt 0) or uint8 (fmt 1) RGBA."""
    f = np.ascontiguousarray(field, np.float32)
    c = np.ascontiguousarray(ct, np.uint8)
    out = np.empty(f.shape + (4,), np.float32 if fmt == 0 else np.uint8)
    _lib(32).orc_colormap(f.ctypes.data, c.ctypes.data, f.size, int(cmap), float(lo), float(hi), int(fmt),
                          out.ctypes.data)
    return out
