"""ctypes handle on the reference's own FP32 CUDA solver (TEST INFRASTRUCTURE).

oracle/_ref/libfvm_ref.so is the UNMODIFIED reference src/solver.cu plus
oracle/ref_harness.cu, built by oracle/build_ref.sh.  It needs a GPU; tests
use it on the GPU box to pin the oracle and the CUDA library to the
reference's own kernels.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "fvm-airidynamic-simulator_b200"))
from fvm_b200.abi import SimParams  # noqa: E402

REF_LIB = os.path.join(HERE, "_ref", "libfvm_ref.so")
REF_BENCH = os.path.join(HERE, "_ref", "kernel_benchmark")
_lib = None


def available():
    return os.path.exists(REF_LIB)


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(REF_LIB)
        vp, i, f = C.c_void_p, C.c_int, C.c_float
        P = C.POINTER(SimParams)
        lib.ref_create.restype = vp
        lib.ref_create.argtypes = [P]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_steps.argtypes = [vp, P, i, i]
        lib.ref_compute_dt.argtypes = [vp, P]
        lib.ref_compute_dt.restype = f
        lib.ref_read_fields.argtypes = [vp] + [vp] * 5
        lib.ref_write_fields.argtypes = [vp] + [vp] * 5
        lib.ref_read_primitives.argtypes = [vp] + [vp] * 4
        lib.ref_read_geometry.argtypes = [vp, vp, vp]
        lib.ref_max_temperature.argtypes = [vp]
        lib.ref_max_temperature.restype = f
        lib.ref_max_mach.argtypes = [vp]
        lib.ref_max_mach.restype = f
        lib.ref_update_obstacle.argtypes = [vp, P]
        lib.ref_time_steps.argtypes = [vp, P, i, i]
        lib.ref_time_steps.restype = f
        assert lib.ref_sizeof_params() == C.sizeof(SimParams)
        _lib = lib
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class RefSolver:
    def __init__(self, params):
        self.lib = _load()
        self.params = SimParams.from_buffer_copy(params)
        self.nx, self.ny = params.nx, params.ny
        self.h = self.lib.ref_create(C.byref(self.params))

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def steps(self, n, dt=None, recompute=False):
        if dt is not None:
            self.params.dt = dt
        rc = self.lib.ref_steps(self.h, C.byref(self.params), int(n), 1 if recompute else 0)
        assert rc == 0, f"reference step failed: cudaError {rc}"

    def compute_dt(self):
        return self.lib.ref_compute_dt(self.h, C.byref(self.params))

    def fields(self):
        out = [np.empty(self.nx * self.ny, np.float32) for _ in range(5)]
        self.lib.ref_read_fields(self.h, *[_p(a) for a in out])
        return np.stack([a.reshape(self.ny, self.nx) for a in out])

    def write_fields(self, U):
        U = [np.ascontiguousarray(U[k], dtype=np.float32).reshape(-1) for k in range(5)]
        self.lib.ref_write_fields(self.h, *[_p(a) for a in U])

    def primitives(self):
        out = [np.empty(self.nx * self.ny, np.float32) for _ in range(4)]
        self.lib.ref_read_primitives(self.h, *[_p(a) for a in out])
        return np.stack([a.reshape(self.ny, self.nx) for a in out])

    def geometry(self):
        sdf = np.empty(self.nx * self.ny, np.float32)
        ct = np.empty(self.nx * self.ny, np.uint8)
        self.lib.ref_read_geometry(self.h, _p(sdf), _p(ct))
        return sdf.reshape(self.ny, self.nx), ct.reshape(self.ny, self.nx)

    def time_steps(self, warmup, steps):
        return self.lib.ref_time_steps(self.h, C.byref(self.params), int(warmup), int(steps))
