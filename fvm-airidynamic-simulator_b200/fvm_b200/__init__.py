"""fvm_b200 -- Python handle on the B200 compressible-flow hot path.

A thin ctypes layer over the C ABI in include/fvm_b200.h (libfvm_b200.so,
built in-tree for sm_100a).  `Solver` mirrors the reference's host class
`CFDSolver` (reference: src/include/solver.cuh:22-257): initialize, reset,
step, updateObstacleGeometry, computeStableTimeStep, field readback and the
statistics calls, with the same argument meaning.  Errors raise FvmError
instead of exiting.  There is no CPU fallback: without the CUDA library or a
device every call fails.
"""
import ctypes as C
import os

import numpy as np

from .abi import (SimParams, Ext, Diag, KernelTime, Result, ServerStats, Shedding, STATUS, params_default, compute_derived,
                  ext_default, workload)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfvm_b200.so")

# Every symbol include/fvm_b200.h declares.
EXPORTS = [
    "fvm_last_error", "fvm_params_compute_derived", "fvm_params_default", "fvm_ext_default",
    "fvm_create", "fvm_destroy", "fvm_set_stream", "fvm_initialize", "fvm_resize", "fvm_reset",
    "fvm_update_obstacle", "fvm_set_ext", "fvm_step", "fvm_steps", "fvm_compute_dt", "fvm_queue_dt",
    "fvm_read_dt", "fvm_synchronize", "fvm_get_cell_types", "fvm_get_sdf", "fvm_read_fields",
    "fvm_read_region", "fvm_read_region_geometry",
    "fvm_write_fields", "fvm_read_primitives", "fvm_field_to_device", "fvm_set_display_field",
    "fvm_cell_types_to_device",
    "fvm_vector_arrows", "fvm_max_temperature", "fvm_max_mach", "fvm_memory_usage", "fvm_gpu_mem_info",
    "fvm_diagnostics", "fvm_shock_standoff", "fvm_set_kernel_timing", "fvm_kernel_times",
    "fvm_launch_count", "fvm_batch_create", "fvm_batch_destroy", "fvm_batch_set_stream", "fvm_batch_add",
    "fvm_batch_remove", "fvm_batch_count", "fvm_batch_step", "fvm_batch_synchronize", "fvm_batch_instance",
    "fvm_batch_read_fields", "fvm_batch_diagnostics", "fvm_batch_nonfinite_count", "fvm_batch_memory_usage",
    "fvm_batch_launch_count",
    "fvm_batch_instance_bytes", "fvm_batch_retire", "fvm_batch_trim", "fvm_server_create", "fvm_server_submit",
    "fvm_server_poll", "fvm_server_wait", "fvm_server_drain", "fvm_server_get_stats", "fvm_server_destroy",
    "fvm_state_max_noalloc", "fvm_shedding_stats", "fvm_colormap_to_device", "fvm_colormap_table",
    "fvm_save_checkpoint", "fvm_load_checkpoint", "fvm_checkpoint_info", "fvm_autotune", "fvm_get_tune",
    "fvm_set_tune", "fvm_nonfinite_count", "fvm_debug_stage1", "fvm_debug_ghost_table",
    "fvm_debug_wait_timeout", "fvm_build_info",
]


class FvmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{STATUS.get(code, code)}] {msg}")
        self.code = code


_lib = None


def load_library(path=None):
    """Load libfvm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FvmError(8, f"CUDA library not built: {path} (run __graft_entry__.build())")
    lib = C.CDLL(path)
    vp, i, f, sz = C.c_void_p, C.c_int, C.c_float, C.c_size_t
    fp = C.POINTER(C.c_float)
    Pp = C.POINTER(SimParams)
    lib.fvm_last_error.restype = C.c_char_p
    lib.fvm_build_info.restype = C.c_char_p
    lib.fvm_params_default.argtypes = [Pp]
    lib.fvm_params_default.restype = None
    lib.fvm_params_compute_derived.argtypes = [Pp]
    lib.fvm_params_compute_derived.restype = None
    lib.fvm_ext_default.argtypes = [C.POINTER(Ext)]
    lib.fvm_ext_default.restype = None
    lib.fvm_create.argtypes = [C.POINTER(vp)]
    lib.fvm_destroy.argtypes = [vp]
    lib.fvm_set_stream.argtypes = [vp, vp]
    lib.fvm_initialize.argtypes = [vp, Pp, C.POINTER(Ext)]
    lib.fvm_resize.argtypes = [vp, i, i]
    lib.fvm_reset.argtypes = [vp, Pp]
    lib.fvm_update_obstacle.argtypes = [vp, Pp]
    lib.fvm_set_ext.argtypes = [vp, C.POINTER(Ext)]
    lib.fvm_step.argtypes = [vp, Pp]
    lib.fvm_steps.argtypes = [vp, Pp, i]
    lib.fvm_compute_dt.argtypes = [vp, Pp, fp]
    lib.fvm_queue_dt.argtypes = [vp, Pp]
    lib.fvm_read_dt.argtypes = [vp, Pp, fp]
    lib.fvm_synchronize.argtypes = [vp]
    lib.fvm_get_cell_types.argtypes = [vp, vp]
    lib.fvm_get_sdf.argtypes = [vp, vp]
    lib.fvm_read_fields.argtypes = [vp] + [vp] * 5
    lib.fvm_read_region.argtypes = [vp, i, i, i, i] + [vp] * 5
    lib.fvm_read_region_geometry.argtypes = [vp, i, i, i, i, vp, vp]
    lib.fvm_write_fields.argtypes = [vp] + [vp] * 5
    lib.fvm_read_primitives.argtypes = [vp] + [vp] * 4
    lib.fvm_field_to_device.argtypes = [vp, i, vp]
    lib.fvm_set_display_field.argtypes = [vp, i, vp]
    lib.fvm_colormap_to_device.argtypes = [vp, i, i, f, f, vp, i]
    lib.fvm_colormap_table.argtypes = [i, vp]
    lib.fvm_save_checkpoint.argtypes = [vp, Pp, C.c_char_p]
    lib.fvm_load_checkpoint.argtypes = [vp, C.c_char_p, Pp]
    lib.fvm_checkpoint_info.argtypes = [C.c_char_p, Pp, C.POINTER(Ext)]
    lib.fvm_cell_types_to_device.argtypes = [vp, vp]
    lib.fvm_vector_arrows.argtypes = [vp, vp, i, i, f, f, f, f, C.POINTER(i)]
    lib.fvm_max_temperature.argtypes = [vp, fp]
    lib.fvm_max_mach.argtypes = [vp, fp]
    lib.fvm_memory_usage.argtypes = [vp, C.POINTER(sz)]
    lib.fvm_gpu_mem_info.argtypes = [C.POINTER(sz), C.POINTER(sz)]
    lib.fvm_diagnostics.argtypes = [vp, C.POINTER(Diag)]
    lib.fvm_shock_standoff.argtypes = [vp, C.POINTER(C.c_double)]
    lib.fvm_set_kernel_timing.argtypes = [vp, i]
    lib.fvm_kernel_times.argtypes = [vp, C.POINTER(KernelTime), i, C.POINTER(i)]
    lib.fvm_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.fvm_debug_stage1.argtypes = [vp, f, i] + [vp] * 5
    lib.fvm_autotune.argtypes = [vp, Pp, i, fp]
    lib.fvm_batch_create.argtypes = [C.POINTER(vp), C.POINTER(Ext)]
    lib.fvm_batch_destroy.argtypes = [vp]
    lib.fvm_batch_set_stream.argtypes = [vp, vp]
    lib.fvm_batch_add.argtypes = [vp, Pp, C.POINTER(i)]
    lib.fvm_batch_remove.argtypes = [vp, i]
    lib.fvm_batch_count.argtypes = [vp, C.POINTER(i)]
    lib.fvm_batch_step.argtypes = [vp, i]
    lib.fvm_batch_synchronize.argtypes = [vp]
    lib.fvm_batch_instance.argtypes = [vp, i, Pp]
    lib.fvm_batch_read_fields.argtypes = [vp, i] + [vp] * 5
    lib.fvm_batch_diagnostics.argtypes = [vp, i, C.POINTER(Diag)]
    lib.fvm_batch_nonfinite_count.argtypes = [vp, i, C.POINTER(C.c_ulonglong)]
    lib.fvm_batch_memory_usage.argtypes = [vp, C.POINTER(sz)]
    lib.fvm_batch_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.fvm_batch_instance_bytes.argtypes = [i, i]
    lib.fvm_batch_instance_bytes.restype = sz
    lib.fvm_state_max_noalloc.argtypes = [vp, i, i, sz, sz, i, fp, vp]
    dp = C.POINTER(C.c_double)
    lib.fvm_shedding_stats.argtypes = [dp, dp, dp, i, C.c_double, C.c_double, C.POINTER(Shedding)]
    lib.fvm_batch_retire.argtypes = [vp, i]
    lib.fvm_batch_trim.argtypes = [vp, sz, C.POINTER(sz)]
    lib.fvm_server_create.argtypes = [C.POINTER(vp), C.POINTER(Ext), sz, i, i]
    lib.fvm_server_submit.argtypes = [vp, Pp, i, vp, vp, vp, vp, vp, C.POINTER(C.c_longlong)]
    lib.fvm_server_poll.argtypes = [vp, C.POINTER(Result), i, C.POINTER(i)]
    lib.fvm_server_wait.argtypes = [vp, C.c_longlong, C.c_double, C.POINTER(Result)]
    lib.fvm_server_drain.argtypes = [vp, C.c_double]
    lib.fvm_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
    lib.fvm_server_destroy.argtypes = [vp]
    lib.fvm_get_tune.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    lib.fvm_set_tune.argtypes = [vp, i, i, i]
    lib.fvm_nonfinite_count.argtypes = [vp, C.POINTER(C.c_ulonglong), i]
    lib.fvm_debug_wait_timeout.argtypes = [vp, C.c_longlong]
    lib.fvm_debug_ghost_table.argtypes = [vp, vp, i, C.POINTER(i)]
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        raise FvmError(rc, _lib.fvm_last_error().decode(errors="replace"))


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Solver:
    """One solve on the GPU (the reference CFDSolver's public surface)."""

    def __init__(self, params=None, ext=None):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.fvm_create(C.byref(h)))
        self.h = h
        self.params = None
        self.ext = None
        if params is not None:
            self.initialize(params, ext)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # lifecycle -----------------------------------------------------------
    def initialize(self, params, ext=None):
        self.params = params
        self.ext = ext if ext is not None else ext_default()
        _check(self.lib.fvm_initialize(self.h, C.byref(self.params), C.byref(self.ext)))

    def reset(self, params=None):
        if params is not None:
            self.params = params
        _check(self.lib.fvm_reset(self.h, C.byref(self.params)))

    def resize(self, nx, ny):
        _check(self.lib.fvm_resize(self.h, int(nx), int(ny)))

    def update_obstacle(self, params):
        self.params = params
        _check(self.lib.fvm_update_obstacle(self.h, C.byref(self.params)))

    def set_ext(self, ext):
        self.ext = ext
        _check(self.lib.fvm_set_ext(self.h, C.byref(self.ext)))

    def set_stream(self, stream_handle):
        _check(self.lib.fvm_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    # stepping --------------------------------------------------------------
    def step(self, n=1):
        _check(self.lib.fvm_steps(self.h, C.byref(self.params), int(n)))

    def compute_dt(self):
        dt = C.c_float()
        _check(self.lib.fvm_compute_dt(self.h, C.byref(self.params), C.byref(dt)))
        return dt.value

    def synchronize(self):
        _check(self.lib.fvm_synchronize(self.h))

    @property
    def shape(self):
        return (self.params.ny, self.params.nx)

    # readback --------------------------------------------------------------
    def fields(self):
        n = self.params.nx * self.params.ny
        out = [np.empty(n, np.float32) for _ in range(5)]
        _check(self.lib.fvm_read_fields(self.h, *[_p(a) for a in out]))
        return np.stack([a.reshape(self.shape) for a in out])

    def read_region(self, i0, j0, w, h):
        """Conserved fields of the window [i0, i0+w) x [j0, j0+h): (5, h, w) float32."""
        out = [np.empty(w * h, np.float32) for _ in range(5)]
        _check(self.lib.fvm_read_region(self.h, int(i0), int(j0), int(w), int(h), *[_p(a) for a in out]))
        return np.stack([a.reshape(h, w) for a in out])

    def read_region_geometry(self, i0, j0, w, h):
        """(sdf float32 (h, w), cell classes uint8 (h, w)) of the window."""
        sdf = np.empty(w * h, np.float32)
        ct = np.empty(w * h, np.uint8)
        _check(self.lib.fvm_read_region_geometry(self.h, int(i0), int(j0), int(w), int(h), _p(sdf), _p(ct)))
        return sdf.reshape(h, w), ct.reshape(h, w)

    def write_fields(self, U):
        U = [np.ascontiguousarray(U[k], dtype=np.float32).reshape(-1) for k in range(5)]
        _check(self.lib.fvm_write_fields(self.h, *[_p(a) for a in U]))

    def primitives(self):
        n = self.params.nx * self.params.ny
        out = [np.empty(n, np.float32) for _ in range(4)]
        _check(self.lib.fvm_read_primitives(self.h, *[_p(a) for a in out]))
        return np.stack([a.reshape(self.shape) for a in out])

    def cell_types(self):
        out = np.empty(self.params.nx * self.params.ny, np.uint8)
        _check(self.lib.fvm_get_cell_types(self.h, _p(out)))
        return out.reshape(self.shape)

    def sdf(self):
        out = np.empty(self.params.nx * self.params.ny, np.float32)
        _check(self.lib.fvm_get_sdf(self.h, _p(out)))
        return out.reshape(self.shape)

    def field_to_device(self, kind, dev_ptr):
        _check(self.lib.fvm_field_to_device(self.h, int(kind), C.c_void_p(dev_ptr)))

    def set_display_field(self, kind, dev_ptr):
        """Register (or, with dev_ptr 0 / None, unregister) a device buffer
        that every step's last passes fill with derived field `kind`."""
        _check(self.lib.fvm_set_display_field(self.h, int(kind), C.c_void_p(dev_ptr or None)))

    def save_checkpoint(self, path):
        """Write the solve (state, parameters, time-step state) to a checkpoint file."""
        _check(self.lib.fvm_save_checkpoint(self.h, C.byref(self.params), os.fsencode(path)))

    def load_checkpoint(self, path):
        """Restore a checkpoint into this handle; returns (and adopts) the saved parameters."""
        p = SimParams()
        _check(self.lib.fvm_load_checkpoint(self.h, os.fsencode(path), C.byref(p)))
        self.params = p
        return p

    def colormap_to_device(self, kind, colormap, min_val, max_val, dev_ptr, fmt=0):
        """RGBA image of a derived field into a device buffer (fmt 0: float4, 1: uchar4 per cell)."""
        _check(self.lib.fvm_colormap_to_device(self.h, int(kind), int(colormap), float(min_val), float(max_val),
                                               C.c_void_p(dev_ptr), int(fmt)))

    def cell_types_to_device(self, dev_ptr):
        _check(self.lib.fvm_cell_types_to_device(self.h, C.c_void_p(dev_ptr)))

    def vector_arrows(self, dev_ptr, max_vertices, step, u_inf, max_len, head_angle, head_len):
        n = C.c_int()
        _check(self.lib.fvm_vector_arrows(self.h, C.c_void_p(dev_ptr), int(max_vertices), int(step),
                                          float(u_inf), float(max_len), float(head_angle), float(head_len),
                                          C.byref(n)))
        return n.value

    # statistics / diagnostics -------------------------------------------
    def max_temperature(self):
        v = C.c_float()
        _check(self.lib.fvm_max_temperature(self.h, C.byref(v)))
        return v.value

    def max_mach(self):
        v = C.c_float()
        _check(self.lib.fvm_max_mach(self.h, C.byref(v)))
        return v.value

    def memory_usage(self):
        v = C.c_size_t()
        _check(self.lib.fvm_memory_usage(self.h, C.byref(v)))
        return v.value

    def diagnostics(self):
        d = Diag()
        _check(self.lib.fvm_diagnostics(self.h, C.byref(d)))
        return d

    def shock_standoff(self):
        v = C.c_double()
        _check(self.lib.fvm_shock_standoff(self.h, C.byref(v)))
        return v.value

    def set_kernel_timing(self, on):
        _check(self.lib.fvm_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        cap = 32
        arr = (KernelTime * cap)()
        n = C.c_int()
        _check(self.lib.fvm_kernel_times(self.h, arr, cap, C.byref(n)))
        return {arr[k].name.decode(): (arr[k].launches, arr[k].total_ms) for k in range(min(n.value, cap))}

    def debug_stage1(self, dt, with_ghost=True):
        n = self.params.nx * self.params.ny
        out = [np.empty(n, np.float32) for _ in range(5)]
        _check(self.lib.fvm_debug_stage1(self.h, float(dt), 1 if with_ghost else 0, *[_p(x) for x in out]))
        return np.stack([x.reshape(self.shape) for x in out])

    def debug_ghost_table(self):
        n = C.c_int()
        _check(self.lib.fvm_debug_ghost_table(self.h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 7), np.int32)
        _check(self.lib.fvm_debug_ghost_table(self.h, _p(out), n.value, C.byref(n)))
        return out[:n.value]

    def autotune(self, steps=6):
        """Pick the fastest launch tuning for this grid class (see fvm_autotune)."""
        ms = C.c_float()
        _check(self.lib.fvm_autotune(self.h, C.byref(self.params), int(steps), C.byref(ms)))
        return ms.value

    def nonfinite_count(self, reset=False):
        """(cell, step) pairs that came out of a step non-finite (see fvm_nonfinite_count)."""
        v = C.c_ulonglong()
        _check(self.lib.fvm_nonfinite_count(self.h, C.byref(v), 1 if reset else 0))
        return v.value

    def set_tune(self, threads, ring, rows):
        """Pin the launch tuning (see fvm_set_tune)."""
        _check(self.lib.fvm_set_tune(self.h, int(threads), int(ring), int(rows)))

    def tune(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.fvm_get_tune(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def launch_count(self):
        v = C.c_longlong()
        _check(self.lib.fvm_launch_count(self.h, C.byref(v)))
        return v.value


class Batch:
    """Many independent solves advanced together (fvm_batch_* in the C ABI)."""

    def __init__(self, ext=None):
        self.lib = load_library()
        h = C.c_void_p()
        self.ext = ext if ext is not None else ext_default()
        _check(self.lib.fvm_batch_create(C.byref(h), C.byref(self.ext)))
        self.h = h
        self.shapes = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        _check(self.lib.fvm_batch_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    def add(self, params):
        i = C.c_int()
        _check(self.lib.fvm_batch_add(self.h, C.byref(params), C.byref(i)))
        self.shapes[i.value] = (params.ny, params.nx)
        return i.value

    def remove(self, id_):
        _check(self.lib.fvm_batch_remove(self.h, int(id_)))
        self.shapes.pop(id_, None)

    def retire(self, id_):
        """Take an instance out but keep its memory for a later add of the same grid size."""
        _check(self.lib.fvm_batch_retire(self.h, int(id_)))
        self.shapes.pop(id_, None)

    def trim(self, keep_bytes=0):
        """Free retired instances until at most keep_bytes stay parked; returns the bytes parked."""
        v = C.c_size_t()
        _check(self.lib.fvm_batch_trim(self.h, int(keep_bytes), C.byref(v)))
        return v.value

    def count(self):
        n = C.c_int()
        _check(self.lib.fvm_batch_count(self.h, C.byref(n)))
        return n.value

    def step(self, n=1):
        _check(self.lib.fvm_batch_step(self.h, int(n)))

    def synchronize(self):
        _check(self.lib.fvm_batch_synchronize(self.h))

    def instance(self, id_):
        p = SimParams()
        _check(self.lib.fvm_batch_instance(self.h, int(id_), C.byref(p)))
        return p

    def fields(self, id_):
        ny, nx = self.shapes[id_]
        out = [np.empty(nx * ny, np.float32) for _ in range(5)]
        _check(self.lib.fvm_batch_read_fields(self.h, int(id_), *[_p(a) for a in out]))
        return np.stack([a.reshape(ny, nx) for a in out])

    def diagnostics(self, id_):
        d = Diag()
        _check(self.lib.fvm_batch_diagnostics(self.h, int(id_), C.byref(d)))
        return d

    def nonfinite_count(self, id_):
        """Non-finite (cell, step) count of one instance (fvm_batch_nonfinite_count)."""
        v = C.c_ulonglong()
        _check(self.lib.fvm_batch_nonfinite_count(self.h, int(id_), C.byref(v)))
        return v.value

    def memory_usage(self):
        v = C.c_size_t()
        _check(self.lib.fvm_batch_memory_usage(self.h, C.byref(v)))
        return v.value

    def launch_count(self):
        v = C.c_longlong()
        _check(self.lib.fvm_batch_launch_count(self.h, C.byref(v)))
        return v.value


class Server:
    """Continuous-batching request loop (fvm_server_* in the C ABI).

    submit() queues a solve and returns a ticket; the final state lands in
    host arrays owned by this object, handed back by wait()/poll() with the
    result record."""

    def __init__(self, ext=None, budget_bytes=150 * 10**9, max_active=0, chunk_steps=64):
        self.lib = load_library()
        self.ext = ext if ext is not None else ext_default()
        h = C.c_void_p()
        _check(self.lib.fvm_server_create(C.byref(h), C.byref(self.ext), int(budget_bytes), int(max_active),
                                          int(chunk_steps)))
        self.h = h
        self.outputs = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, params, steps, keep_fields=True):
        """Queue a solve of `steps` steps; returns its ticket."""
        t = C.c_longlong()
        if keep_fields:
            arrs = [np.empty((params.ny, params.nx), np.float32) for _ in range(5)]
            ptrs = [_p(a) for a in arrs]
        else:
            arrs, ptrs = None, [None] * 5
        _check(self.lib.fvm_server_submit(self.h, C.byref(params), int(steps), *ptrs, C.byref(t)))
        self.outputs[t.value] = arrs
        return t.value

    def _collect(self, r):
        arrs = self.outputs.pop(r.ticket, None)
        fields = np.stack(arrs) if arrs is not None and r.status == 0 else None
        return r, fields

    def wait(self, ticket, timeout_s=-1.0):
        """(Result, fields or None) of one request."""
        r = Result()
        _check(self.lib.fvm_server_wait(self.h, int(ticket), float(timeout_s), C.byref(r)))
        return self._collect(r)

    def poll(self, cap=256):
        """Finished requests not yet collected: list of (Result, fields or None)."""
        buf = (Result * cap)()
        n = C.c_int()
        _check(self.lib.fvm_server_poll(self.h, buf, int(cap), C.byref(n)))
        return [self._collect(Result.from_buffer_copy(buf[k])) for k in range(n.value)]

    def drain(self, timeout_s=-1.0):
        _check(self.lib.fvm_server_drain(self.h, float(timeout_s)))

    def stats(self):
        st = ServerStats()
        _check(self.lib.fvm_server_get_stats(self.h, C.byref(st)))
        return st


CHECKPOINT_MAGIC = b"FVMB200C"


def read_checkpoint(path):
    """Read a checkpoint file without a GPU: (header dict, fields (5, ny, nx)
    float32).  The header dict holds the saved SimParams / Ext and the
    time-step state; the payload CRC-32 is verified."""
    import struct
    import zlib
    with open(path, "rb") as f:
        head = f.read(256)
        if len(head) != 256 or head[:8] != CHECKPOINT_MAGIC:
            raise FvmError(1, f"{path}: not a checkpoint file")
        version, hbytes, nx, ny, nf, flags = struct.unpack_from("<IIiiII", head, 8)
        next_dt, t_dev, cfl_speed, cfl_nu = struct.unpack_from("<ffff", head, 32)
        payload_bytes, crc = struct.unpack_from("<QI", head, 48)
        if version != 1 or hbytes != 256 or nf != 5 or payload_bytes != nx * ny * 20:
            raise FvmError(8, f"{path}: unsupported checkpoint layout")
        params = SimParams.from_buffer_copy(head, 64)
        ext = Ext.from_buffer_copy(head, 64 + C.sizeof(SimParams))
        data = f.read(payload_bytes)
    if len(data) != payload_bytes or zlib.crc32(data) != crc:
        raise FvmError(1, f"{path}: payload truncated or checksum mismatch")
    fields = np.frombuffer(data, np.float32).reshape(5, ny, nx).copy()
    return {"params": params, "ext": ext, "next_dt": next_dt, "t_device": t_dev, "flags": flags,
            "cfl": (cfl_speed, cfl_nu)}, fields


def checkpoint_info(path):
    """Validate a checkpoint file in the library (no device needed): (SimParams, Ext)."""
    p, e = SimParams(), Ext()
    _check(load_library().fvm_checkpoint_info(os.fsencode(path), C.byref(p), C.byref(e)))
    return p, e


def colormap_table(colormap):
    """(256, 3) float32 colour table of a colormap (fvm_colormap_table)."""
    out = np.empty((256, 3), np.float32)
    _check(load_library().fvm_colormap_table(int(colormap), C.c_void_p(out.ctypes.data)))
    return out


def write_ppm(path, rgba):
    """Write an (ny, nx, 4) uint8 image (row 0 = bottom grid row) as a binary
    PPM with the top row first."""
    img = np.ascontiguousarray(np.asarray(rgba, np.uint8)[::-1, :, :3])
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
        f.write(img.tobytes())


def shedding_stats(t, cd, cl, ref_length, u_inf):
    """Strouhal number and cycle-averaged drag/lift of a force history
    (fvm_shedding_stats); t, cd, cl: equal-length sequences."""
    t, cd, cl = (np.ascontiguousarray(x, dtype=np.float64) for x in (t, cd, cl))
    if not (len(t) == len(cd) == len(cl)):
        raise FvmError(1, "t, cd, cl must have equal lengths")
    out = Shedding()
    dp = C.POINTER(C.c_double)
    _check(load_library().fvm_shedding_stats(t.ctypes.data_as(dp), cd.ctypes.data_as(dp), cl.ctypes.data_as(dp),
                                             len(t), float(ref_length), float(u_inf), C.byref(out)))
    return out


def instance_bytes(nx, ny):
    return load_library().fvm_batch_instance_bytes(int(nx), int(ny))


def gpu_mem_info():
    lib = load_library()
    f, t = C.c_size_t(), C.c_size_t()
    _check(lib.fvm_gpu_mem_info(C.byref(f), C.byref(t)))
    return f.value, t.value


__all__ = ["Solver", "Batch", "Server", "shedding_stats", "read_checkpoint", "write_ppm", "colormap_table", "instance_bytes", "FvmError", "SimParams", "Ext", "Diag", "params_default", "compute_derived",
           "ext_default", "workload", "load_library", "gpu_mem_info", "EXPORTS", "LIB_PATH"]
