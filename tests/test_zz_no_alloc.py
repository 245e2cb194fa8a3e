"""fvm_state_max_noalloc: the maximum temperature / Mach number of a state in
the caller's device memory, computed with the library's fixed scratch (no
allocation).  Checked against the handle-based fvm_max_temperature /
fvm_max_mach on the same state, two calls in a row so the second call runs on
the scratch the first one left behind.  Named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from helpers import gpu_available, small
import fvm_b200

MAX_ROWS = 16384


def _call(lib, ptr, nx, ny, pitch, plane, what):
    out = C.c_float(-1.0)
    rc = lib.fvm_state_max_noalloc(C.c_void_p(ptr), nx, ny, pitch, plane, what, C.byref(out), None)
    return rc, out.value


def test_rejects_rows_beyond_the_fixed_scratch_before_touching_the_device():
    lib = fvm_b200.load_library()
    rc, _ = _call(lib, 0x1000, 64, MAX_ROWS + 1, 64, 64 * (MAX_ROWS + 1), 0)
    assert rc == 1  # FVM_ERR_INVALID, not a CUDA error: nothing was launched
    assert b"exceeds the fixed scratch of 16384 rows" in lib.fvm_last_error()
    rc, _ = _call(lib, 0x1000, 64, 8, 32, 64 * 8, 0)
    assert rc == 1 and b"pitch" in lib.fvm_last_error()
    rc, _ = _call(lib, 0x1000, 64, 8, 64, 64 * 8, 2)
    assert rc == 1


@pytest.mark.gpu
def test_noalloc_max_matches_handle_max_two_calls_in_a_row():
    import torch
    assert gpu_available()
    lib = fvm_b200.load_library()
    p, e = small("euler_m3_circle", 160, 80)
    s = fvm_b200.Solver(p, e)
    nx, ny = p.nx, p.ny
    for _ in range(2):
        s.step(10)
        ref_T, ref_M = s.max_temperature(), s.max_mach()
        U = s.fields()  # (5, ny, nx) float32, host
        # a pitched copy, rows padded to 176 floats, planes 4 rows apart
        pitch, plane = 176, 176 * (ny + 4)
        d = torch.zeros(5 * plane, dtype=torch.float32, device="cuda")
        d.view(5, ny + 4, pitch)[:, :ny, :nx] = torch.from_numpy(np.ascontiguousarray(U)).cuda()
        torch.cuda.synchronize()
        rc, T = _call(lib, d.data_ptr(), nx, ny, pitch, plane, 0)
        assert rc == 0, lib.fvm_last_error()
        rc, M = _call(lib, d.data_ptr(), nx, ny, pitch, plane, 1)
        assert rc == 0, lib.fvm_last_error()
        assert abs(T - ref_T) <= 1e-6 * ref_T, (T, ref_T)
        assert abs(M - ref_M) <= 1e-6 * ref_M, (M, ref_M)


@pytest.mark.gpu
def test_noalloc_max_at_the_row_limit():
    import torch
    lib = fvm_b200.load_library()
    nx, ny = 32, MAX_ROWS
    rho = torch.full((ny, nx), 1.2, dtype=torch.float32, device="cuda")
    T_cells = torch.full((ny, nx), 300.0, device="cuda")
    T_cells[ny - 1, 5] = 700.0
    T_cells[0, 0] = 450.0
    cv = 287.05 / 0.4
    E = rho * cv * T_cells
    U = torch.stack([rho, torch.zeros_like(rho), torch.zeros_like(rho), E, E]).contiguous()
    torch.cuda.synchronize()
    for _ in range(2):
        rc, T = _call(lib, U.data_ptr(), nx, ny, nx, nx * ny, 0)
        assert rc == 0, lib.fvm_last_error()
        assert abs(T - 700.0) <= 1e-3, T


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream_and_works_after():
    import torch
    lib = fvm_b200.load_library()
    nx, ny = 64, 32
    U = torch.ones((5, ny, nx), dtype=torch.float32, device="cuda")
    U[3] *= 2.5e5
    U[4] *= 2.5e5
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    x = torch.zeros(4, device="cuda")
    with torch.cuda.graph(g, stream=st):
        x.add_(1.0)
        out = C.c_float(-1.0)
        rc = lib.fvm_state_max_noalloc(C.c_void_p(U.data_ptr()), nx, ny, nx, nx * ny, 0, C.byref(out),
                                       C.c_void_p(st.cuda_stream))
    assert rc == 4 and b"captured" in lib.fvm_last_error()  # FVM_ERR_STATE, nothing queued
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    rc, T = _call(lib, U.data_ptr(), nx, ny, nx, nx * ny, 0)
    assert rc == 0, lib.fvm_last_error()
    assert abs(T - 2.5e5 * 0.4 / 287.05) <= 1e-3 * T, T
