"""The largest grid class one B200 holds comfortably: 32768 x 16384 cells
(537M cells, ~46 GB of device state), where the fifth field of a state starts
2^31 floats into its buffer, so every offset the kernels form must be 64-bit.

The check is size independent: the update is local (a cell after n steps
depends only on cells within ~6n of it, given dt), so a 200 x 200 window
around a body placed near the far corner of the grid is advanced by the FP32
oracle from the same start state and geometry, and the window's interior
(40 cells from its edges, beyond the reach of the oracle's artificial window
boundaries) must agree within the parity tolerance.  The far corners of the
grid, which no disturbance reaches in that time, must still hold the
freestream state.
"""
import numpy as np
import pytest

from helpers import small, rel_l1, FIELDS

pytestmark = pytest.mark.gpu

from fvm_b200 import Solver, abi  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

NX, NY = 32768, 16384
STEPS = 6
WIN, MARGIN = 200, 40


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info()[0]


def test_largest_grid_window_matches_oracle_and_far_field_is_untouched():
    if _free_bytes() < 64 * 10**9:
        pytest.skip("needs ~46 GB of free device memory")
    probe, _ = small("euler_m3_circle", NX, NY)
    dx, dy = probe.dx, probe.dy
    cx, cy = NX - 400, NY - 400  # body near the far corner: the largest offsets
    p, e = small("euler_m3_circle", NX, NY, obstacle_x=cx * dx, obstacle_y=cy * dy, obstacle_r=24 * dx)
    e.dt_policy = abi.DT_FIXED
    s = Solver(p, e)
    assert s.memory_usage() > 40 * 10**9
    i0, j0 = cx - WIN // 2, cy - WIN // 2
    U0 = s.read_region(i0, j0, WIN, WIN)
    sdf, ct = s.read_region_geometry(i0, j0, WIN, WIN)
    assert ((ct == abi.CELL_SOLID) | (ct == abi.CELL_GHOST)).sum() > 100
    corners = [(NX - 8, NY - 8), (0, NY - 8), (NX - 8, 0), (NX // 2, NY - 8)]
    C0 = [s.read_region(i, j, 8, 8) for i, j in corners]
    p.dt = s.compute_dt()
    s.step(STEPS)
    U = s.read_region(i0, j0, WIN, WIN)
    assert np.isfinite(U).all()

    # the same window through the FP32 oracle: same cell size, geometry and start state
    q, eo = small("euler_m3_circle", WIN, WIN, domain_width=WIN * dx, domain_height=WIN * dy)
    assert q.dx == dx and q.dy == dy
    o = Oracle(q, eo, bits=32)
    o.set_geometry(sdf, ct)
    o.set_fields(U0)
    for _ in range(STEPS):
        o.step(p.dt)
    inner = (slice(None), slice(MARGIN, WIN - MARGIN), slice(MARGIN, WIN - MARGIN))
    l1 = rel_l1(U[inner], o.fields()[inner])
    assert l1.max() <= 1e-4, dict(zip(FIELDS, l1))
    assert np.abs(U[inner] - U0[inner]).max() > 0  # the body has disturbed the window

    for (i, j), c0 in zip(corners, C0):
        c = s.read_region(i, j, 8, 8)
        scale = np.abs(c0).max(axis=(1, 2))
        scale[1:3] = max(scale[1], 1e-30)
        err = (np.abs(c.astype(np.float64) - c0).max(axis=(1, 2)) / np.maximum(scale, 1e-30))
        assert err.max() <= 1e-5, ((i, j), dict(zip(FIELDS, err)))
