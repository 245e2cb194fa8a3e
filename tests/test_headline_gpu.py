"""Parity on the timed workload itself: the Mach-8 blunted cone, Navier-Stokes
with an isothermal wall, van Leer + HLLC, on the full 8192 x 4096 grid
(33.5M cells), the configuration the benchmark measures.

The FP32 oracle cannot advance 33.5M cells in seconds, but the update is local:
within one step a cell depends only on cells at most 10 away (viscous half
step 2, stage 1 2, ghost fill 1, stage 2 2, viscous half step 2, ghost fill 1).
So a window around the nose is read back after a settling run
(fvm_read_region, fvm_read_region_geometry), advanced by the FP32 oracle from
that start state and geometry with the same time steps as the device, and
compared in its interior (MARGIN cells from the window edges, beyond the
reach of the oracle's artificial window boundaries in STEPS steps).  Every
step takes the CFL time step of the current state (the reference
application's per-frame policy; reference CFDSolver::step and its time-step
reduction, src/solver.cu:3289-3412, :3206-3278).

The FP64 outputs of the timed workload (drag and lift over the immersed
boundary, wall heat flux, mass / momentum / energy totals, bow-shock standoff;
no reference counterpart) are checked at the same full size: the oracle
evaluates them in FP64 on the device's own state after 400 steps.
"""
import os

import numpy as np
import pytest

from helpers import small, rel_l1, rel_linf, away_from_walls, FIELDS

pytestmark = pytest.mark.gpu

from fvm_b200 import Solver, abi  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

NX, NY = 8192, 4096
SETTLE, STEPS = 24, 8
REACH = 10  # cells of influence per step
MARGIN = REACH * STEPS + 10
# window: 360 x 600 cells; the nose tip (x = 0.5 L) sits at column 2048 on the
# axis row 2048, the nose radius is ~410 cells; the interior then holds ~90
# columns of the flow ahead of the nose and the wall arc over +-210 rows
WIN_W, WIN_H = 360, 600
I0, J0 = 1878, 1748


def test_cone_8192x4096_window_matches_fp32_oracle():
    p, e = small("ns_hypersonic_cone", NX, NY)
    e.dt_policy = abi.DT_FIXED
    s = Solver(p, e)
    for _ in range(SETTLE):
        p.dt = s.compute_dt()
        s.step(1)
    U0 = s.read_region(I0, J0, WIN_W, WIN_H)
    sdf, ct = s.read_region_geometry(I0, J0, WIN_W, WIN_H)
    inner = (slice(MARGIN, WIN_H - MARGIN), slice(MARGIN, WIN_W - MARGIN))
    wall = (ct == abi.CELL_SOLID) | (ct == abi.CELL_GHOST)
    assert (ct[inner] == abi.CELL_GHOST).sum() >= 200  # the wall arc runs through the interior
    assert (~wall[inner]).sum() >= 100 * 100
    dts = []
    for _ in range(STEPS):
        dts.append(s.compute_dt())
        p.dt = dts[-1]
        s.step(1)
    U = s.read_region(I0, J0, WIN_W, WIN_H)
    assert np.isfinite(U).all()

    q, eo = small("ns_hypersonic_cone", WIN_W, WIN_H, domain_width=WIN_W * p.dx, domain_height=WIN_H * p.dy)
    q.dx, q.dy = p.dx, p.dy  # the cell size exactly, not W / nx rounded again
    q.T_wall, q.adiabatic_wall, q.enable_viscosity = p.T_wall, p.adiabatic_wall, p.enable_viscosity
    o = Oracle(q, eo, bits=32)
    o.set_geometry(sdf, ct)
    o.set_fields(U0)
    for dt in dts:
        o.step(dt)
    R = o.fields()
    Ui, Ri = U[(slice(None),) + inner], R[(slice(None),) + inner]
    l1 = rel_l1(Ui, Ri)
    far = away_from_walls(ct, 3)[inner]
    msg = {"l1": dict(zip(FIELDS, l1)), "linf_far": dict(zip(FIELDS, rel_linf(Ui, Ri, far)))}
    assert l1.max() <= 1e-4, msg
    # the flow in the window is not the freestream: the nose has disturbed it
    dU = np.abs(Ui.astype(np.float64) - U0[(slice(None),) + inner])
    assert dU[0].max() > 1e-3 * np.abs(U0[0]).max()
    # neither side selected the separately evolved internal energy anywhere
    eta_u = Ui[4] / np.where(Ui[3] > 0, Ui[3], 1.0)
    eta_r = Ri[4] / np.where(Ri[3] > 0, Ri[3], 1.0)
    assert not ((eta_u < 1e-3) | (eta_r < 1e-3)).any()


def test_cone_8192x4096_diagnostics_match_fp64_oracle_on_the_device_state():
    p, e = small("ns_hypersonic_cone", NX, NY)
    e.dt_policy = abi.DT_RECOMPUTE
    s = Solver(p, e)
    s.step(400)
    dg, sg = s.diagnostics(), s.shock_standoff()
    o = Oracle(p, e, bits=64, threads=os.cpu_count() or 1)
    o.set_geometry(s.sdf(), s.cell_types())
    o.set_fields(s.fields())
    do, so = o.diagnostics(), o.shock_standoff()
    # per-cell primitives are FP32 on the device and FP64 in the oracle; the
    # sums are FP64 on both sides
    # the body is symmetric about the axis, so lift is measured against drag
    assert abs(dg.force_x - do.force_x) <= 1e-4 * abs(do.force_x), (dg.force_x, do.force_x)
    assert abs(dg.force_y - do.force_y) <= 1e-4 * abs(do.force_x), (dg.force_y, do.force_y)
    assert abs(dg.cd - do.cd) <= 1e-4 * abs(do.cd) and do.cd > 0
    assert abs(dg.wall_heat - do.wall_heat) <= 1e-4 * abs(do.wall_heat), (dg.wall_heat, do.wall_heat)
    for name in ("mass", "mom_x", "energy"):
        g, r = getattr(dg, name), getattr(do, name)
        assert abs(g - r) <= 1e-9 * abs(r), (name, g, r)
    assert abs(dg.mom_y - do.mom_y) <= 1e-9 * abs(do.mom_x)
    # the standoff exists once the bow shock has formed on the axis row
    assert np.isfinite(sg) == np.isfinite(so), (sg, so)
    if np.isfinite(so):
        assert so > 0 and abs(sg - so) <= 5e-3 * so, (sg, so)
