"""Grid shapes the marching kernels treat specially, against the oracle:
odd row and column counts (a tile's last row pair holds one spare row),
grids narrower than one column strip or shorter than one tile, and grids a
few cells thin (every cell on a domain edge, one-sided viscous differences on
both sides).  Also: the results do not depend on the launch tuning (threads
per CTA, ring depth, rows per CTA) -- tiles start on even rows, so every
cell's arithmetic is the same and runs under different tunings are bitwise
equal.  Odd tile heights are rejected: they would move rows between the two
places of the row pair the kernels evaluate together, which are separately
compiled code and can round differently in the last bit.
"""
import numpy as np
import pytest

from helpers import small, rel_l1, FIELDS

pytestmark = pytest.mark.gpu

from fvm_b200 import FvmError, Solver, abi  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

NO_OBSTACLE = {"obstacle_x": -1.0e3}

GRIDS = {
    # name: (workload, nx, ny, overrides)
    "euler_odd_131x67": ("euler_m3_circle", 131, 67, {}),
    "ns_odd_97x33": ("ns_karman_re200", 97, 33, {}),
    "euler_narrow_37x19": ("euler_m3_circle", 37, 19, {}),
    "ns_iso_odd_125x41": ("ns_karman_re200", 125, 41, {"obstacle_shape": abi.SHAPE_DIAMOND, "adiabatic_wall": False,
                                                      "T_wall": 350.0}),
    "ns_thin_40x3": ("ns_karman_re200", 40, 3, dict(NO_OBSTACLE, mach=2.0)),
    "euler_thin_5x40": ("euler_m3_circle", 5, 40, NO_OBSTACLE),
    "ns_one_strip_124x5": ("ns_karman_re200", 124, 5, dict(NO_OBSTACLE, mach=1.5)),
}


def _case(name):
    wl, nx, ny, kw = GRIDS[name]
    p, e = small(wl, nx, ny, **kw)
    return p, e


@pytest.mark.parametrize("name", list(GRIDS))
def test_odd_and_small_grids_match_fp32_oracle(name):
    """30 steps from the same start state: relative L1 <= 1e-4 per field
    against the FP32 oracle."""
    p, e = _case(name)
    s = Solver(p, e)
    o = Oracle(p, e, bits=32)
    o.set_geometry(s.sdf(), s.cell_types())
    o.set_fields(s.fields())
    dt = o.compute_dt()
    p.dt = dt
    s.step(30)
    for _ in range(30):
        o.step(dt)
    U, R = s.fields(), o.fields()
    assert np.isfinite(U).all()
    l1 = rel_l1(U, R)
    assert l1.max() <= 1e-4, dict(zip(FIELDS, l1))


TUNES = [(128, 4, 4), (128, 6, 6), (256, 4, 10), (256, 6, 64), (128, 4, 1000)]


@pytest.mark.parametrize("name", ["euler_odd_131x67", "ns_odd_97x33", "ns_iso_odd_125x41"])
def test_results_do_not_depend_on_launch_tuning(name):
    """12 steps (recomputed dt, so the CFL reductions are exercised) under
    five launch tunings, including a tile taller than the grid and grids whose
    last tile has an odd row count: states, time step and simulated time
    bitwise equal."""
    ref = None
    for tune in TUNES:
        p, e = _case(name)
        e.dt_policy = abi.DT_RECOMPUTE
        s = Solver(p, e)
        s.set_tune(*tune)
        assert s.tune() == tune
        s.step(12)
        got = (s.fields(), p.dt, p.t_current)
        if ref is None:
            ref = got
            continue
        assert np.array_equal(got[0].view(np.uint32), ref[0].view(np.uint32)), tune
        assert got[1] == ref[1] and got[2] == ref[2], (tune, got[1:], ref[1:])


def test_set_tune_rejects_unsupported_shapes():
    p, e = _case("euler_odd_131x67")
    s = Solver(p, e)
    before = s.tune()
    for bad in [(64, 4, 16), (128, 5, 16), (128, 4, 3), (512, 6, 16), (128, 4, 5), (256, 6, 33)]:
        with pytest.raises(FvmError):
            s.set_tune(*bad)
    assert s.tune() == before
