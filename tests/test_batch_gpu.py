"""Batched solves (fvm_batch_*): every instance's result equals the same solve
run alone, bit for bit, while instances of different sizes, Mach numbers,
obstacles and Euler/NS mix in one persistent launch per stage."""
import numpy as np
import pytest

from helpers import small

pytestmark = pytest.mark.gpu

import fvm_b200  # noqa: E402
from fvm_b200 import abi  # noqa: E402


def _mix():
    cases = [
        small("euler_m3_circle", 160, 80),
        small("ns_karman_re200", 200, 100),
        small("euler_m3_circle", 128, 64, obstacle_shape=abi.SHAPE_STAR, obstacle_r=0.15, mach=2.0),
        small("ns_karman_re200", 144, 72, obstacle_shape=abi.SHAPE_DIAMOND, adiabatic_wall=False, T_wall=350.0),
    ]
    out = []
    for p, e in cases:
        e.dt_policy = abi.DT_RECOMPUTE
        out.append((p, e))
    return out


def _solo(p, e, steps):
    s = fvm_b200.Solver(abi.SimParams.from_buffer_copy(p), abi.Ext.from_buffer_copy(e))
    s.step(steps)
    return s.fields(), s.params


def test_batched_instances_equal_solo_runs_bitwise():
    mix = _mix()
    e0 = abi.Ext.from_buffer_copy(mix[0][1])
    b = fvm_b200.Batch(e0)
    ids = [b.add(p) for p, _ in mix]
    b.step(25)
    b.synchronize()
    for (p, e), i in zip(mix, ids):
        U, ps = _solo(p, e0, 25)
        B = b.fields(i)
        assert np.array_equal(U.view(np.uint32), B.view(np.uint32)), i
        q = b.instance(i)
        assert q.step == 25 and q.t_current == ps.t_current and q.dt == ps.dt
        assert b.nonfinite_count(i) == 0


def test_batch_add_remove_mid_run():
    mix = _mix()
    e0 = abi.Ext.from_buffer_copy(mix[0][1])
    b = fvm_b200.Batch(e0)
    ids = [b.add(p) for p, _ in mix[:3]]
    b.step(6)
    b.remove(ids[1])
    late = b.add(mix[3][0])
    b.step(7)
    assert b.count() == 3
    for k, steps in ((0, 13), (2, 13)):
        U, _ = _solo(mix[k][0], e0, steps)
        assert np.array_equal(U.view(np.uint32), b.fields(ids[k]).view(np.uint32))
    U, _ = _solo(mix[3][0], e0, 7)
    assert np.array_equal(U.view(np.uint32), b.fields(late).view(np.uint32))


def test_batch_launches_per_step_do_not_grow_with_instances():
    e = abi.ext_default()
    e.dt_policy = abi.DT_RECOMPUTE
    b = fvm_b200.Batch(e)
    rng = abi.SeededStream(11)
    for _ in range(12):
        p, _ = abi.uneven_instance(rng, sizes=(64, 128))
        b.add(p)
    b.step(1)
    n0 = b.launch_count()
    b.step(5)
    per = (b.launch_count() - n0) / 5
    assert per in (4, 6)
    for i in range(12):
        assert np.isfinite(b.fields(i)).all()
    d = b.diagnostics(0)
    assert np.isfinite(d.mass) and d.mass > 0
