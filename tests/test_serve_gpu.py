"""Request loop (fvm_server_*): continuous batching.  Every served result must
equal the same solve run alone (bit for bit: the batched kernels compute each
cell exactly as the single-solve ones), whatever else shares the batch, when
it was admitted, or whether its instance memory was reused."""
import threading
import time

import numpy as np
import pytest

from helpers import small

pytestmark = pytest.mark.gpu

import fvm_b200  # noqa: E402
from fvm_b200 import abi  # noqa: E402


def _ext():
    e = abi.ext_default()
    e.dt_policy = abi.DT_RECOMPUTE
    return e


def _requests():
    return [
        (small("euler_m3_circle", 160, 80)[0], 23),
        (small("ns_karman_re200", 192, 96)[0], 9),
        (small("euler_m3_circle", 128, 64, obstacle_shape=abi.SHAPE_STAR, obstacle_r=0.15, mach=2.0)[0], 31),
        (small("ns_karman_re200", 144, 72, obstacle_shape=abi.SHAPE_DIAMOND, adiabatic_wall=False,
               T_wall=350.0)[0], 14),
        (small("euler_m3_circle", 160, 80, mach=5.0)[0], 5),
        (small("euler_m3_circle", 96, 48, obstacle_shape=abi.SHAPE_TRIANGLE, obstacle_r=0.12)[0], 17),
    ]


_solo_cache = {}


def _solo(p, steps):
    key = (bytes(p), steps)
    if key not in _solo_cache:
        s = fvm_b200.Solver(abi.SimParams.from_buffer_copy(p), _ext())
        s.step(steps)
        _solo_cache[key] = (s.fields(), s.params.t_current)
        s.close()
    return _solo_cache[key]


def _check(res, fields, p, steps):
    assert res.status == 0, res.status
    assert res.steps == steps
    U, t = _solo(p, steps)
    assert np.array_equal(U.view(np.uint32), fields.view(np.uint32))
    assert res.t_final == np.float32(t)
    assert res.admit_s >= res.submit_s and res.done_s >= res.admit_s


def test_served_results_equal_solo_runs_with_staggered_arrivals():
    reqs = _requests()
    srv = fvm_b200.Server(_ext(), chunk_steps=4)
    tickets = {}

    def client():
        for k, (p, n) in enumerate(reqs):
            tickets[srv.submit(p, n)] = k
            time.sleep(0.003 * (k % 3))

    th = threading.Thread(target=client)
    th.start()
    th.join()
    srv.drain(timeout_s=120)
    got = {}
    for res, fields in srv.poll():
        got[res.ticket] = (res, fields)
    assert len(got) == len(reqs)
    for t, k in tickets.items():
        res, fields = got[t]
        _check(res, fields, *reqs[k])
    st = srv.stats()
    assert st.completed == len(reqs) and st.pending == 0 and st.active == 0
    assert st.batched_steps >= max(n for _, n in reqs)
    assert st.step_ms_p99 >= st.step_ms_p50 > 0
    srv.close()


def test_budget_admits_one_at_a_time_and_rejects_oversize():
    reqs = _requests()[:4]
    biggest = max(fvm_b200.instance_bytes(p.nx, p.ny) for p, _ in reqs)
    srv = fvm_b200.Server(_ext(), budget_bytes=biggest + 1, chunk_steps=8)
    huge, _ = small("euler_m3_circle", 1024, 512)
    t_huge = srv.submit(huge, 3)
    tickets = [srv.submit(p, n) for p, n in reqs]
    res, fields = srv.wait(t_huge, timeout_s=60)
    assert res.status == 7 and fields is None  # FVM_ERR_BUDGET
    spans = []
    for t, (p, n) in zip(tickets, reqs):
        res, fields = srv.wait(t, timeout_s=120)
        _check(res, fields, p, n)
        spans.append((res.admit_s, res.done_s))
    # one admitted solve at a time: each admission after the previous completion
    for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
        assert a1 >= d0
    st = srv.stats()
    assert st.rejected == 1
    assert st.active_bytes == 0 and st.parked_bytes + st.active_bytes <= biggest + 1
    srv.close()


def test_parked_instances_are_reused_with_identical_results():
    p, _ = small("euler_m3_circle", 160, 80)
    q, _ = small("euler_m3_circle", 160, 80, obstacle_shape=abi.SHAPE_CAPSULE, mach=4.0)
    srv = fvm_b200.Server(_ext(), chunk_steps=16)
    r1, f1 = srv.wait(srv.submit(p, 11))
    _check(r1, f1, p, 11)
    assert srv.stats().parked_bytes > 0
    r2, f2 = srv.wait(srv.submit(q, 13))  # reuses the parked 160x80 instance
    _check(r2, f2, q, 13)
    r3, f3 = srv.wait(srv.submit(p, 11))
    _check(r3, f3, p, 11)
    assert np.array_equal(f1.view(np.uint32), f3.view(np.uint32))
    srv.close()


def test_slot_limit_and_many_requests():
    reqs = _requests() * 2
    srv = fvm_b200.Server(_ext(), max_active=2, chunk_steps=64)
    tickets = [srv.submit(p, n) for p, n in reqs]
    for t, (p, n) in zip(tickets, reqs):
        res, fields = srv.wait(t, timeout_s=120)
        _check(res, fields, p, n)
    srv.close()
