"""CPU oracle self-checks (no GPU): precision agreement, symmetry, freestream
preservation, CFL formula, geometry classes."""
import numpy as np
import pytest

from helpers import small, rel_l1, rel_linf
from fvm_b200 import abi
from oracle.oracle import Oracle


def test_fp32_tracks_fp64():
    p, e = small("euler_m3_circle", 128, 64)
    a, b = Oracle(p, e, bits=64), Oracle(p, e, bits=32)
    dt = a.compute_dt()
    for _ in range(50):
        a.step(dt)
        b.step(dt)
    assert rel_l1(b.fields(), a.fields()).max() < 1e-5


@pytest.mark.parametrize("wl", ["euler_m3_circle", "ns_karman_re200"])
def test_freestream_preserved_without_obstacle(wl):
    p, e = small(wl, 96, 48)
    p.obstacle_x = -100.0 * p.domain_width  # far outside: every cell is fluid
    o = Oracle(p, e, bits=64)
    U0 = o.fields()
    _, ct = o.geometry()
    assert not ((ct == abi.CELL_SOLID) | (ct == abi.CELL_GHOST)).any()
    o.run(30)
    assert rel_linf(o.fields(), U0).max() < 1e-12


def test_mirror_symmetry_of_a_symmetric_pulse():
    """Without obstacle, a pulse symmetric about y = H/2 stays symmetric (the
    y-direction reconstruction, Riemann solver and NRBC are mirror images).
    With an obstacle the reference method is not mirror-symmetric: wall faces
    carry the pressure of the bottom cell (src/solver.cu:1679), which is the
    fluid cell below a body and the ghost cell above it."""
    p, e = small("euler_m3_circle", 128, 64)
    p.obstacle_x = -100.0 * p.domain_width
    o = Oracle(p, e, bits=64)
    o.set_fields(_pulse_state(p, amp=0.05))
    o.run(40)
    U = o.fields()
    M = U[:, ::-1].copy()
    M[2] = -M[2]
    assert rel_linf(U, M).max() < 1e-12


def test_cfl_formula_matches_read_time_step_result():
    p, e = small("ns_karman_re200", 64, 32)
    o = Oracle(p, e, bits=64)
    ms, mn = o.cfl_maxima()
    mind = min(p.dx, p.dy)
    expect = min(p.cfl * mind / (ms + 1e-10), p.cfl_visc * mind * mind / (mn + 1e-10))
    assert o.compute_dt() == pytest.approx(expect, rel=1e-12)


@pytest.mark.parametrize("shape", [abi.SHAPE_CIRCLE, abi.SHAPE_STAR, abi.SHAPE_DIAMOND, abi.SHAPE_CAPSULE,
                                   abi.SHAPE_TRIANGLE, abi.SHAPE_STARSHIP, abi.SHAPE_CONE_CAPSULE])
def test_cell_classes_follow_the_band_rule(shape):
    p, e = small("euler_m3_circle", 200, 100, obstacle_shape=shape, obstacle_r=0.15, obstacle_rotation=0.4)
    if shape == abi.SHAPE_CONE_CAPSULE:
        e.cone_length = 0.2
    o = Oracle(p, e, bits=64)
    sdf, ct = o.geometry()
    band = 1.5 * max(p.dx, p.dy)
    inner = ct[:, 1:-1]
    d = sdf[:, 1:-1]
    assert ((inner == abi.CELL_SOLID) == (d < -band)).all()
    assert ((inner == abi.CELL_GHOST) == ((d >= -band) & (d < band))).all()
    assert (ct[:, 0] == abi.CELL_INFLOW).all() and (ct[:, -1] == abi.CELL_OUTFLOW).all()
    assert (inner == abi.CELL_SOLID).any() and (inner == abi.CELL_GHOST).any()


def _pulse_state(p, amp=0.01, width_cells=6.0):
    """Uniform freestream plus a Gaussian isentropic pressure/density pulse."""
    ny, nx = p.ny, p.nx
    x = (np.arange(nx) + 0.5) * p.dx
    y = (np.arange(ny) + 0.5) * p.dy
    X, Y = np.meshgrid(x, y)
    r2 = ((X - 0.5 * p.domain_width) ** 2 + (Y - 0.5 * p.domain_height) ** 2) / (width_cells * p.dx) ** 2
    g = 1.4
    pr = p.p_inf * (1.0 + amp * np.exp(-r2))
    rho = p.rho_inf * (pr / p.p_inf) ** (1.0 / g)
    u = np.full_like(rho, p.u_inf)
    e = pr / (g - 1.0)
    return np.stack([rho, rho * u, 0.0 * rho, e + 0.5 * rho * u * u, e])


def test_ausm_and_hllc_agree_on_a_smooth_acoustic_pulse():
    """Both Riemann solvers converge to the same smooth solution: on a resolved
    acoustic pulse in a uniform M0.3 stream the perturbations agree closely."""
    p, e = small("ns_karman_re200", 128, 64)
    p.enable_viscosity = False
    p.obstacle_x = -100.0 * p.domain_width
    U0 = _pulse_state(p)
    runs = []
    for scheme in (abi.FLUX_HLLC, abi.FLUX_AUSM_PLUS):
        e2 = abi.Ext.from_buffer_copy(e)
        e2.flux_scheme = scheme
        o = Oracle(p, e2, bits=64)
        o.set_fields(U0)
        dt = o.compute_dt()
        for _ in range(40):
            o.step(dt)
        runs.append(o.fields())
    base = np.stack([p.rho_inf, p.rho_inf * p.u_inf, 0.0, 0, 0])
    dh = runs[0][0] - p.rho_inf
    da = runs[1][0] - p.rho_inf
    assert np.abs(dh).max() > 1e-4 * p.rho_inf
    assert np.linalg.norm(da - dh) / np.linalg.norm(dh) < 0.05
