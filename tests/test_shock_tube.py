"""Sod's shock tube on the FP64 oracle against the exact Riemann solution
(no GPU): every flux / limiter pair within 1 % of the density jump (L1 over
the window), the shock within two cells of its exact place, the error
falling with the grid, and the exact solver itself against the star states
Toro 2009 tabulates (Table 4.3)."""
import pytest

from shock_tube import setup, errors
from exact_riemann import star_state
from fvm_b200 import abi
from oracle.oracle import Oracle


@pytest.mark.parametrize("left, right, p_star, u_star", [
    ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.30313, 0.92745),
    ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), 0.00189, 0.0),
    ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), 460.894, 19.5975),
    ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), 1691.64, 8.68975),
])
def test_exact_solver_matches_published_star_states(left, right, p_star, u_star):
    p, u = star_state(left, right)
    assert p == pytest.approx(p_star, rel=5e-5, abs=1e-5)
    assert u == pytest.approx(u_star, rel=5e-5, abs=1e-5)


def _run(n, flux, limiter):
    p, e, U, dt, t_end = setup(n, flux, limiter)
    o = Oracle(p, e, bits=64)
    o.set_fields(U)
    for _ in range(200):
        o.step(dt)
    return errors(o.fields(), n, t_end)


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_AUSM_PLUS])
@pytest.mark.parametrize("limiter", [abi.LIMITER_MINMOD, abi.LIMITER_VAN_LEER])
def test_oracle_sod_matches_exact_solution(flux, limiter):
    err_rho, err_u, shock_cells, band = _run(200, flux, limiter)
    assert err_rho < 1e-2 and err_u < 2e-2, (err_rho, err_u)
    assert shock_cells <= 2
    assert band < 1e-9  # the compared rows are still the 1-D problem


def test_oracle_sod_error_falls_with_the_grid():
    e100 = _run(100, abi.FLUX_HLLC, abi.LIMITER_MINMOD)[0]
    e200 = _run(200, abi.FLUX_HLLC, abi.LIMITER_MINMOD)[0]
    assert e200 < 0.7 * e100, (e100, e200)
