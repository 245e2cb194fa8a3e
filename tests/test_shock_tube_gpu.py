"""Sod's shock tube through the CUDA kernels (C ABI): after 100 steps the
whole state against the FP32 oracle from the same start state (L1 <= 1e-4
through the shock, contact and rarefaction, the parity bound of 100-step
runs), after 200 the window against the exact Riemann solution (the
tolerances of the oracle's own test)."""
import numpy as np
import pytest

from helpers import rel_l1, FIELDS
from shock_tube import setup, errors, STEPS

pytestmark = pytest.mark.gpu

from fvm_b200 import Solver, abi  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_AUSM_PLUS])
@pytest.mark.parametrize("limiter", [abi.LIMITER_MINMOD, abi.LIMITER_VAN_LEER])
def test_sod_matches_exact_solution_and_fp32_oracle(flux, limiter):
    n = 200
    p, e, U, dt, t_end = setup(n, flux, limiter)
    s = Solver(p, e)
    s.write_fields(U)
    o = Oracle(p, e, bits=32)
    o.set_fields(U)
    half = STEPS // 2
    s.step(half)
    for _ in range(half):
        o.step(dt)
    l1 = rel_l1(s.fields(), o.fields())
    assert l1.max() <= 1e-4, dict(zip(FIELDS, l1))
    s.step(STEPS - half)
    G = s.fields()
    assert np.isfinite(G).all()
    err_rho, err_u, shock_cells, band = errors(G, n, t_end)
    assert err_rho < 1e-2 and err_u < 2e-2, (err_rho, err_u)
    assert shock_cells <= 2
    assert band < 1e-5 * np.abs(G[0]).max()
