"""Sod's shock tube (Sod 1978, J. Comput. Phys. 27:1) in SI units on the 2-D
grid: left state rho = 1 kg/m^3, p = 1e5 Pa, right state rho = 0.125 kg/m^3,
p = 1e4 Pa, both at rest, the diaphragm at x = L/2 of a square domain of side
L = 1 m without obstacle.  The freestream of the run is the right state at
rest, so the outflow and top / bottom conditions see a consistent far field
on the right; the inflow condition at i = 0 imposes the right state against
the left one and sends a wave in from the left edge, and the top / bottom
conditions do the same over the left half.  At t = 0.2 L / c_L those waves
have travelled 0.2 L, so the middle row over x in [0.3 L, 0.95 L] (the
rarefaction head is at 0.3 L, the shock near 0.80 L) is the exact Riemann
problem's solution, compared with exact_riemann.sample."""
import numpy as np

from helpers import small
from exact_riemann import sample
from fvm_b200 import abi

R_GAS = 287.05
LEFT = (1.0, 0.0, 1e5)
RIGHT = (0.125, 0.0, 1e4)
STEPS = 200


def setup(n, flux, limiter):
    """(params, ext, initial state [5, n, n] float32, dt, t_end)."""
    p, e = small("euler_m3_circle", n, n, domain_width=1.0, domain_height=1.0, mach=0.0, p_inf=RIGHT[2],
                 T_inf=RIGHT[2] / (RIGHT[0] * R_GAS), flux_scheme=flux, limiter=limiter)
    p.obstacle_x = -100.0  # far outside: every cell is fluid
    abi.compute_derived(p)
    x = (np.arange(n) + 0.5) * p.dx
    left = x < 0.5
    U = np.zeros((5, n, n), dtype=np.float32)
    U[0] = np.where(left, LEFT[0], RIGHT[0])[None, :]
    U[3] = (np.where(left, LEFT[2], RIGHT[2]) / 0.4)[None, :]  # E = p / (gamma - 1) at rest
    U[4] = U[3]
    t_end = 0.2 / np.sqrt(1.4 * LEFT[2] / LEFT[0])
    p.dt = t_end / STEPS  # CFL <= 0.37 over the run
    return p, e, U, p.dt, t_end


def errors(U, n, t_end):
    """Mean |rho - exact| over the window as a fraction of the density jump,
    mean |u - exact| as a fraction of the star velocity, the cell distance of
    the shock from its exact place, and the largest deviation of the middle
    band of rows from the middle row."""
    x = (np.arange(n) + 0.5) / n
    rho = U[0, n // 2].astype(np.float64)
    u = U[1, n // 2] / rho
    re, ue, _ = sample(LEFT, RIGHT, (x - 0.5) / t_end)
    w = (x > 0.3) & (x < 0.95)
    err_rho = np.abs(rho - re)[w].mean() / (LEFT[0] - RIGHT[0])
    u_star = ue.max()
    err_u = np.abs(u - ue)[w].mean() / u_star
    # shock: where rho falls through the mean of the post-shock and right densities
    rho_post = re[(x > 0.7) & (x < 0.75)].mean()
    mid = 0.5 * (rho_post + RIGHT[0])
    right_half = np.where(x > 0.6)[0]
    i_num = right_half[np.argmax(rho[right_half] < mid)]
    i_ex = right_half[np.argmax(re[right_half] < mid)]
    band = U[0, n // 2 - n // 10:n // 2 + n // 10].astype(np.float64)
    return err_rho, err_u, abs(int(i_num) - int(i_ex)), np.abs(band - rho[None, :]).max()
