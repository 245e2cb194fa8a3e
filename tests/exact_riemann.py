"""Exact solution of the 1-D Riemann problem for the Euler equations of an
ideal gas, restated from the published method of E. F. Toro, "Riemann
Solvers and Numerical Methods for Fluid Dynamics" (3rd ed., Springer 2009),
chapter 4: the pressure function f(p) = f_L(p) + f_R(p) + (u_R - u_L), with
shock (Rankine-Hugoniot) and rarefaction (isentropic) branches per side,
solved for the star pressure by Newton iteration from the primitive-variable
guess, and the wave pattern sampled at x/t.  Test infrastructure: the
analytic reference for shock-tube checks of the solver and the oracle."""
import math

import numpy as np


def _side(p, rho_k, p_k, c_k, g):
    """f_K(p) and its derivative (Toro 2009, eqs. 4.6-4.7 and 4.37)."""
    if p > p_k:  # shock
        a = 2.0 / ((g + 1.0) * rho_k)
        b = (g - 1.0) / (g + 1.0) * p_k
        q = math.sqrt(a / (p + b))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (b + p))
    # rarefaction
    r = (p / p_k) ** ((g - 1.0) / (2.0 * g))
    return 2.0 * c_k / (g - 1.0) * (r - 1.0), 1.0 / (rho_k * c_k) * (p / p_k) ** (-(g + 1.0) / (2.0 * g))


def star_state(left, right, g=1.4, tol=1e-12, max_iter=100):
    """Star-region pressure and velocity for left / right = (rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    # primitive-variable guess (Toro eq. 4.47), kept positive
    p = max(tol, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(max_iter):
        fl, dl = _side(p, rl, pl, cl, g)
        fr, dr = _side(p, rr, pr, cr, g)
        p_new = max(tol, p - (fl + fr + ur - ul) / (dl + dr))
        if abs(p_new - p) <= tol * 0.5 * (p_new + p):
            p = p_new
            break
        p = p_new
    fl, _ = _side(p, rl, pl, cl, g)
    fr, _ = _side(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(left, right, xi, g=1.4):
    """(rho, u, p) arrays at the similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    ps, us = star_state(left, right, g)
    gm, gp = (g - 1.0) / (g + 1.0), 2.0 / (g + 1.0)
    xi = np.asarray(xi, dtype=np.float64)
    rho, u, p = np.empty_like(xi), np.empty_like(xi), np.empty_like(xi)
    for n, s in enumerate(xi.ravel()):
        if s <= us:  # left of the contact
            if ps > pl:  # left shock
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                if s <= sl:
                    val = (rl, ul, pl)
                else:
                    val = (rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps)
            else:  # left rarefaction
                head = ul - cl
                cs = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                tail = us - cs
                if s <= head:
                    val = (rl, ul, pl)
                elif s >= tail:
                    val = (rl * (ps / pl) ** (1.0 / g), us, ps)
                else:  # inside the fan
                    c = gp * (cl + 0.5 * (g - 1.0) * (ul - s))
                    uu = gp * (cl + 0.5 * (g - 1.0) * ul + s)
                    val = (rl * (c / cl) ** (2.0 / (g - 1.0)), uu, pl * (c / cl) ** (2.0 * g / (g - 1.0)))
        else:  # right of the contact
            if ps > pr:  # right shock
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                if s >= sr:
                    val = (rr, ur, pr)
                else:
                    val = (rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps)
            else:  # right rarefaction
                head = ur + cr
                cs = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                tail = us + cs
                if s >= head:
                    val = (rr, ur, pr)
                elif s <= tail:
                    val = (rr * (ps / pr) ** (1.0 / g), us, ps)
                else:
                    c = gp * (cr - 0.5 * (g - 1.0) * (ur - s))
                    uu = gp * (-cr + 0.5 * (g - 1.0) * ur + s)
                    val = (rr * (c / cr) ** (2.0 / (g - 1.0)), uu, pr * (c / cr) ** (2.0 * g / (g - 1.0)))
        rho.flat[n], u.flat[n], p.flat[n] = val
    return rho, u, p
