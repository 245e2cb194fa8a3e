"""Shared test helpers: workload builders, parity metrics, wall masks."""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "fvm-airidynamic-simulator_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from fvm_b200 import abi  # noqa: E402

FIELDS = ("rho", "rho_u", "rho_v", "E", "rho_e")


def small(name, nx, ny, **kw):
    p, e = abi.workload(name, nx, ny)
    for k, v in kw.items():
        if hasattr(e, k):
            setattr(e, k, v)
        else:
            setattr(p, k, v)
    abi.compute_derived(p)
    if "obstacle_y" in kw:
        p.obstacle_y = kw["obstacle_y"]
    return p, e


def _scales(b, mask=None, kind="max"):
    """Per-field normalisation: the field's own magnitude for rho, E, rho_e;
    the momentum magnitude |(rho_u, rho_v)| for both momentum components
    (rho_v alone is ~0 in the freestream)."""
    b = b.astype(np.float64)
    red = np.max if kind == "max" else np.mean
    sel = (lambda x: x[mask]) if mask is not None else (lambda x: x)
    mom = red(sel(np.hypot(b[1], b[2])))
    return np.array([red(sel(np.abs(b[0]))), mom, mom, red(sel(np.abs(b[3]))), red(sel(np.abs(b[4])))])


def rel_linf(a, b, mask=None):
    """Per-field max|a-b| / scale, scale = max magnitude (see _scales)."""
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    m = np.array([(d[k][mask] if mask is not None else d[k]).max() for k in range(5)])
    return m / np.maximum(_scales(b, mask, "max"), 1e-300)


def rel_l1(a, b, mask=None):
    """Per-field mean|a-b| / mean magnitude (see _scales)."""
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    m = np.array([(d[k][mask] if mask is not None else d[k]).mean() for k in range(5)])
    return m / np.maximum(_scales(b, mask, "mean"), 1e-300)


def away_from_walls(ct, dist=2):
    """True for cells at least `dist` cells (Chebyshev) from any solid/ghost cell."""
    wall = (ct == abi.CELL_SOLID) | (ct == abi.CELL_GHOST)
    near = wall.copy()
    for dj in range(-dist, dist + 1):
        for di in range(-dist, dist + 1):
            near |= np.roll(np.roll(wall, dj, axis=0), di, axis=1)
    return ~near


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
