"""The oracle against golden outputs of the reference's own FP32 CUDA solver.

tests/golden/ref_*.npz were produced by tests/golden/make_golden.py, which runs
the unmodified reference src/solver.cu (oracle/_ref) on a GPU: per case the
SimParams bytes, the reference's SDF and cell classes, its state after reset
and after N fixed-dt steps.  CPU only.
"""
import glob
import os

import numpy as np
import pytest

from helpers import REPO, rel_l1, rel_linf, away_from_walls, FIELDS
from fvm_b200 import abi
from oracle.oracle import Oracle

GOLDEN = os.path.join(REPO, "tests", "golden")
DYN = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))
DYN = [f for f in DYN if "U1" in np.load(f).files]
SHAPES = [f for f in sorted(glob.glob(os.path.join(GOLDEN, "ref_shape_*.npz")))]


def _params(z):
    return abi.SimParams.from_buffer_copy(z["params"].tobytes())


def test_fixtures_present():
    assert len(DYN) >= 5 and len(SHAPES) == 6


@pytest.mark.parametrize("path", DYN, ids=[os.path.basename(f)[4:-4] for f in DYN])
def test_oracle_fp64_reproduces_reference_steps(path):
    """FP64 oracle from the reference's start state and geometry: after N
    reference steps the conserved fields agree to relative L1 <= 1e-4 (the
    reference is FP32 fast-math and its ghost-cell kernel is order dependent)."""
    z = np.load(path)
    p = _params(z)
    o = Oracle(p, abi.ext_default(), bits=64)
    o.set_geometry(z["sdf"], z["ct"])
    o.set_fields(z["U0"])
    for _ in range(int(z["steps"])):
        o.step(float(z["dt"]))
    U = o.fields()
    l1 = rel_l1(z["U1"], U)
    assert l1.max() <= 1e-4, dict(zip(FIELDS, l1))
    far = away_from_walls(z["ct"], 3)
    linf = rel_linf(z["U1"], U, far)
    assert linf.max() <= 1e-3, dict(zip(FIELDS, linf))


@pytest.mark.parametrize("mistake", ["ausm_plus_flux", "dt_plus_1pct"])
@pytest.mark.parametrize("path", DYN, ids=[os.path.basename(f)[4:-4] for f in DYN])
def test_a_planted_mistake_fails_the_golden_check(path, mistake):
    """The check above is sensitive: the FP64 oracle with a mistake planted
    in it (AUSM+ in place of the reference's HLLC, or every step 1 % too
    long) misses the reference's state by more than the L1 tolerance."""
    z = np.load(path)
    p = _params(z)
    e = abi.ext_default()
    dt = float(z["dt"])
    if mistake == "ausm_plus_flux":
        e.flux_scheme = abi.FLUX_AUSM_PLUS
    else:
        dt *= 1.01
    o = Oracle(p, e, bits=64)
    o.set_geometry(z["sdf"], z["ct"])
    o.set_fields(z["U0"])
    for _ in range(int(z["steps"])):
        o.step(dt)
    assert rel_l1(z["U1"], o.fields()).max() > 1e-4


@pytest.mark.parametrize("path", DYN, ids=[os.path.basename(f)[4:-4] for f in DYN])
def test_oracle_reset_matches_reference_away_from_ghosts(path):
    """Freestream + boundary conditions: identical to the reference except at
    ghost cells, whose values in the reference depend on launch scheduling."""
    z = np.load(path)
    p = _params(z)
    o = Oracle(p, abi.ext_default(), bits=32)
    o.set_geometry(z["sdf"], z["ct"])
    o.reinit()
    U = o.fields()
    not_ghost = z["ct"] != abi.CELL_GHOST
    assert rel_linf(z["U0"], U, not_ghost).max() <= 1e-6


@pytest.mark.parametrize("path", SHAPES, ids=[os.path.basename(f)[10:-4] for f in SHAPES])
def test_oracle_masks_match_reference(path):
    """Cell classes of the FP32 oracle (libm, IEEE) against the reference's
    fast-math kernel: equal except at cells within rounding of the band edge."""
    z = np.load(path)
    p = _params(z)
    o = Oracle(p, abi.ext_default(), bits=32)
    sdf, ct = o.compute_sdf()
    diff = ct != z["ct"]
    band = 1.5 * max(p.dx, p.dy)
    if diff.any():
        d = z["sdf"][diff].astype(np.float64)
        assert np.min(np.minimum(np.abs(np.abs(d) - band), np.abs(d))) < 1e-5 * band
    assert diff.sum() <= 3
    scale = max(p.domain_width, p.domain_height)
    assert np.abs(sdf.astype(np.float64) - z["sdf"]).max() <= 1e-5 * scale
