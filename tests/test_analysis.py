"""fvm_shedding_stats (host code in the library): Strouhal number and
cycle-averaged force coefficients of a lift/drag history (CPU)."""
import math

import numpy as np
import pytest

from helpers import REPO  # noqa: F401  (puts the package on sys.path)
import fvm_b200


def _history(f=1250.0, cycles=9.3, n_per=80, a=0.7, cd0=1.84, b=0.05, phase=0.4, cl0=0.02):
    t = np.linspace(0.0, cycles / f, int(cycles * n_per) + 1) + 3e-4
    cl = cl0 + a * np.sin(2 * math.pi * f * t + phase)
    cd = cd0 + b * np.sin(4 * math.pi * f * t + 2 * phase)
    return t, cd, cl


def test_sinusoidal_history_gives_exact_statistics():
    f, D, U = 1250.0, 0.02, 125.0
    t, cd, cl = _history(f=f)
    st = fvm_b200.shedding_stats(t, cd, cl, D, U)
    assert st.cycles in (8, 9)
    assert st.strouhal == pytest.approx(f * D / U, rel=1e-4)
    assert st.period == pytest.approx(1.0 / f, rel=1e-4)
    assert st.cd_mean == pytest.approx(1.84, rel=1e-4)
    assert st.cl_mean == pytest.approx(0.02, abs=1e-3)
    assert st.cl_rms == pytest.approx(0.7 / math.sqrt(2.0), rel=1e-3)


def test_partial_cycles_do_not_bias_the_means():
    f = 900.0
    for cycles in (5.1, 5.5, 5.9):
        t, cd, cl = _history(f=f, cycles=cycles, b=0.3)
        st = fvm_b200.shedding_stats(t, cd, cl, 1.0, 1.0)
        assert st.cd_mean == pytest.approx(1.84, rel=2e-4), cycles


def test_errors():
    t, cd, cl = _history()
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.shedding_stats(t[:2], cd[:2], cl[:2], 1.0, 1.0)
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.shedding_stats(t[::-1], cd, cl, 1.0, 1.0)
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.shedding_stats(t, cd, np.full_like(cl, 0.5), 1.0, 1.0)  # no crossing
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.shedding_stats(t, cd, cl, 0.0, 1.0)
