"""C-ABI library: loads, exports every declared symbol, struct layouts (CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helpers import REPO, gpu_available
import fvm_b200
from fvm_b200 import abi

HEADER = os.path.join(REPO, "include", "fvm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = fvm_b200.load_library()
    names = declared_functions()
    assert set(names) == set(fvm_b200.EXPORTS), set(names) ^ set(fvm_b200.EXPORTS)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_simparams_layout_is_the_reference_layout():
    # offsets of the reference struct SimParams (src/include/common.h:50-102)
    expect = dict(nx=0, ny=4, dx=8, dy=12, domain_width=16, domain_height=20, mach=24, T_inf=28, p_inf=32,
                  rho_inf=36, u_inf=40, v_inf=44, c_inf=48, obstacle_x=52, obstacle_y=56, obstacle_r=60,
                  obstacle_rotation=64, obstacle_shape=68, wing_rotation=72, cfl=76, dt=80, t_current=84,
                  step=88, enable_viscosity=92, cfl_visc=96, adiabatic_wall=100, T_wall=104, paused=108)
    for name, off in expect.items():
        assert getattr(abi.SimParams, name).offset == off, name
    assert C.sizeof(abi.SimParams) == 112


def test_compute_derived_matches_host_float_arithmetic():
    lib = fvm_b200.load_library()
    for wl in ("euler_m3_circle", "ns_karman_re200", "ns_hypersonic_cone"):
        p, _ = abi.workload(wl, 300, 150)
        q = abi.SimParams.from_buffer_copy(p)
        lib.fvm_params_compute_derived(C.byref(q))
        for f in ("rho_inf", "c_inf", "u_inf", "dx", "dy", "obstacle_y"):
            assert np.float32(getattr(q, f)) == np.float32(getattr(p, f)), (wl, f)


def test_defaults_match_reference_initialisers():
    lib = fvm_b200.load_library()
    q = abi.SimParams()
    lib.fvm_params_default(C.byref(q))
    p = abi.params_default()
    assert bytes(q) == bytes(p)
    e = abi.Ext()
    lib.fvm_ext_default(C.byref(e))
    d = abi.ext_default()
    assert (e.flux_scheme, e.limiter, e.dt_policy) == (d.flux_scheme, d.limiter, d.dt_policy)
    assert np.float32(e.prandtl) == np.float32(0.71)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_create_without_device_reports_cuda_error():
    with pytest.raises(fvm_b200.FvmError) as ei:
        fvm_b200.Solver()
    assert ei.value.code == 2


def test_build_info_names_the_target():
    lib = fvm_b200.load_library()
    assert b"sm_100a" in lib.fvm_build_info()


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    # no CPU fallback: without the built CUDA library the package refuses to run
    monkeypatch.setattr(fvm_b200, "_lib", None)
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.load_library(str(tmp_path / "absent.so"))
