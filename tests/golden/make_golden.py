"""Generate golden fixtures from the reference's own FP32 CUDA solver.

Runs oracle/_ref/libfvm_ref.so (the unmodified reference src/solver.cu built
by oracle/build_ref.sh) on a CUDA device for small seeded cases and stores,
per case, the parameters, the reference's SDF and cell classes, its state
after reset and after N fixed-dt steps, into tests/golden/ref_<case>.npz.
The CPU tests (tests/test_golden.py) check the oracle against these files.

Usage (GPU box):  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "fvm-airidynamic-simulator_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

from fvm_b200 import abi  # noqa: E402
from helpers import small  # noqa: E402
from oracle import ref as refmod  # noqa: E402

# case: (workload, nx, ny, overrides, steps)
CASES = {
    "euler_circle": ("euler_m3_circle", 96, 48, {}, 20),
    "euler_star": ("euler_m3_circle", 96, 48, {"obstacle_shape": abi.SHAPE_STAR, "obstacle_r": 0.2,
                                               "obstacle_rotation": 0.3}, 20),
    "ns_karman": ("ns_karman_re200", 96, 48, {}, 20),
    "ns_isothermal_triangle": ("ns_karman_re200", 96, 48, {"obstacle_shape": abi.SHAPE_TRIANGLE,
                                                           "r_rel": 0.1, "adiabatic_wall": False,
                                                           "T_wall": 400.0}, 20),
    "kernel_benchmark": ("reference_benchmark", 128, 64, {}, 10),
}
# geometry-only cases (masks of every reference shape)
SHAPES = {
    f"shape_{n}": ("euler_m3_circle", 211, 107, {"obstacle_shape": s, "obstacle_r": 0.17, "obstacle_rotation": 0.7,
                                                "wing_rotation": 0.4})
    for n, s in [("circle", 0), ("star", 1), ("diamond", 2), ("capsule", 3), ("triangle", 4), ("starship", 5)]
}


def params_array(p):
    return np.frombuffer(bytes(p), dtype=np.uint8).copy()


def main():
    assert refmod.available(), "build oracle/_ref first (oracle/build_ref.sh)"
    for name, (wl, nx, ny, kw, steps) in CASES.items():
        kw = dict(kw)
        r_rel = kw.pop("r_rel", None)
        p, _ = small(wl, nx, ny, **kw)
        if r_rel is not None:  # obstacle size relative to the domain height
            p.obstacle_r = r_rel * p.domain_height
        r = refmod.RefSolver(p)
        sdf, ct = r.geometry()
        U0 = r.fields()
        dt = r.compute_dt()
        r.steps(steps, dt=dt)
        U1 = r.fields()
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), params=params_array(r.params), sdf=sdf, ct=ct,
                            U0=U0, U1=U1, dt=np.float32(dt), steps=np.int32(steps))
        r.close()
        print("wrote", name, "dt", dt)
    for name, (wl, nx, ny, kw) in SHAPES.items():
        p, _ = small(wl, nx, ny, **kw)
        r = refmod.RefSolver(p)
        sdf, ct = r.geometry()
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), params=params_array(p), sdf=sdf, ct=ct)
        r.close()
        print("wrote", name)


if __name__ == "__main__":
    main()
