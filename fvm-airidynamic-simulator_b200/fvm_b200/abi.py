"""ctypes mirror of include/fvm_b200.h (structures and enums only).

`SimParams` is byte-for-byte the reference's `struct SimParams`
(reference: src/include/common.h:50-102, 112 bytes).  Nothing here loads a
shared library, so host-side code and CPU tests can use it without a GPU.
"""
import ctypes as C
import math

import numpy as np

# enum fvm_shape (0..5 = reference ObstacleShape, src/include/common.h:39-47)
SHAPE_CIRCLE, SHAPE_STAR, SHAPE_DIAMOND, SHAPE_CAPSULE, SHAPE_TRIANGLE, SHAPE_STARSHIP, SHAPE_CONE_CAPSULE = range(7)
# enum CellType (src/include/common.h:105-111)
CELL_FLUID, CELL_SOLID, CELL_GHOST, CELL_INFLOW, CELL_OUTFLOW = range(5)
FLUX_HLLC, FLUX_AUSM_PLUS = 0, 1
LIMITER_MINMOD, LIMITER_VAN_LEER = 0, 1
DT_FIXED, DT_RECOMPUTE = 0, 1
FIELD_TEMPERATURE, FIELD_PRESSURE, FIELD_DENSITY, FIELD_VELOCITY_MAG, FIELD_MACH = range(5)
CMAP_JET, CMAP_HOT, CMAP_PLASMA, CMAP_INFERNO, CMAP_VIRIDIS = range(5)
RGBA_F32, RGBA_U8 = 0, 1

STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "ALLOC", 4: "STATE", 5: "TIMEOUT",
          6: "NONFINITE", 7: "BUDGET", 8: "UNSUPPORTED"}

GAMMA = np.float32(1.4)
R_GAS = np.float32(287.05)


class SimParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_float), ("dy", C.c_float),
        ("domain_width", C.c_float), ("domain_height", C.c_float),
        ("mach", C.c_float), ("T_inf", C.c_float), ("p_inf", C.c_float),
        ("rho_inf", C.c_float), ("u_inf", C.c_float), ("v_inf", C.c_float), ("c_inf", C.c_float),
        ("obstacle_x", C.c_float), ("obstacle_y", C.c_float), ("obstacle_r", C.c_float),
        ("obstacle_rotation", C.c_float),
        ("obstacle_shape", C.c_int),
        ("wing_rotation", C.c_float),
        ("cfl", C.c_float), ("dt", C.c_float), ("t_current", C.c_float),
        ("step", C.c_int),
        ("enable_viscosity", C.c_bool),
        ("cfl_visc", C.c_float),
        ("adiabatic_wall", C.c_bool),
        ("T_wall", C.c_float),
        ("paused", C.c_bool),
    ]


assert C.sizeof(SimParams) == 112


class Ext(C.Structure):
    _fields_ = [
        ("flux_scheme", C.c_int), ("limiter", C.c_int), ("prandtl", C.c_float),
        ("dt_policy", C.c_int), ("cone_half_angle", C.c_float), ("cone_length", C.c_float),
        ("ref_length", C.c_float), ("reserved", C.c_int * 8),
    ]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "force_x", "force_y", "cd", "cl", "mass", "mom_x", "mom_y", "energy",
        "wall_heat", "wall_heat_max")] + [("reserved", C.c_double * 6)]


class Result(C.Structure):
    """fvm_result: the outcome of one served request."""
    _fields_ = [("ticket", C.c_longlong), ("status", C.c_int), ("steps", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("t_final", C.c_float), ("dt_last", C.c_float), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double), ("diag", Diag)]


class ServerStats(C.Structure):
    """fvm_server_stats."""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("rejected", C.c_longlong),
                ("batched_steps", C.c_longlong), ("active", C.c_int), ("pending", C.c_int),
                ("budget_bytes", C.c_size_t), ("active_bytes", C.c_size_t), ("parked_bytes", C.c_size_t),
                ("cell_updates", C.c_double), ("busy_s", C.c_double), ("step_ms_p50", C.c_double),
                ("step_ms_p99", C.c_double), ("step_ms_mean", C.c_double), ("reserved", C.c_double * 4)]


class Shedding(C.Structure):
    """fvm_shedding: vortex-shedding statistics of a force history."""
    _fields_ = [("strouhal", C.c_double), ("period", C.c_double), ("cd_mean", C.c_double), ("cl_mean", C.c_double),
                ("cl_rms", C.c_double), ("cycles", C.c_int), ("reserved", C.c_int)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_longlong), ("total_ms", C.c_double)]


def params_default():
    """SimParams with the reference's default member initialisers (src/include/common.h:53-90)."""
    p = SimParams()
    p.nx, p.ny, p.dx, p.dy = 512, 256, 1.0, 1.0
    p.domain_width, p.domain_height = 10.0, 5.0
    p.mach, p.T_inf, p.p_inf = 3.0, 300.0, 101325.0
    p.obstacle_x, p.obstacle_y, p.obstacle_r = 2.5, 2.5, 0.5
    p.obstacle_shape = SHAPE_CIRCLE
    p.cfl, p.dt = 0.5, 1e-6
    p.enable_viscosity, p.cfl_visc = False, 0.4
    p.adiabatic_wall, p.T_wall, p.paused = True, 300.0, True
    return p


def compute_derived(p):
    """SimParams::computeDerived (src/include/common.h:93-101) in float32 arithmetic."""
    f = np.float32
    p.rho_inf = float(f(p.p_inf) / (R_GAS * f(p.T_inf)))
    p.c_inf = float(np.sqrt(GAMMA * R_GAS * f(p.T_inf), dtype=np.float32))
    p.u_inf = float(f(p.mach) * f(p.c_inf))
    p.dx = float(f(p.domain_width) / f(p.nx))
    p.dy = float(f(p.domain_height) / f(p.ny))
    p.obstacle_y = float(f(p.domain_height) / f(2.0))
    return p


def ext_default():
    """Extension knobs that reproduce the reference (HLLC, minmod, Pr 0.71, fixed dt)."""
    e = Ext()
    e.flux_scheme, e.limiter, e.prandtl, e.dt_policy = FLUX_HLLC, LIMITER_MINMOD, 0.71, DT_FIXED
    e.cone_half_angle, e.cone_length, e.ref_length = math.radians(15.0), 0.3, 0.0
    return e


def sutherland(T):
    """Sutherland viscosity with the reference constants (src/include/common.h:13-15)."""
    return 1.716e-5 * (T / 273.15) ** 1.5 * (273.15 + 110.4) / (T + 110.4)


def workload(name, nx=None, ny=None):
    """Seeded SI parameter sets for the benchmark workloads.

    The reference runs in dimensional SI units with absolute clamps
    (src/solver.cu:10-14), so non-dimensional workload descriptions are mapped
    to SI: freestream T=300 K, p=101325 Pa, and the length scale L chosen so
    that the stated Reynolds number holds on the stated length.  Returns
    (SimParams, Ext).
      euler_m3_circle      : [0,2]x[0,1], M3, circle r=0.08 at (0.4,0.5), Euler, L=1 m
      ns_karman_re200      : [0,2]x[0,1], M0.3, Re_D=200 (D=0.1 L), circle r=0.05, no-slip adiabatic
      ns_hypersonic_cone   : [0,2]x[0,1], M8, Re=1e5 on the nose diameter 0.2 L, isothermal
                             T_w = 600 K, blunted cone (nose r=0.1 L, tip at x=0.5 L)
      reference_benchmark  : the reference KernelBenchmark case (src/test/kernel_benchmark.cu:69-83)
    """
    p = params_default()
    e = ext_default()
    p.T_inf, p.p_inf = 300.0, 101325.0
    if name == "euler_m3_circle":
        L = 1.0
        p.nx, p.ny = nx or 512, ny or 256
        p.mach, p.enable_viscosity = 3.0, False
        p.domain_width, p.domain_height = 2.0 * L, 1.0 * L
        p.obstacle_x, p.obstacle_r, p.obstacle_shape = 0.4 * L, 0.08 * L, SHAPE_CIRCLE
        p.cfl = 0.5
    elif name == "ns_karman_re200":
        p.nx, p.ny = nx or 2048, ny or 1024
        p.mach, p.enable_viscosity, p.adiabatic_wall = 0.3, True, True
        compute_derived(p)
        D = 200.0 * sutherland(300.0) / (p.rho_inf * p.u_inf)
        L = D / 0.1
        p.domain_width, p.domain_height = 2.0 * L, 1.0 * L
        p.obstacle_x, p.obstacle_r, p.obstacle_shape = 0.4 * L, 0.05 * L, SHAPE_CIRCLE
        p.cfl = 0.5
        e.prandtl = 0.72
        e.ref_length = D
    elif name == "ns_hypersonic_cone":
        p.nx, p.ny = nx or 8192, ny or 4096
        p.mach, p.enable_viscosity, p.adiabatic_wall = 8.0, True, False
        compute_derived(p)
        D = 1e5 * sutherland(300.0) / (p.rho_inf * p.u_inf)
        L = D / 0.2
        p.domain_width, p.domain_height = 2.0 * L, 1.0 * L
        rn = 0.1 * L
        p.obstacle_x, p.obstacle_r, p.obstacle_shape = 0.5 * L + rn, rn, SHAPE_CONE_CAPSULE
        p.T_wall = 600.0
        p.cfl = 0.4
        e.limiter, e.flux_scheme = LIMITER_VAN_LEER, FLUX_HLLC
        e.cone_half_angle, e.cone_length = math.radians(15.0), 0.3 * L
        e.ref_length = 2.0 * rn
    elif name == "reference_benchmark":
        p.nx, p.ny = nx or 1024, ny or 512
        p.mach, p.enable_viscosity = 3.0, True
        p.cfl, p.cfl_visc = 0.5, 0.4
        p.obstacle_shape, p.obstacle_r = SHAPE_CIRCLE, 0.5
        p.domain_width, p.domain_height = 10.0, 5.0
    else:
        raise ValueError(f"unknown workload {name!r}")
    if nx:
        p.nx = nx
    if ny:
        p.ny = ny
    compute_derived(p)
    return p, e


def _splitmix64(state):
    """One step of splitmix64: returns (new_state, 64-bit output)."""
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


class SeededStream:
    """Deterministic uniform numbers from splitmix64 (platform independent)."""

    def __init__(self, seed):
        self.s = int(seed) & 0xFFFFFFFFFFFFFFFF

    def uniform(self, lo=0.0, hi=1.0):
        self.s, z = _splitmix64(self.s)
        return lo + (hi - lo) * ((z >> 11) * (1.0 / (1 << 53)))

    def log_uniform(self, lo, hi):
        return math.exp(self.uniform(math.log(lo), math.log(hi)))

    def choice(self, seq):
        return seq[min(int(self.uniform() * len(seq)), len(seq) - 1)]


def uneven_instance(rng, sizes=(128, 256, 512, 1024), mach=(0.3, 6.0), re=(1e2, 1e5), p_viscous=0.5):
    """One synthetic solve of the uneven-batch workload: nx drawn from `sizes`,
    ny = nx/2, Mach log-uniform, Euler or Navier-Stokes (Re log-uniform on the
    obstacle diameter), obstacle from the reference shapes 0-4 with size
    0.03-0.1 of the domain height and a random rotation.  SI mapping as in
    `workload`: freestream 300 K / 101325 Pa; L = 1 m for Euler, L from the
    Reynolds number for Navier-Stokes.  Returns (SimParams, Ext)."""
    p = params_default()
    e = ext_default()
    nx = int(rng.choice(list(sizes)))
    p.nx, p.ny = nx, nx // 2
    p.T_inf, p.p_inf = 300.0, 101325.0
    p.mach = rng.log_uniform(*mach)
    viscous = rng.uniform() < p_viscous
    size = rng.uniform(0.03, 0.1)
    p.obstacle_shape = int(rng.choice([SHAPE_CIRCLE, SHAPE_STAR, SHAPE_DIAMOND, SHAPE_CAPSULE, SHAPE_TRIANGLE]))
    p.obstacle_rotation = rng.uniform(0.0, 2.0 * math.pi)
    reynolds = rng.log_uniform(*re)
    p.enable_viscosity = viscous
    compute_derived(p)
    if viscous:
        L = reynolds * sutherland(300.0) / (p.rho_inf * p.u_inf * 2.0 * size)
    else:
        L = 1.0
    p.domain_width, p.domain_height = 2.0 * L, 1.0 * L
    p.obstacle_x, p.obstacle_r = 0.4 * L, size * L
    p.cfl = 0.5
    compute_derived(p)
    e.ref_length = 2.0 * size * L
    e.dt_policy = DT_RECOMPUTE
    return p, e
