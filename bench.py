"""Benchmark: cell-updates/s of the SSP-RK2 step on one B200 per rank.

Workload (default): the hypersonic blunted-cone Navier-Stokes case on an
8192x4096 grid (33.5M cells): Mach 8, Re 1e5 on the nose diameter, isothermal
wall at 600 K, van Leer + HLLC, SSP-RK2, SI units (freestream 300 K,
101325 Pa).  Inputs are seeded synthetic states (freestream start, then
`--settle` steps), resident in HBM; every state (670 MB) exceeds L2, so no
flush is needed between timed steps.

Multi-GPU: one process per GPU, each advancing an independent solve of the
same size (replicas; weak scaling, no data-path collective).  Timing: CUDA
events on the launching stream, barrier + synchronize around the timed
region, max over ranks.

--impl reference times the reference method on the host cores: the CPU
restatement of the reference kernel chain (oracle/liborc64.so, all threads)
on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "fvm-airidynamic-simulator_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

from fvm_b200 import abi  # noqa: E402

WORKLOADS = {
    "ns_hypersonic_cone": (8192, 4096),
    "ns_karman_re200": (2048, 1024),
    "euler_m3_circle": (512, 256),
    "reference_benchmark": (1024, 512),
}
# Algorithmic HBM bytes per cell for each launch of the step (5 conserved
# fields of 4 B, mask 1 B): input state read once, output written once,
# blend partner read once.
KERNEL_BYTES = {"stage1": 41, "stage2": 61, "viscous_pre": 41, "viscous_post": 41}
STEP_BYTES_FUSED = 102  # compulsory bytes per cell-update of a fused 5-field RK2 step


def load_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if ws > 1:
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local, dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_reference(params, ext, steps_budget_s=20.0, sample_nx=None, sample_ny=None):
    """Time the FP64 CPU restatement on a bounded sample of the workload."""
    from oracle.oracle import Oracle
    nx0, ny0 = params.nx, params.ny
    nx = sample_nx or max(64, nx0 // 8)
    ny = sample_ny or max(32, ny0 // 8)
    p, e = abi.SimParams.from_buffer_copy(params), abi.Ext.from_buffer_copy(ext)
    p.nx, p.ny = nx, ny
    abi.compute_derived(p)
    threads = os.cpu_count() or 1
    o = Oracle(p, e, bits=64, threads=threads)
    dt = o.compute_dt()
    o.step(dt)  # warm
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(dt)
        n += 1
        el = time.perf_counter() - t0
        if el >= steps_budget_s or n >= 200:
            break
    rate = nx * ny * n / el
    return rate, threads, f"{nx}x{ny} grid of the same workload (1/{nx0 // nx} resolution), {n} FP64 steps in {el:.1f} s"


def run_reference_arm(args, params, ext, ws, rank, dist):
    if rank != 0:
        return
    budget = float(os.environ.get("FVM_CPU_BUDGET_S", "10"))
    rates = []
    for _ in range(args.warmup):
        cpu_reference(params, ext, steps_budget_s=min(2.0, budget))
    sample = ""
    threads = 1
    for _ in range(args.steps):
        r, threads, sample = cpu_reference(params, ext, steps_budget_s=budget / max(1, args.steps))
        rates.append(r)
    value = statistics.median(rates)
    ms_per_step = params.nx * params.ny / value * 1e3
    line = {
        "impl": "reference", "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded freestream start)",
        "config": {"workload": args.workload, "nx": params.nx, "ny": params.ny},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--settle", type=int, default=20)
    ap.add_argument("--impl", default="fvm", choices=["fvm", "reference"])
    ap.add_argument("--workload", default="ns_hypersonic_cone", choices=sorted(WORKLOADS))
    ap.add_argument("--nx", type=int, default=0)
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="skip the launch-shape autotuner")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    ws, rank, local, dist = dist_setup()
    nx, ny = WORKLOADS[args.workload]
    nx, ny = args.nx or nx, args.ny or ny
    params, ext = abi.workload(args.workload, nx, ny)

    if args.impl == "reference":
        run_reference_arm(args, params, ext, ws, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    import fvm_b200
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    s = fvm_b200.Solver(params, ext)
    s.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        # settle into a non-uniform flow, fixed dt from the start state
        params.dt = s.compute_dt()
        s.step(args.settle)
        if not args.no_autotune:
            s.autotune(steps=4)  # launch shape for this grid class (untimed)
        s.step(args.warmup)
        torch.cuda.synchronize()

        # ---- timed region (device-resident): K steps
        s.set_kernel_timing(False)
        barrier(dist)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        n0 = s.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = s.launch_count() - n0
        ms = ev0.elapsed_time(ev1)
        clk = clocks.stop()
        barrier(dist)
        ms_max = max_over_ranks(ms, dist)

        # ---- per-kernel times (separate pass, events around each launch)
        s.set_kernel_timing(True)
        s.step(max(4, args.steps // 4))
        s.synchronize()
        ktimes = s.kernel_times()
        s.set_kernel_timing(False)

        # ---- end to end through the C ABI with host buffers: upload state,
        # K steps, download state
        import ctypes as C
        U = s.fields()
        host = [torch.from_numpy(np.ascontiguousarray(U[k])).pin_memory() for k in range(5)]
        out = [torch.empty_like(h).pin_memory() for h in host]
        lib = s.lib
        barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fvm_b200._check(lib.fvm_write_fields(s.h, *[C.c_void_p(h.data_ptr()) for h in host]))
        fvm_b200._check(lib.fvm_steps(s.h, C.byref(s.params), args.steps))
        fvm_b200._check(lib.fvm_read_fields(s.h, *[C.c_void_p(o.data_ptr()) for o in out]))
        e2e_s = time.perf_counter() - t0
        e2e_max = max_over_ranks(e2e_s, dist)
        assert all(np.isfinite(o.numpy()).all() for o in out), "non-finite state after the e2e run"

    cells = nx * ny
    value = cells * args.steps * ws / (ms_max / 1e3)
    e2e_value = cells * args.steps * ws / e2e_max
    hbm, peak_kind = load_peaks()
    # dominant kernel by total time
    dom = max(((k, v) for k, v in ktimes.items() if k in KERNEL_BYTES), key=lambda kv: kv[1][1])
    dom_name, (dom_n, dom_ms) = dom
    dom_avg_ms = dom_ms / dom_n
    achieved = KERNEL_BYTES[dom_name] * cells / (dom_avg_ms / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get(args.workload, {}).get(dom_name)
    except Exception:
        pass
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        budget = float(os.environ.get("FVM_CPU_BUDGET_S", "15"))
        r, threads, sample = cpu_reference(params, ext, steps_budget_s=budget)
        cpu = {"value": r, "unit": "cell-updates/s", "cores": threads, "kind": "port", "sample": sample}
    step_gbs = value / ws * STEP_BYTES_FUSED / 1e9
    if rank == 0:
        line = {
            "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded freestream start, settled)",
            "config": {"workload": args.workload, "nx": nx, "ny": ny,
                       "viscous": bool(params.enable_viscosity),
                       "flux": ["hllc", "ausm+"][ext.flux_scheme], "limiter": ["minmod", "van_leer"][ext.limiter],
                       "parallelism": f"replicas x{ws}", "l2": "inputs > L2 (670 MB per state), no flush",
                       "tune": dict(zip(("threads", "ring", "rows_per_cta"), s.tune()))},
            "hbm_gbs_per_gpu_at_102B": step_gbs,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "kernel": dom_name,
                         "algorithmic_bytes_per_cell": KERNEL_BYTES[dom_name], "peak_kind": peak_kind},
            "kernels": {k: {"launches": v[0], "avg_ms": v[1] / v[0]} for k, v in ktimes.items()},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": cells * 20 / args.steps, "d2h_bytes_per_step": cells * 20 / args.steps},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
