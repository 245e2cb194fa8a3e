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
    # many-solve workloads (own code paths below)
    "batched_uneven": (0, 0),
    "serving": (0, 0),
    # the stated runs of the three single-solve configurations and their outputs
    "config_outputs": (0, 0),
}
BATCH_SEED, SERVE_SEED = 4, 5
# Algorithmic HBM bytes per cell for each launch of the step (5 conserved
# fields of 4 B, mask 1 B): input state read once, output written once,
# blend partner read once.
KERNEL_BYTES = {"stage1": 41, "stage2": 61, "viscous_pre": 41, "viscous_post": 41}
STEP_BYTES_FUSED = 102  # compulsory bytes per cell-update of a fused 5-field RK2 step
# Navier-Stokes: the two Strang viscous half steps are passes of their own
# (41 B each: state in, state out, mask)
STEP_BYTES_NS = 184
# DRAM bytes (read + write) per launch measured by ncu on the 4096x2048 case
# and scaled by the cell count to 8192x4096 (profiles/marching_kernels_*.md).
MEASURED_TRAFFIC = {
    ("ns_hypersonic_cone", 8192, 4096): {"stage1": 1250917376, "stage2": 1926714368,
                                         "viscous_pre": 1254623232, "viscous_post": 1235197952},
}


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


def uneven_batch(n, seed=BATCH_SEED):
    """The uneven batched workload: n seeded solves, nx in {128,256,512,1024},
    ny = nx/2, Mach log-uniform 0.3-6, Euler or NS (Re log-uniform 1e2-1e5)
    with p = 0.5, obstacle from the five reference shapes, size 0.03-0.1,
    random rotation; each solve keeps its own CFL time step."""
    rng = abi.SeededStream(seed)
    return [abi.uneven_instance(rng) for _ in range(n)]


def serving_requests(n, lam, seed=SERVE_SEED):
    """Poisson arrivals at rate lam [1/s]: (arrival_s, params, steps); grid
    nx in {256,512,1024,2048}, ny = nx/2, Mach log-uniform 0.3-8, Euler or NS
    (Re log-uniform 1e2-1e5), obstacle as the uneven batch, steps uniform in
    200-5000."""
    import math
    rng = abi.SeededStream(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += -math.log(1.0 - rng.uniform()) / lam
        p, _ = abi.uneven_instance(rng, sizes=(256, 512, 1024, 2048), mach=(0.3, 8.0))
        out.append((t, p, int(rng.uniform(200, 5001))))
    return out


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def solo_rate(torch, fvm_b200, p, ext, stream, steps):
    """Device time of `steps` single-solve steps (graphs warmed for both parities)."""
    s = fvm_b200.Solver(abi.SimParams.from_buffer_copy(p), ext)
    s.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        s.step(3)
        s.step(3)
        ev0, ev1 = _events(torch)
        ev0.record(stream)
        s.step(steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    s.close()
    return ms


def bench_batched(n_inst=256, steps=20, warmup=5, solo_steps=10):
    """Batched step over the uneven workload vs the same solves one at a time."""
    import torch
    import fvm_b200
    insts = uneven_batch(n_inst)
    ext = insts[0][1]
    cells = [p.nx * p.ny for p, _ in insts]
    total = sum(cells)
    stream = torch.cuda.Stream()
    b = fvm_b200.Batch(ext)
    b.set_stream(stream.cuda_stream)
    ids = [b.add(p) for p, _ in insts]
    with torch.cuda.stream(stream):
        b.step(warmup)
        torch.cuda.synchronize()
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        time.sleep(0.2)
        n0 = b.launch_count()
        ev0, ev1 = _events(torch)
        ev0.record(stream)
        b.step(steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        launches = b.launch_count() - n0
        clk = clocks.stop()
    finite = all(np.isfinite(b.diagnostics(i).mass) for i in ids)
    # end to end through the API with host buffers: admit every solve (reusing
    # the parked instances), `steps` batched steps, final states to host memory
    outs = {i: [np.empty(p.nx * p.ny, np.float32) for _ in range(5)] for i, (p, _) in enumerate(insts)}
    for i in ids:
        b.retire(i)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids2 = [b.add(p) for p, _ in insts]
    b.step(steps)
    for k, i in enumerate(ids2):
        fvm_b200._check(b.lib.fvm_batch_read_fields(b.h, i, *[fvm_b200._p(a) for a in outs[k]]))
    e2e_s = time.perf_counter() - t0
    b.close()
    # one solve at a time through the single-solve path (device time only)
    solo_ms = 0.0
    for p, e in insts:
        solo_ms += solo_rate(torch, fvm_b200, p, e, stream, solo_steps)
    rate = total * steps / (ms / 1e3)
    solo = total * solo_steps / (solo_ms / 1e3)
    visc = sum(c for c, (p, _) in zip(cells, insts) if p.enable_viscosity)
    step_bytes = 102 * (total - visc) + 184 * visc
    return {
        "value": rate, "unit": "cell-updates/s", "ms_per_step": ms / steps, "instances": n_inst,
        "cells": total, "steps": steps, "warmup": warmup,
        "solves_per_s_at_500_steps": n_inst / (500 * ms / steps / 1e3),
        "one_at_a_time": {"value": solo, "unit": "cell-updates/s",
                          "sample": f"each of the {n_inst} solves alone, {solo_steps} steps, device time summed"},
        "speedup_vs_one_at_a_time": rate / solo,
        "step_gbs": step_bytes / (ms / steps / 1e3) / 1e9,
        "e2e": {"value": total * steps / e2e_s, "unit": "cell-updates/s",
                "h2d_bytes_per_step": n_inst * 112 / steps, "d2h_bytes_per_step": total * 20 / steps,
                "includes": "admission of every solve (instance reuse), steps, final states to host"},
        "gpu_launches": launches, "finite": bool(finite), "clocks": clk,
    }


def one_at_a_time(torch, fvm_b200, reqs, ext, stream):
    """The same arrivals served one solve at a time on this GPU, first come
    first served: each request waits for its arrival and for the previous
    solve, then a single-solve handle is created, stepped, its FP64
    diagnostics read to the host and the handle destroyed.  Wall-clock times
    like the server's.  Returns (sorted completion latencies, span, work)."""
    t0 = time.perf_counter()
    lat, work, done = [], 0, 0.0
    for t, p, n in reqs:
        now = time.perf_counter() - t0
        if now < t:
            time.sleep(t - now)
        s = fvm_b200.Solver(abi.SimParams.from_buffer_copy(p), ext)
        s.set_stream(stream.cuda_stream)
        s.step(n)
        s.diagnostics()
        s.close()
        done = time.perf_counter() - t0
        lat.append(done - t)
        work += p.nx * p.ny * n
    return sorted(lat), done - reqs[0][0], work


def bench_serving(lams=(10.0, 100.0, 1000.0), n_req=48, chunk=64, budget=150 * 10**9, class_steps=20):
    """Continuous-batching request loop on Poisson arrivals, against the same
    arrivals served one solve at a time on the same GPU (measured)."""
    import torch
    import fvm_b200
    stream = torch.cuda.Stream()
    ext = abi.ext_default()
    ext.dt_policy = abi.DT_RECOMPUTE
    # single-solve rate per (grid, viscous) class: what batching can gain on a mix
    class_rate = {}
    rng = abi.SeededStream(SERVE_SEED + 1)
    for nx in (256, 512, 1024, 2048):
        for visc in (False, True):
            while True:
                p, _ = abi.uneven_instance(rng, sizes=(nx,), mach=(0.3, 8.0))
                if bool(p.enable_viscosity) == visc:
                    break
            ms = solo_rate(torch, fvm_b200, p, ext, stream, class_steps)
            class_rate[(nx, visc)] = p.nx * p.ny * class_steps / (ms / 1e3)
    q = lambda v, f: v[min(len(v) - 1, int(round(f * (len(v) - 1))))] if v else None  # noqa: E731
    sweep = []
    for lam in lams:
        reqs = serving_requests(n_req, lam)
        srv = fvm_b200.Server(ext, budget_bytes=budget, chunk_steps=chunk)
        import threading
        clk_srv = ClockSampler(torch.cuda.current_device())
        clk_srv.start()
        t_start = time.perf_counter()

        def client():
            for t, p, n in reqs:
                d = t_start + t - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                srv.submit(p, n, keep_fields=False)

        th = threading.Thread(target=client)
        th.start()
        th.join()
        srv.drain()
        res = [r for r, _ in srv.poll(cap=n_req)]
        st = srv.stats()
        srv.close()
        clocks_served = clk_srv.stop()
        ok = [r for r in res if r.status == 0]
        work = sum(r.nx * r.ny * r.steps for r in ok)
        span = max(r.done_s for r in res) - min(r.submit_s for r in res)
        lat = sorted(r.done_s - r.submit_s for r in ok)
        clk_solo = ClockSampler(torch.cuda.current_device())
        clk_solo.start()
        solo_lat, solo_span, solo_work = one_at_a_time(torch, fvm_b200, reqs, ext, stream)
        clocks_solo = clk_solo.stop()
        # every request at its class's single-solve rate: the work-weighted
        # single-solve rate, the one-at-a-time rate without set-up or idle time
        solo_model_s = sum(p.nx * p.ny * n / class_rate[(p.nx, bool(p.enable_viscosity))] for _, p, n in reqs)
        sweep.append({
            "lambda_per_s": lam, "requests": n_req, "completed_ok": len(ok), "failed": len(res) - len(ok),
            "value": work / span, "unit": "cell-updates/s",
            "completion_s_p50": q(lat, 0.5), "completion_s_p99": q(lat, 0.99),
            "step_ms_p50": st.step_ms_p50, "step_ms_p99": st.step_ms_p99,
            "device_busy_frac": st.busy_s / span,
            "one_at_a_time": {"value": solo_work / solo_span, "unit": "cell-updates/s",
                              "completion_s_p50": q(solo_lat, 0.5), "completion_s_p99": q(solo_lat, 0.99),
                              "measured": "same arrivals, one single-solve handle at a time, FIFO, wall clock",
                              "clocks": clocks_solo},
            "clocks": clocks_served,
            "speedup_vs_one_at_a_time": (work / span) / (solo_work / solo_span),
            "single_solve_rate_work_weighted": solo_work / solo_model_s,
            "batched_steps": st.batched_steps,
        })
    return {"sweep": sweep, "class_rates": {f"{k[0]}x{k[0] // 2}{'_ns' if k[1] else '_euler'}": v
                                            for k, v in class_rate.items()},
            "budget_bytes": budget, "chunk_steps": chunk}


def reference_cuda(grids=((8192, 4096), (1024, 512)), steps=20):
    """The reference's own FP32 CUDA KernelBenchmark (src/test/kernel_benchmark.cu,
    built unmodified from the reference sources into oracle/_ref/) beside the
    same case through this library's CFDSolver shim, on this GPU: ms per step
    of each (each program's own host-clock timing of its timed steps), with
    the clocks seen."""
    ref_bin = os.path.join(REPO, "oracle", "_ref", "kernel_benchmark")
    own_bin = os.path.join(PKG, "fvm_b200", "lib", "kernel_benchmark")
    if not (os.path.exists(ref_bin) and os.path.exists(own_bin)):
        return {"unavailable": "reference KernelBenchmark or shim benchmark not built"}

    def avg_ms(cmd):
        # the reference prints "Total time: X ms" over "Running benchmark (N
        # steps)" with two decimals; the total keeps more of them than its
        # per-step line.  The shim prints "Avg per step: X ms" with four.
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        total, n, avg = None, None, None
        for ln in out.stdout.splitlines():
            ln = ln.strip()
            if ln.startswith("Total time:"):
                total = float(ln.split()[2])
            elif "Running benchmark (" in ln:
                n = int(ln.split("(")[1].split()[0])
            elif ln.startswith("Avg per step:"):
                avg = float(ln.split()[3])
        if total is not None and n:
            return total / n
        if avg is not None:
            return avg
        raise RuntimeError(f"{cmd[0]}: no timing line (rc {out.returncode}): {out.stderr[-200:]}")

    clocks = ClockSampler(0)
    clocks.start()
    rows = []
    for nx, ny in grids:
        r = avg_ms([ref_bin, str(nx), str(ny)])
        o = avg_ms([own_bin, str(nx), str(ny), str(steps)])
        rows.append({"grid": f"{nx}x{ny}", "reference_ms_per_step": r, "this_ms_per_step": o, "speedup": r / o})
    return {"case": "reference KernelBenchmark: NS Mach 3 circle, HLLC + minmod, fixed dt, one step() per step",
            "rows": rows, "clocks": clocks.stop()}


def grid_scaling(torch, fvm_b200, nx=4096, ny=2048, steps=20, settle=20):
    """The cone workload at another grid size (autotuned launch shape): device
    time per step and per kernel, to set beside the 8192x4096 figures."""
    params, ext = abi.workload("ns_hypersonic_cone", nx, ny)
    ext.dt_policy = abi.DT_RECOMPUTE
    stream = torch.cuda.Stream()
    s = fvm_b200.Solver(params, ext)
    s.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        s.step(settle)
        s.autotune(steps=4)
        s.step(5)
        ev0, ev1 = _events(torch)
        ev0.record(stream)
        s.step(steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        s.set_kernel_timing(True)
        s.step(10)
        s.synchronize()
        kt = s.kernel_times()
        s.set_kernel_timing(False)
    tune = dict(zip(("threads", "ring", "rows_per_cta"), s.tune()))
    s.close()
    return {"grid": f"{nx}x{ny}", "cells": nx * ny, "ms_per_step": ms, "cell_updates_per_s": nx * ny / (ms / 1e3),
            "kernels": {k: {"launches": v[0], "avg_ms": v[1] / v[0]} for k, v in kt.items()}, "tune": tune}


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


def run_config_outputs(args, ws, rank, local):
    """The stated runs and outputs of the single-solve configurations, each
    timed on the device: Euler Mach-3 circle 512x256 for 200 steps (AUSM+ and
    HLLC); Re-200 vortex street 2048x1024 for 20000 steps (drag / lift
    history, Strouhal number when the history holds whole shedding cycles);
    Mach-8 blunted cone 8192x4096 for 2000 steps (standoff, wall heat flux)."""
    import torch
    import fvm_b200
    torch.cuda.set_device(local)
    out = {}

    def timed(s, n, every=None, sample=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        done = 0
        while done < n:
            k = min(every or n, n - done)
            e0.record()
            s.step(k)
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
            done += k
            if sample:
                sample(s)
        return total

    for flux, tag in ((abi.FLUX_AUSM_PLUS, "ausm+"), (abi.FLUX_HLLC, "hllc")):
        p, e = abi.workload("euler_m3_circle", 512, 256)
        e.flux_scheme, e.dt_policy = flux, abi.DT_RECOMPUTE
        s = fvm_b200.Solver(p, e)
        ms = timed(s, 200)
        d = s.diagnostics()
        out[f"c1_euler_m3_circle_512x256_200steps_{tag}"] = {
            "ms_total": ms, "cell_updates_per_s": 512 * 256 * 200 / (ms / 1e3), "cd": d.cd, "cl": d.cl,
            "mass": d.mass, "t_end_s": s.params.t_current}
        s.close()
    p, e = abi.workload("ns_karman_re200", 2048, 1024)
    e.dt_policy = abi.DT_RECOMPUTE
    s = fvm_b200.Solver(p, e)
    hist = []
    ms = timed(s, 20000, every=20, sample=lambda x: hist.append((x.params.t_current, x.diagnostics())))
    t = np.array([h[0] for h in hist])
    cd = np.array([h[1].cd for h in hist])
    cl = np.array([h[1].cl for h in hist])
    D, U = e.ref_length, p.u_inf
    c2 = {"ms_total": ms, "cell_updates_per_s": 2048 * 1024 * 20000 / (ms / 1e3),
          "t_end_over_D_per_U": float(t[-1] / (D / U)), "cd_final": float(cd[-1]), "cl_final": float(cl[-1]),
          "cd_mean_last_quarter": float(cd[3 * len(cd) // 4:].mean())}
    try:
        st = fvm_b200.shedding_stats(t[len(t) // 2:], cd[len(t) // 2:], cl[len(t) // 2:], D, U)
        c2.update({"strouhal": st.strouhal, "cd_cycle_mean": st.cd_mean, "shedding_cycles": st.cycles})
    except fvm_b200.FvmError:
        c2["strouhal"] = None  # no whole shedding cycle yet in the stated 20000 steps
    out["c2_ns_karman_re200_2048x1024_20000steps"] = c2
    s.close()
    p, e = abi.workload("ns_hypersonic_cone", 8192, 4096)
    e.dt_policy = abi.DT_RECOMPUTE
    s = fvm_b200.Solver(p, e)
    ms = timed(s, 2000)
    d = s.diagnostics()
    out["c3_ns_hypersonic_cone_8192x4096_2000steps"] = {
        "ms_total": ms, "cell_updates_per_s": 8192 * 4096 * 2000 / (ms / 1e3), "standoff_m": s.shock_standoff(),
        "standoff_over_nose_radius": s.shock_standoff() / p.obstacle_r, "wall_heat_w_per_m": d.wall_heat,
        "wall_heat_max_w_per_m2": d.wall_heat_max, "cd": d.cd, "t_end_s": s.params.t_current}
    s.close()
    if rank == 0:
        c3 = out["c3_ns_hypersonic_cone_8192x4096_2000steps"]
        print(json.dumps({"metric": "cell_updates_per_s", "value": c3["cell_updates_per_s"] * ws,
                          "unit": "cell-updates/s", "n_gpus": ws, "steps": 2000, "warmup": 0,
                          "ms_per_step": c3["ms_total"] / 2000, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic (freestream start)",
                          "config": {"workload": "config_outputs"}, "outputs": out}), flush=True)


def run_many_solves(args, ws, rank, local, dist):
    """batched_uneven / serving: one line per run on rank 0 (other ranks run
    replicas of the same work; weak scaling)."""
    if args.impl == "reference":
        if rank != 0:
            return
        # the reference method on the host cores, one solve at a time, on a
        # bounded sample of the same solves
        if args.workload == "batched_uneven":
            sample = [p for p, _ in uneven_batch(args.instances)]
        else:
            sample = [p for _, p, _ in serving_requests(args.requests, 100.0)]
        budget = float(os.environ.get("FVM_CPU_BUDGET_S", "10"))
        cu, secs, used, threads = 0.0, 0.0, 0, 1
        from oracle.oracle import Oracle
        e = abi.ext_default()
        e.dt_policy = abi.DT_RECOMPUTE
        threads = os.cpu_count() or 1
        for p in sample:
            o = Oracle(p, e, bits=64, threads=threads)
            dt = o.compute_dt()
            o.step(dt)
            t0 = time.perf_counter()
            n = 0
            while n < 3 or (time.perf_counter() - t0) < budget / 8 and n < 20:
                o.step(o.compute_dt())
                n += 1
            secs += time.perf_counter() - t0
            cu += p.nx * p.ny * n
            used += 1
            if secs >= budget:
                break
        value = cu / secs
        line = {"impl": "reference", "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded solves)", "config": {"workload": args.workload},
                "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                                 "sample": f"first {used} solves of the workload, one at a time, FP64"},
                "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    barrier(dist)
    if args.workload == "batched_uneven":
        r = bench_batched(n_inst=args.instances, steps=args.steps, warmup=args.warmup)
        ms = max_over_ranks(r["ms_per_step"], dist)
        value = r["cells"] * ws / (ms / 1e3)
        hbm, peak_kind = load_peaks()
        line = {
            "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded solves)",
            "config": {"workload": "batched_uneven", "instances": args.instances, "cells": r["cells"],
                       "dt": "per-solve CFL", "l2": f"inputs > L2 ({r['cells'] * 20 / 1e6:.0f} MB per state set)"},
            "roofline": {"bound": "hbm", "achieved": r["step_gbs"], "peak": hbm, "unit": "GB/s",
                         "frac": r["step_gbs"] / hbm, "traffic": None, "kernel": "whole batched step",
                         "algorithmic_bytes_per_cell": "102 (Euler) / 184 (NS)", "peak_kind": peak_kind},
            "solves_per_s_at_500_steps": r["solves_per_s_at_500_steps"],
            "one_at_a_time": r["one_at_a_time"], "speedup_vs_one_at_a_time": r["speedup_vs_one_at_a_time"],
            "cpu_baseline": None, "e2e": r["e2e"], "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "finite": r["finite"],
        }
    else:
        lams = tuple(float(x) for x in args.lambdas.split(","))
        r = bench_serving(lams=lams, n_req=args.requests)
        top = r["sweep"][-1]
        value = top["value"] * ws  # replicas of the same request stream
        line = {
            "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": None, "warmup": None, "ms_per_step": top["step_ms_p50"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Poisson requests)",
            "config": {"workload": "serving", "requests_per_rate": args.requests, "lambdas": list(lams),
                       "budget_bytes": r["budget_bytes"], "chunk_steps": r["chunk_steps"]},
            "latency": {"completion_s_p50": top["completion_s_p50"], "completion_s_p99": top["completion_s_p99"],
                        "step_ms_p50": top["step_ms_p50"], "step_ms_p99": top["step_ms_p99"]},
            "sweep": r["sweep"], "class_rates": r["class_rates"],
            # per batched step: each request's parameters in (112 B), its result record out (184 B)
            "e2e": {"value": value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": args.requests * 112 / max(1, top["batched_steps"]),
                    "d2h_bytes_per_step": args.requests * 184 / max(1, top["batched_steps"]),
                    "includes": "submit from host to final diagnostics on host"},
        }
    if rank == 0:
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
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the batched and serving summaries")
    ap.add_argument("--instances", type=int, default=256, help="batched_uneven: number of solves")
    ap.add_argument("--requests", type=int, default=48, help="serving: requests per arrival rate")
    ap.add_argument("--lambdas", default="10,100,1000", help="serving: arrival rates [1/s]")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    ws, rank, local, dist = dist_setup()
    if args.workload == "config_outputs" and args.impl == "fvm":
        run_config_outputs(args, ws, rank, local)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.workload in ("batched_uneven", "serving"):
        run_many_solves(args, ws, rank, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    # the reference arm of config_outputs times the cone case's CPU restatement
    wl = "ns_hypersonic_cone" if args.workload == "config_outputs" else args.workload
    nx, ny = WORKLOADS[wl]
    nx, ny = args.nx or nx, args.ny or ny
    params, ext = abi.workload(wl, nx, ny)

    if args.impl == "reference":
        run_reference_arm(args, params, ext, ws, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    import fvm_b200
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    # every step takes the CFL time step of its own start state (reduced on
    # the device, fused into the step's last kernels): the flow stays within
    # the stability limit while the bow shock forms
    ext.dt_policy = abi.DT_RECOMPUTE
    s = fvm_b200.Solver(params, ext)
    s.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        # settle into a non-uniform flow
        s.step(args.settle)
        if not args.no_autotune:
            s.autotune(steps=4)  # launch shape for this grid class (untimed)
        # W warm-up steps as W-1 and 1: the first call captures the two-step
        # graphs, the second the one-step graphs (both buffer parities each),
        # so the timed steps replay graphs and capture none
        s.step(max(args.warmup - 1, 2))
        s.step(1)
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

        # ---- colour image of the Mach field (headless renderer pass), RGBA8
        img = torch.empty((nx * ny, 4), dtype=torch.uint8, device="cuda")
        for _ in range(3):
            s.colormap_to_device(abi.FIELD_MACH, abi.CMAP_JET, 0.0, 10.0, img.data_ptr(), abi.RGBA_U8)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(10):
            s.colormap_to_device(abi.FIELD_MACH, abi.CMAP_JET, 0.0, 10.0, img.data_ptr(), abi.RGBA_U8)
        c1.record(stream)
        torch.cuda.synchronize()
        cmap_ms = c0.elapsed_time(c1) / 10
        del img

        # ---- end to end through the C ABI, the reference application's
        # frame loop (src/main.cpp:285-367, one step per frame): step with the
        # time step read back at the end of the previous frame, the Mach
        # field into a device buffer (the display buffer), maximum
        # temperature and Mach number to the host at most every 0.25 s (the
        # first frame included), the next time step queued, the stream
        # synchronized, the time step read back
        import ctypes as C
        lib = s.lib
        e_fixed = abi.Ext.from_buffer_copy(ext)
        e_fixed.dt_policy = abi.DT_FIXED
        s.set_ext(e_fixed)
        field = torch.empty(nx * ny, dtype=torch.float32, device="cuda")
        dt_c, tmax, mmax = C.c_float(), C.c_float(), C.c_float()
        stats_reads = [0, -1.0]

        def frame():
            s.params.dt = dt_c.value
            fvm_b200._check(lib.fvm_steps(s.h, C.byref(s.params), 1))
            fvm_b200._check(lib.fvm_field_to_device(s.h, abi.FIELD_MACH, C.c_void_p(field.data_ptr())))
            now = time.perf_counter()
            if stats_reads[1] < 0 or now - stats_reads[1] >= 0.25:
                fvm_b200._check(lib.fvm_max_temperature(s.h, C.byref(tmax)))
                fvm_b200._check(lib.fvm_max_mach(s.h, C.byref(mmax)))
                stats_reads[0] += 1
                stats_reads[1] = now
            fvm_b200._check(lib.fvm_queue_dt(s.h, C.byref(s.params)))
            fvm_b200._check(lib.fvm_synchronize(s.h))  # the app's cudaDeviceSynchronize
            fvm_b200._check(lib.fvm_read_dt(s.h, C.byref(s.params), C.byref(dt_c)))

        def frame_loop(display):
            # display: the Mach buffer registered as the solver's display
            # field (fvm_set_display_field), so the step's last passes write
            # it and the frame's fvm_field_to_device finds it fresh; otherwise
            # a separate derived-field pass per frame
            fvm_b200._check(lib.fvm_set_display_field(s.h, abi.FIELD_MACH,
                                                      C.c_void_p(field.data_ptr() if display else None)))
            fvm_b200._check(lib.fvm_compute_dt(s.h, C.byref(s.params), C.byref(dt_c)))
            for _ in range(args.warmup):
                frame()
            barrier(dist)
            torch.cuda.synchronize()
            stats_reads[:] = [0, -1.0]
            t0 = time.perf_counter()
            for _ in range(args.steps):
                frame()
            secs = time.perf_counter() - t0
            assert np.isfinite(tmax.value) and np.isfinite(mmax.value) and dt_c.value > 0
            return max_over_ranks(secs, dist), stats_reads[0]

        sep_max, _ = frame_loop(False)
        app_max, app_stats_reads = frame_loop(True)
        fvm_b200._check(lib.fvm_set_display_field(s.h, abi.FIELD_MACH, None))
        s.set_ext(ext)
        s.step(3)  # captures the step graphs again (a new policy drops them)
        torch.cuda.synchronize()

        # ---- end to end with the whole state through host memory: upload
        # the state from pinned host buffers, K steps, download the state
        U = s.fields()
        host = [torch.from_numpy(np.ascontiguousarray(U[k])).pin_memory() for k in range(5)]
        out = [torch.empty_like(h).pin_memory() for h in host]
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
    app_value = cells * args.steps * ws / app_max
    sep_value = cells * args.steps * ws / sep_max
    hbm, peak_kind = load_peaks()
    # dominant kernel by total time
    dom = max(((k, v) for k, v in ktimes.items() if k in KERNEL_BYTES), key=lambda kv: kv[1][1])
    dom_name, (dom_n, dom_ms) = dom
    dom_avg_ms = dom_ms / dom_n
    achieved = KERNEL_BYTES[dom_name] * cells / (dom_avg_ms / 1e3) / 1e9
    traffic = MEASURED_TRAFFIC.get((args.workload, nx, ny), {}).get(dom_name)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        budget = float(os.environ.get("FVM_CPU_BUDGET_S", "15"))
        r, threads, sample = cpu_reference(params, ext, steps_budget_s=budget)
        cpu = {"value": r, "unit": "cell-updates/s", "cores": threads, "kind": "port", "sample": sample}
    step_bytes = STEP_BYTES_NS if params.enable_viscosity else STEP_BYTES_FUSED
    step_gbs = value / ws * step_bytes / 1e9
    tune = dict(zip(("threads", "ring", "rows_per_cta"), s.tune()))
    s.close()
    extras = {}
    if rank == 0 and ws == 1 and not args.no_extras:
        import torch
        for name, fn in (("reference_cuda", reference_cuda),
                         ("scaling_4096x2048", lambda: grid_scaling(torch, fvm_b200)),
                         ("batched", lambda: bench_batched(n_inst=args.instances, steps=10, warmup=args.warmup)),
                         ("serving", lambda: bench_serving(lams=(10.0, 100.0, 1000.0), n_req=args.requests))):
            try:
                extras[name] = fn()
            except Exception as exc:  # reported, never hides the main line
                extras[name] = {"error": repr(exc)}
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
                       "tune": tune},
            "step_hbm": {"gbs_per_gpu": step_gbs, "algorithmic_bytes_per_cell": step_bytes,
                         "frac": step_gbs / hbm,
                         "basis": "whole step: 5 conserved fields in and out of every pass, mask bytes"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "kernel": dom_name,
                         "algorithmic_bytes_per_cell": KERNEL_BYTES[dom_name], "peak_kind": peak_kind},
            "kernels": {k: {"launches": v[0], "avg_ms": v[1] / v[0]} for k, v in ktimes.items()},
            "cpu_baseline": cpu,
            # per frame: dt and simulated time to the device as 8 B of kernel
            # arguments; the 176-byte device-scalar block back by fvm_queue_dt and
            # again by fvm_synchronize (error word), 4 B per statistic read
            "e2e": {"value": app_value, "unit": "cell-updates/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": 2 * 176 + 8 * app_stats_reads / args.steps,
                    "ms_per_frame": app_max / args.steps * 1e3,
                    "protocol": "reference app frame loop, one step per frame: fvm_steps(1) with the host's dt, "
                                "Mach field into a device buffer (registered once as the display field, "
                                "written by the step's last passes; fvm_field_to_device per frame), max T and "
                                "max Mach to host every 0.25 s, fvm_queue_dt + fvm_synchronize + fvm_read_dt "
                                "(dt to host)",
                    "separate_field_pass": {"value": sep_value, "ms_per_frame": sep_max / args.steps * 1e3,
                                            "protocol": "the same frames with a derived-field pass per frame"}},
            "e2e_state_roundtrip": {"value": e2e_value, "unit": "cell-updates/s", "steps_per_roundtrip": args.steps,
                                    "h2d_bytes_per_step": cells * 20 / args.steps,
                                    "d2h_bytes_per_step": cells * 20 / args.steps,
                                    "includes": "whole state from pinned host memory, K steps, whole state back"},
            "gpu_launches": launches,
            "clocks": clk,
            # Mach field (reads rho, rho_u, rho_v, rho_e = 16 B + class 1 B, writes 4 B per cell)
            "colormap": {"field": "mach", "format": "rgba8", "ms_per_image": cmap_ms,
                         "gbs": 21 * cells / (cmap_ms / 1e3) / 1e9,
                         "frac": 21 * cells / (cmap_ms / 1e3) / 1e9 / hbm},
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
