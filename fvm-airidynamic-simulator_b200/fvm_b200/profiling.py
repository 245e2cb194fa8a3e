"""Summaries of Nsight Compute exports for the library's kernels.

    python -m fvm_b200.profiling launches <ncu --csv launch-list file>
    python -m fvm_b200.profiling raw <ncu -i X.ncu-rep --page raw --csv output file>

`launches` aggregates a `--metrics gpu__time_duration.sum` launch list per
kernel (launches, total time, share).  `raw` prints the metrics the design
notes use (duration, DRAM bytes and throughput, issue activity, warps, top
stall reasons) per captured launch.
"""
import collections
import csv
import sys

_UNIT = {"ns": 1e-6, "nsecond": 1e-6, "us": 1e-3, "usecond": 1e-3, "ms": 1.0, "msecond": 1.0, "s": 1e3,
         "second": 1e3}


def _kernel(name):
    name = name.replace("void ", "")
    base = name.split("(")[0]
    return base.replace("fvm::", "")


def launches(path):
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    hdr = rows[hi]
    ki, mi, vi, ui = (hdr.index(k) for k in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    agg = collections.OrderedDict()
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[mi] != "gpu__time_duration.sum":
            continue
        ms = float(r[vi].replace(",", "")) * _UNIT.get(r[ui].strip(), 1e-6)
        a = agg.setdefault(_kernel(r[ki]), [0, 0.0])
        a[0] += 1
        a[1] += ms
    tot = sum(v[1] for v in agg.values()) or 1.0
    out = ["| kernel | launches | total ms | mean ms | share |", "|---|---|---|---|---|"]
    for k, (n, ms) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        out.append(f"| `{k}` | {n} | {ms:.3f} | {ms / n:.4f} | {100 * ms / tot:.1f} % |")
    return "\n".join(out)


RAW = [
    ("gpu__time_duration.sum", "duration"),
    ("dram__bytes_read.sum", "DRAM read"),
    ("dram__bytes_write.sum", "DRAM write"),
    ("gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "DRAM throughput % of peak"),
    ("sm__throughput.avg.pct_of_peak_sustained_elapsed", "SM throughput % of peak"),
    ("smsp__issue_active.avg.pct_of_peak_sustained_active", "issue active %"),
    ("smsp__inst_executed.sum", "warp instructions"),
    ("sm__warps_active.avg.per_cycle_active", "warps active / SM"),
    ("launch__registers_per_thread", "registers / thread"),
    ("launch__occupancy_limit_shared_mem", "CTA limit (smem)"),
    ("sm__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active", "XU (MUFU) pipe %"),
    ("sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active", "FMA pipe %"),
    ("l1tex__data_bank_conflicts_pipe_lsu_mem_shared.sum", "smem bank conflicts"),
]


def raw(path):
    rows = list(csv.reader(open(path)))
    hdr, units, data = rows[0], rows[1], rows[2:]
    idx = {h: i for i, h in enumerate(hdr)}
    out = []
    for d in data:
        out.append(f"### `{_kernel(d[idx['Kernel Name']])}`")
        out.append("| metric | value |")
        out.append("|---|---|")
        for key, label in RAW:
            if key in idx:
                out.append(f"| {label} (`{key}`) | {d[idx[key]]} {units[idx[key]]} |")
        stalls = {h: float(v) for h, v in zip(hdr, d)
                  if h.startswith("smsp__average_warps_issue_stalled_") and h.endswith("_per_issue_active.ratio")
                  and v not in ("", "n/a")}
        top = sorted(stalls.items(), key=lambda kv: -kv[1])[:6]
        out.append("| top stalls per issued instruction | " + ", ".join(
            f"{h[len('smsp__average_warps_issue_stalled_'):-len('_per_issue_active.ratio')]} {v:.2f}"
            for h, v in top) + " |")
        out.append("")
    return "\n".join(out)


if __name__ == "__main__":
    mode, path = sys.argv[1], sys.argv[2]
    print(launches(path) if mode == "launches" else raw(path))
