"""Benchmark of the whole conformer pipeline: ``generate_conformers_nk(run_mmff=True)``.

DG (4-D) -> retry -> stereo checks -> collapse -> ETK -> MMFF94 for N synthetic
molecules x k conformers (heavy atoms 10-30), the reference's automatic
iteration budgets, wall-clock time of the call (the molecules are generated
beforehand; their DG/ETK/MMFF terms are extracted inside the call, as the
reference extracts with RDKit inside its).  The reference publishes
"DG + ETK + MMFF" at 614 conformers/s for 20 x 50 and 1,250 for 1000 x 10 on an
M3 Max (docs/BENCHMARKS.md:44-61).

Per workload: conformers/s of the call (median of ``--repeats`` after one
warm-up call), the fraction converged by the reference's rule (every stage),
the seconds of each part (embedding host / GPU, ETK host / GPU, MMFF), and the
host CPU: the metric-matrix starts come from LAPACK's ``eigh`` on the host,
whose last-bit rounding can differ between CPU models, so the converged
fraction may move by a few conformers between machines.

Usage: python -m mlxmolkit_b200.pipeline_bench [--workloads 20x50,1000x10] [--repeats 3]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import synth
from .conformer_pipeline_v2 import generate_conformers_nk


def _host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def run(n_mols: int, k: int, repeats: int, seed: int = 0) -> dict:
    import torch
    mols = synth.make_molecules(n_mols, 1, seed, 10, 30)
    generate_conformers_nk(mols, k, run_mmff=True)                 # warm-up: library load, first launches
    times, parts, res = [], [], None
    for _ in range(repeats):
        tm = {}
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = generate_conformers_nk(mols, k, run_mmff=True, timings=tm)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
        parts.append(tm)
    i = int(np.argsort(times)[len(times) // 2])
    conv = np.concatenate([r.converged for r in res.molecules])
    return {"workload": f"{n_mols}x{k} synthetic, heavy atoms 10-30", "conformers": int(res.total_conformers),
            "seconds": times[i], "conf_per_s": res.total_conformers / times[i],
            "converged": float(conv.mean()), "parts_s": {k2: round(v, 4) for k2, v in parts[i].items()},
            "host_cpu": _host_cpu(), "host_threads": os.cpu_count()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="20x50,1000x10")
    ap.add_argument("--repeats", type=int, default=3)
    a = ap.parse_args()
    for w in a.workloads.split(","):
        n, k = (int(v) for v in w.split("x"))
        print(json.dumps(run(n, k, a.repeats)), flush=True)


if __name__ == "__main__":
    main()
