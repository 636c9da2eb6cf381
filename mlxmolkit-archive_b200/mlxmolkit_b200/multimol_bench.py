"""Benchmark of ``mmff_optimize_metal_multi_mol`` (the reference's multi-molecule L-BFGS)
and ``mmff_optimize_metal_fused_multi_mol`` (its fused steepest descent).

The small workload: 50 seeded molecules x 50 conformers (heavy atoms 10-30,
MMFF94).  It reports ms per conformer and how many conformers end within
0.1 kcal/mol of the FP64 minimum from the same start (each leg: one untimed
warm-up call, then the median of ``--repeats`` timed calls): an all-FP64 dense BFGS
with RDKit's optimizer constants and 2000 iterations, computed once.  These are
the quantities of the reference's published MULTI and FUSED rows (ms/conf and
"within 0.1 kcal/mol" out of 2500, docs/BENCHMARKS.md:22-27).  The energies compared
are the multi-mol result's own (mega-kernel term constants) against the FP64
minimum with the same constants.

Usage: python -m mlxmolkit_b200.multimol_bench [--iters 1000,2000] [--fused-iters 200,500,1000,2000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import mmff_minimize as mm
from . import synth
from .mmff_metal_optimizer import mmff_optimize_metal_fused_multi_mol, mmff_optimize_metal_multi_mol
from .mmff_params import extract_mmff_params


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", default="1000,2000")
    ap.add_argument("--fused-iters", default="200,500,1000,2000")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--threads", default="0", help="multi-mol threads per conformer: a comma list of 0/64/128/256")
    ap.add_argument("--scale", type=float, default=1.0)
    a = ap.parse_args()
    import torch
    wl = synth.make_workload("small", seed=0, scale=a.scale)
    params = [extract_mmff_params(m) for m in wl.mols]
    counts = [m.GetNumConformers() for m in wl.mols]
    start = [np.stack([c.pos.copy() for c in m.GetConformers()]) for m in wl.mols]
    pos = np.concatenate([s.reshape(-1) for s in start]).astype(np.float32)
    ref = mm.Minimizer(params, counts).minimize(pos, max_iters=2000, precision="fp64", consts=mm.RDKIT_CONSTS,
                                                mode=mm.MODE_MEGA)
    C = int(sum(counts))
    out = {"workload": f"small-50x50-heavy10-30 x scale {a.scale}", "conformers": C, "runs": []}
    legs = [("multi", int(v), int(t)) for v in a.iters.split(",") if v for t in a.threads.split(",")] + \
           [("fused", int(v), 0) for v in a.fused_iters.split(",") if v]
    def run(fn, iters):
        for m, s in zip(wl.mols, start):                  # every run starts from the same coordinates
            for c, x in zip(m.GetConformers(), s):
                c.pos[:] = x
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = fn([(m, None) for m in wl.mols], max_iters=iters)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t

    for api, iters, threads in legs:
        if api == "multi":
            def fn(specs, max_iters, _t=threads):
                return mmff_optimize_metal_multi_mol(specs, max_iters=max_iters, threads=_t)
        else:
            fn = mmff_optimize_metal_fused_multi_mol
        run(fn, iters)                                    # untimed warm-up, as the reference's script does
        times = []
        for _ in range(a.repeats):
            r, t = run(fn, iters)
            times.append(t)
        dt = float(np.median(times))
        e = np.concatenate([mr.energies for mr in r.mol_results]).astype(np.float64)
        d = np.abs(e - ref.energies)
        out["runs"].append({"api": api, "max_iters": iters, "threads": threads or "auto", "seconds": dt, "ms_per_conformer": dt * 1e3 / C,
                            "within_0.1_kcal": int(np.sum(d <= 0.1)), "mean_abs_dE": float(d.mean()),
                            "n_iters": int(r.mol_results[0].n_iters),
                            "converged": (int(sum(int(mr.converged.sum()) for mr in r.mol_results))
                                          if api == "multi" else None)})
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
