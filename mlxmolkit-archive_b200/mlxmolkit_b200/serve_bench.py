"""Serving benchmark: Poisson arrivals, mixed sizes, p50/p99 latency.

Each request is one seeded molecule (heavy atoms 10-80, MMFF94 / MMFF94s at
random) with k ~ U{1..50} conformers.  Requests arrive as a Poisson stream at a
given rate of conformers per second; ``MMFFServer`` admits them by device
memory budget, runs them concurrently on CUDA streams and completes each one
when its kernel ends.  For every swept rate the run reports the achieved
throughput (converged conformers / s), p50 / p99 request latency, and whether
the server kept up (queue drained within the run).  Molecules are drawn from
a pre-generated pool so request generation does not throttle the arrivals.

Converged conformers are counted two ways: by exit status, and by the rule of
``convergence.py`` (within 0.1 kcal/mol of an FP64 minimum).  A request's
result depends only on its molecule and starting coordinates, never on the
mix it was served in, so every request of one pool molecule returns the same
energies; the run checks that, and evaluates the rule once per pool molecule
(FP64 minima from the pool's starts and from the returned coordinates),
weighted by how often the molecule was served.

Usage: python -m mlxmolkit_b200.serve_bench --rates 500,2000,8000 --duration 20
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import synth
from .convergence import RULE
from .serve import MMFFServer, poisson_stream


def make_pool(n_mols: int, seed: int = 4):
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, 51, size=n_mols)
    mols = synth.make_molecules(n_mols, [int(k) for k in ks], seed, 10, 80, max_atoms=170)
    variants = ["MMFF94" if rng.random() < 0.5 else "MMFF94s" for _ in range(n_mols)]
    return mols, variants


def rule_converged(pool, first: dict) -> tuple:
    """Per pool molecule served: the rule's converged mask of its conformers (the result of its
    first request, ``first[j]``).  Dense BFGS below 150 atoms, L-BFGS m=8 from 150 on, as served."""
    import torch
    from . import mmff_minimize as mm
    from .convergence import converged, fp64_minima
    from .mmff_params import extract_mmff_params
    mols, variants = pool
    masks, parts = {}, {}
    for hist in (0, mm.LBFGS_M):
        idx = [j for j in sorted(first) if (mols[j].GetNumAtoms() >= mm.LBFGS_ATOM_THRESHOLD) == bool(hist)]
        if not idx:
            continue
        params = [extract_mmff_params(mols[j], mmff_variant=variants[j]) for j in idx]
        counts = [len(first[j].energies) for j in idx]
        m = mm.BinnedMinimizer(params, counts)
        start = np.concatenate([np.stack([c.pos for c in mols[j].GetConformers()]).reshape(-1) for j in idx])
        ret = np.concatenate([first[j].positions.reshape(-1) for j in idx])
        e = np.concatenate([first[j].energies for j in idx])
        e_same = fp64_minima(m, torch.from_numpy(start.astype(np.float32)).cuda(), hist)
        e_basin = fp64_minima(m, torch.from_numpy(ret.astype(np.float32)).cuda(), hist)
        mask, pp = converged(e, e_same, e_basin)
        parts["lbfgs" if hist else "dense"] = pp
        off = np.concatenate([[0], np.cumsum(counts)])
        for t, j in enumerate(idx):
            masks[j] = mask[off[t]:off[t + 1]]
    return masks, parts


def run_rate(pool, rate: float, duration: float, budget: int, seed: int = 0) -> dict:
    mols, variants = pool
    srv = MMFFServer(hbm_budget_bytes=budget)

    def make_request(i):
        j = i % len(mols)
        m = mols[j]
        xyz = np.stack([c.pos for c in m.GetConformers()])
        return m, xyz, variants[j]

    t0 = time.perf_counter()
    futures = poisson_stream(srv, make_request, rate, duration, seed=seed)
    results = [f.result() for f in futures]
    t1 = time.perf_counter()
    srv.close()
    lat = np.array([r.latency for r in results])
    atoms = np.array([r.positions.shape[1] for r in results])
    per_class = {}
    for name, sel in (("dense_bfgs_lt150_atoms", atoms < 150), ("lbfgs_150_atoms_up", atoms >= 150)):
        if sel.any():
            per_class[name] = {"requests": int(sel.sum()), "p50_ms": float(np.percentile(lat[sel], 50) * 1e3),
                               "p99_ms": float(np.percentile(lat[sel], 99) * 1e3)}
    confs = sum(len(r.energies) for r in results)
    conv = sum(int(r.converged.sum()) for r in results)
    wall = t1 - t0
    first, same = {}, 0
    for i, r in enumerate(results):
        j = i % len(mols)
        if j not in first:
            first[j] = r
        else:
            same += int(np.array_equal(r.energies, first[j].energies) and np.array_equal(r.positions, first[j].positions))
    repeats = len(results) - len(first)
    masks, parts = rule_converged(pool, first)
    conv_rule = sum(int(masks[i % len(mols)].sum()) for i in range(len(results)))
    return {"rate_confs_per_s": rate, "requests": len(results), "conformers": confs,
            "converged": conv, "wall_s": wall, "converged_per_s": conv / wall,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "kept_up": bool(wall <= duration * 1.2 + 5.0), "peak_mem_bytes": int(srv.peak_in_use),
            "launches": int(srv.launches), "mean_latency_ms": float(lat.mean() * 1e3), "per_class": per_class,
            "converged_frac": conv / max(confs, 1),
            "converged_by": "exit status (gradient, TOLX, slope or line-search exit)",
            "converged_rule": {"rule": RULE, "converged": conv_rule, "per_s": conv_rule / wall,
                               "frac": conv_rule / max(confs, 1), "parts_per_pool_molecule": parts,
                               "pool_molecules_served": len(first),
                               "repeat_requests_identical": f"{same} of {repeats}"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="500,2000,8000")
    ap.add_argument("--duration", type=float, default=20.0)
    ap.add_argument("--pool", type=int, default=300)
    ap.add_argument("--budget-gb", type=float, default=16.0)
    a = ap.parse_args()
    pool = make_pool(a.pool)
    rows = [run_rate(pool, float(r), a.duration, int(a.budget_gb * (1 << 30))) for r in a.rates.split(",")]
    print(json.dumps({"serving": rows}), flush=True)


if __name__ == "__main__":
    main()
