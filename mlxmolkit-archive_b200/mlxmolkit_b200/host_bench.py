"""Host-side steps of ``generate_conformers_nk`` for N synthetic molecules x k conformers, timed
on the CPU alone (no GPU needed).

Each step is what the pipeline does on the host around its GPU stages
(conformer_pipeline_v2.py): DG terms with the metric-matrix starts (process
pool), ETK term extraction and MMFF typing + packing (pool), the 3-D batch with its ETK terms,
the DG and ETK device tables (host threads; also timed on one thread), the
re-centring of the 1-2 / 1-3 bounds, and the merge of the per-molecule MMFF
packs.  Seconds are the median of ``--repeats`` after one warm-up pass (which
also starts the pool).

Usage: python -m mlxmolkit_b200.host_bench [--workloads 1000x10] [--repeats 3]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import conformer_pipeline_v2 as cp
from . import synth
from .pack import merge_packed
from .shared_batch import add_etk_to_batch, dg_device_arrays, etk_device_arrays, pack_shared_dg_batch


def _steps(mols, ks):
    """One pass over the host steps; returns {step: seconds}."""
    t = {}

    def timed(name, fn):
        t0 = time.perf_counter()
        out = fn()
        t[name] = time.perf_counter() - t0
        return out

    dgp, b4, x4 = timed("dg_terms_and_starts", lambda: cp._dg_terms_and_positions(mols, ks, 42, dim=4))
    etk = timed("etk_terms", lambda: cp._pmap(cp._etk_terms, [(m, p.bounds_mat) for m, p in zip(mols, dgp)]))
    mmff = timed("mmff_packs", lambda: cp._pmap(cp._mmff_pack, [(m, "MMFF94") for m in mols]))
    timed("dg_tables", lambda: dg_device_arrays(b4))
    timed("dg_tables_1_thread", lambda: dg_device_arrays(b4, workers=1))

    def batch3():
        b = pack_shared_dg_batch(dgp, ks, dim=3)
        add_etk_to_batch(b, etk)
        return b

    b3 = timed("pack_3d_with_etk", batch3)
    timed("etk_tables", lambda: etk_device_arrays(b3))
    timed("etk_tables_1_thread", lambda: etk_device_arrays(b3, workers=1))
    x3 = x4.reshape(-1, 4)[:, :3].reshape(-1).copy()
    timed("recentre_bounds", lambda: cp._recenter_bounds(b3, x3))
    timed("merge_mmff_packs", lambda: merge_packed([k for k in mmff if k is not None]))
    return t


def run(n_mols: int, k: int, repeats: int, seed: int = 0) -> dict:
    mols = synth.make_molecules(n_mols, 1, seed, 10, 30)
    ks = [k] * n_mols
    _steps(mols, ks)                                        # warm-up: pool start, imports
    passes = [_steps(mols, ks) for _ in range(repeats)]
    med = {s: float(np.median([p[s] for p in passes])) for s in passes[0]}
    return {"workload": f"{n_mols}x{k} synthetic, heavy atoms 10-30", "host_threads": os.cpu_count(),
            "seconds": {s: round(v, 4) for s, v in med.items()}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="1000x10")
    ap.add_argument("--repeats", type=int, default=3)
    a = ap.parse_args()
    for w in a.workloads.split(","):
        n, k = (int(v) for v in w.split("x"))
        print(json.dumps(run(n, k, a.repeats)), flush=True)


if __name__ == "__main__":
    main()
