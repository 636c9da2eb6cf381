"""Autotuner of the size-binned launch.

For every size class (bin of atom counts) it times the optimizer kernel on a
sample of that class's conformers and picks the fastest launch form:

* inverse Hessian in shared memory (up to 74 atoms): each CTA size (64, 128,
  256 threads per conformer) at each persistent occupancy (CTAs per SM);
* inverse Hessian in a global slot: the register-cached streamed form at 1
  CTA/SM, or the register-lean form at 1-2 CTAs/SM (256 threads) or 1 CTA/SM
  (512 threads).

It writes the table that ``BinnedMinimizer`` reads (``tuning.json`` next to
this file, or the path given):

    {"bins": {"24": {"threads": 64, "ctas_per_sm": 6, "lean": true}, ...},
     "device": "...", "timings": {...}}

Usage: python -m mlxmolkit_b200.autotune [--scale 0.1] [--out path]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import mmff_minimize as mm


def _bin_of(n: int, bins) -> int:
    for hi in bins:
        if n <= hi:
            return hi
    return bins[-1]


def tune(params, counts, pos, bins=mm.DEFAULT_BINS, max_iters: int = 1000, per_bin: int = 3000,
         reps: int = 2, verbose: bool = True) -> dict:
    import torch
    n_atoms = np.array([p.n_atoms for p in params])
    mol_bin = np.array([_bin_of(int(n), bins) for n in n_atoms])
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    table, timings = {}, {}
    starts = np.concatenate([[0], np.cumsum(3 * n_atoms * np.asarray(counts))])
    for hi in bins:
        mols = np.nonzero(mol_bin == hi)[0]
        if len(mols) == 0:
            continue
        # sample whole molecules until the bin sample holds per_bin conformers
        take, tot = [], 0
        for mi in mols:
            take.append(mi)
            tot += counts[mi]
            if tot >= per_bin:
                break
        sp = [params[i] for i in take]
        sc = [counts[i] for i in take]
        sx = np.concatenate([pos[starts[i]: starts[i + 1]] for i in take])
        m = mm.Minimizer(sp, sc)
        nmax = int(max(p.n_atoms for p in sp))
        if nmax <= 74:
            # inverse Hessian in shared memory: CTA size x persistent occupancy
            cands = [(t, cps, True) for t in (64, 128, 256) if not (t == 64 and nmax > 42)
                     for cps in (1, 2, 3, 4, 6, 8, 12, 16) if t * cps <= 2048]
        else:
            # global slot, streamed rows: register-cached columns at 1 CTA/SM, or the
            # register-lean form at 1-2 CTAs/SM (256 threads) or 1 CTA/SM (512 threads)
            cands = [(256, 1, False), (256, 1, True), (256, 2, True), (512, 1, True)]
        x0 = torch.from_numpy(sx.astype(np.float32)).cuda()
        best = None
        for t, cps, lean in cands:
            work = x0.clone()
            kw = dict(max_iters=max_iters, threads=t, ctas_per_sm=cps, hpass_lean=lean)
            try:
                m.minimize_device(work, **kw)   # warm
                torch.cuda.synchronize()
            except Exception:
                continue
            ts = []
            for _ in range(reps):
                work.copy_(x0)
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record()
                m.minimize_device(work, **kw)
                e.record()
                torch.cuda.synchronize()
                ts.append(s.elapsed_time(e))
            ms = float(np.min(ts))
            timings[f"{hi}/{t}/{cps}/{'lean' if lean else 'cols'}"] = ms
            if verbose:
                print(f"bin <= {hi:4d} atoms ({sum(sc)} confs): threads {t:3d} ctas/SM {cps:2d} "
                      f"lean {int(lean)}: {ms:8.2f} ms", flush=True)
            if best is None or ms < best[0] * 0.995:
                best = (ms, t, cps, lean)
        if best:
            table[str(hi)] = {"threads": best[1], "ctas_per_sm": best[2], "lean": best[3], "ms_sample": best[0],
                              "sample_conformers": int(sum(sc))}
    return {"bins": table, "device": torch.cuda.get_device_name(), "sms": sms, "timings": timings,
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.1)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "tuning.json"))
    ap.add_argument("--per-bin", type=int, default=3000)
    a = ap.parse_args()
    from . import synth
    from .mmff_params import extract_mmff_params
    wl = synth.make_workload("druglike", seed=11, scale=a.scale)
    params = [extract_mmff_params(m, mmff_variant=v) for m, v in zip(wl.mols, wl.variants)]
    counts = [m.GetNumConformers() for m in wl.mols]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m in wl.mols])
    res = tune(params, counts, pos, max_iters=wl.max_iters, per_bin=a.per_bin)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print("wrote", a.out, json.dumps(res["bins"]))


if __name__ == "__main__":
    main()
