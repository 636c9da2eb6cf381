"""Precision study on the drug-like workload (2000 molecules x 10 conformers, heavy atoms 8-70).

Runs the same inputs three ways on the GPU:

* ``fp64``  -- every term, gradient, vector and the inverse Hessian in FP64 (the GPU oracle);
* ``mixed`` -- the chosen form: FP32 terms, gradients and BFGS update; FP64 energy sums,
  Armijo comparisons and convergence tests; FP64 line-search energies once the FP32
  ones stall;
* ``fp32``  -- everything FP32.

For every conformer it reports |dE| against the FP64 result and the RMS gradient at
exit (FP64 gradient of the returned coordinates), and prints one JSON summary.

Usage: python -m mlxmolkit_b200.precision_study [--scale 0.1] [--max-iters 1000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import mmff_minimize as mm
from . import synth
from .mmff_params import extract_mmff_params


def run(scale: float = 0.1, max_iters: int = 1000, seed: int = 0) -> dict:
    import torch
    wl = synth.make_workload("druglike", seed=seed, scale=scale)
    params = [extract_mmff_params(m, mmff_variant=v) for m, v in zip(wl.mols, wl.variants)]
    counts = [m.GetNumConformers() for m in wl.mols]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1)
                          for m in wl.mols]).astype(np.float32)
    m = mm.BinnedMinimizer(params, counts, tuning=mm.load_tuning())
    start = torch.from_numpy(pos).cuda()
    out = {}
    for name, kw in (("fp64", dict(precision="fp64", consts=mm.RDKIT_CONSTS)),
                     ("mixed", dict(precision="mixed")),
                     ("mixed_no_fp64_polish", dict(precision="mixed", polish64=False)),
                     ("fp32", dict(precision="fp32"))):
        x = start.clone()
        torch.cuda.synchronize()
        t = time.perf_counter()
        e, st, it = m.minimize_device(x, max_iters=max_iters, **kw)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        _, g = m.energy_grad(x.cpu().numpy(), precision="fp64")
        rms = np.empty(m.confs.n_conf)
        for c in range(m.confs.n_conf):
            n3 = 3 * params[m.conf_mol[c]].n_atoms
            gc = g[m.conf_coord[c]: m.conf_coord[c] + n3].astype(np.float64)
            rms[c] = np.sqrt(np.mean(gc * gc))
        out[name] = dict(e=e.cpu().numpy(), st=st.cpu().numpy(), it=it.cpu().numpy(), rms=rms, s=dt)
    ref = out["fp64"]["e"]
    summary = {"workload": f"druglike-2000x10-heavy8-70 x scale {scale}", "conformers": int(len(ref)),
               "max_iters": max_iters}
    for name, r in out.items():
        d = np.abs(r["e"] - ref)
        summary[name] = {"seconds": r["s"], "within_0.1_kcal": float(np.mean(d <= 0.1)),
                         "within_0.1_one_sided": float(np.mean(r["e"] - ref <= 0.1)),
                         "mean_abs_dE": float(d.mean()), "p99_abs_dE": float(np.quantile(d, 0.99)),
                         "rms_grad_exit_median": float(np.median(r["rms"])),
                         "rms_grad_exit_p99": float(np.quantile(r["rms"], 0.99)),
                         "iters_mean": float(r["it"].mean()),
                         "status_counts": np.bincount(r["st"], minlength=6).tolist()}
    return summary


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.1)
    ap.add_argument("--max-iters", type=int, default=1000)
    a = ap.parse_args()
    print(json.dumps(run(a.scale, a.max_iters)), flush=True)


if __name__ == "__main__":
    main()
