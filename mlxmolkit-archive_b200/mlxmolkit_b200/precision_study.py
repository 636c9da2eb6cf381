"""Precision study on the drug-like workload (2000 molecules x 10 conformers, heavy atoms 8-70).

Runs the same inputs three ways on the GPU:

* ``fp64``  -- every term, gradient, vector and the inverse Hessian in FP64 (the GPU oracle);
* ``mixed`` -- the chosen form: FP32 terms, gradients and BFGS update; FP64 energy sums,
  Armijo comparisons and convergence tests;
* ``mixed_fp64_polish`` -- the same, with FP64 line-search energies once the FP32 ones
  stall (the L-BFGS default);
* ``fp32``  -- everything FP32.

For every conformer it reports |dE| against the FP64 minimum from the same start, whether it
is converged by the rule of ``convergence.py`` (within 0.1 kcal/mol of an FP64 minimum: the
same-start one or its own basin's), and the RMS gradient at exit (``mmffb_fp64_check``: the
FP64 gradient at the returned coordinates); one JSON summary.

Usage: python -m mlxmolkit_b200.precision_study [--scale 0.1] [--max-iters 1000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import mmff_minimize as mm
from . import synth
from .convergence import RULE, converged, fp64_minima
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
    e_same = fp64_minima(m, start)
    out = {}
    for name, kw in (("fp64", dict(precision="fp64", consts=mm.RDKIT_CONSTS)),
                     ("mixed", dict(precision="mixed")),
                     ("mixed_fp64_polish", dict(precision="mixed", polish64=True)),
                     ("fp32", dict(precision="fp32"))):
        x = start.clone()
        torch.cuda.synchronize()
        t = time.perf_counter()
        e, st, it = m.minimize_device(x, max_iters=max_iters, **kw)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        _, _, rms = m.fp64_check_device(x, e)
        e = e.cpu().numpy()
        mask, parts = converged(e, e_same, fp64_minima(m, x))
        out[name] = dict(e=e, st=st.cpu().numpy(), it=it.cpu().numpy(), rms=rms.cpu().numpy(), s=dt,
                         conv=float(mask.mean()), parts=parts)
    summary = {"workload": f"druglike-2000x10-heavy8-70 x scale {scale}", "conformers": int(len(e_same)),
               "max_iters": max_iters, "converged_rule": RULE}
    for name, r in out.items():
        d = np.abs(r["e"] - e_same)
        summary[name] = {"seconds": r["s"], "converged": r["conv"], "converged_parts": r["parts"],
                         "mean_abs_dE_same_start": float(d.mean()), "p99_abs_dE_same_start": float(np.quantile(d, 0.99)),
                         "rms_grad_exit_median": float(np.median(r["rms"])),
                         "rms_grad_exit_p99": float(np.quantile(r["rms"], 0.99)),
                         "iters_mean": float(r["it"].mean()),
                         "status_counts": np.bincount(r["st"], minlength=7).tolist()}
    return summary


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.1)
    ap.add_argument("--max-iters", type=int, default=1000)
    a = ap.parse_args()
    print(json.dumps(run(a.scale, a.max_iters)), flush=True)


if __name__ == "__main__":
    main()
