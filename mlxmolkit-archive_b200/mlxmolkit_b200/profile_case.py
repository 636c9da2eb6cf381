"""Small profiling case of the optimizer kernels, sized for an ncu capture.

One size-binned minimisation of ``--mols`` seeded drug-like molecules x ``--k``
conformers (heavy atoms ``--lo``-``--hi``, default 8-70, at most 150 atoms),
mixed precision, dense BFGS, at most 1000 iterations.  At the defaults
(60 x 10) the global-slot size class holds about 300 conformers of 75-150
atoms, whose inverse-Hessian slots (one per CTA, 296 CTAs) take more than the
126 MB L2, so DRAM counters keep their meaning, while the device holds well
under 1 GB.  Small heavy-atom ranges fill the GPU with one shared-memory size
class instead: ``--lo 4 --hi 8`` (up to 24 atoms), ``--lo 10 --hi 16``
(25-48 atoms), each with enough conformers for every SM.

``--lbfgs`` runs the large workload's optimizer instead: L-BFGS m = 8, at most
3000 iterations, molecules built like the large workload's (30 % macrocycles,
at most 20 rotatable bonds).  ``--lbfgs --mols 40 --k 8 --lo 60 --hi 75
--max-atoms 170`` is one launch of the 150-170-atom class (320 conformers),
whose instance keeps the L-BFGS history in shared memory at 2 CTAs per SM.
``--lbfgs --keep-target --mols 40 --k 8 --lo 95 --hi 125 --max-atoms 288`` is one
launch of the 171-288-atom class (186-284 atoms), whose instance keeps the history
in a global slot at 2 CTAs per SM.

Usage: python -m mlxmolkit_b200.profile_case [--mols 60] [--k 10] [--lo 8] [--hi 70] [--repeat 1]
                                             [--lbfgs] [--max-atoms 150]
"""
from __future__ import annotations

import argparse

import numpy as np

from . import mmff_minimize as mm
from . import synth
from .mmff_params import extract_mmff_params
from .roofline import algorithmic_bytes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mols", type=int, default=60)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--lo", type=int, default=8, help="fewest heavy atoms")
    ap.add_argument("--hi", type=int, default=70, help="most heavy atoms")
    ap.add_argument("--lbfgs", action="store_true", help="L-BFGS m = 8 on large-workload-like molecules")
    ap.add_argument("--max-atoms", type=int, default=150)
    ap.add_argument("--keep-target", action="store_true",
                    help="with --lbfgs: the large workload's generator (heavy-atom count kept across redraws)")
    a = ap.parse_args()
    import torch
    if a.lbfgs:
        mols = synth.make_molecules(a.mols, a.k, a.seed, a.lo, a.hi, macro_frac=0.3, max_rotatable=20,
                                    max_atoms=a.max_atoms, ring_density=0.12, keep_target=a.keep_target)
    else:
        mols = synth.make_molecules(a.mols, a.k, a.seed, a.lo, a.hi, max_atoms=a.max_atoms)
    hist, max_iters = (mm.LBFGS_M, 3000) if a.lbfgs else (0, 1000)
    params = [extract_mmff_params(m) for m in mols]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1)
                          for m in mols]).astype(np.float32)
    m = mm.BinnedMinimizer(params, [a.k] * len(mols))
    x0 = torch.from_numpy(pos).cuda()
    evals = torch.zeros(m.confs.n_conf, dtype=torch.int32, device=x0.device)
    for _ in range(a.repeat):
        x = x0.clone()
        e, st, it = m.minimize_device(x, max_iters=max_iters, history_m=hist, time_bins=True, evals=evals)
        torch.cuda.synchronize()
        e, it, ev = e.cpu().numpy(), it.cpu().numpy(), evals.cpu().numpy()
        if not np.isfinite(e).all():
            raise SystemExit("non-finite energies")
        bins = [{"max_atoms": hi, "conformers": len(sel), "ms": round(ms, 2),
                 "algorithmic_bytes": algorithmic_bytes(params, m.conf_mol[sel], it[sel], ev[sel], hist)}
                for hi, sel, ms in m.bin_times_ms()]
        print(f"ok: {len(e)} conformers, mean iterations {it.mean():.1f}, size classes {bins}", flush=True)


if __name__ == "__main__":
    main()
