"""Benchmark of the distance-geometry (DG) stage: ``dg_minimize_shared`` on the GPU.

The stage as ``generate_conformers_nk`` runs it (mlxmolkit/conformer_pipeline_v2.py:172-221):
metric-matrix starts, the 4-D minimisation with the automatic iteration budget
max(300, 300 + 20 * max_atoms) (fourth-dimension weight 0.1, chiral weight 1.0),
then the 4-D -> 3-D collapse of 200 iterations (weights 1.0 / 0.2).  The ETK leg
continues from there as the pipeline's stage 3 (:260-290): the first three
coordinates, then ``etk_minimize_shared``'s kernel with the budget
max(150, 150 + 10 * max_atoms) (the reference's "DG + ETK" rows).  Inputs are
seeded synthetic molecules (heavy atoms 10-30; bounds and chirality from
``dg_extract.synth_dg_params``); the reference quotes its DG-only throughput on
20 molecules x 50 conformers (docs/BENCHMARKS.md:44-50), and 1000 x 10 is its
scale row.

Per workload it reports:
  * ``conf_per_s``: both minimisations with the positions resident in HBM, timed
    with CUDA events on the launching stream (median of ``--repeats`` after one
    warm-up run);
  * ``e2e_conf_per_s``: the same through ``dg_minimize_shared`` with host arrays
    (tables packed and uploaded, positions copied both ways, every call);
  * ``converged``: the fraction of conformers with status 0 after the 4-D stage;
  * ``dg_etk_conf_per_s``: DG, collapse, 3-D extraction and ETK, all on the device.

The FP64 CPU baseline of the same stages is ``bench.py --workload dg``; agreement
with the FP64 restatement is what tests/test_gpu_dg.py and tests/test_gpu_etk.py check.

Usage: python -m mlxmolkit_b200.dg_bench [--workloads 20x50,1000x10] [--tpm auto|32,64,...]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import synth
from .conformer_metal import DGDeviceBatch, dg_minimize_shared
from .dg_extract import metric_matrix_positions, synth_dg_params
from .etk_extract import synth_etk_params
from .etk_metal import ETKDeviceBatch
from .shared_batch import add_etk_to_batch, pack_shared_dg_batch


def _auto_iters(max_atoms: int, base: int, scale: float) -> int:
    return max(base, int(base + scale * max_atoms))      # conformer_pipeline_v2.py:123-126


def _workload(n_mols: int, k: int, seed: int):
    mols = synth.make_molecules(n_mols, 1, seed, 10, 30)
    params = [synth_dg_params(m) for m in mols]
    b4 = pack_shared_dg_batch(params, [k] * n_mols, dim=4)
    x0 = metric_matrix_positions(b4, [p.bounds_mat for p in params], seed=42, dim=4)
    max_atoms = max(p.n_atoms for p in params)
    complexity = max(max_atoms, int(max(len(p.dist_idx1) for p in params) ** 0.5))
    b3 = pack_shared_dg_batch(params, [k] * n_mols, dim=3)
    add_etk_to_batch(b3, [synth_etk_params(m, p.bounds_mat) for m, p in zip(mols, params)])
    return b4, x0, _auto_iters(complexity, 300, 20.0), max_atoms, b3, _auto_iters(complexity, 150, 10.0)


def _sub_batch(b, confs):
    """The conformers ``confs`` of batch b as a batch of their own (a CPU baseline's sample)."""
    mols = sorted(set(int(b.conf_to_mol[c]) for c in confs))
    from .dg_extract import DGParams
    ps = []
    for m in mols:
        d0, d1 = b.dist_term_starts[m], b.dist_term_starts[m + 1]
        c0, c1 = b.chiral_term_starts[m], b.chiral_term_starts[m + 1]
        f0, f1 = b.fourth_term_starts[m], b.fourth_term_starts[m + 1]
        ps.append(DGParams(int(b.mol_n_atoms[m]), b.dist_idx1[d0:d1], b.dist_idx2[d0:d1], b.dist_lb2[d0:d1],
                           b.dist_ub2[d0:d1], b.dist_weight[d0:d1], b.chiral_idx1[c0:c1], b.chiral_idx2[c0:c1],
                           b.chiral_idx3[c0:c1], b.chiral_idx4[c0:c1], b.chiral_vol_lower[c0:c1],
                           b.chiral_vol_upper[c0:c1], b.fourth_idx[f0:f1]))
    counts = [sum(1 for c in confs if int(b.conf_to_mol[c]) == m) for m in mols]
    ordered = [c for m in mols for c in confs if int(b.conf_to_mol[c]) == m]
    return pack_shared_dg_batch(ps, counts, dim=b.dim), ordered


def run(n_mols: int, k: int, repeats: int, seed: int = 0, tpm=None, hist_mode: int = 0) -> dict:
    import torch
    b4, x0, iters, max_atoms, b3, etk_iters = _workload(n_mols, k, seed)
    C = b4.n_confs_total
    dev = DGDeviceBatch(b4)
    p1 = dev.params(iters, 1e-4, 1.0, 0.1, tpm=tpm, hist_mode=hist_mode)
    p2 = dev.params(200, 1e-4, 0.2, 1.0, tpm=tpm, hist_mode=hist_mode)
    start = torch.from_numpy(x0).cuda()
    pos = torch.empty_like(start)
    it = torch.empty(C, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()

    def stage(record=None):
        pos.copy_(start)
        e1, s1 = dev.minimize_device(pos, p1, iters=it)
        s1 = s1.clone()
        dev.minimize_device(pos, p2)
        return e1, s1

    stage()
    times = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(st)
        e1, s1 = stage()
        ev1.record(st)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1) / 1e3)
    # positions are reset inside the timed region by a device copy of C * n * 4 floats (< 1 % of it)
    t_dev = float(np.median(times))
    s1n = s1.cpu().numpy()
    itn = it.cpu().numpy()

    e2e = []
    for _ in range(max(1, repeats // 2)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        xa, _, _ = dg_minimize_shared(b4, x0, max_iters=iters, chiral_weight=1.0, fourth_dim_weight=0.1, tpm=tpm)
        dg_minimize_shared(b4, xa, max_iters=200, chiral_weight=0.2, fourth_dim_weight=1.0, tpm=tpm)
        e2e.append(time.perf_counter() - t)
    t_e2e = float(np.median(e2e))

    # DG + ETK on the device: the 3-D start is the collapsed 4-D result's first three coordinates
    edev = ETKDeviceBatch(b3)
    p3 = edev.params(etk_iters, 1e-4, 0.0, 0.0, tpm=tpm, hist_mode=hist_mode)
    it3 = torch.empty(C, dtype=torch.int32, device="cuda")

    def dg_etk():
        stage()
        pos3 = pos.view(-1, 4)[:, :3].contiguous().view(-1)
        e3, s3 = edev.minimize_device(pos3, p3, iters=it3)
        return e3, s3

    dg_etk()
    times = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(st)
        e3, s3 = dg_etk()
        ev1.record(st)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1) / 1e3)
    t_dg_etk = float(np.median(times))
    s3n, it3n = s3.cpu().numpy(), it3.cpu().numpy()

    out = {"workload": f"{n_mols}x{k} synthetic, heavy atoms 10-30", "conformers": C, "max_atoms": max_atoms,
           "threads_per_conformer": tpm or "auto", "history": ("auto", "shared", "device")[hist_mode],
           "dg_max_iters": iters, "seconds": t_dev, "conf_per_s": C / t_dev, "ms_per_conf": t_dev * 1e3 / C,
           "e2e_seconds": t_e2e, "e2e_conf_per_s": C / t_e2e, "converged": float(np.mean(s1n == 0)),
           "mean_iters": float(itn.mean()), "max_iters_hit": int(np.sum(itn >= iters)),
           "etk_max_iters": etk_iters, "dg_etk_seconds": t_dg_etk, "dg_etk_conf_per_s": C / t_dg_etk,
           "etk_converged": float(np.mean(s3n == 0)), "etk_mean_iters": float(it3n.mean())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="20x50,1000x10")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--tpm", default="auto", help="threads per conformer: auto or a comma list of 32/64/128/256")
    ap.add_argument("--history", default="0", help="L-BFGS history: comma list of 0 (auto) / 1 (shared) / 2 (device)")
    a = ap.parse_args()
    tpms = [None] if a.tpm == "auto" else [int(v) for v in a.tpm.split(",")]
    for w in a.workloads.split(","):
        n, k = (int(v) for v in w.split("x"))
        for tpm in tpms:
            for hm in (int(v) for v in a.history.split(",")):
                print(json.dumps(run(n, k, a.repeats, tpm=tpm, hist_mode=hm)), flush=True)


if __name__ == "__main__":
    main()
