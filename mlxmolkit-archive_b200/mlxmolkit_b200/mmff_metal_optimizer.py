"""Multi-molecule MMFF optimisation entry points of the reference, on B200.

``mmff_optimize_metal_multi_mol`` and ``mmff_optimize_metal_fused_multi_mol``
keep the reference signatures (mlxmolkit/mmff_metal_optimizer.py:217-225,
543-548) and result types (:34-44, :210-214), plus an additive
``mmff_variant`` keyword (default "MMFF94", the reference's only variant).

multi_mol runs the reference's own algorithm (:217-535) on the GPU:
L-BFGS with ``lbfgs_m`` pairs on the ``grad_scale``-scaled gradient, no line
search, each atom's step capped at ``max_step_per_atom``.  Every ``eval_freq``
iterations it keeps the best-seen positions and marks the conformers whose
largest per-atom scaled-gradient norm is at or below ``grad_tol``; the batch
stops when all are.  It then returns every conformer to its best-seen
positions and runs a polish pass of ``max_iters // 4`` iterations from a fresh
history, stopping when every conformer is under ``grad_tol`` at a check point.
The result holds the best-seen positions and their energies, the gradient
norms of the last iterate, the iteration of each conformer's first passing
check and the sticky converged flags of the main loop, as the reference's.
The iterations run inside ``mmffb_multimol_step`` launches (one per
``eval_freq`` iterations, state resident on the device); the host reads one
counter per check point, where the reference synchronises too.

The energies use the constants of the reference's mega kernel
(mmff_metal_kernel.py:274-280), like the reference entry point.

fused: Barzilai-Borwein steepest descent with the +1 kcal/mol energy guard
and the per-atom step cap (mmff_metal_kernel.py:792-1076), ``grad_norms``
zero and ``n_iters = max_iters`` as in the reference (:642-650).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from . import mmff_minimize as mm
from .mmff_params import extract_mmff_params


@dataclass
class MetalBatchResult:
    """Result of one molecule's conformers (mlxmolkit/mmff_metal_optimizer.py:34-44)."""

    energies: np.ndarray
    positions: np.ndarray
    grad_norms: np.ndarray
    n_iters: int
    n_conformers: int
    per_conf_iters: Optional[np.ndarray] = None
    converged: Optional[np.ndarray] = None


@dataclass
class MultiMolResult:
    """Result of multi-molecule optimisation (mlxmolkit/mmff_metal_optimizer.py:210-214)."""

    mol_results: list


def _collect(mol_specs, mmff_variant: str):
    mols, conf_ids, params, counts, pos = [], [], [], [], []
    for mol, cids in mol_specs:
        if cids is None:
            cids = [c.GetId() for c in mol.GetConformers()]
        cids = list(cids)
        if not cids:
            raise ValueError("molecule without conformers")
        mols.append(mol)
        conf_ids.append(cids)
        params.append(extract_mmff_params(mol, conf_id=cids[0], mmff_variant=mmff_variant))
        counts.append(len(cids))
        for cid in cids:
            conf = mol.GetConformer(cid)
            xyz = np.asarray(conf.pos if hasattr(conf, "pos") else conf.GetPositions(), dtype=np.float64)
            pos.append(xyz.reshape(-1))
    return mols, conf_ids, params, counts, np.concatenate(pos).astype(np.float32)


def _write_back(mol, cids, xyz):
    for k, cid in enumerate(cids):
        conf = mol.GetConformer(cid)
        if hasattr(conf, "pos"):
            conf.pos[:] = xyz[k].astype(np.float64)
        else:
            for a in range(xyz.shape[1]):
                conf.SetAtomPosition(a, xyz[k, a].astype(float).tolist())


class _MultiMolRun:
    """Device state of one multi-molecule L-BFGS run (the reference's loop variables)."""

    def __init__(self, m: mm.Minimizer, pos: np.ndarray, lbfgs_m: int, grad_scale: float,
                 max_step_per_atom: float, grad_tol: float, mode=mm.MODE_MEGA, threads: int = 0):
        import torch
        self.torch, self.m, self.L = torch, m, _lib.load()
        dev = m.batch.device
        C = m.confs.n_conf
        self.hist_m = int(lbfgs_m)
        if not 1 <= self.hist_m <= 16:
            raise ValueError("lbfgs_m must be in 1..16")
        self.x = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float32)).to(dev)
        self.g = torch.zeros_like(self.x)
        self.best_x = torch.zeros_like(self.x)
        self.e = torch.zeros(C, dtype=torch.float64, device=dev)
        self.best_e = torch.zeros_like(self.e)
        self.bd, self.cd = m.batch.desc(), m.confs.desc()
        hf = self.L.mmffb_multimol_hist_floats(ctypes.byref(self.cd), self.hist_m)
        self.hist = torch.zeros(max(C * hf, 1), dtype=torch.float32, device=dev)
        self.rho = torch.zeros(max(C * self.hist_m, 1), dtype=torch.float32, device=dev)
        ints = lambda k: torch.zeros(max(k, 1), dtype=torch.int32, device=dev)
        self.hcount, self.converged, self.conv_iter, self.pending = ints(C), ints(C), ints(C), ints(1)
        self.state = _lib.MMFFMultiMolState(*(t.data_ptr() for t in (
            self.x, self.g, self.best_x, self.e, self.best_e, self.hist, self.rho, self.hcount,
            self.converged, self.conv_iter, self.pending)))
        self.prm = _lib.MMFFMultiMolParams(self.hist_m, float(grad_scale), float(max_step_per_atom),
                                           float(grad_tol), (ctypes.c_double * 4)(*mode), int(threads))

    def step(self, phase: int, n_iters: int = 0, it_end: int = 0, max_iters: int = 0) -> None:
        rc = self.L.mmffb_multimol_step(ctypes.byref(self.bd), ctypes.byref(self.cd), ctypes.byref(self.prm),
                                        ctypes.byref(self.state), phase, n_iters, it_end, max_iters,
                                        ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "mmffb_multimol_step")

    def _loop(self, total: int, eval_freq: int, check_phase: int, max_iters: int) -> int:
        """Run ``total`` iterations in chunks ending at the check points (every eval_freq
        iterations); returns the iteration count at which every conformer passed, or total."""
        it = 0
        while it < total:
            n = min(eval_freq - it % eval_freq, total - it)
            check = (it + n) % eval_freq == 0
            if check:
                self.pending.zero_()
            self.step(check_phase if check else _lib.MM_RUN, n, it + n, max_iters)
            it += n
            if check and int(self.pending.item()) == 0:
                return it
        return total

    def run(self, max_iters: int, eval_freq: int) -> int:
        self.step(_lib.MM_START, 0, 0, max_iters)
        iters_used = self._loop(max_iters, eval_freq, _lib.MM_MAIN_CHECK, max_iters)   # :346-410
        self.step(_lib.MM_REVERT, 0, 0, max_iters)                                     # :412-428
        self._loop(max_iters // 4, eval_freq, _lib.MM_POLISH_CHECK, max_iters)         # :430-483
        self.torch.cuda.synchronize()
        return iters_used


def mmff_optimize_metal_multi_mol(
    mol_specs,
    max_iters: int = 200,
    eval_freq: int = 10,
    max_step_per_atom: float = 0.3,
    lbfgs_m: int = 10,
    grad_scale: float = 0.1,
    grad_tol: float = 1e-4,
    mmff_variant: str = "MMFF94",
    threads: int = 0,
) -> MultiMolResult:
    """Optimise many molecules' conformers with the reference's multi-molecule L-BFGS.

    ``threads`` (additive) fixes the threads per conformer (64, 128 or 256); 0 chooses them
    from the batch."""
    if eval_freq < 1:
        raise ValueError("eval_freq must be >= 1")
    mols, conf_ids, params, counts, pos = _collect(mol_specs, mmff_variant)
    m = mm.Minimizer(params, counts)
    run = _MultiMolRun(m, pos, lbfgs_m, grad_scale, max_step_per_atom, grad_tol, threads=threads)
    iters_used = run.run(int(max_iters), int(eval_freq))
    best_x = run.best_x.cpu().numpy()
    best_e = run.best_e.cpu().numpy()
    g_last = run.g.cpu().numpy()
    conv = run.converged.cpu().numpy()[: m.confs.n_conf].astype(bool)
    per_iters = run.conv_iter.cpu().numpy()[: m.confs.n_conf].astype(np.int32)
    results, cursor = [], 0
    for mi, (mol, cids) in enumerate(zip(mols, conf_ids)):
        k = len(cids)
        n = int(params[mi].n_atoms)
        sl = slice(cursor, cursor + k)
        start = int(m.conf_coord[cursor])
        xyz = best_x[start: start + 3 * n * k].reshape(k, n, 3)
        gl = g_last[start: start + 3 * n * k].reshape(k, n, 3).astype(np.float64)
        gn = np.sqrt((gl * gl).sum(-1)).max(axis=1) if n else np.zeros(k)
        _write_back(mol, cids, xyz)
        results.append(MetalBatchResult(
            energies=best_e[sl].astype(np.float32), positions=xyz.copy(), grad_norms=gn.astype(np.float32),
            n_iters=int(iters_used), n_conformers=k, per_conf_iters=per_iters[sl].copy(),
            converged=conv[sl].copy()))
        cursor += k
    return MultiMolResult(mol_results=results)


def mmff_optimize_metal_fused_multi_mol(
    mol_specs,
    max_iters: int = 500,
    max_step: float = 0.3,
    grad_lr: float = 0.1,
    mmff_variant: str = "MMFF94",
) -> MultiMolResult:
    """Barzilai-Borwein steepest descent for every conformer, one launch."""
    mols, conf_ids, params, counts, pos = _collect(mol_specs, mmff_variant)
    m = mm.Minimizer(params, counts)
    xo, e = m.fused_sd(pos, max_iters=max_iters, max_step=max_step, grad_lr=grad_lr, mode=mm.MODE_MEGA)
    results, cursor = [], 0
    for mi, (mol, cids) in enumerate(zip(mols, conf_ids)):
        k = len(cids)
        n = int(params[mi].n_atoms)
        start = int(m.conf_coord[cursor])
        xyz = xo[start: start + 3 * n * k].reshape(k, n, 3)
        _write_back(mol, cids, xyz)
        en = e[cursor: cursor + k].astype(np.float32)
        results.append(MetalBatchResult(energies=en, positions=xyz.copy(), grad_norms=en * 0,
                                        n_iters=int(max_iters), n_conformers=k))
        cursor += k
    return MultiMolResult(mol_results=results)
