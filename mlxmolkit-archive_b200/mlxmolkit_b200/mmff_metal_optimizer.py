"""Multi-molecule MMFF optimisation entry points of the reference, on B200.

``mmff_optimize_metal_multi_mol`` and ``mmff_optimize_metal_fused_multi_mol``
keep the reference signatures (mlxmolkit/mmff_metal_optimizer.py:217-225,
543-548) and result types (:34-44, :210-214), plus an additive
``mmff_variant`` keyword (default "MMFF94", the reference's only variant).

multi_mol: every conformer is minimised inside one persistent kernel launch
(dense BFGS up to 150 atoms, L-BFGS with ``lbfgs_m`` pairs above) with the
reference's convergence rule -- the largest per-atom norm of the gradient
scaled by ``grad_scale`` at or below ``grad_tol``, tested every ``eval_freq``
iterations (:334-359, :405-416).  Preserved behaviour:

* ``converged[i] == (grad_norms[i] <= grad_tol)``, ``grad_norms`` being that
  per-atom norm at the returned coordinates;
* ``per_conf_iters`` is the iteration at which a conformer met ``grad_tol``
  (``max_iters`` if it never did), so ``grad_tol=0`` gives ``max_iters``;
* each conformer stops on its own, so raising ``max_iters`` past
  convergence does not change the answer;
* coordinates are written back into each molecule's conformers (:514-519).

The energies use the constants of the reference's mega kernel
(mmff_metal_kernel.py:274-280), like the reference entry point.

fused: Barzilai-Borwein steepest descent with the +1 kcal/mol energy guard
and the per-atom step cap (mmff_metal_kernel.py:792-1076), ``grad_norms``
zero and ``n_iters = max_iters`` as in the reference (:642-650).
"""
from __future__ import annotations

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


def _atom_grad_norms(m: mm.Minimizer, positions: np.ndarray, grad_scale: float, mode) -> np.ndarray:
    _, g = m.energy_grad(positions, precision="mixed", mode=mode)
    out = np.empty(m.confs.n_conf)
    for c in range(m.confs.n_conf):
        n = int(m.params_list[m.conf_mol[c]].n_atoms)
        gc = g[m.conf_coord[c]: m.conf_coord[c] + 3 * n].reshape(n, 3) * grad_scale
        out[c] = np.sqrt((gc.astype(np.float64) ** 2).sum(1)).max() if n else 0.0
    return out


def mmff_optimize_metal_multi_mol(
    mol_specs,
    max_iters: int = 200,
    eval_freq: int = 10,
    max_step_per_atom: float = 0.3,
    lbfgs_m: int = 10,
    grad_scale: float = 0.1,
    grad_tol: float = 1e-4,
    mmff_variant: str = "MMFF94",
) -> MultiMolResult:
    """Optimise many molecules' conformers in one persistent GPU launch.

    ``max_step_per_atom`` is accepted for signature compatibility; the line
    search of the in-kernel optimizer controls the step length instead.
    """
    mols, conf_ids, params, counts, pos = _collect(mol_specs, mmff_variant)
    m = mm.Minimizer(params, counts)
    big = max(p.n_atoms for p in params) >= mm.LBFGS_ATOM_THRESHOLD
    hist = max(1, min(int(lbfgs_m), 16)) if big else 0
    r = m.minimize(pos, max_iters=max_iters, grad_tol=grad_tol, history_m=hist, mode=mm.MODE_MEGA,
                   exit_test=_lib.EXIT_ATOM_NORM, check_every=max(1, int(eval_freq)),
                   atom_grad_scale=grad_scale)
    gn = _atom_grad_norms(m, r.positions, grad_scale, mm.MODE_MEGA)
    conv = gn <= grad_tol
    per_iters = np.where(conv, np.minimum(r.iters, max_iters), max_iters).astype(np.int32)
    results, cursor = [], 0
    for mi, (mol, cids) in enumerate(zip(mols, conf_ids)):
        k = len(cids)
        n = int(params[mi].n_atoms)
        sl = slice(cursor, cursor + k)
        start = int(m.conf_coord[cursor])
        xyz = r.positions[start: start + 3 * n * k].reshape(k, n, 3)
        _write_back(mol, cids, xyz)
        results.append(MetalBatchResult(
            energies=r.energies[sl].astype(np.float32), positions=xyz.copy(),
            grad_norms=gn[sl].astype(np.float32),
            n_iters=int(per_iters.max()) if conv.all() else int(max_iters), n_conformers=k,
            per_conf_iters=per_iters[sl].copy(), converged=conv[sl].copy()))
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
