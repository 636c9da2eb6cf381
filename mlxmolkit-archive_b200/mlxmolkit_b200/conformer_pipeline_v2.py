"""``generate_conformers_nk(run_mmff=True)`` with the MMFF stage on B200.

Signature and result types of mlxmolkit/conformer_pipeline_v2.py:41-56,
357-372.  The distance-geometry / ETK embedding stages of the reference
(:172-290) are outside this package: molecules are embedded on the host --
with RDKit's ETKDG for SMILES input, or taken as given for molecules that
already carry conformers (RDKit ``Mol`` or ``SynthMol``) -- and the MMFF stage
runs on the GPU:

* parameters are extracted once per molecule from its first conformer
  (:299-317);
* iterations default to 200 + 15 * (largest atom count) when
  ``mmff_max_iters`` is 0 (:123-126, :169-170);
* ``mmff_use_lbfgs=None`` picks L-BFGS per size class -- molecules of 150 or
  more atoms run L-BFGS (m = 8), smaller ones dense BFGS -- where the
  reference switched the whole call on its largest molecule (:448-452);
  an explicit True / False applies to every molecule;
* a molecule whose MMFF typing fails keeps its embedded coordinates and is
  reported unconverged, as the reference's chunk fallback does (:312-316).
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import mmff_minimize as mm
from .mmff_params import extract_mmff_params


@dataclass
class ConformerResult:
    """Result for one molecule."""
    n_atoms: int
    positions_3d: List[np.ndarray]
    energies: List[float]
    converged: List[bool]


@dataclass
class PipelineResult:
    """Result for the full N x k pipeline."""
    molecules: List[ConformerResult]
    total_conformers: int
    total_time: float
    n_batches: int


def _auto_iters(max_atoms: int, base: int = 200, scale: float = 15.0) -> int:
    return max(base, int(base + scale * max_atoms))


def _embed(item, k: int, seed: int):
    """(molecule, list of (N,3) float64 conformer coordinates)."""
    if isinstance(item, str):
        from rdkit import Chem
        from rdkit.Chem import AllChem
        mol = Chem.MolFromSmiles(item)
        if mol is None:
            raise ValueError(f"Invalid SMILES: {item}")
        mol = Chem.AddHs(mol)
        params = AllChem.ETKDGv3()
        params.randomSeed = seed
        cids = list(AllChem.EmbedMultipleConfs(mol, k, params))
        return mol, [np.asarray(mol.GetConformer(c).GetPositions(), dtype=np.float64) for c in cids]
    confs = item.GetConformers()
    if not confs:
        raise ValueError("molecule without conformers and no embedder for it")
    xyz = [np.asarray(c.pos if hasattr(c, "pos") else c.GetPositions(), dtype=np.float64) for c in confs]
    return item, xyz[:k] if k else xyz


def generate_conformers_nk(
    smiles_list: Sequence,
    n_confs_per_mol=10,
    *,
    max_confs_per_batch: Optional[int] = None,
    max_memory_bytes: Optional[int] = None,
    dg_max_iters: int = 0,
    etk_max_iters: int = 0,
    fourth_dim_weight: float = 0.1,
    chiral_weight: float = 1.0,
    variant: str = "ETKDGv2",
    run_mmff: bool = False,
    mmff_max_iters: int = 0,
    mmff_use_lbfgs: Optional[bool] = None,
    mmff_variant: str = "MMFF94",
) -> PipelineResult:
    """N molecules x k conformers; MMFF94/94s refinement on the GPU when ``run_mmff``."""
    t0 = time.time()
    N = len(smiles_list)
    ks = [n_confs_per_mol] * N if isinstance(n_confs_per_mol, int) else list(n_confs_per_mol)
    embedded = [_embed(item, int(k), 42 + i) for i, (item, k) in enumerate(zip(smiles_list, ks))]
    results = [ConformerResult(n_atoms=m.GetNumAtoms(), positions_3d=[x.copy() for x in xs],
                               energies=[0.0] * len(xs), converged=[True] * len(xs))
               for m, xs in embedded]
    n_batches = 0
    if run_mmff and N:
        params, ok = [], []
        for (mol, xs) in embedded:
            try:
                params.append(extract_mmff_params(mol, conf_id=mol.GetConformers()[0].GetId(),
                                                  mmff_variant=mmff_variant))
                ok.append(len(xs) > 0)
            except Exception:
                params.append(None)
                ok.append(False)
        for i, good in enumerate(ok):
            if not good:
                results[i].converged = [False] * len(results[i].positions_3d)
        idx = [i for i, g in enumerate(ok) if g]
        if idx:
            max_atoms = max(params[i].n_atoms for i in idx)
            iters = mmff_max_iters if mmff_max_iters > 0 else _auto_iters(max_atoms)
            if mmff_use_lbfgs is None:
                groups = [[i for i in idx if params[i].n_atoms < mm.LBFGS_ATOM_THRESHOLD],
                          [i for i in idx if params[i].n_atoms >= mm.LBFGS_ATOM_THRESHOLD]]
                hists = [0, mm.LBFGS_M]
            else:
                groups, hists = [idx], [mm.LBFGS_M if mmff_use_lbfgs else 0]
            for grp, hist in zip(groups, hists):
                if not grp:
                    continue
                n_batches += 1
                m = mm.Minimizer([params[i] for i in grp], [len(embedded[i][1]) for i in grp])
                pos = np.concatenate([np.stack(embedded[i][1]).reshape(-1) for i in grp]).astype(np.float32)
                r = m.minimize(pos, max_iters=iters, grad_tol=1e-4, history_m=hist)
                cursor = 0
                for i in grp:
                    n = params[i].n_atoms
                    k = len(embedded[i][1])
                    start = int(m.conf_coord[cursor])
                    xyz = r.positions[start: start + 3 * n * k].reshape(k, n, 3).astype(np.float64)
                    results[i].positions_3d = [xyz[c] for c in range(k)]
                    results[i].energies = [float(v) for v in r.energies[cursor: cursor + k]]
                    results[i].converged = [bool(v) for v in r.converged[cursor: cursor + k]]
                    cursor += k
    return PipelineResult(molecules=results, total_conformers=sum(len(r.positions_3d) for r in results),
                          total_time=time.time() - t0, n_batches=max(n_batches, 1))
