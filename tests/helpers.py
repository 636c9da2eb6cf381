"""Shared helpers of the test-suite: fixture molecules and small seeded workloads."""
from __future__ import annotations

import numpy as np

from mlxmolkit_b200 import synth
from mlxmolkit_b200.mmff_params import MMFFParams, TERM_FIELDS, extract_mmff_params


def golden_mol(golden, mi: int) -> synth.SynthMol:
    pre = f"m{mi}_"
    bonds = [(int(i), int(j), float(o)) for i, j, o in golden[pre + "bonds"]]
    mol = synth.SynthMol(list(golden[pre + "elements"]), bonds, golden[pre + "aromatic"].astype(bool),
                         golden[pre + "ring_of"].tolist(), name=f"golden-{mi}")
    synth.assign_types(mol)
    for c in golden[pre + "pos"]:
        mol.AddConformer(c)
    return mol


def golden_params(golden, mi: int, variant: str = "MMFF94") -> MMFFParams:
    """The reference extraction's term lists stored in the fixture."""
    vp = f"m{mi}_{variant}_"
    n = len(golden[f"m{mi}_elements"])
    p = MMFFParams(n_atoms=n)
    for f in TERM_FIELDS:
        setattr(p, f, golden[vp + f])
    p.ele_diel_model = int(golden[vp + "ele_diel_model"])
    return p


def small_workload(n_mols=6, k=3, seed=5, lo=6, hi=24, variant="MMFF94"):
    mols = synth.make_molecules(n_mols, k, seed, lo, hi, workers=1)
    params = [extract_mmff_params(m, mmff_variant=variant) for m in mols]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m in mols])
    return mols, params, [k] * n_mols, pos


# ---- distance-geometry stage ----

def all_pairs_dg(n: int, lb: float = 1.0, ub: float = 4.0):
    """All-pair distance constraints, weight 1/(ub^2 - lb^2): the constraint sets of the
    reference's DG tests (tests/test_conformer_metal.py:22-43)."""
    from mlxmolkit_b200.dg_extract import DGParams
    iu, ju = np.triu_indices(n, 1)
    m = len(iu)
    z = np.zeros(0, dtype=np.int32)
    return DGParams(n_atoms=n, dist_idx1=iu.astype(np.int32), dist_idx2=ju.astype(np.int32),
                    dist_lb2=np.full(m, lb * lb, np.float32), dist_ub2=np.full(m, ub * ub, np.float32),
                    dist_weight=np.full(m, 1.0 / max(ub * ub - lb * lb, 1e-8), np.float32),
                    chiral_idx1=z, chiral_idx2=z, chiral_idx3=z, chiral_idx4=z,
                    chiral_vol_lower=np.zeros(0, np.float32), chiral_vol_upper=np.zeros(0, np.float32),
                    fourth_idx=np.arange(n, dtype=np.int32))


def dg_golden_mol(g, mi: int) -> synth.SynthMol:
    pre = f"s{mi}_"
    bonds = [(int(i), int(j), float(o)) for i, j, o in g[pre + "bonds"]]
    mol = synth.SynthMol(list(g[pre + "elements"]), bonds, g[pre + "aromatic"].astype(bool),
                         g[pre + "ring_of"].tolist(), name=f"dg-golden-{mi}")
    synth.assign_types(mol)
    mol.AddConformer(g[pre + "pos"])
    mol.chiral_tags = {int(c): str(t) for c, t in zip(g[pre + "chiral_centers"], g[pre + "chiral_tags"])}
    return mol


def dg_synth_params(n_mols: int, seed: int, lo: int = 8, hi: int = 30):
    """DG terms of seeded synthetic molecules (stand-in bounds and chirality)."""
    from mlxmolkit_b200.dg_extract import synth_dg_params
    mols = synth.make_molecules(n_mols, 1, seed, lo, hi, workers=1)
    return [synth_dg_params(m) for m in mols]
