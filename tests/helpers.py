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
