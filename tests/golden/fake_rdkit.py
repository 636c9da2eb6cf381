"""A stand-in ``rdkit`` package that lets the reference's own Python run on SynthMol molecules.

Used only by ``make_golden.py`` (and the reference-pinning tests when the
reference checkout is present) to execute the reference's
``extract_mmff_params`` and numpy energy on the synthetic molecules of this
package.  It provides the few names those files import: ``Chem.HybridizationType``,
``Chem.GetDistanceMatrix`` and ``Chem.rdForceFieldHelpers.MMFFGetMoleculeProperties``.
"""
from __future__ import annotations

import sys
import types


def install():
    from mlxmolkit_b200 import synth
    rdkit = types.ModuleType("rdkit")
    chem = types.ModuleType("rdkit.Chem")
    ff = types.ModuleType("rdkit.Chem.rdForceFieldHelpers")
    chem.HybridizationType = synth.HybridizationType
    chem.GetDistanceMatrix = lambda mol: mol.distance_matrix()
    chem.Mol = synth.SynthMol
    ff.MMFFGetMoleculeProperties = synth.MMFFGetMoleculeProperties
    chem.rdForceFieldHelpers = ff
    # the distance-geometry modules: chirality read from a SynthMol's ``chiral_tags`` dict
    # ({atom: "CW" | "CCW" | "OTHER"}), stereo assignment a no-op, rdDistGeom and mlx.core empty
    chem.ChiralType = _ChiralType
    chem.AssignStereochemistry = lambda mol, cleanIt=True, force=True: None
    synth.SynthAtom.GetChiralTag = lambda atom: _ChiralType.BY_NAME.get(
        (getattr(atom._mol, "chiral_tags", None) or {}).get(atom.GetIdx()), _ChiralType.CHI_UNSPECIFIED)
    synth.SynthMol.GetRingInfo = lambda mol: _RingInfo(mol)
    dg = types.ModuleType("rdkit.Chem.rdDistGeom")
    chem.rdDistGeom = dg
    rdkit.Chem = chem
    mlx = types.ModuleType("mlx")
    mlx.core = types.ModuleType("mlx.core")
    sys.modules.update({"rdkit": rdkit, "rdkit.Chem": chem, "rdkit.Chem.rdForceFieldHelpers": ff,
                        "rdkit.Chem.rdDistGeom": dg, "mlx": mlx, "mlx.core": mlx.core})
    return rdkit


class _ChiralType:
    CHI_UNSPECIFIED, CHI_TETRAHEDRAL_CW, CHI_TETRAHEDRAL_CCW, CHI_OTHER = "unspec", "cw", "ccw", "other"
    BY_NAME = {"CW": CHI_TETRAHEDRAL_CW, "CCW": CHI_TETRAHEDRAL_CCW, "OTHER": CHI_OTHER}


def import_reference(ref_root: str):
    """Import the reference's extraction and numpy energy modules from ``ref_root``."""
    install()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    import importlib
    params = importlib.import_module("mlxmolkit.mmff_params")
    vec = importlib.import_module("mlxmolkit.mmff_energy_vectorized")
    return params, vec


class _RingInfo:
    """RingInfo over a SynthMol's ring ids (``ring_of``: one ring per atom, -1 outside rings)."""

    def __init__(self, mol):
        self.ring_of = list(mol.ring_of)

    def NumAtomRings(self, idx):
        return 1 if self.ring_of[idx] >= 0 else 0

    def IsAtomInRingOfSize(self, idx, size):
        r = self.ring_of[idx]
        return r >= 0 and sum(1 for x in self.ring_of if x == r) == size
