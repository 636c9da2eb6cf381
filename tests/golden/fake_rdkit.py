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
    rdkit.Chem = chem
    sys.modules.update({"rdkit": rdkit, "rdkit.Chem": chem, "rdkit.Chem.rdForceFieldHelpers": ff})
    return rdkit


def import_reference(ref_root: str):
    """Import the reference's extraction and numpy energy modules from ``ref_root``."""
    install()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    import importlib
    params = importlib.import_module("mlxmolkit.mmff_params")
    vec = importlib.import_module("mlxmolkit.mmff_energy_vectorized")
    return params, vec
