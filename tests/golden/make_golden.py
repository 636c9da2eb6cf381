"""Generate the golden fixture that pins term extraction and energies to the reference.

Run from the repository root with the reference checkout available:

    python tests/golden/make_golden.py /root/reference

It builds a handful of seeded synthetic molecules (mlxmolkit_b200.synth),
runs the REFERENCE's own ``extract_mmff_params`` (mlxmolkit/mmff_params.py)
and numpy energy/gradient (mlxmolkit/mmff_energy_vectorized.py) on them
through the stand-in ``rdkit`` module of ``fake_rdkit.py``, and stores the
molecule graphs, coordinates, term lists and energies in
``tests/golden/ref_mmff_synth.npz``.  The tests compare this package's
extraction and the FP64 oracle against that file, so they need neither the
reference nor RDKit at run time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mlxmolkit-archive_b200"))
sys.path.insert(0, HERE)

import fake_rdkit  # noqa: E402
from mlxmolkit_b200 import synth  # noqa: E402
from mlxmolkit_b200.mmff_params import TERM_FIELDS  # noqa: E402

# (seed, heavy_lo, heavy_hi, macrocycle) of the fixture molecules
SPECS = [(101, 6, 10, False), (102, 12, 20, False), (103, 20, 30, False), (104, 30, 45, False),
         (105, 14, 18, True), (106, 40, 60, False), (107, 8, 14, False), (108, 25, 35, False)]


def main(ref_root: str) -> None:
    rp, rv = fake_rdkit.import_reference(ref_root)
    out = {}
    for mi, (seed, lo, hi, macro) in enumerate(SPECS):
        rng = np.random.default_rng(seed)
        mol = synth.generate_molecule(rng, lo, hi, macrocycle=macro, name=f"golden-{mi}")
        for c in synth.embed_conformers(mol, 3, rng):
            mol.AddConformer(c)
        pre = f"m{mi}_"
        out[pre + "elements"] = np.array(mol.elements)
        out[pre + "bonds"] = np.array([(b._i, b._j, b.order) for b in mol.bonds], dtype=np.float64)
        out[pre + "aromatic"] = mol.aromatic.astype(np.int8)
        out[pre + "ring_of"] = np.array(mol.ring_of, dtype=np.int32)
        pos = np.stack([c.pos for c in mol.GetConformers()])
        out[pre + "pos"] = pos
        for variant in ("MMFF94", "MMFF94s"):
            p = rp.extract_mmff_params(mol, mmff_variant=variant)
            vp = f"{pre}{variant}_"
            for f in TERM_FIELDS:
                out[vp + f] = getattr(p, f)
            out[vp + "ele_diel_model"] = np.array(p.ele_diel_model)
            e, g = rv.mmff_energy_grad_batch(p, pos)
            out[vp + "ref_energy"] = np.asarray(e, dtype=np.float64)
            out[vp + "ref_grad"] = np.asarray(g, dtype=np.float32)
    out["n_mols"] = np.array(len(SPECS))
    np.savez_compressed(os.path.join(HERE, "ref_mmff_synth.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_mmff_synth.npz"), "molecules:", len(SPECS))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
