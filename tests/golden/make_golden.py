"""Generate the golden fixtures that pin term extraction and energies to the reference.

Run from the repository root with the path of a reference checkout:

    python tests/golden/make_golden.py <reference-root>            # both sets
    python tests/golden/make_golden.py <reference-root> drug       # ref_mmff_synth.npz only
    python tests/golden/make_golden.py <reference-root> large      # ref_mmff_large.npz only

It builds seeded synthetic molecules (mlxmolkit_b200.synth), runs the
REFERENCE's own ``extract_mmff_params`` (mlxmolkit/mmff_params.py) and numpy
energy/gradient (mlxmolkit/mmff_energy_vectorized.py) on them through the
stand-in ``rdkit`` module of ``fake_rdkit.py``, and stores the molecule graphs,
coordinates, term lists and energies:

* ``ref_mmff_synth.npz``: 8 drug-like molecules of 16-111 atoms, 3 conformers each;
* ``ref_mmff_large.npz``: 6 molecules of 130-380 atoms, 2 conformers each -- the
  dense-BFGS class of 112-170 atoms and the L-BFGS sizes of the large workload
  (macrocycles, up to 20 rotatable bonds) up to a 400-atom molecule.

The tests compare this package's extraction, the FP64 oracle and the GPU
kernels against these files, so they need neither the reference nor RDKit at
run time.
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

# (seed, heavy_lo, heavy_hi, macrocycle, generator options) of the fixture molecules
SPECS = {
    "drug": [(101, 6, 10, False, {}), (102, 12, 20, False, {}), (103, 20, 30, False, {}),
             (104, 30, 45, False, {}), (105, 14, 18, True, {}), (106, 40, 60, False, {}),
             (107, 8, 14, False, {}), (108, 25, 35, False, {})],
    "large": [(202, 52, 58, False, dict(max_atoms=170)),
              (212, 60, 68, False, dict(max_atoms=170)),
              (203, 64, 80, True, dict(ring_density=0.12, max_rotatable=20)),
              (204, 90, 110, False, dict(ring_density=0.12, max_rotatable=20)),
              (205, 120, 140, True, dict(ring_density=0.12)),
              (206, 150, 160, False, dict(max_atoms=400))],
}
CONFS = {"drug": 3, "large": 2}
OUT = {"drug": "ref_mmff_synth.npz", "large": "ref_mmff_large.npz"}


def build(ref_root: str, which: str) -> None:
    rp, rv = fake_rdkit.import_reference(ref_root)
    out = {}
    for mi, (seed, lo, hi, macro, kw) in enumerate(SPECS[which]):
        rng = np.random.default_rng(seed)
        mol = synth.generate_molecule(rng, lo, hi, macrocycle=macro, name=f"golden-{which}-{mi}",
                                      max_tries=200, **kw)
        for c in synth.embed_conformers(mol, CONFS[which], rng):
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
        print(f"{which} molecule {mi}: {mol.GetNumAtoms()} atoms", flush=True)
    out["n_mols"] = np.array(len(SPECS[which]))
    path = os.path.join(HERE, OUT[which])
    np.savez_compressed(path, **out)
    print("wrote", path, "molecules:", len(SPECS[which]))


def main(argv) -> None:
    if not argv:
        raise SystemExit("usage: make_golden.py <reference-root> [drug|large]")
    for which in (argv[1:] or ["drug", "large"]):
        build(argv[0], which)


if __name__ == "__main__":
    main(sys.argv[1:])
