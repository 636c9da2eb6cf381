"""Generate the golden fixture that pins the DG stage's host side to the reference.

Run from the repository root with the reference checkout available:

    python tests/golden/make_golden_dg.py <reference-root>

Through the stand-in ``rdkit`` / ``mlx`` modules of ``fake_rdkit.py`` it runs
the REFERENCE's own mlxmolkit/dg_extract.py (``extract_dg_params``,
``metric_matrix_positions``) and mlxmolkit/shared_batch.py
(``pack_shared_dg_batch``, ``init_random_positions``) on

  * the all-pairs constraint sets of the reference's DG tests
    (tests/test_conformer_metal.py:22-43), and
  * seeded synthetic molecules whose bounds matrix and chiral tags come from
    this package's stand-ins (``synth_bounds_matrix``, ``synth_chiral_tags``),
    and their ETK terms (``etk_extract.synth_etk_params``) through the
    reference's ``add_etk_to_batch`` (mlxmolkit/shared_batch.py:204-296), and the
    reference's stereo checks (mlxmolkit/stereo_checks_metal.py:102-141,
    ``extract_tetrahedral_data``) on their conformers as embedded, mirrored and
    flattened,

and stores the inputs and the reference's outputs in
``tests/golden/ref_dg_batches.npz``.  The tests compare this package's
functions with that file; they need neither the reference nor RDKit.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mlxmolkit-archive_b200"))
sys.path.insert(0, HERE)

import fake_rdkit  # noqa: E402
from mlxmolkit_b200 import synth  # noqa: E402
from mlxmolkit_b200.dg_extract import synth_bounds_matrix, synth_chiral_tags  # noqa: E402
from mlxmolkit_b200.etk_extract import synth_etk_params  # noqa: E402

BATCH_FIELDS = ("conf_atom_starts", "conf_to_mol", "mol_n_atoms", "dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2",
                "dist_weight", "dist_term_starts", "chiral_idx1", "chiral_idx2", "chiral_idx3", "chiral_idx4",
                "chiral_vol_lower", "chiral_vol_upper", "chiral_term_starts", "fourth_idx", "fourth_term_starts")
ETK_FIELDS = ("torsion_idx", "torsion_V", "torsion_signs", "improper_idx", "improper_weight", "dist12_idx1",
              "dist12_idx2", "dist12_lb", "dist12_ub", "dist12_weight", "dist13_idx1", "dist13_idx2", "dist13_lb",
              "dist13_ub", "dist13_weight", "dist14_idx1", "dist14_idx2", "dist14_lb", "dist14_ub", "dist14_weight")
ETK_BATCH = ["etk_torsion_idx", "etk_torsion_V", "etk_torsion_signs", "etk_torsion_term_starts", "etk_improper_idx",
             "etk_improper_weight", "etk_improper_term_starts"] + [
    f"etk_dist{t}_{f}" for t in ("12", "13", "14") for f in ("idx1", "idx2", "lb", "ub", "weight", "term_starts")]
PARAM_FIELDS = ("dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2", "dist_weight", "chiral_idx1", "chiral_idx2",
                "chiral_idx3", "chiral_idx4", "chiral_vol_lower", "chiral_vol_upper", "fourth_idx")
# (seed, heavy_lo, heavy_hi) of the synthetic molecules, and their conformer counts
SYNTH = [(201, 8, 12), (202, 14, 20), (203, 22, 30)]
SYNTH_K = [2, 3, 1]
ALLPAIRS = [(5, 1.0, 4.0), (8, 1.0, 4.0), (6, 1.5, 3.0)]
ALLPAIRS_K = [3, 2, 2]


def _all_pairs(DGParams, n, lb, ub):
    iu, ju = np.triu_indices(n, 1)
    m = len(iu)
    z = np.zeros(0, dtype=np.int32)
    return DGParams(n_atoms=n, dist_idx1=iu.astype(np.int32), dist_idx2=ju.astype(np.int32),
                    dist_lb2=np.full(m, lb * lb, np.float32), dist_ub2=np.full(m, ub * ub, np.float32),
                    dist_weight=np.full(m, 1.0 / max(ub * ub - lb * lb, 1e-8), np.float32),
                    chiral_idx1=z, chiral_idx2=z, chiral_idx3=z, chiral_idx4=z,
                    chiral_vol_lower=np.zeros(0, np.float32), chiral_vol_upper=np.zeros(0, np.float32),
                    fourth_idx=np.arange(n, dtype=np.int32))


def main(ref_root: str) -> None:
    fake_rdkit.install()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    rdg = importlib.import_module("mlxmolkit.dg_extract")
    rsb = importlib.import_module("mlxmolkit.shared_batch")
    retk = importlib.import_module("mlxmolkit.etk_extract")
    rst = importlib.import_module("mlxmolkit.stereo_checks_metal")
    out = {}

    # all-pairs sets of the reference's tests
    ap = [_all_pairs(rdg.DGParams, *spec) for spec in ALLPAIRS]
    b = rsb.pack_shared_dg_batch(ap, ALLPAIRS_K, dim=4)
    for f in BATCH_FIELDS:
        out["ap_" + f] = np.asarray(getattr(b, f))
    out["ap_init_seed7"] = rsb.init_random_positions(b, seed=7)

    # synthetic molecules through the reference's extraction
    params, bms, etks, mols = [], [], [], []
    for mi, (seed, lo, hi) in enumerate(SYNTH):
        rng = np.random.default_rng(seed)
        mol = synth.generate_molecule(rng, lo, hi, name=f"dg-golden-{mi}")
        for c in synth.embed_conformers(mol, 1, rng):
            mol.AddConformer(c)
        bm = synth_bounds_matrix(mol)
        mol.chiral_tags = synth_chiral_tags(mol)
        p = rdg.extract_dg_params(mol, bm)
        pre = f"s{mi}_"
        out[pre + "elements"] = np.array(mol.elements)
        out[pre + "bonds"] = np.array([(bd._i, bd._j, bd.order) for bd in mol.bonds], dtype=np.float64)
        out[pre + "aromatic"] = mol.aromatic.astype(np.int8)
        out[pre + "ring_of"] = np.array(mol.ring_of, dtype=np.int32)
        out[pre + "pos"] = mol.GetConformers()[0].pos
        out[pre + "bounds_mat"] = bm
        out[pre + "chiral_centers"] = np.array(sorted(mol.chiral_tags), dtype=np.int32)
        out[pre + "chiral_tags"] = np.array([mol.chiral_tags[k] for k in sorted(mol.chiral_tags)])
        for f in PARAM_FIELDS:
            out[pre + "ref_" + f] = np.asarray(getattr(p, f))
        params.append(p)
        bms.append(bm)
        mols.append(mol)
        tet = rdg.extract_tetrahedral_data(mol)
        out[pre + "ref_tetrahedral"] = np.array(tet[:5], dtype=np.int32).reshape(5, -1)
        ep = synth_etk_params(mol, bm)
        for f in ETK_FIELDS:
            out[pre + "etk_" + f] = np.asarray(getattr(ep, f))
        etks.append(retk.ETKParams(n_atoms=ep.n_atoms, **{f: getattr(ep, f) for f in ETK_FIELDS}))
    b = rsb.pack_shared_dg_batch(params, SYNTH_K, dim=4)
    for f in BATCH_FIELDS:
        out["sy_" + f] = np.asarray(getattr(b, f))
    out["sy_metric_seed42"] = rdg.metric_matrix_positions(b, bms, seed=42, dim=4)
    out["sy_metric_seed5_dim3"] = rdg.metric_matrix_positions(rsb.pack_shared_dg_batch(params, SYNTH_K, dim=3),
                                                              bms, seed=5, dim=3)
    # stereo checks: conformer j of a molecule as embedded (j = 0), mirrored (1: chirality inverted),
    # flattened onto z = 0 (2: planar centres)
    pos4 = np.zeros((int(b.conf_atom_starts[-1]), 4), np.float32)
    c = 0
    for mol, k in zip(mols, SYNTH_K):
        x = np.asarray(mol.GetConformers()[0].pos, dtype=np.float32)
        for j in range(k):
            y = x.copy()
            if j == 1:
                y[:, 0] = -y[:, 0]
            elif j == 2:
                y[:, 2] = 0.0
            a0 = int(b.conf_atom_starts[c])
            pos4[a0:a0 + len(x), :3] = y
            c += 1
    out["sy_stereo_pos4"] = pos4.reshape(-1)
    out["sy_stereo_passed"] = rst.run_stereo_checks(pos4.reshape(-1), params, mols, b.conf_atom_starts,
                                                    b.conf_to_mol, list(range(len(mols))), b.n_confs_total, dim=4)
    b3 = rsb.pack_shared_dg_batch(params, SYNTH_K, dim=3)
    rsb.add_etk_to_batch(b3, etks)
    for f in ETK_BATCH:
        out["sy3_" + f] = np.asarray(getattr(b3, f))
    np.savez_compressed(os.path.join(HERE, "ref_dg_batches.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_dg_batches.npz"), "arrays:", len(out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden_dg.py <reference-root>")
    main(sys.argv[1])
