"""MMFF94/94s term tables of one molecule, extracted once and shared by its conformers.

``MMFFParams`` has the field names, dtypes and term order of the reference
dataclass (mlxmolkit/mmff_params.py:30-80), plus two optional per-atom arrays
(``atom_type``, ``partial_charge``) that let the packer express the O(N^2)
non-bonded pair table as per-atom data (see ``pack.py``).

``extract_mmff_params`` reproduces the reference enumeration
(mlxmolkit/mmff_params.py:100-322) term for term and in the same order:

* bonds in bond order, parameters from ``GetMMFFBondStretchParams`` (:129-146);
* angles per centre atom, neighbour pairs ii<jj, linear flag from SP
  hybridization (:148-173);
* stretch-bend per non-SP centre when both stretch-bend and angle parameters
  exist, r0 from the bond table with 1.5 A default (:175-210);
* out-of-plane for degree-3 centres, the three permutations
  (n0,c,n1,n2) (n0,c,n2,n1) (n1,c,n2,n0) with one koop (:212-238);
* torsions per bond (i2,i3) over neighbours i1 of i2 and i4 of i3 with
  i1 != i3, i4 != i2, i4 != i1 (:240-270);
* van der Waals + electrostatics over i<j with topological distance >= 3 and
  conformer distance <= ``non_bonded_thresh``; vdW from the donor-acceptor
  scaled slots [2], [3]; electrostatics when both |q| > 1e-10, charge term
  q_i*q_j rounded to float32 and the 1-4 flag (:272-320).

The non-bonded double loop is vectorised with numpy: the pair order (row-major
over i<j) and every value are identical to the reference's Python loop.  It
works on RDKit molecules (through ``rdForceFieldHelpers``) and on the
synthetic ``SynthMol`` molecules of this package.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

RELATION_1_2 = 0
RELATION_1_3 = 1
RELATION_1_4 = 2
RELATION_1_X = 3


def _i32():
    return field(default_factory=lambda: np.empty(0, dtype=np.int32))


def _f32():
    return field(default_factory=lambda: np.empty(0, dtype=np.float32))


@dataclass
class MMFFParams:
    """All MMFF94 parameters for a molecule, stored as flat numpy arrays."""

    n_atoms: int

    bond_idx1: np.ndarray = _i32()
    bond_idx2: np.ndarray = _i32()
    bond_kb: np.ndarray = _f32()
    bond_r0: np.ndarray = _f32()

    angle_idx1: np.ndarray = _i32()
    angle_idx2: np.ndarray = _i32()
    angle_idx3: np.ndarray = _i32()
    angle_ka: np.ndarray = _f32()
    angle_theta0: np.ndarray = _f32()
    angle_is_linear: np.ndarray = _i32()

    strbend_idx1: np.ndarray = _i32()
    strbend_idx2: np.ndarray = _i32()
    strbend_idx3: np.ndarray = _i32()
    strbend_kba_ijk: np.ndarray = _f32()
    strbend_kba_kji: np.ndarray = _f32()
    strbend_r0_ij: np.ndarray = _f32()
    strbend_r0_kj: np.ndarray = _f32()
    strbend_theta0: np.ndarray = _f32()

    oop_idx1: np.ndarray = _i32()
    oop_idx2: np.ndarray = _i32()
    oop_idx3: np.ndarray = _i32()
    oop_idx4: np.ndarray = _i32()
    oop_koop: np.ndarray = _f32()

    torsion_idx1: np.ndarray = _i32()
    torsion_idx2: np.ndarray = _i32()
    torsion_idx3: np.ndarray = _i32()
    torsion_idx4: np.ndarray = _i32()
    torsion_V1: np.ndarray = _f32()
    torsion_V2: np.ndarray = _f32()
    torsion_V3: np.ndarray = _f32()

    vdw_idx1: np.ndarray = _i32()
    vdw_idx2: np.ndarray = _i32()
    vdw_R_star: np.ndarray = _f32()
    vdw_eps: np.ndarray = _f32()

    ele_idx1: np.ndarray = _i32()
    ele_idx2: np.ndarray = _i32()
    ele_charge_term: np.ndarray = _f32()
    ele_diel_model: int = 1
    ele_is_1_4: np.ndarray = _i32()

    # per-atom extras (not in the reference dataclass): MMFF atom type and the
    # float64 partial charge the electrostatic charge terms were formed from
    atom_type: Optional[np.ndarray] = None
    partial_charge: Optional[np.ndarray] = None

    def term_counts(self) -> dict:
        return {"bond": len(self.bond_idx1), "angle": len(self.angle_idx1),
                "strbend": len(self.strbend_idx1), "oop": len(self.oop_idx1),
                "torsion": len(self.torsion_idx1), "vdw": len(self.vdw_idx1),
                "ele": len(self.ele_idx1)}


TERM_FIELDS = [
    "bond_idx1", "bond_idx2", "bond_kb", "bond_r0",
    "angle_idx1", "angle_idx2", "angle_idx3", "angle_ka", "angle_theta0", "angle_is_linear",
    "strbend_idx1", "strbend_idx2", "strbend_idx3", "strbend_kba_ijk", "strbend_kba_kji",
    "strbend_r0_ij", "strbend_r0_kj", "strbend_theta0",
    "oop_idx1", "oop_idx2", "oop_idx3", "oop_idx4", "oop_koop",
    "torsion_idx1", "torsion_idx2", "torsion_idx3", "torsion_idx4",
    "torsion_V1", "torsion_V2", "torsion_V3",
    "vdw_idx1", "vdw_idx2", "vdw_R_star", "vdw_eps",
    "ele_idx1", "ele_idx2", "ele_charge_term", "ele_is_1_4",
]


def _props_for(mol, mmff_variant: str):
    from . import synth
    if isinstance(mol, synth.SynthMol):
        return synth.SynthMMFFProperties(mol, mmff_variant), True
    from rdkit.Chem import rdForceFieldHelpers   # real RDKit molecule
    return rdForceFieldHelpers.MMFFGetMoleculeProperties(mol, mmffVariant=mmff_variant), False


def _topological_distance(mol) -> np.ndarray:
    from . import synth
    if isinstance(mol, synth.SynthMol):
        return mol.distance_matrix()
    from rdkit import Chem
    return Chem.GetDistanceMatrix(mol)


def _conformer_xyz(mol, conf_id: int) -> np.ndarray:
    conf = mol.GetConformer(conf_id)
    if hasattr(conf, "pos"):
        return np.asarray(conf.pos, dtype=np.float64)
    return np.asarray(conf.GetPositions(), dtype=np.float64)


def _is_sp(atom) -> bool:
    return str(atom.GetHybridization()) == "SP"


def extract_mmff_params(mol, conf_id: int = 0, non_bonded_thresh: float = 100.0,
                        mmff_variant: str = "MMFF94") -> MMFFParams:
    """MMFF94 or MMFF94s term tables of ``mol`` (RDKit ``Mol`` or ``SynthMol``).

    Raises ``ValueError`` when MMFF properties cannot be computed, like the
    reference (mlxmolkit/mmff_params.py:122-124).
    """
    mp, is_synth = _props_for(mol, mmff_variant)
    if mp is None:
        raise ValueError("Could not compute MMFF properties for molecule")
    n_atoms = mol.GetNumAtoms()
    p = MMFFParams(n_atoms=n_atoms)
    atoms = [mol.GetAtomWithIdx(i) for i in range(n_atoms)]
    nbrs = [[x.GetIdx() for x in a.GetNeighbors()] for a in atoms]
    sp = [_is_sp(a) for a in atoms]

    # --- 1. bonds ---
    b1, b2, bk, br = [], [], [], []
    bond_r0 = {}
    bond_list = [(b.GetBeginAtomIdx(), b.GetEndAtomIdx()) for b in mol.GetBonds()]
    for i, j in bond_list:
        res = mp.GetMMFFBondStretchParams(mol, i, j)
        if res:
            _, kb, r0 = res
            b1.append(i); b2.append(j); bk.append(kb); br.append(r0)
            bond_r0[(i, j)] = r0
            bond_r0[(j, i)] = r0
    p.bond_idx1 = np.array(b1, dtype=np.int32)
    p.bond_idx2 = np.array(b2, dtype=np.int32)
    p.bond_kb = np.array(bk, dtype=np.float32)
    p.bond_r0 = np.array(br, dtype=np.float32)

    # --- 2. angles and 3. stretch-bend (one pass over centres) ---
    a1, a2, a3, aka, at0, alin = [], [], [], [], [], []
    s1, s2, s3, sij, skj, srij, srkj, st0 = [], [], [], [], [], [], [], []
    for c in range(n_atoms):
        nb = nbrs[c]
        if len(nb) < 2:
            continue
        lin = 1 if sp[c] else 0
        for ii in range(len(nb)):
            for jj in range(ii + 1, len(nb)):
                i, j = nb[ii], nb[jj]
                res = mp.GetMMFFAngleBendParams(mol, i, c, j)
                if res:
                    _, ka, t0 = res
                    a1.append(i); a2.append(c); a3.append(j)
                    aka.append(ka); at0.append(t0); alin.append(lin)
                if sp[c]:
                    continue
                rsb = mp.GetMMFFStretchBendParams(mol, i, c, j)
                if rsb and res:
                    _, kij, kkj = rsb
                    s1.append(i); s2.append(c); s3.append(j)
                    sij.append(kij); skj.append(kkj)
                    srij.append(bond_r0.get((i, c), 1.5))
                    srkj.append(bond_r0.get((j, c), 1.5))
                    st0.append(res[2])
    p.angle_idx1 = np.array(a1, dtype=np.int32)
    p.angle_idx2 = np.array(a2, dtype=np.int32)
    p.angle_idx3 = np.array(a3, dtype=np.int32)
    p.angle_ka = np.array(aka, dtype=np.float32)
    p.angle_theta0 = np.array(at0, dtype=np.float32)
    p.angle_is_linear = np.array(alin, dtype=np.int32)
    p.strbend_idx1 = np.array(s1, dtype=np.int32)
    p.strbend_idx2 = np.array(s2, dtype=np.int32)
    p.strbend_idx3 = np.array(s3, dtype=np.int32)
    p.strbend_kba_ijk = np.array(sij, dtype=np.float32)
    p.strbend_kba_kji = np.array(skj, dtype=np.float32)
    p.strbend_r0_ij = np.array(srij, dtype=np.float32)
    p.strbend_r0_kj = np.array(srkj, dtype=np.float32)
    p.strbend_theta0 = np.array(st0, dtype=np.float32)

    # --- 4. out-of-plane ---
    o1, o2, o3, o4, ok = [], [], [], [], []
    for c in range(n_atoms):
        nb = nbrs[c]
        if len(nb) != 3:
            continue
        res = mp.GetMMFFOopBendParams(mol, nb[0], c, nb[1], nb[2])
        if res is None:
            continue
        for (x1, x3, x4) in ((nb[0], nb[1], nb[2]), (nb[0], nb[2], nb[1]),
                             (nb[1], nb[2], nb[0])):
            o1.append(x1); o2.append(c); o3.append(x3); o4.append(x4); ok.append(res)
    p.oop_idx1 = np.array(o1, dtype=np.int32)
    p.oop_idx2 = np.array(o2, dtype=np.int32)
    p.oop_idx3 = np.array(o3, dtype=np.int32)
    p.oop_idx4 = np.array(o4, dtype=np.int32)
    p.oop_koop = np.array(ok, dtype=np.float32)

    # --- 5. torsions ---
    t1, t2, t3, t4, v1, v2, v3 = [], [], [], [], [], [], []
    for i2, i3 in bond_list:
        for i1 in nbrs[i2]:
            if i1 == i3:
                continue
            for i4 in nbrs[i3]:
                if i4 == i2 or i4 == i1:
                    continue
                res = mp.GetMMFFTorsionParams(mol, i1, i2, i3, i4)
                if res:
                    _, V1, V2, V3 = res
                    t1.append(i1); t2.append(i2); t3.append(i3); t4.append(i4)
                    v1.append(V1); v2.append(V2); v3.append(V3)
    p.torsion_idx1 = np.array(t1, dtype=np.int32)
    p.torsion_idx2 = np.array(t2, dtype=np.int32)
    p.torsion_idx3 = np.array(t3, dtype=np.int32)
    p.torsion_idx4 = np.array(t4, dtype=np.int32)
    p.torsion_V1 = np.array(v1, dtype=np.float32)
    p.torsion_V2 = np.array(v2, dtype=np.float32)
    p.torsion_V3 = np.array(v3, dtype=np.float32)

    # --- 6 & 7. non-bonded (vectorised double loop) ---
    dm = _topological_distance(mol)
    xyz = _conformer_xyz(mol, conf_id)
    ii, jj = np.triu_indices(n_atoms, k=1)
    d_top = dm[ii, jj]
    keep = d_top >= 3
    ii, jj, d_top = ii[keep], jj[keep], d_top[keep]
    diff = xyz[ii] - xyz[jj]
    dist = np.sqrt(diff[:, 0] ** 2 + diff[:, 1] ** 2 + diff[:, 2] ** 2)
    keep = ~(dist > non_bonded_thresh)
    ii, jj, d_top = ii[keep], jj[keep], d_top[keep]
    is14 = (d_top == 3)

    if is_synth:
        R, E = mp.vdw_scaled_matrix(ii, jj)
        vmask = np.ones(len(ii), dtype=bool)
    else:
        R = np.zeros(len(ii)); E = np.zeros(len(ii)); vmask = np.zeros(len(ii), dtype=bool)
        for t, (i, j) in enumerate(zip(ii.tolist(), jj.tolist())):
            res = mp.GetMMFFVdWParams(i, j)
            if res:
                vmask[t] = True
                R[t], E[t] = res[2], res[3]
    p.vdw_idx1 = ii[vmask].astype(np.int32)
    p.vdw_idx2 = jj[vmask].astype(np.int32)
    p.vdw_R_star = np.asarray(R, dtype=np.float64)[vmask].astype(np.float32)
    p.vdw_eps = np.asarray(E, dtype=np.float64)[vmask].astype(np.float32)

    q = np.array([mp.GetMMFFPartialCharge(i) for i in range(n_atoms)], dtype=np.float64)
    emask = (np.abs(q[ii]) > 1e-10) & (np.abs(q[jj]) > 1e-10)
    p.ele_idx1 = ii[emask].astype(np.int32)
    p.ele_idx2 = jj[emask].astype(np.int32)
    p.ele_charge_term = (q[ii[emask]] * q[jj[emask]]).astype(np.float32)
    p.ele_is_1_4 = is14[emask].astype(np.int32)
    p.ele_diel_model = 0

    p.atom_type = np.array([mp.GetMMFFAtomType(i) for i in range(n_atoms)], dtype=np.int32)
    p.partial_charge = q
    return p
