"""ETK (experimental-torsion knowledge) terms of the 3-D embedding stage.

Mirror of the reference's mlxmolkit/etk_extract.py: ``ETKParams`` (:51-84) with
the same fields.  The reference fills them from RDKit --
``GetExperimentalTorsions`` (CSD torsion preferences), hybridisation, ring
information and the bounds matrix (:130-428) -- which is not available here.
``synth_etk_params`` is a synthetic stand-in for the seeded molecules of
``synth.py`` that produces the same term families with the reference's
weights and tolerances:

  * torsion preferences on rotatable single bonds (6-term Fourier form; a
    3-fold term for sp3-sp3, a 2-fold planar term for sp2-sp2, a 6-fold term
    otherwise) and ring-planarity torsions V1 = 100, s1 = -1 on aromatic ring
    bonds (:228-238);
  * impropers at sp2 C / N / O centres with exactly three neighbours, all three
    neighbour permutations, weight 10, x 50/6 next to a terminal sp2 oxygen
    (:257-292);
  * 1-2 and 1-3 flat-bottom terms at the bounds-matrix midpoint +- 0.01 A, force
    constant 100 (:300-345);
  * 1-4 terms at the bounds with weight 1, and long-range terms (topological
    distance >= 4) at weight 10, first occurrence of a pair kept (:346-405).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BOND_TOL = 0.01
BOND_FC = 100.0
ANGLE_FC = 100.0
IMPROPER_WEIGHT = 10.0
RING_PLANARITY_FC = 100.0
DIST14_WEIGHT = 1.0
LONG_RANGE_WEIGHT = 10.0


@dataclass
class ETKParams:
    """ETK terms of one molecule (etk_extract.py:51-84)."""
    n_atoms: int
    torsion_idx: np.ndarray      # (n, 4) int32
    torsion_V: np.ndarray        # (n, 6) float32
    torsion_signs: np.ndarray    # (n, 6) int32
    improper_idx: np.ndarray     # (n, 4) int32: centre, three neighbours
    improper_weight: np.ndarray  # (n,) float32
    dist12_idx1: np.ndarray
    dist12_idx2: np.ndarray
    dist12_lb: np.ndarray
    dist12_ub: np.ndarray
    dist12_weight: np.ndarray
    dist13_idx1: np.ndarray
    dist13_idx2: np.ndarray
    dist13_lb: np.ndarray
    dist13_ub: np.ndarray
    dist13_weight: np.ndarray
    dist14_idx1: np.ndarray
    dist14_idx2: np.ndarray
    dist14_lb: np.ndarray
    dist14_ub: np.ndarray
    dist14_weight: np.ndarray


def _hyb(atom) -> str:
    return str(atom.GetHybridization()).split(".")[-1]


def synth_etk_params(mol, bounds_mat: np.ndarray) -> ETKParams:
    """ETK terms of a ``synth`` molecule from its bounds matrix (see the module doc)."""
    bm = np.asarray(bounds_mat, dtype=np.float64)
    n = int(mol.GetNumAtoms())
    atoms = list(mol.GetAtoms())
    nbrs = [[x.GetIdx() for x in a.GetNeighbors()] for a in atoms]
    ring_of = list(getattr(mol, "ring_of", [-1] * n))
    arom = np.asarray(getattr(mol, "aromatic", np.zeros(n, bool)), dtype=bool)

    tq, tv, ts = [], [], []
    seen_ring = set()
    for bd in mol.GetBonds():
        b, c = bd.GetBeginAtomIdx(), bd.GetEndAtomIdx()
        same_ring = ring_of[b] >= 0 and ring_of[b] == ring_of[c]
        others_b = [x for x in nbrs[b] if x != c]
        others_c = [x for x in nbrs[c] if x != b]
        if not others_b or not others_c:
            continue
        heavy_b = [x for x in others_b if atoms[x].GetSymbol() != "H"] or others_b
        heavy_c = [x for x in others_c if atoms[x].GetSymbol() != "H"] or others_c
        a, d = heavy_b[0], heavy_c[0]
        if same_ring and arom[b] and arom[c]:
            key = (min(b, c), max(b, c))
            if key not in seen_ring:
                seen_ring.add(key)
                tq.append([a, b, c, d]), tv.append([0, RING_PLANARITY_FC, 0, 0, 0, 0]), ts.append([0, -1, 0, 0, 0, 0])
            continue
        if same_ring or bd.GetBondTypeAsDouble() != 1.0:
            continue
        hb, hc = _hyb(atoms[b]), _hyb(atoms[c])
        if hb == "SP3" and hc == "SP3":
            v, s = [0, 0, 2.5, 0, 0, 0], [0, 0, 1, 0, 0, 0]
        elif hb == "SP2" and hc == "SP2":
            v, s = [0, 6.0, 0, 0, 0, 0], [0, -1, 0, 0, 0, 0]
        else:
            v, s = [0, 0, 0, 0, 0, 0.6], [0, 0, 0, 0, 0, 1]
        tq.append([a, b, c, d]), tv.append(v), ts.append(s)

    iq, iw = [], []
    for a in atoms:
        if a.GetSymbol() not in ("C", "N", "O") or _hyb(a) != "SP2" or len(nbrs[a.GetIdx()]) != 3:
            continue
        w = IMPROPER_WEIGHT
        if a.GetSymbol() == "C" and any(atoms[x].GetSymbol() == "O" and _hyb(atoms[x]) == "SP2" and
                                        len(nbrs[x]) == 1 for x in nbrs[a.GetIdx()]):
            w = IMPROPER_WEIGHT * (50.0 / 6.0)
        c0 = a.GetIdx()
        n0, n1, n2 = nbrs[c0]
        for p in ((n0, n1, n2), (n1, n2, n0), (n2, n0, n1)):
            iq.append([c0, *p]), iw.append(w)

    def pairs(cand):
        """(i, j) arrays of the candidate pairs whose bounds are both positive, order kept."""
        c = np.asarray(cand, dtype=np.int64).reshape(-1, 2)
        keep = (bm[c[:, 0], c[:, 1]] > 0) & (bm[c[:, 1], c[:, 0]] > 0) if len(c) else np.zeros(0, bool)
        return c[keep, 0], c[keep, 1]

    bonds = [(bd.GetBeginAtomIdx(), bd.GetEndAtomIdx()) for bd in mol.GetBonds()]
    i12, j12 = pairs([(min(i, j), max(i, j)) for i, j in bonds])
    i13, j13 = pairs([(nb[x], nb[y]) for nb in (sorted(v) for v in nbrs)
                      for x in range(len(nb)) for y in range(x + 1, len(nb))])
    # 1-4 pairs (a < d) through each bond b-c, first occurrence kept
    a14, d14 = pairs([(a, d) for b, c in bonds for a in nbrs[b] if a != c for d in nbrs[c] if d != b and a < d])
    if len(a14):
        _, first = np.unique(a14 * n + d14, return_index=True)
        first.sort()
        a14, d14 = a14[first], d14[first]
    topo = np.asarray(mol.distance_matrix())
    iu, ju = np.triu_indices(n, 1)                 # row-major, as the reference's double loop
    keep = (topo[iu, ju] >= 4) & (bm[iu, ju] > 0) & (bm[ju, iu] > 0)
    if len(a14):
        taken = np.zeros((n, n), dtype=bool)
        taken[a14, d14] = True
        keep &= ~taken[iu, ju]
    iL, jL = iu[keep], ju[keep]
    i14, j14 = np.concatenate([a14, iL]), np.concatenate([d14, jL])
    w14 = np.concatenate([np.full(len(a14), DIST14_WEIGHT), np.full(len(iL), LONG_RANGE_WEIGHT)])

    def mid(i, j):
        return 0.5 * (bm[j, i] + bm[i, j])

    def i32(x, shape=(0,)):
        return np.array(x, dtype=np.int32).reshape(-1, *shape[1:]) if len(x) else np.zeros(shape, np.int32)

    def f32(x, shape=(0,)):
        return np.array(x, dtype=np.float32).reshape(-1, *shape[1:]) if len(x) else np.zeros(shape, np.float32)

    return ETKParams(
        n_atoms=n,
        torsion_idx=i32(tq, (0, 4)), torsion_V=f32(tv, (0, 6)), torsion_signs=i32(ts, (0, 6)),
        improper_idx=i32(iq, (0, 4)), improper_weight=f32(iw),
        dist12_idx1=i32(i12), dist12_idx2=i32(j12),
        dist12_lb=f32(mid(i12, j12) - BOND_TOL), dist12_ub=f32(mid(i12, j12) + BOND_TOL),
        dist12_weight=f32(np.full(len(i12), BOND_FC)),
        dist13_idx1=i32(i13), dist13_idx2=i32(j13),
        dist13_lb=f32(mid(i13, j13) - BOND_TOL), dist13_ub=f32(mid(i13, j13) + BOND_TOL),
        dist13_weight=f32(np.full(len(i13), ANGLE_FC)),
        dist14_idx1=i32(i14), dist14_idx2=i32(j14),
        dist14_lb=f32(bm[j14, i14]), dist14_ub=f32(bm[i14, j14]),
        dist14_weight=f32(w14),
    )
