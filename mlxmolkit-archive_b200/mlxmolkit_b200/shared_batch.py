"""N molecules x k conformers with distance-geometry constraints stored once per molecule.

Mirror of the reference's mlxmolkit/shared_batch.py: ``SharedConstraintBatch``
(:23-96, same fields and meaning), ``pack_shared_dg_batch`` (:103-201) and
``init_random_positions`` (:298-309).  Constraint atom indices are local to
their molecule; conformer c of molecule ``conf_to_mol[c]`` has its
coordinates at ``conf_atom_starts[c] * dim``.

``add_etk_to_batch`` (:204-296) adds a molecule list's ETK terms.

``dg_device_arrays`` and ``etk_device_arrays`` turn a batch into the device
layout of include/mmffb200_dg.h: 16-byte distance records for the energy, the
same terms listed under each of their atoms for the gradient, incidence rows
of the multi-atom terms, fourth-dimension counts per atom row, and a
largest-first conformer order.  Host-only numpy: no device is touched here.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .dg_extract import DGParams
from .etk_extract import ETKParams


@dataclass
class SharedConstraintBatch:
    """N molecules x k conformers with shared constraints (shared_batch.py:23-96)."""

    n_mols: int
    n_confs_total: int
    n_confs_per_mol: List[int]
    dim: int

    conf_atom_starts: np.ndarray      # (C+1,) int32
    conf_to_mol: np.ndarray           # (C,) int32
    mol_n_atoms: np.ndarray           # (N,) int32

    dist_idx1: np.ndarray
    dist_idx2: np.ndarray
    dist_lb2: np.ndarray
    dist_ub2: np.ndarray
    dist_weight: np.ndarray
    dist_term_starts: np.ndarray      # (N+1,) int32

    chiral_idx1: np.ndarray
    chiral_idx2: np.ndarray
    chiral_idx3: np.ndarray
    chiral_idx4: np.ndarray
    chiral_vol_lower: np.ndarray
    chiral_vol_upper: np.ndarray
    chiral_term_starts: np.ndarray    # (N+1,) int32

    fourth_idx: np.ndarray
    fourth_term_starts: np.ndarray    # (N+1,) int32

    # ETK terms of the 3-D stage (shared_batch.py:59-89); not used by the DG stage
    etk_torsion_idx: Optional[np.ndarray] = None
    etk_torsion_V: Optional[np.ndarray] = None
    etk_torsion_signs: Optional[np.ndarray] = None
    etk_torsion_term_starts: Optional[np.ndarray] = None
    etk_improper_idx: Optional[np.ndarray] = None
    etk_improper_weight: Optional[np.ndarray] = None
    etk_improper_term_starts: Optional[np.ndarray] = None
    etk_dist12_idx1: Optional[np.ndarray] = None
    etk_dist12_idx2: Optional[np.ndarray] = None
    etk_dist12_lb: Optional[np.ndarray] = None
    etk_dist12_ub: Optional[np.ndarray] = None
    etk_dist12_weight: Optional[np.ndarray] = None
    etk_dist12_term_starts: Optional[np.ndarray] = None
    etk_dist13_idx1: Optional[np.ndarray] = None
    etk_dist13_idx2: Optional[np.ndarray] = None
    etk_dist13_lb: Optional[np.ndarray] = None
    etk_dist13_ub: Optional[np.ndarray] = None
    etk_dist13_weight: Optional[np.ndarray] = None
    etk_dist13_term_starts: Optional[np.ndarray] = None
    etk_dist14_idx1: Optional[np.ndarray] = None
    etk_dist14_idx2: Optional[np.ndarray] = None
    etk_dist14_lb: Optional[np.ndarray] = None
    etk_dist14_ub: Optional[np.ndarray] = None
    etk_dist14_weight: Optional[np.ndarray] = None
    etk_dist14_term_starts: Optional[np.ndarray] = None

    @property
    def n_atoms_total(self) -> int:
        return int(self.conf_atom_starts[-1])

    @property
    def total_coords(self) -> int:
        return self.n_atoms_total * self.dim


def _cat(arrays, dtype) -> np.ndarray:
    arrays = [np.asarray(a) for a in arrays if len(a)]
    return np.concatenate(arrays).astype(dtype) if arrays else np.zeros(0, dtype=dtype)


def _starts(counts) -> np.ndarray:
    out = np.zeros(len(counts) + 1, dtype=np.int32)
    out[1:] = np.cumsum(np.asarray(counts, dtype=np.int64))
    return out


def pack_shared_dg_batch(dg_params_list: List[DGParams], n_confs_per_mol: List[int],
                         dim: int = 4) -> SharedConstraintBatch:
    """Pack N molecules x k conformers; constraints once per molecule, local indices."""
    if len(n_confs_per_mol) != len(dg_params_list):
        raise ValueError("one conformer count per molecule is required")
    counts = [int(k) for k in n_confs_per_mol]
    mol_n_atoms = np.array([p.n_atoms for p in dg_params_list], dtype=np.int32)
    conf_to_mol = np.repeat(np.arange(len(counts), dtype=np.int32), counts).astype(np.int32)
    conf_atom_starts = _starts(mol_n_atoms[conf_to_mol]) if len(conf_to_mol) else np.zeros(1, np.int32)
    P = dg_params_list
    return SharedConstraintBatch(
        n_mols=len(P), n_confs_total=int(sum(counts)), n_confs_per_mol=counts, dim=dim,
        conf_atom_starts=conf_atom_starts, conf_to_mol=conf_to_mol, mol_n_atoms=mol_n_atoms,
        dist_idx1=_cat([p.dist_idx1 for p in P], np.int32),
        dist_idx2=_cat([p.dist_idx2 for p in P], np.int32),
        dist_lb2=_cat([p.dist_lb2 for p in P], np.float32),
        dist_ub2=_cat([p.dist_ub2 for p in P], np.float32),
        dist_weight=_cat([p.dist_weight for p in P], np.float32),
        dist_term_starts=_starts([len(p.dist_idx1) for p in P]),
        chiral_idx1=_cat([p.chiral_idx1 for p in P], np.int32),
        chiral_idx2=_cat([p.chiral_idx2 for p in P], np.int32),
        chiral_idx3=_cat([p.chiral_idx3 for p in P], np.int32),
        chiral_idx4=_cat([p.chiral_idx4 for p in P], np.int32),
        chiral_vol_lower=_cat([p.chiral_vol_lower for p in P], np.float32),
        chiral_vol_upper=_cat([p.chiral_vol_upper for p in P], np.float32),
        chiral_term_starts=_starts([len(p.chiral_idx1) for p in P]),
        fourth_idx=_cat([p.fourth_idx for p in P], np.int32),
        fourth_term_starts=_starts([len(p.fourth_idx) for p in P]),
    )


def init_random_positions(batch: SharedConstraintBatch, seed: int = 42) -> np.ndarray:
    """Independent standard-normal coordinates for every conformer (flat, float32)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal(int(batch.conf_atom_starts[-1]) * batch.dim).astype(np.float32)


def _term_mol(starts: np.ndarray) -> np.ndarray:
    return np.repeat(np.arange(len(starts) - 1, dtype=np.int64), np.diff(starts))


def dg_device_arrays(batch: SharedConstraintBatch) -> dict:
    """The device layout of include/mmffb200_dg.h as numpy arrays (validated)."""
    if batch.dim not in (3, 4):
        raise ValueError(f"dim must be 3 or 4, got {batch.dim}")
    n_atoms = np.asarray(batch.mol_n_atoms, dtype=np.int64)
    if len(n_atoms) and (n_atoms.min() < 1 or n_atoms.max() > 1024):
        raise ValueError("molecules must have 1..1024 atoms")
    base = np.zeros(len(n_atoms), dtype=np.int64)
    if len(n_atoms):
        base[1:] = np.cumsum(n_atoms)[:-1]
    rows = int(n_atoms.sum())

    ds = np.asarray(batch.dist_term_starts, dtype=np.int64)
    dm = _term_mol(ds)
    i1 = np.asarray(batch.dist_idx1, dtype=np.int64)
    i2 = np.asarray(batch.dist_idx2, dtype=np.int64)
    if len(i1) and (min(i1.min(), i2.min()) < 0 or np.any(i1 >= n_atoms[dm]) or np.any(i2 >= n_atoms[dm])):
        raise ValueError("distance term atom index out of range for its molecule")
    lb2 = np.asarray(batch.dist_lb2, dtype=np.float32)
    ub2 = np.asarray(batch.dist_ub2, dtype=np.float32)
    w = np.asarray(batch.dist_weight, dtype=np.float32)
    dist_rec = np.empty((len(i1), 4), dtype=np.float32)
    dist_rec[:, 0] = (i1 | (i2 << 16)).astype(np.int32).view(np.float32)
    dist_rec[:, 1], dist_rec[:, 2], dist_rec[:, 3] = lb2, ub2, w
    # every distance term under both of its atoms; a stable sort keeps term order within a row
    row = np.concatenate([base[dm] + i1, base[dm] + i2])
    other = np.concatenate([i2, i1])
    order = np.argsort(row, kind="stable")
    dinc_rec = np.empty((len(row), 4), dtype=np.float32)
    dinc_rec[:, 0] = other[order].astype(np.int32).view(np.float32)
    dinc_rec[:, 1] = np.concatenate([lb2, lb2])[order]
    dinc_rec[:, 2] = np.concatenate([ub2, ub2])[order]
    dinc_rec[:, 3] = np.concatenate([w, w])[order]
    dinc_starts = _starts(np.bincount(row, minlength=rows)[:rows])

    cs = np.asarray(batch.chiral_term_starts, dtype=np.int64)
    cm = _term_mol(cs)
    quads = np.stack([np.asarray(getattr(batch, f"chiral_idx{k}"), dtype=np.int64) for k in (1, 2, 3, 4)], axis=1) \
        if len(cm) else np.zeros((0, 4), np.int64)
    if len(quads) and (quads.min() < 0 or np.any(quads >= n_atoms[cm][:, None])):
        raise ValueError("chiral term atom index out of range for its molecule")
    chiral_bounds = np.stack([np.asarray(batch.chiral_vol_lower, np.float32),
                              np.asarray(batch.chiral_vol_upper, np.float32)], axis=1) \
        if len(cm) else np.zeros((0, 2), np.float32)
    crow = (base[cm][:, None] + quads).reshape(-1)
    cterm = np.repeat(np.arange(len(quads), dtype=np.int64), 4)
    crole = np.tile(np.arange(4, dtype=np.int64), len(quads))
    corder = np.argsort(crow, kind="stable")
    cinc_rec = np.stack([cterm[corder], crole[corder]], axis=1).astype(np.int32) if len(crow) \
        else np.zeros((0, 2), np.int32)
    cinc_starts = _starts(np.bincount(crow, minlength=rows)[:rows])

    fs = np.asarray(batch.fourth_term_starts, dtype=np.int64)
    fm = _term_mol(fs)
    fi = np.asarray(batch.fourth_idx, dtype=np.int64)
    if len(fi) and (fi.min() < 0 or np.any(fi >= n_atoms[fm])):
        raise ValueError("fourth-dimension atom index out of range for its molecule")
    fourth_count = np.bincount(base[fm] + fi, minlength=rows)[:rows].astype(np.int32)

    conf_to_mol = np.asarray(batch.conf_to_mol, dtype=np.int32)
    conf_order = np.argsort(-n_atoms[conf_to_mol], kind="stable").astype(np.int32) if len(conf_to_mol) \
        else np.zeros(0, np.int32)
    return dict(
        conf_to_mol=conf_to_mol, conf_atom_starts=np.asarray(batch.conf_atom_starts, dtype=np.int32),
        conf_order=conf_order, mol_n_atoms=n_atoms.astype(np.int32), mol_atom_base=base.astype(np.int32),
        dist_starts=ds.astype(np.int32), dist_rec=dist_rec, dinc_starts=dinc_starts, dinc_rec=dinc_rec,
        chiral_starts=cs.astype(np.int32), chiral_quads=quads.astype(np.int32),
        chiral_bounds=chiral_bounds.astype(np.float32), cinc_starts=cinc_starts, cinc_rec=cinc_rec,
        fourth_count=fourth_count, max_atoms=int(n_atoms.max()) if len(n_atoms) else 1,
    )


def add_etk_to_batch(batch: SharedConstraintBatch, etk_params_list: List[ETKParams]) -> None:
    """Set the batch's etk_* fields from one ETKParams per molecule (in place)."""
    if len(etk_params_list) != batch.n_mols:
        raise ValueError("one ETKParams per molecule is required")
    P = etk_params_list

    def rows(name, width, dtype):
        parts = [np.asarray(getattr(p, name)).reshape(-1, width) for p in P if len(getattr(p, name))]
        return np.concatenate(parts).astype(dtype) if parts else np.zeros((0, width), dtype)

    batch.etk_torsion_idx = rows("torsion_idx", 4, np.int32)
    batch.etk_torsion_V = rows("torsion_V", 6, np.float32)
    batch.etk_torsion_signs = rows("torsion_signs", 6, np.float32)
    batch.etk_torsion_term_starts = _starts([len(p.torsion_idx) for p in P])
    batch.etk_improper_idx = rows("improper_idx", 4, np.int32)
    batch.etk_improper_weight = _cat([p.improper_weight for p in P], np.float32)
    batch.etk_improper_term_starts = _starts([len(p.improper_idx) for p in P])
    for tag in ("12", "13", "14"):
        setattr(batch, f"etk_dist{tag}_idx1", _cat([getattr(p, f"dist{tag}_idx1") for p in P], np.int32))
        setattr(batch, f"etk_dist{tag}_idx2", _cat([getattr(p, f"dist{tag}_idx2") for p in P], np.int32))
        for f in ("lb", "ub", "weight"):
            setattr(batch, f"etk_dist{tag}_{f}", _cat([getattr(p, f"dist{tag}_{f}") for p in P], np.float32))
        setattr(batch, f"etk_dist{tag}_term_starts", _starts([len(getattr(p, f"dist{tag}_idx1")) for p in P]))


def _conf_arrays(batch: SharedConstraintBatch, n_atoms: np.ndarray, base: np.ndarray) -> dict:
    conf_to_mol = np.asarray(batch.conf_to_mol, dtype=np.int32)
    conf_order = np.argsort(-n_atoms[conf_to_mol], kind="stable").astype(np.int32) if len(conf_to_mol) \
        else np.zeros(0, np.int32)
    return dict(conf_to_mol=conf_to_mol, conf_atom_starts=np.asarray(batch.conf_atom_starts, dtype=np.int32),
                conf_order=conf_order, mol_n_atoms=n_atoms.astype(np.int32), mol_atom_base=base.astype(np.int32),
                max_atoms=int(n_atoms.max()) if len(n_atoms) else 1)


def _atoms_and_base(batch):
    n_atoms = np.asarray(batch.mol_n_atoms, dtype=np.int64)
    if len(n_atoms) and (n_atoms.min() < 1 or n_atoms.max() > 1024):
        raise ValueError("molecules must have 1..1024 atoms")
    base = np.zeros(len(n_atoms), dtype=np.int64)
    if len(n_atoms):
        base[1:] = np.cumsum(n_atoms)[:-1]
    return n_atoms, base, int(n_atoms.sum())


def _pair_tables(starts, i1, i2, a, b, w, n_atoms, base, rows, what):
    """16-byte pair records {i | j << 16, a, b, w} and their per-atom incidence rows."""
    starts = np.asarray(starts, dtype=np.int64)
    tm = _term_mol(starts)
    i1 = np.asarray(i1, dtype=np.int64)
    i2 = np.asarray(i2, dtype=np.int64)
    if len(i1) and (min(i1.min(), i2.min()) < 0 or np.any(i1 >= n_atoms[tm]) or np.any(i2 >= n_atoms[tm])):
        raise ValueError(f"{what} term atom index out of range for its molecule")
    rec = np.empty((len(i1), 4), dtype=np.float32)
    rec[:, 0] = (i1 | (i2 << 16)).astype(np.int32).view(np.float32)
    rec[:, 1], rec[:, 2], rec[:, 3] = a, b, w
    row = np.concatenate([base[tm] + i1, base[tm] + i2])
    order = np.argsort(row, kind="stable")
    inc = np.empty((len(row), 4), dtype=np.float32)
    inc[:, 0] = np.concatenate([i2, i1])[order].astype(np.int32).view(np.float32)
    for k, v in ((1, a), (2, b), (3, w)):
        inc[:, k] = np.concatenate([v, v])[order]
    return rec, _starts(np.bincount(row, minlength=rows)[:rows]), inc


def _quad_incidence(starts, quads, n_atoms, base, rows, what):
    tm = _term_mol(np.asarray(starts, dtype=np.int64))
    quads = np.asarray(quads, dtype=np.int64).reshape(-1, 4)
    if len(quads) and (quads.min() < 0 or np.any(quads >= n_atoms[tm][:, None])):
        raise ValueError(f"{what} term atom index out of range for its molecule")
    crow = (base[tm][:, None] + quads).reshape(-1)
    cterm = np.repeat(np.arange(len(quads), dtype=np.int64), 4)
    crole = np.tile(np.arange(4, dtype=np.int64), len(quads))
    order = np.argsort(crow, kind="stable")
    inc = np.stack([cterm[order], crole[order]], axis=1).astype(np.int32) if len(crow) else np.zeros((0, 2), np.int32)
    return inc, _starts(np.bincount(crow, minlength=rows)[:rows])


def etk_device_arrays(batch: SharedConstraintBatch) -> dict:
    """The ETK terms in the device layout of include/mmffb200_dg.h (MMFFETKTermsDev), validated.

    Per molecule the flat-bottom list is its 1-2, then 1-3, then 1-4 terms; the Fourier list is
    its torsions, then its impropers as Fourier terms (V1 = w, s1 = -1, etk_metal.py:105-124)."""
    if batch.dim != 3:
        raise ValueError("the ETK stage is 3-D")
    if batch.etk_torsion_term_starts is None:
        raise ValueError("the batch has no ETK terms (add_etk_to_batch)")
    n_atoms, base, rows = _atoms_and_base(batch)
    M = int(batch.n_mols)
    fb_parts = []
    for m in range(M):
        for tag in ("12", "13", "14"):
            st = np.asarray(getattr(batch, f"etk_dist{tag}_term_starts"))
            sl = slice(int(st[m]), int(st[m + 1]))
            fb_parts.append([np.asarray(getattr(batch, f"etk_dist{tag}_{f}"))[sl]
                             for f in ("idx1", "idx2", "lb", "ub", "weight")])
    fb = [np.concatenate([p[k] for p in fb_parts]) if fb_parts else np.zeros(0) for k in range(5)]
    fb_counts = [sum(int(np.diff(np.asarray(getattr(batch, f"etk_dist{tag}_term_starts")))[m])
                     for tag in ("12", "13", "14")) for m in range(M)]
    fb_starts = _starts(fb_counts)
    fb_rec, fbinc_starts, fbinc_rec = _pair_tables(fb_starts, fb[0], fb[1], np.asarray(fb[2], np.float32),
                                                   np.asarray(fb[3], np.float32), np.asarray(fb[4], np.float32),
                                                   n_atoms, base, rows, "flat-bottom")
    ts, isx = np.asarray(batch.etk_torsion_term_starts), np.asarray(batch.etk_improper_term_starts)
    tq = np.asarray(batch.etk_torsion_idx).reshape(-1, 4)
    tV = np.asarray(batch.etk_torsion_V, np.float32).reshape(-1, 6)
    tS = np.asarray(batch.etk_torsion_signs, np.float32).reshape(-1, 6)
    iq = np.asarray(batch.etk_improper_idx).reshape(-1, 4)
    iw = np.asarray(batch.etk_improper_weight, np.float32)
    quads, coef, counts = [], [], []
    for m in range(M):
        t0, t1, i0, i1 = int(ts[m]), int(ts[m + 1]), int(isx[m]), int(isx[m + 1])
        quads += [tq[t0:t1], iq[i0:i1]]
        imp = np.zeros((i1 - i0, 12), np.float32)
        imp[:, 1] = iw[i0:i1]
        imp[:, 7] = -1.0
        coef += [np.concatenate([tV[t0:t1], tS[t0:t1]], axis=1), imp]
        counts.append((t1 - t0) + (i1 - i0))
    tor_quads = np.concatenate(quads).astype(np.int32) if quads else np.zeros((0, 4), np.int32)
    tor_coef = np.concatenate(coef).astype(np.float32) if coef else np.zeros((0, 12), np.float32)
    tor_starts = _starts(counts)
    tinc_rec, tinc_starts = _quad_incidence(tor_starts, tor_quads, n_atoms, base, rows, "torsion")
    out = _conf_arrays(batch, n_atoms, base)
    out.update(fb_starts=fb_starts, fb_rec=fb_rec, fbinc_starts=fbinc_starts, fbinc_rec=fbinc_rec,
               tor_starts=tor_starts, tor_quads=tor_quads, tor_coef=tor_coef, tinc_starts=tinc_starts,
               tinc_rec=tinc_rec, max_tor=int(max(counts)) if counts else 0)
    return out
