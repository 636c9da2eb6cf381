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

import os

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


def _stable_order(row: np.ndarray) -> np.ndarray:
    """The stable sorting permutation of ``row`` (non-negative int64): an unstable sort of the
    unique keys row * len + position, which is the same permutation and faster."""
    n = len(row)
    if n == 0 or int(row.max()) >= (1 << 62) // n:
        return np.argsort(row, kind="stable")
    return np.argsort(row * n + np.arange(n, dtype=np.int64))


def _incidence_rows(rec: np.ndarray, i1: np.ndarray, i2: np.ndarray, row: np.ndarray):
    """Each 16-byte pair record under both of its atoms, in ``row`` order (term order within a
    row), its first word replaced by the other atom's index; and the permutation used (incidence
    row p holds record order[p] mod len(rec))."""
    m = len(rec)
    both = np.concatenate([rec, rec])
    both[:m, 0] = i2.astype(np.int32).view(np.float32)
    both[m:, 0] = i1.astype(np.int32).view(np.float32)
    order = _stable_order(row)
    return both[order], order


def _dg_view(batch: SharedConstraintBatch, m0: int, m1: int) -> dict:
    """The DG term arrays of molecules [m0, m1), starts relative to molecule m0."""
    v = {"n_atoms": np.asarray(batch.mol_n_atoms, dtype=np.int64)[m0:m1]}

    def part(starts_name, names):
        st = np.asarray(getattr(batch, starts_name), dtype=np.int64)
        a, b = int(st[m0]), int(st[m1])
        return st[m0:m1 + 1] - a, [np.asarray(getattr(batch, nm))[a:b] for nm in names]

    v["ds"], v["dist"] = part("dist_term_starts", ("dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2", "dist_weight"))
    v["cs"], v["chiral"] = part("chiral_term_starts", ("chiral_idx1", "chiral_idx2", "chiral_idx3", "chiral_idx4",
                                                       "chiral_vol_lower", "chiral_vol_upper"))
    v["fs"], (v["fi"],) = part("fourth_term_starts", ("fourth_idx",))
    return v


def _dg_tables(v: dict) -> dict:
    """The DG device tables of one run of molecules (``_dg_view``), rows and terms counted from
    the run's first molecule."""
    n_atoms = v["n_atoms"]
    base = np.zeros(len(n_atoms), dtype=np.int64)
    if len(n_atoms):
        base[1:] = np.cumsum(n_atoms)[:-1]
    rows = int(n_atoms.sum())

    ds = v["ds"]
    dm = _term_mol(ds)
    i1 = np.asarray(v["dist"][0], dtype=np.int64)
    i2 = np.asarray(v["dist"][1], dtype=np.int64)
    if len(i1) and (min(i1.min(), i2.min()) < 0 or np.any(i1 >= n_atoms[dm]) or np.any(i2 >= n_atoms[dm])):
        raise ValueError("distance term atom index out of range for its molecule")
    dist_rec = np.empty((len(i1), 4), dtype=np.float32)
    dist_rec[:, 0] = (i1 | (i2 << 16)).astype(np.int32).view(np.float32)
    for k in (1, 2, 3):
        dist_rec[:, k] = np.asarray(v["dist"][k + 1], dtype=np.float32)
    # every distance term under both of its atoms, term order kept within a row
    row = np.concatenate([base[dm] + i1, base[dm] + i2])
    dinc_rec, _ = _incidence_rows(dist_rec, i1, i2, row)
    dinc_starts = _starts(np.bincount(row, minlength=rows)[:rows])

    cs = v["cs"]
    cm = _term_mol(cs)
    quads = np.stack([np.asarray(v["chiral"][k], dtype=np.int64) for k in range(4)], axis=1) \
        if len(cm) else np.zeros((0, 4), np.int64)
    if len(quads) and (quads.min() < 0 or np.any(quads >= n_atoms[cm][:, None])):
        raise ValueError("chiral term atom index out of range for its molecule")
    chiral_bounds = np.stack([np.asarray(v["chiral"][4], np.float32), np.asarray(v["chiral"][5], np.float32)],
                             axis=1) if len(cm) else np.zeros((0, 2), np.float32)
    crow = (base[cm][:, None] + quads).reshape(-1)
    cterm = np.repeat(np.arange(len(quads), dtype=np.int64), 4)
    crole = np.tile(np.arange(4, dtype=np.int64), len(quads))
    corder = _stable_order(crow)
    cinc_rec = np.stack([cterm[corder], crole[corder]], axis=1).astype(np.int32) if len(crow) \
        else np.zeros((0, 2), np.int32)
    cinc_starts = _starts(np.bincount(crow, minlength=rows)[:rows])

    fm = _term_mol(v["fs"])
    fi = np.asarray(v["fi"], dtype=np.int64)
    if len(fi) and (fi.min() < 0 or np.any(fi >= n_atoms[fm])):
        raise ValueError("fourth-dimension atom index out of range for its molecule")
    fourth_count = np.bincount(base[fm] + fi, minlength=rows)[:rows].astype(np.int32)
    return dict(dist_starts=ds.astype(np.int32), dist_rec=dist_rec, dinc_starts=dinc_starts, dinc_rec=dinc_rec,
                chiral_starts=cs.astype(np.int32), chiral_quads=quads.astype(np.int32),
                chiral_bounds=chiral_bounds.astype(np.float32), cinc_starts=cinc_starts, cinc_rec=cinc_rec,
                fourth_count=fourth_count)


def _runs_by_terms(per_mol: np.ndarray, parts: int):
    """Contiguous runs of molecules with about equal numbers of terms (``per_mol`` per molecule)."""
    M = len(per_mol)
    cuts = np.searchsorted(np.cumsum(per_mol), np.arange(1, parts) * (per_mol.sum() / parts), side="right")
    bounds = np.unique(np.concatenate([[0], np.clip(cuts, 1, M - 1), [M]])) if M > 1 else np.array([0, M])
    return [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:])]


def _map_runs(fn, runs):
    """``fn`` over the runs, on host threads when there is more than one (numpy releases the
    interpreter lock in the large sorts and gathers)."""
    if len(runs) == 1:
        return [fn(runs[0])]
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(runs)) as ex:
        return list(ex.map(fn, runs))


def _default_workers(n_terms: int) -> int:
    return min(16, os.cpu_count() or 1, max(1, n_terms // 65536))


def dg_device_arrays(batch: SharedConstraintBatch, workers: Optional[int] = None) -> dict:
    """The device layout of include/mmffb200_dg.h as numpy arrays (validated).  Large batches
    are built as runs of molecules on host threads (``workers``, default up to 16) and merged;
    the result does not depend on the split."""
    if batch.dim not in (3, 4):
        raise ValueError(f"dim must be 3 or 4, got {batch.dim}")
    n_atoms, base, _ = _atoms_and_base(batch)
    M = len(n_atoms)
    ds = np.asarray(batch.dist_term_starts, dtype=np.int64)
    w = _default_workers(int(ds[-1])) if workers is None else int(workers)
    runs = _runs_by_terms(np.diff(ds), max(1, min(w, M))) if M else [(0, 0)]
    parts = _map_runs(lambda r: _dg_tables(_dg_view(batch, *r)), runs)
    if len(parts) == 1:
        out = parts[0]
    else:
        cat = lambda k: np.concatenate([p[k] for p in parts])
        counts = lambda k: np.concatenate([np.diff(p[k]) for p in parts])
        chiral_starts = _starts(counts("chiral_starts"))
        cinc = []
        for p, (m0, _) in zip(parts, runs):
            c = p["cinc_rec"].copy()
            c[:, 0] += chiral_starts[m0]
            cinc.append(c)
        out = dict(dist_starts=_starts(counts("dist_starts")), dist_rec=cat("dist_rec"),
                   dinc_starts=_starts(counts("dinc_starts")), dinc_rec=cat("dinc_rec"),
                   chiral_starts=chiral_starts, chiral_quads=cat("chiral_quads"),
                   chiral_bounds=cat("chiral_bounds"), cinc_starts=_starts(counts("cinc_starts")),
                   cinc_rec=np.concatenate(cinc), fourth_count=cat("fourth_count"))
    out.update(_conf_arrays(batch, n_atoms, base))
    return out


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
    """16-byte pair records {i | j << 16, a, b, w}, their per-atom incidence rows, and the
    incidence permutation (``_incidence_rows``)."""
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
    inc, order = _incidence_rows(rec, i1, i2, row)
    return rec, _starts(np.bincount(row, minlength=rows)[:rows]), inc, order


def _quad_incidence(starts, quads, n_atoms, base, rows, what):
    tm = _term_mol(np.asarray(starts, dtype=np.int64))
    quads = np.asarray(quads, dtype=np.int64).reshape(-1, 4)
    if len(quads) and (quads.min() < 0 or np.any(quads >= n_atoms[tm][:, None])):
        raise ValueError(f"{what} term atom index out of range for its molecule")
    crow = (base[tm][:, None] + quads).reshape(-1)
    cterm = np.repeat(np.arange(len(quads), dtype=np.int64), 4)
    crole = np.tile(np.arange(4, dtype=np.int64), len(quads))
    order = _stable_order(crow)
    inc = np.stack([cterm[order], crole[order]], axis=1).astype(np.int32) if len(crow) else np.zeros((0, 2), np.int32)
    return inc, _starts(np.bincount(crow, minlength=rows)[:rows])


_FB_FAMILIES = ("12", "13", "14")


def _etk_view(batch: SharedConstraintBatch, m0: int, m1: int) -> dict:
    """The ETK term arrays of molecules [m0, m1), starts relative to molecule m0."""
    v = {"n_atoms": np.asarray(batch.mol_n_atoms, dtype=np.int64)[m0:m1]}

    def part(starts_name, arrays):
        st = np.asarray(getattr(batch, starts_name), dtype=np.int64)
        a, b = int(st[m0]), int(st[m1])
        return st[m0:m1 + 1] - a, [x[a:b] for x in arrays]

    for t in _FB_FAMILIES:
        names = [f"etk_dist{t}_{f}" for f in ("idx1", "idx2", "lb", "ub", "weight")]
        v[f"st{t}"], v[f"d{t}"] = part(f"etk_dist{t}_term_starts", [np.asarray(getattr(batch, n)) for n in names])
    v["st_tor"], (v["tq"], v["tV"], v["tS"]) = part(
        "etk_torsion_term_starts", [np.asarray(batch.etk_torsion_idx).reshape(-1, 4),
                                    np.asarray(batch.etk_torsion_V, np.float32).reshape(-1, 6),
                                    np.asarray(batch.etk_torsion_signs, np.float32).reshape(-1, 6)])
    v["st_imp"], (v["iq"], v["iw"]) = part(
        "etk_improper_term_starts", [np.asarray(batch.etk_improper_idx).reshape(-1, 4),
                                     np.asarray(batch.etk_improper_weight, np.float32)])
    return v


def _etk_tables(v: dict) -> dict:
    """The device tables of one run of molecules (``_etk_view``), rows and terms counted from
    the run's first molecule."""
    n_atoms = v["n_atoms"]
    base = np.zeros(len(n_atoms), dtype=np.int64)
    if len(n_atoms):
        base[1:] = np.cumsum(n_atoms)[:-1]
    rows = int(n_atoms.sum())
    M = len(n_atoms)

    def interleave(starts_list):
        """Concatenate per-family term arrays molecule by molecule (family order kept within a
        molecule): the permutation of the family-major concatenation, and per-molecule counts."""
        mol = np.concatenate([_term_mol(st) for st in starts_list])
        fam = np.concatenate([np.full(int(st[-1]), k) for k, st in enumerate(starts_list)])
        order = np.lexsort((np.arange(len(mol)), fam, mol))
        counts = np.bincount(mol, minlength=M)[:M] if len(mol) else np.zeros(M, np.int64)
        return order, counts

    order, fb_counts = interleave([v[f"st{t}"] for t in _FB_FAMILIES])

    def cat(k, dtype):
        return np.concatenate([np.asarray(v[f"d{t}"][k], dtype=dtype) for t in _FB_FAMILIES])[order]

    fb_starts = _starts(fb_counts)
    fb_rec, fbinc_starts, fbinc_rec, inc_order = _pair_tables(
        fb_starts, cat(0, np.int64), cat(1, np.int64), cat(2, np.float32), cat(3, np.float32),
        cat(4, np.float32), n_atoms, base, rows, "flat-bottom")
    imp = np.zeros((len(v["iq"]), 12), np.float32)
    imp[:, 1] = v["iw"]
    imp[:, 7] = -1.0
    torder, counts = interleave([v["st_tor"], v["st_imp"]])
    tor_quads = np.concatenate([v["tq"], v["iq"]]).astype(np.int32)[torder].reshape(-1, 4)
    tor_coef = np.concatenate([np.concatenate([v["tV"], v["tS"]], axis=1), imp]).astype(np.float32)[torder]
    tor_starts = _starts(counts)
    tinc_rec, tinc_starts = _quad_incidence(tor_starts, tor_quads, n_atoms, base, rows, "torsion")
    # where each flat-bottom term sits, for patching its bounds in place (fb_bounds_patch):
    # fb_row[t] is the record of term t of the 12 | 13 | 14 concatenation, and fbinc_pos[r] and
    # fbinc_pos[r + len(fb_rec)] are record r's two incidence rows
    fb_row = np.empty(len(order), np.int64)
    fb_row[order] = np.arange(len(order), dtype=np.int64)
    fbinc_pos = np.empty(len(inc_order), np.int64)
    fbinc_pos[inc_order] = np.arange(len(inc_order), dtype=np.int64)
    return dict(fb_starts=fb_starts, fb_rec=fb_rec, fbinc_starts=fbinc_starts, fbinc_rec=fbinc_rec,
                tor_starts=tor_starts, tor_quads=tor_quads, tor_coef=tor_coef.reshape(-1, 12),
                tinc_starts=tinc_starts, tinc_rec=tinc_rec, max_tor=int(counts.max()) if len(counts) else 0,
                fb_row=fb_row, fbinc_pos=fbinc_pos,
                fam_sizes=[int(v[f"st{t}"][-1]) for t in _FB_FAMILIES])


def _etk_runs(batch: SharedConstraintBatch, parts: int):
    """Contiguous runs of molecules with about equal numbers of flat-bottom terms."""
    return _runs_by_terms(sum(np.diff(np.asarray(getattr(batch, f"etk_dist{t}_term_starts"), dtype=np.int64))
                              for t in _FB_FAMILIES), parts)


def _merge_etk(parts, runs, batch) -> dict:
    """One batch's tables from its runs' tables: records concatenate, starts re-accumulate, and
    the term and record indices the runs counted locally move to the batch's numbering."""
    cat = lambda k: np.concatenate([p[k] for p in parts])
    counts = lambda k: np.concatenate([np.diff(p[k]) for p in parts])
    fb_starts, tor_starts = _starts(counts("fb_starts")), _starts(counts("tor_starts"))
    tinc = []
    for p, (m0, _) in zip(parts, runs):
        t = p["tinc_rec"].copy()
        t[:, 0] += tor_starts[m0]
        tinc.append(t)
    total = sum(len(p["fb_row"]) for p in parts)
    fb_row = np.empty(total, np.int64)
    fbinc_pos = np.empty(2 * total, np.int64)
    fam_off = np.concatenate([[0], np.cumsum([int(np.asarray(getattr(batch, f"etk_dist{t}_term_starts"))[-1])
                                              for t in _FB_FAMILIES])])
    for p, (m0, _) in zip(parts, runs):
        rec0, mc = int(fb_starts[m0]), len(p["fb_rec"])
        local = 0
        for f, t in enumerate(_FB_FAMILIES):
            g0 = int(fam_off[f]) + int(np.asarray(getattr(batch, f"etk_dist{t}_term_starts"))[m0])
            n = p["fam_sizes"][f]
            fb_row[g0:g0 + n] = p["fb_row"][local:local + n] + rec0
            local += n
        fbinc_pos[rec0:rec0 + mc] = p["fbinc_pos"][:mc] + 2 * rec0
        fbinc_pos[total + rec0:total + rec0 + mc] = p["fbinc_pos"][mc:] + 2 * rec0
    return dict(fb_starts=fb_starts, fb_rec=cat("fb_rec"), fbinc_starts=_starts(counts("fbinc_starts")),
                fbinc_rec=cat("fbinc_rec"), tor_starts=tor_starts, tor_quads=cat("tor_quads"),
                tor_coef=cat("tor_coef"), tinc_starts=_starts(counts("tinc_starts")),
                tinc_rec=np.concatenate(tinc) if tinc else np.zeros((0, 2), np.int32),
                max_tor=max(p["max_tor"] for p in parts), fb_row=fb_row, fbinc_pos=fbinc_pos)


def etk_device_arrays(batch: SharedConstraintBatch, workers: Optional[int] = None) -> dict:
    """The ETK terms in the device layout of include/mmffb200_dg.h (MMFFETKTermsDev), validated.

    Per molecule the flat-bottom list is its 1-2, then 1-3, then 1-4 terms; the Fourier list is
    its torsions, then its impropers as Fourier terms (V1 = w, s1 = -1, etk_metal.py:105-124).
    Large batches are built as runs of molecules on host threads (``workers``, default up to 16)
    and merged; the result does not depend on the split."""
    if batch.dim != 3:
        raise ValueError("the ETK stage is 3-D")
    if batch.etk_torsion_term_starts is None:
        raise ValueError("the batch has no ETK terms (add_etk_to_batch)")
    n_atoms, base, _ = _atoms_and_base(batch)
    M = int(batch.n_mols)
    n_fb = sum(int(np.asarray(getattr(batch, f"etk_dist{t}_term_starts"))[-1]) for t in _FB_FAMILIES)
    w = _default_workers(n_fb) if workers is None else int(workers)
    runs = _etk_runs(batch, max(1, min(w, M))) if M else [(0, 0)]
    parts = _map_runs(lambda r: _etk_tables(_etk_view(batch, *r)), runs)
    if len(parts) == 1:
        out = parts[0]
        del out["fam_sizes"]
    else:
        out = _merge_etk(parts, runs, batch)
    out.update(_conf_arrays(batch, n_atoms, base))
    return out


def fb_bounds_patch(arrs: dict, batch: SharedConstraintBatch, tags=("12", "13")):
    """The writes that bring ``etk_device_arrays``' flat-bottom tables up to date after the
    bounds of the ``tags`` families changed in the batch (the pipeline's re-centred 1-2 / 1-3
    terms; the term lists themselves unchanged): (record rows, incidence rows, (T, 2) float32
    lb / ub).  Column 1 and 2 of ``fb_rec[rows]`` and of ``fbinc_rec[inc_rows]`` take the values,
    the latter once per atom of a term (values repeated)."""
    fams = ("12", "13", "14")
    if list(tags) != list(fams[:len(tags)]):
        raise ValueError("the patched families must lead the 12 | 13 | 14 order")
    lb = np.concatenate([np.asarray(getattr(batch, f"etk_dist{t}_lb"), np.float32) for t in tags])
    ub = np.concatenate([np.asarray(getattr(batch, f"etk_dist{t}_ub"), np.float32) for t in tags])
    rows = arrs["fb_row"][:len(lb)]
    m = len(arrs["fb_rec"])
    inc_rows = np.concatenate([arrs["fbinc_pos"][rows], arrs["fbinc_pos"][rows + m]])
    return rows, inc_rows, np.stack([lb, ub], axis=1)


def patch_fb_bounds(arrs: dict, batch: SharedConstraintBatch, tags=("12", "13")) -> None:
    """``fb_bounds_patch`` applied to the host tables (in place)."""
    rows, inc_rows, vals = fb_bounds_patch(arrs, batch, tags)
    arrs["fb_rec"][rows, 1:3] = vals
    arrs["fbinc_rec"][inc_rows, 1:3] = np.concatenate([vals, vals])
