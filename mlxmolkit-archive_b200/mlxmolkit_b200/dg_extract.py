"""Distance-geometry (DG) parameters per molecule, and the DG initial embedding.

Mirror of the reference's mlxmolkit/dg_extract.py:
  * ``DGParams`` (:20-53): the same fields;
  * ``extract_dg_params`` (:173-283): the same rules that turn a distance-bounds
    matrix into terms -- every pair i < j with positive bounds whose linear
    spread ub - lb is at most 5 A, weight 1, squared bounds -- plus the fixed
    signed chiral-volume windows ([5, 100], [2, 100] for 3-coordinate centres,
    negated for the other handedness) and one fourth-dimension term per atom;
  * ``metric_matrix_positions`` (:56-103): random distances within the bounds,
    double-centred Gram matrix, top-``dim`` eigenvectors scaled by sqrt(lambda),
    a uniform [-1, 1] column where an eigenvalue is not positive.  The random
    draws are taken in the reference's order (one uniform per upper-triangle
    pair, then the uniform columns), so a seed gives the reference's starts.

RDKit is not available here, so the bounds matrix of RDKit's
``GetMoleculeBoundsMatrix`` (which ``get_bounds_matrix`` wraps, :151-170) and
its chiral tags have no source.  ``synth_bounds_matrix`` and
``synth_chiral_tags`` are a synthetic stand-in for the seeded molecules of
``synth.py``: bounds from the topology and the embedded conformer (tight 1-2
and 1-3, a band for 1-4, van der Waals floors and path-length ceilings
beyond), chirality from the conformer's signed volumes.  They give constraint
sets of the reference's structure and size; they do not reproduce RDKit's
numbers.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

# linear bound spread above which a pair is left out of the DG error function (dg_extract.py:203-207)
BASIN_THRESH = 5.0


@dataclass
class DGParams:
    """Distance-geometry terms of one molecule (dg_extract.py:20-53)."""
    n_atoms: int
    dist_idx1: np.ndarray
    dist_idx2: np.ndarray
    dist_lb2: np.ndarray
    dist_ub2: np.ndarray
    dist_weight: np.ndarray
    chiral_idx1: np.ndarray
    chiral_idx2: np.ndarray
    chiral_idx3: np.ndarray
    chiral_idx4: np.ndarray
    chiral_vol_lower: np.ndarray
    chiral_vol_upper: np.ndarray
    fourth_idx: np.ndarray
    bounds_mat: Optional[np.ndarray] = None


CHI_CW, CHI_CCW, CHI_OTHER = "CW", "CCW", "OTHER"


def extract_dg_params(mol, bounds_mat: np.ndarray, dim: int = 4, basin_size_tol: float = 1e8,
                      chiral_tags: Optional[dict] = None) -> DGParams:
    """DG terms from a bounds matrix (upper bounds above the diagonal, lower bounds below).

    ``chiral_tags`` maps a centre atom to CW / CCW / OTHER; when it is None the
    molecule's own ``chiral_tags`` attribute is used if it has one.
    """
    bm = np.asarray(bounds_mat, dtype=np.float64)
    n = int(mol.GetNumAtoms())
    iu, ju = np.triu_indices(n, 1)
    ub, lb = bm[iu, ju], bm[ju, iu]
    keep = (ub > 0) & (lb > 0) & ~(ub - lb > BASIN_THRESH)
    iu, ju, ub, lb = iu[keep], ju[keep], ub[keep], lb[keep]

    tags = chiral_tags if chiral_tags is not None else getattr(mol, "chiral_tags", None) or {}
    quads, lo, hi = [], [], []
    for center in sorted(tags):
        nb = [a.GetIdx() for a in mol.GetAtomWithIdx(center).GetNeighbors()]
        if len(nb) < 3:
            continue
        if len(nb) == 3:
            q, lo_mag = (nb[0], nb[1], nb[2], center), 2.0
        else:
            q, lo_mag = (nb[0], nb[1], nb[2], nb[3]), 5.0
        tag = tags[center]
        if tag == CHI_CCW:
            lo.append(lo_mag), hi.append(100.0)
        elif tag == CHI_CW:
            lo.append(-100.0), hi.append(-lo_mag)
        else:
            lo.append(-100.0), hi.append(100.0)
        quads.append(q)
    qa = np.array(quads, dtype=np.int32).reshape(-1, 4)
    return DGParams(
        n_atoms=n,
        dist_idx1=iu.astype(np.int32), dist_idx2=ju.astype(np.int32),
        dist_lb2=(lb * lb).astype(np.float32), dist_ub2=(ub * ub).astype(np.float32),
        dist_weight=np.ones(len(iu), dtype=np.float32),
        chiral_idx1=qa[:, 0].copy(), chiral_idx2=qa[:, 1].copy(), chiral_idx3=qa[:, 2].copy(),
        chiral_idx4=qa[:, 3].copy(),
        chiral_vol_lower=np.array(lo, dtype=np.float32), chiral_vol_upper=np.array(hi, dtype=np.float32),
        fourth_idx=np.arange(n, dtype=np.int32),
        bounds_mat=bm.astype(np.float32),
    )


def _metric_embed(bmat: np.ndarray, rng: np.random.Generator, dim: int) -> np.ndarray:
    n = int(bmat.shape[0])
    if n <= 1:
        return np.zeros((n, dim), np.float32)
    iu, ju = np.triu_indices(n, 1)
    upper = bmat[iu, ju].astype(np.float64)
    lower = np.minimum(bmat[ju, iu].astype(np.float64), upper)
    d = lower + rng.random(len(upper)) * (upper - lower)
    d2 = np.zeros((n, n))
    d2[iu, ju] = d2[ju, iu] = d * d
    gram = -0.5 * (d2 - d2.mean(axis=1, keepdims=True) - d2.mean(axis=0, keepdims=True) + d2.mean())
    evals, evecs = np.linalg.eigh(gram)
    top = np.argsort(evals)[::-1][:dim]
    # a non-positive eigenvalue -- or none at all, for fewer atoms than dimensions -- takes a
    # uniform [-1, 1] column
    cols = [evecs[:, top[k]] * np.sqrt(evals[top[k]]) if k < len(top) and evals[top[k]] > 0.0
            else 1.0 - 2.0 * rng.random(n) for k in range(dim)]
    return np.stack(cols, axis=1).astype(np.float32)


def _metric_embed_sequential(batch, bounds_mats, rng, dim, out, first: int) -> None:
    starts = np.asarray(batch.conf_atom_starts)
    for c in range(first, int(batch.n_confs_total)):
        a0, a1 = int(starts[c]), int(starts[c + 1])
        bm = bounds_mats[int(batch.conf_to_mol[c])]
        if bm is None:
            out[a0 * dim:a1 * dim] = rng.standard_normal((a1 - a0) * dim).astype(np.float32)
        else:
            out[a0 * dim:a1 * dim] = _metric_embed(np.asarray(bm), rng, dim).reshape(-1)


def uniform_draws(seed: int, offset: int, count: int) -> np.ndarray:
    """Draws ``offset`` .. ``offset + count`` of ``np.random.default_rng(seed).random``, without
    drawing the ones before (the PCG64 state jumped ahead; one 64-bit step per double)."""
    bg = np.random.PCG64(seed)
    bg.advance(int(offset))
    return np.random.Generator(bg).random(int(count))


def embed_conformers(bmat: np.ndarray, u: np.ndarray, k: int, dim: int):
    """Metric-matrix coordinates of ``k`` conformers of one molecule in one batched ``eigh``,
    from their ``k * n(n-1)/2`` uniform distance draws ``u`` (conformer-major, row-major upper
    triangle).  Returns ((k, n * dim) float32, j): j is the first conformer that needs the extra
    uniform column of a non-positive eigenvalue (k when none does); rows from j on are unset."""
    bm = np.asarray(bmat, dtype=np.float64)
    n = bm.shape[0]
    iu, ju = np.triu_indices(n, 1)
    upper = bm[iu, ju]
    lower = np.minimum(bm[ju, iu], upper)
    d = lower[None, :] + np.asarray(u).reshape(k, -1) * (upper - lower)[None, :]
    d2 = np.zeros((k, n, n))
    d2[:, iu, ju] = d2[:, ju, iu] = d * d
    gram = -0.5 * (d2 - d2.mean(axis=2, keepdims=True) - d2.mean(axis=1, keepdims=True)
                   + d2.mean(axis=(1, 2), keepdims=True))
    evals, evecs = np.linalg.eigh(gram)
    out = np.zeros((k, n * dim), np.float32)
    for j in range(k):
        top = np.argsort(evals[j])[::-1][:dim]
        if len(top) < dim or np.any(evals[j][top] <= 0.0):
            return out, j
        out[j] = (evecs[j][:, top] * np.sqrt(evals[j][top])).astype(np.float32).reshape(-1)
    return out, k


def pair_draw_offsets(n_atoms_per_conf) -> np.ndarray:
    """Start of each conformer's distance draws in the batch's draw sequence (length C + 1)."""
    n = np.asarray(n_atoms_per_conf, dtype=np.int64)
    return np.concatenate([[0], np.cumsum(n * (n - 1) // 2)])


def finish_sequentially(batch, bounds_mats, seed: int, dim: int, out: np.ndarray, first: int) -> None:
    """The reference's sequence from conformer ``first`` on, when that conformer needs an extra
    uniform column: the generator is set to its state before that conformer's draws."""
    offs = pair_draw_offsets(np.diff(np.asarray(batch.conf_atom_starts)))
    rng = np.random.Generator(np.random.PCG64(seed))
    rng.bit_generator.advance(int(offs[first]))
    _metric_embed_sequential(batch, bounds_mats, rng, dim, out, first)


def metric_matrix_positions(batch, bounds_mats, seed: int = 42, dim: int = 4) -> np.ndarray:
    """Metric-matrix initial coordinates of every conformer (flat, atom-major, float32).

    The draws follow the reference's order conformer by conformer.  When every molecule has a
    bounds matrix, the distances of all conformers are drawn at once and each molecule's
    conformers are decomposed in one batched ``eigh``; that equals the sequential result as long
    as no conformer needs the extra uniform column of a non-positive eigenvalue.  From the first
    conformer that does, the rest is redone sequentially from the same generator state."""
    rng = np.random.default_rng(seed)
    starts = np.asarray(batch.conf_atom_starts)
    C = int(batch.n_confs_total)
    out = np.zeros(int(starts[-1]) * dim, np.float32)
    mols = [int(m) for m in np.asarray(batch.conf_to_mol)[:C]]
    if C == 0 or any(bounds_mats[m] is None for m in set(mols)) or \
            any(np.asarray(bounds_mats[m]).shape[0] <= 1 for m in set(mols)):
        _metric_embed_sequential(batch, bounds_mats, rng, dim, out, 0)
        return out
    offs = pair_draw_offsets(np.diff(starts[:C + 1]))
    u = rng.random(int(offs[-1]))
    runs, c = [], 0
    while c < C:                                   # runs of consecutive conformers of one molecule
        e = c
        while e < C and mols[e] == mols[c]:
            e += 1
        runs.append((c, e))
        c = e

    def embed_run(run):
        """Writes the run's coordinates; returns the index of its first conformer that needs the
        extra uniform column (C when none does)."""
        c, e = run
        xyz, j = embed_conformers(bounds_mats[mols[c]], u[offs[c]:offs[e]], e - c, dim)
        out[int(starts[c]) * dim:int(starts[c + j]) * dim] = xyz[:j].reshape(-1)
        return c + j if j < e - c else C

    workers = min(len(runs), os.cpu_count() or 1, 16)
    if workers > 1:
        from concurrent.futures import ThreadPoolExecutor     # eigh releases the interpreter lock
        try:                                                   # one BLAS thread per worker
            from threadpoolctl import threadpool_limits
            limit = threadpool_limits(1)
        except ImportError:
            limit = None
        try:
            with ThreadPoolExecutor(workers) as ex:
                bad = min(ex.map(embed_run, runs))
        finally:
            if limit is not None:
                limit.restore_original_limits()
    else:
        bad = min((embed_run(r) for r in runs), default=C)
    if bad < C:                                    # the reference's sequence from the first extra draw on
        finish_sequentially(batch, bounds_mats, seed, dim, out, bad)
    return out


# van der Waals radii (A) of the generator's elements, for the non-bonded lower bounds
_VDW = {"H": 1.10, "C": 1.70, "N": 1.55, "O": 1.52, "F": 1.47, "S": 1.80, "Cl": 1.75, "Br": 1.85, "P": 1.80}


def synth_bounds_matrix(mol, conf_id: int = 0) -> np.ndarray:
    """Synthetic stand-in for RDKit's bounds matrix of a ``synth`` molecule (see the module doc)."""
    pos = np.asarray(mol.GetConformer(conf_id).GetPositions(), dtype=np.float64)
    n = len(pos)
    dist = np.sqrt(((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1))
    topo = np.asarray(mol.distance_matrix())
    path = np.full((n, n), np.inf)
    np.fill_diagonal(path, 0.0)
    for b in mol.GetBonds():
        i, j = b.GetBeginAtomIdx(), b.GetEndAtomIdx()
        path[i, j] = path[j, i] = dist[i, j]
    # shortest bond-path lengths: Floyd-Warshall (the relaxation path[i,k] + path[k,j] in k order;
    # row and column k do not change in pass k, so in place equals pass by pass, bit for bit)
    from scipy.sparse.csgraph import floyd_warshall
    path = np.asarray(floyd_warshall(path, directed=False))
    rad = np.array([_VDW.get(a.GetSymbol(), 1.7) for a in mol.GetAtoms()])
    lb = np.where(topo == 1, dist - 0.01,
         np.where(topo == 2, dist - 0.04,
         np.where(topo == 3, np.maximum(dist - 0.6, 2.0), 0.7 * (rad[:, None] + rad[None, :]))))
    ub = np.where(topo == 1, dist + 0.01,
         np.where(topo == 2, dist + 0.04,
         np.where(topo == 3, dist + 0.6, np.maximum(path, dist + 0.1))))
    lb = np.minimum(lb, dist)                            # the embedded conformer stays feasible
    bm = np.zeros((n, n))
    iu, ju = np.triu_indices(n, 1)
    bm[iu, ju] = ub[iu, ju]
    bm[ju, iu] = lb[iu, ju]
    return bm


def synth_chiral_tags(mol, conf_id: int = 0) -> dict:
    """Chiral tags for a ``synth`` molecule: 4-coordinate centres with at most one hydrogen,
    handedness from the embedded conformer's signed volume (positive = CCW window)."""
    pos = np.asarray(mol.GetConformer(conf_id).GetPositions(), dtype=np.float64)
    tags = {}
    for a in mol.GetAtoms():
        nb = [x.GetIdx() for x in a.GetNeighbors()]
        if len(nb) != 4 or sum(mol.GetAtomWithIdx(k).GetSymbol() == "H" for k in nb) > 1:
            continue
        v1, v2, v3 = (pos[nb[k]] - pos[nb[3]] for k in range(3))
        vol = float(np.dot(v1, np.cross(v2, v3)))
        if abs(vol) >= 5.0:
            tags[a.GetIdx()] = CHI_CCW if vol > 0 else CHI_CW
    return tags


def synth_dg_params(mol, conf_id: int = 0) -> DGParams:
    """DG terms of a ``synth`` molecule: the stand-in bounds and tags through ``extract_dg_params``."""
    return extract_dg_params(mol, synth_bounds_matrix(mol, conf_id), chiral_tags=synth_chiral_tags(mol, conf_id))
