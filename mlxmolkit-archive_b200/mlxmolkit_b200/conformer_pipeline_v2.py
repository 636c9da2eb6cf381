"""``generate_conformers_nk``: distance geometry, ETK and MMFF on B200.

Signature and result types of mlxmolkit/conformer_pipeline_v2.py:41-56,
357-372, plus one additive keyword, ``embed``.

Embedding (``embed="auto"`` picks per molecule):
* ``"device"`` -- the reference's stages (:172-290) on the GPU, for ``synth``
  molecules: DG terms from the molecule's bounds (``dg_extract.synth_dg_params``,
  the synthetic stand-in for RDKit's bounds matrix), metric-matrix starts (seed
  42), the 4-D DG minimisation with the budget max(300, 300 + 20 * complexity),
  a second pass at twice the budget for the conformers that did not converge
  when some but not all failed (improved results kept), the 4-D -> 3-D collapse
  (200 iterations, weights 1.0 / 0.2), the 1-2 / 1-3 ETK bounds re-centred on the
  3-D distances (:224-258: a molecule's terms take its last conformer's
  distances, as there), then ETK (budget max(150, 150 + 10 * complexity)) unless
  ``variant == "DG"``.  The stereo checks of :197-209 run on the GPU after the
  DG passes (``stereo_checks.run_stereo_checks``); a conformer that fails them
  is reported unconverged;
* ``"host"`` -- RDKit's ETKDG for SMILES input; molecules that carry conformers
  (RDKit ``Mol`` or ``SynthMol``) are taken as given.

MMFF stage (``run_mmff``), on the GPU:

* parameters are extracted once per molecule from its first conformer
  (:299-317);
* iterations default to 200 + 15 * (largest atom count) when
  ``mmff_max_iters`` is 0 (:123-126, :169-170);
* ``mmff_use_lbfgs=None`` picks L-BFGS per size class -- molecules of 150 or
  more atoms run L-BFGS (m = 8), smaller ones dense BFGS -- where the
  reference switched the whole call on its largest molecule (:448-452);
  an explicit True / False applies to every molecule;
* a molecule whose MMFF typing fails keeps its embedded coordinates and is
  reported unconverged, as the reference's chunk fallback does (:312-316).
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import mmff_minimize as mm
from .mmff_params import extract_mmff_params
from .pack import merge_packed


@dataclass
class ConformerResult:
    """Result for one molecule."""
    n_atoms: int
    positions_3d: List[np.ndarray]
    energies: List[float]
    converged: List[bool]


@dataclass
class PipelineResult:
    """Result for the full N x k pipeline."""
    molecules: List[ConformerResult]
    total_conformers: int
    total_time: float
    n_batches: int


def _auto_iters(max_atoms: int, base: int = 200, scale: float = 15.0) -> int:
    """The reference's iteration budgets (conformer_pipeline_v2.py:123-126)."""
    return max(base, int(base + scale * max_atoms))


def _embed(item, k: int, seed: int):
    """(molecule, list of (N,3) float64 conformer coordinates)."""
    if isinstance(item, str):
        from rdkit import Chem
        from rdkit.Chem import AllChem
        mol = Chem.MolFromSmiles(item)
        if mol is None:
            raise ValueError(f"Invalid SMILES: {item}")
        mol = Chem.AddHs(mol)
        params = AllChem.ETKDGv3()
        params.randomSeed = seed
        cids = list(AllChem.EmbedMultipleConfs(mol, k, params))
        return mol, [np.asarray(mol.GetConformer(c).GetPositions(), dtype=np.float64) for c in cids]
    confs = item.GetConformers()
    if not confs:
        raise ValueError("molecule without conformers and no embedder for it")
    xyz = [np.asarray(c.pos if hasattr(c, "pos") else c.GetPositions(), dtype=np.float64) for c in confs]
    return item, xyz[:k] if k else xyz


# Term extraction is independent per molecule and runs in Python: batches of at least
# _POOL_MIN molecules map it over a persistent pool of spawned host processes (spawn, so
# that it is safe after CUDA has been initialised in this process).
_POOL = None
_POOL_MIN = 64


def _pool_for(n_items: int):
    """The process pool when a batch of ``n_items`` molecules uses it, else None."""
    global _POOL
    workers = min(16, os.cpu_count() or 1)
    if n_items < _POOL_MIN or workers < 2:
        return None
    if _POOL is None:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        _POOL = ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn"))
    return _POOL


def _chunk(n_items: int) -> int:
    return max(1, n_items // (4 * min(16, os.cpu_count() or 1)))


def _pmap(fn, items):
    pool = _pool_for(len(items))
    if pool is None:
        return [fn(x) for x in items]
    return list(pool.map(fn, items, chunksize=_chunk(len(items))))


def _pmap_async(fn, items):
    """Queue ``fn`` over ``items`` on the pool now (in-process at the call, for small batches);
    returns a function that waits for and returns the results."""
    pool = _pool_for(len(items))
    if pool is None:
        return lambda: [fn(x) for x in items]
    it = pool.map(fn, items, chunksize=_chunk(len(items)))
    return lambda: list(it)


def _dg_terms(mol):
    from .dg_extract import synth_dg_params
    return synth_dg_params(mol)


_ONE_BLAS_THREAD = None


def _dg_terms_and_starts(item):
    """A molecule's DG terms and the metric-matrix starts of its k conformers, from its slice of
    the batch's draw sequence (``dg_extract.embed_conformers``): (params, (k, n * dim) float32,
    index of the first conformer that needs an extra uniform column, k when none), or
    (params, None, 0) for a molecule the batched form does not cover."""
    global _ONE_BLAS_THREAD
    from .dg_extract import embed_conformers, synth_dg_params, uniform_draws
    if _ONE_BLAS_THREAD is None:                  # the pool's processes share the cores
        try:
            from threadpoolctl import threadpool_limits
            _ONE_BLAS_THREAD = threadpool_limits(1)
        except ImportError:
            _ONE_BLAS_THREAD = False
    mol, k, seed, offset, dim = item
    p = synth_dg_params(mol)
    n = int(p.n_atoms)
    if p.bounds_mat is None or n <= 1 or k == 0:
        return p, None, 0
    xyz, j = embed_conformers(p.bounds_mat, uniform_draws(seed, offset, k * n * (n - 1) // 2), k, dim)
    return p, xyz, j


def _dg_terms_and_positions(mols, ks, seed: int, dim: int = 4):
    """DG terms, the packed batch and its metric-matrix starts (``metric_matrix_positions``'s
    result); on the process pool for large batches, each task one molecule's terms and starts."""
    from .dg_extract import metric_matrix_positions, pair_draw_offsets
    from .shared_batch import pack_shared_dg_batch
    if _pool_for(len(mols)) is None:
        dgp = [_dg_terms(m) for m in mols]
        b4 = pack_shared_dg_batch(dgp, ks, dim=dim)
        return dgp, b4, metric_matrix_positions(b4, [p.bounds_mat for p in dgp], seed=seed, dim=dim)
    first = np.concatenate([[0], np.cumsum(ks)]).astype(np.int64)
    offs = pair_draw_offsets(np.repeat([m.GetNumAtoms() for m in mols], ks))
    res = _pmap(_dg_terms_and_starts, [(m, int(k), seed, int(offs[first[i]]), dim)
                                       for i, (m, k) in enumerate(zip(mols, ks))])
    dgp = [r[0] for r in res]
    b4 = pack_shared_dg_batch(dgp, ks, dim=dim)
    bounds = [p.bounds_mat for p in dgp]
    out = _assemble_starts(res, ks, b4, seed, dim)
    return dgp, b4, out if out is not None else metric_matrix_positions(b4, bounds, seed=seed, dim=dim)


def _assemble_starts(res, ks, b4, seed: int, dim: int):
    """The batch's starts from the per-molecule results of ``_dg_terms_and_starts``, equal to
    ``metric_matrix_positions``; None when a molecule needs that function's sequential form."""
    from .dg_extract import finish_sequentially
    if any(r[1] is None for r, k in zip(res, ks) if k > 0) or \
            not np.array_equal(np.diff(np.asarray(b4.conf_atom_starts)), np.repeat([r[0].n_atoms for r in res], ks)):
        return None
    first = np.concatenate([[0], np.cumsum(ks)]).astype(np.int64)
    starts = np.asarray(b4.conf_atom_starts)
    C = int(b4.n_confs_total)
    out = np.zeros(int(starts[-1]) * dim, np.float32)
    bad = C
    for i, (_, xyz, j) in enumerate(res):
        c0 = int(first[i])
        if xyz is None:
            continue
        out[int(starts[c0]) * dim:int(starts[c0 + j]) * dim] = xyz[:j].reshape(-1)
        if j < xyz.shape[0]:                       # later conformers' draws shift: redo from here
            bad = c0 + j
            break
    if bad < C:
        finish_sequentially(b4, [r[0].bounds_mat for r in res], seed, dim, out, bad)
    return out


def _etk_terms(mol_and_bounds):
    from .etk_extract import synth_etk_params
    mol, bm = mol_and_bounds
    return synth_etk_params(mol, bm)


def _mmff_pack(mol_and_variant):
    """The molecule's packed MMFF tables, typed from its first conformer, or None when typing or
    packing fails.  Only the tables travel back from a pool process: they hold everything the
    minimiser reads, the atom count included."""
    from .pack import pack_molecules
    mol, variant = mol_and_variant
    try:
        p = extract_mmff_params(mol, conf_id=mol.GetConformers()[0].GetId(), mmff_variant=variant)
        return pack_molecules([p])
    except Exception:
        return None


def _recenter_bounds(b3, pos3: np.ndarray) -> None:
    """Re-centre each molecule's 1-2 / 1-3 ETK bounds on the measured 3-D distances, keeping
    their half-widths (conformer_pipeline_v2.py:224-258; the last conformer of a molecule wins)."""
    C = int(b3.n_confs_total)
    conf_mol = np.asarray(b3.conf_to_mol, dtype=np.int64)[:C]
    last = np.full(int(b3.n_mols), -1, np.int64)
    last[conf_mol] = np.arange(C, dtype=np.int64)             # the last write of a molecule wins
    first_atom = np.asarray(b3.conf_atom_starts, dtype=np.int64)[np.maximum(last, 0)]
    X = np.asarray(pos3).reshape(-1, 3).astype(np.float64)
    for tag in ("12", "13"):
        st = np.asarray(getattr(b3, f"etk_dist{tag}_term_starts"), dtype=np.int64)
        tm = np.repeat(np.arange(len(st) - 1, dtype=np.int64), np.diff(st))
        sel = np.nonzero(last[tm] >= 0)[0]                    # molecules with a conformer
        if len(sel) == 0:
            continue
        i1 = np.asarray(getattr(b3, f"etk_dist{tag}_idx1"), dtype=np.int64)[sel]
        i2 = np.asarray(getattr(b3, f"etk_dist{tag}_idx2"), dtype=np.int64)[sel]
        lb, ub = getattr(b3, f"etk_dist{tag}_lb"), getattr(b3, f"etk_dist{tag}_ub")
        a0 = first_atom[tm[sel]]
        d = np.linalg.norm(X[a0 + i1] - X[a0 + i2], axis=1)
        hw = (ub[sel].astype(np.float64) - lb[sel]) / 2.0
        lb[sel] = (d - hw).astype(np.float32)
        ub[sel] = (d + hw).astype(np.float32)


def _embed_on_device(mols, ks, *, dg_max_iters, etk_max_iters, fourth_dim_weight, chiral_weight, variant,
                     seed: int = 42, timings: Optional[dict] = None, after_host=None):
    """DG -> retry -> stereo checks -> collapse -> (ETK) on the GPU, positions resident on the device
    between the stages; returns per molecule a list of (N, 3) conformers, whether each conformer's
    DG and ETK stages converged, its DG + ETK energy (:333-341), and what ``after_host`` -- called
    once the stages' own host work is queued, before the first launch -- returned."""
    import torch
    from .conformer_metal import DGDeviceBatch
    from .etk_metal import ETKDeviceBatch
    from .shared_batch import add_etk_to_batch, pack_shared_dg_batch
    from .stereo_checks import TetrahedralTable, stereo_check_device
    tick = time.perf_counter()

    def lap(name):
        nonlocal tick
        if timings is not None:
            torch.cuda.synchronize()
            now = time.perf_counter()
            timings[name] = timings.get(name, 0.0) + now - tick
            tick = now

    dgp, b4, x4 = _dg_terms_and_positions(list(mols), ks, seed, dim=4)
    if variant != "DG":                          # extracted on the pool while the GPU runs DG
        etk_terms = _pmap_async(_etk_terms, [(m, p.bounds_mat) for m, p in zip(mols, dgp)])
    background = after_host() if after_host is not None else None
    C = b4.n_confs_total
    max_atoms = max(p.n_atoms for p in dgp)
    complexity = max(max_atoms, int(max(len(p.dist_idx1) for p in dgp) ** 0.5))
    dg_iters = dg_max_iters if dg_max_iters > 0 else _auto_iters(complexity, 300, 20.0)
    etk_iters = etk_max_iters if etk_max_iters > 0 else _auto_iters(complexity, 150, 10.0)
    lap("dg_host")
    dev4 = DGDeviceBatch(b4)
    pos4 = torch.from_numpy(x4).cuda()
    e4, s4 = dev4.minimize_device(pos4, dev4.params(dg_iters, 1e-4, chiral_weight, fourth_dim_weight))
    e4, s4 = e4[:C].clone(), s4[:C].clone()
    failed = s4 != 0
    # while the GPU runs DG: the stereo table and the ETK tables, built here and uploaded on a
    # side stream (a copy on this stream would wait for DG); the ETK bounds are patched in once
    # they are re-centred on the 3-D distances
    main, side = torch.cuda.current_stream(), torch.cuda.Stream()
    with torch.cuda.stream(side):
        tet = TetrahedralTable(mols)
        dev3 = None
        if variant != "DG":
            b3 = pack_shared_dg_batch(dgp, ks, dim=3)
            add_etk_to_batch(b3, etk_terms())
            dev3 = ETKDeviceBatch(b3)
    main.wait_stream(side)
    for t in [tet.starts, tet.quads] + (list(dev3.dev.values()) if dev3 is not None else []):
        t.record_stream(main)
    n_failed = int(failed.sum().item())
    if 0 < n_failed < C:                                         # :186-200, warm start from the first pass
        pos2 = pos4.clone()
        e2, s2 = dev4.minimize_device(pos2, dev4.params(2 * dg_iters, 1e-4, chiral_weight, fourth_dim_weight))
        better = failed & ((s2[:C] == 0) | (e2[:C] < e4))
        counts = torch.from_numpy(np.diff(np.asarray(b4.conf_atom_starts)).astype(np.int64) * 4).cuda()
        mask = torch.repeat_interleave(better, counts)
        pos4 = torch.where(mask, pos2, pos4)
        e4 = torch.where(better, e2[:C], e4)
        s4 = torch.where(better, s2[:C], s4)
    passed = stereo_check_device(dev4, tet, pos4)[:C]                     # :197-209
    s4 = torch.where(passed != 0, s4, torch.full_like(s4, 2))
    dev4.minimize_device(pos4, dev4.params(200, 1e-4, 0.2, 1.0))            # collapse, :211-215
    pos3 = pos4.view(-1, 4)[:, :3].contiguous().view(-1)
    lap("dg_gpu")
    e3 = torch.zeros(C, dtype=torch.float32, device="cuda")
    s3 = torch.zeros(C, dtype=torch.int32, device="cuda")
    if variant != "DG":
        _recenter_bounds(b3, pos3.cpu().numpy())
        dev3.refresh_bounds()
        lap("etk_host")
        e3, s3 = dev3.minimize_device(pos3, dev3.params(etk_iters, 1e-4, 0.0, 0.0))
        e3, s3 = e3[:C], s3[:C]
        lap("etk_gpu")
    p3 = pos3.cpu().numpy()
    ok = ((s4 == 0) & (s3 == 0)).cpu().numpy()
    en = (e4.double() + e3.double()).cpu().numpy()
    confs, oks, energy, c = [], [], [], 0
    for m, k in zip(mols, ks):
        n = m.GetNumAtoms()
        confs.append([p3[int(b4.conf_atom_starts[c + j]) * 3:(int(b4.conf_atom_starts[c + j]) + n) * 3]
                      .reshape(n, 3).astype(np.float64) for j in range(k)])
        oks.append([bool(v) for v in ok[c:c + k]])
        energy.append([float(v) for v in en[c:c + k]])
        c += k
    return confs, oks, energy, background


def generate_conformers_nk(
    smiles_list: Sequence,
    n_confs_per_mol=10,
    *,
    max_confs_per_batch: Optional[int] = None,
    max_memory_bytes: Optional[int] = None,
    dg_max_iters: int = 0,
    etk_max_iters: int = 0,
    fourth_dim_weight: float = 0.1,
    chiral_weight: float = 1.0,
    variant: str = "ETKDGv2",
    run_mmff: bool = False,
    mmff_max_iters: int = 0,
    mmff_use_lbfgs: Optional[bool] = None,
    mmff_variant: str = "MMFF94",
    embed: str = "auto",
    timings: Optional[dict] = None,
) -> PipelineResult:
    """N molecules x k conformers: embedding (DG + ETK on the GPU for ``synth`` molecules) and
    MMFF94/94s refinement on the GPU when ``run_mmff``.  ``timings`` (additive), when a dict,
    receives the seconds of the device embedding's host and GPU parts."""
    if embed not in ("auto", "device", "host"):
        raise ValueError("embed must be 'auto', 'device' or 'host'")
    t0 = time.time()
    N = len(smiles_list)
    ks = [n_confs_per_mol] * N if isinstance(n_confs_per_mol, int) else list(n_confs_per_mol)
    on_device = [embed == "device" or (embed == "auto" and hasattr(item, "distance_matrix")) for item in smiles_list]
    if embed == "device" and not all(hasattr(item, "distance_matrix") for item in smiles_list):
        raise ValueError("embed='device' needs synth molecules: their bounds matrices come from the stand-in "
                         "extraction (RDKit's bounds matrix is not available)")
    embedded = [None] * N
    dg_ok = [None] * N
    dg_e = [None] * N
    dev_idx = [i for i in range(N) if on_device[i]]
    # molecules that carry their own conformer are MMFF-typed from it whatever the embedding, so
    # their extraction is queued behind the embedding's host work and runs during its GPU stages
    pre_idx = [i for i in range(N) if not isinstance(smiles_list[i], str)] if run_mmff else []
    pre_packs = None
    if dev_idx:
        def queue_mmff():
            return _pmap_async(_mmff_pack, [(smiles_list[i], mmff_variant) for i in pre_idx]) if pre_idx else None

        confs, ok, en, pre_packs = _embed_on_device(
            [smiles_list[i] for i in dev_idx], [int(ks[i]) for i in dev_idx], dg_max_iters=dg_max_iters,
            etk_max_iters=etk_max_iters, fourth_dim_weight=fourth_dim_weight, chiral_weight=chiral_weight,
            variant=variant, timings=timings, after_host=queue_mmff)
        for j, i in enumerate(dev_idx):
            embedded[i] = (smiles_list[i], confs[j])
            dg_ok[i], dg_e[i] = ok[j], en[j]
    for i in range(N):
        if embedded[i] is None:
            embedded[i] = _embed(smiles_list[i], int(ks[i]), 42 + i)
    results = [ConformerResult(n_atoms=m.GetNumAtoms(), positions_3d=[x.copy() for x in xs],
                               energies=list(dg_e[i]) if dg_e[i] else [0.0] * len(xs),
                               converged=list(dg_ok[i]) if dg_ok[i] else [True] * len(xs))
               for i, (m, xs) in enumerate(embedded)]
    n_batches = 0
    t_mmff = time.perf_counter()
    if run_mmff and N:
        packs = [None] * N
        if pre_packs is not None:
            for i, k in zip(pre_idx, pre_packs()):
                packs[i] = k
        done = set(pre_idx) if pre_packs is not None else set()
        rest = [i for i in range(N) if i not in done]
        for i, k in zip(rest, _pmap(_mmff_pack, [(embedded[i][0], mmff_variant) for i in rest])):
            packs[i] = k
        ok = [k is not None and len(xs) > 0 for k, (_, xs) in zip(packs, embedded)]
        for i, good in enumerate(ok):
            if not good:
                results[i].converged = [False] * len(results[i].positions_3d)
        idx = [i for i, g in enumerate(ok) if g]
        n_at = {i: int(packs[i].n_atoms[0]) for i in idx}
        if idx:
            max_atoms = max(n_at.values())
            iters = mmff_max_iters if mmff_max_iters > 0 else _auto_iters(max_atoms)
            if mmff_use_lbfgs is None:
                groups = [[i for i in idx if n_at[i] < mm.LBFGS_ATOM_THRESHOLD],
                          [i for i in idx if n_at[i] >= mm.LBFGS_ATOM_THRESHOLD]]
                hists = [0, mm.LBFGS_M]
            else:
                groups, hists = [idx], [mm.LBFGS_M if mmff_use_lbfgs else 0]
            for grp, hist in zip(groups, hists):
                if not grp:
                    continue
                n_batches += 1
                m = mm.Minimizer(None, [len(embedded[i][1]) for i in grp], packed=merge_packed([packs[i] for i in grp]))
                pos = np.concatenate([np.stack(embedded[i][1]).reshape(-1) for i in grp]).astype(np.float32)
                r = m.minimize(pos, max_iters=iters, grad_tol=1e-4, history_m=hist)
                cursor = 0
                for i in grp:
                    n = n_at[i]
                    k = len(embedded[i][1])
                    start = int(m.conf_coord[cursor])
                    xyz = r.positions[start: start + 3 * n * k].reshape(k, n, 3).astype(np.float64)
                    results[i].positions_3d = [xyz[c] for c in range(k)]
                    results[i].energies = [float(v) for v in r.energies[cursor: cursor + k]]
                    conv = [bool(v) for v in r.converged[cursor: cursor + k]]
                    if dg_ok[i] is not None:                  # an embedding failure stays a failure
                        conv = [a and b for a, b in zip(conv, dg_ok[i])]
                    results[i].converged = conv
                    cursor += k
    if timings is not None and run_mmff:
        timings["mmff"] = timings.get("mmff", 0.0) + time.perf_counter() - t_mmff
    return PipelineResult(molecules=results, total_conformers=sum(len(r.positions_3d) for r in results),
                          total_time=time.time() - t0, n_batches=max(n_batches, 1))
