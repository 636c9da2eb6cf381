"""Pack MMFF term tables into the device layout of ``include/mmffb200.h``.

Molecule-shared tables: the k conformers of a molecule reference one copy of
its terms through ``conf_mol`` (the reference replicates every table k times,
mlxmolkit/mmff_minimize.py:99-144).

Bonded terms become 16-byte records in chunks of 32 per term type, packed so
that inside a chunk no two terms share an atom in the same role; the kernel
then scatters each role's gradient without atomics.

Non-bonded terms are not stored pair by pair.  The packer checks that the
extracted pair lists (mlxmolkit/mmff_params.py:272-320) are exactly what
per-atom data reproduce --

* every vdW pair's (R*, eps) equals a table entry indexed by the two atoms'
  MMFF types (bit for bit in float32);
* every electrostatic pair's charge term equals float32(q_i * q_j) of the
  float64 partial charges, and every vdW pair absent from the electrostatic
  list has a zero charge product --

and then emits one class x class (R*, eps) table, per-atom class and charge,
and two bit rows per atom (non-bonded pair, 1-4 pair).  Pair tables that
cannot be expressed this way raise ``ValueError``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

MOL_DESC_INTS = 16
(MD_N, MD_ATOM_OFF, MD_NCLS, MD_CLS_OFF, MD_MASK_OFF, MD_DIEL, MD_B_OFF, MD_B_NCH, MD_A_OFF,
 MD_A_NCH, MD_S_OFF, MD_S_NCH, MD_O_OFF, MD_O_NCH, MD_T_OFF, MD_T_NCH) = range(16)
INVALID = np.uint32(0xFFFFFFFF)
MAX_ATOMS = 1024


@dataclass
class PackedBatch:
    mol_desc: np.ndarray      # int32 (M, 16)
    bonded: np.ndarray        # uint32 (R, 4)
    atom_cls: np.ndarray      # int32 (total atoms)
    atom_q: np.ndarray        # float64 (total atoms)
    cls_tab: np.ndarray       # float32 (T, 2)
    pair_mask: np.ndarray     # uint32 (words)
    n_atoms: np.ndarray       # int32 (M,)

    @property
    def n_mols(self) -> int:
        return int(self.mol_desc.shape[0])

    @property
    def max_atoms(self) -> int:
        return int(self.n_atoms.max()) if len(self.n_atoms) else 0

    @property
    def max_classes(self) -> int:
        return int(self.mol_desc[:, MD_NCLS].max()) if len(self.mol_desc) else 1

    def nbytes(self) -> int:
        return sum(a.nbytes for a in (self.mol_desc, self.bonded, self.atom_cls, self.atom_q,
                                      self.cls_tab, self.pair_mask))


def _chunk(role_atoms: np.ndarray, flip_perm=None):
    """Chunk id (and orientation) of every term: the native chunker of libmmffb200.so.

    Same rule and result as ``chunk_reference`` below, which the tests compare it with.
    """
    from . import _lib
    ra = np.ascontiguousarray(role_atoms, dtype=np.int32)
    T, R = ra.shape
    out = np.empty(T, dtype=np.int64)
    flipped = np.zeros(T, dtype=np.uint8)
    fp = None if flip_perm is None else np.ascontiguousarray(flip_perm, dtype=np.int32)
    n_atoms = int(ra.max()) + 1 if T else 1
    rc = _lib.load().mmffb_pack_chunk(T, R, ra.ctypes.data, None if fp is None else fp.ctypes.data, n_atoms,
                                      out.ctypes.data, flipped.ctypes.data)
    if rc < 0:
        raise ValueError(f"mmffb_pack_chunk failed ({rc})")
    return out, flipped.astype(bool)


def chunk_reference(role_atoms: np.ndarray, flip_perm=None):
    """Chunk id (and orientation) of every term (the rule in Python).

    At most 32 terms per chunk and, per role, no atom twice in a chunk.
    role_atoms: (T, R) int.  flip_perm: the role permutation of the term's
    equivalent reversed form (None if it has none); a term that does not fit a
    chunk in its given orientation may enter it reversed.  Greedy first fit in
    term order, one integer bitset of used atoms per role and chunk.
    Returns (chunk ids, reversed flags).
    """
    T, R = role_atoms.shape
    out = np.empty(T, dtype=np.int64)
    flipped = np.zeros(T, dtype=bool)
    fill: list[int] = []
    used: list[list[int]] = []
    first_open = 0
    for t, atoms in enumerate(role_atoms.tolist()):
        forms = [[1 << a for a in atoms]]
        if flip_perm is not None:
            forms.append([1 << atoms[q] for q in flip_perm])
        c = first_open
        nch = len(fill)
        pick = -1
        while c < nch:
            if fill[c] < 32:
                u = used[c]
                for fi, bits in enumerate(forms):
                    ok = True
                    for r in range(R):
                        if u[r] & bits[r]:
                            ok = False
                            break
                    if ok:
                        pick = fi
                        break
                if pick >= 0:
                    break
            c += 1
        if c == nch:
            fill.append(0)
            used.append([0] * R)
            pick = 0
        fill[c] += 1
        u = used[c]
        bits = forms[pick]
        for r in range(R):
            u[r] |= bits[r]
        out[t] = c
        flipped[t] = pick == 1
        while first_open < len(fill) and fill[first_open] >= 32:
            first_open += 1
    return out, flipped


def _place(chunk_ids: np.ndarray, recs: list[np.ndarray]) -> tuple[np.ndarray, int]:
    """Scatter per-term records (one (T,4) uint32 array per 16-byte half) into chunks."""
    T = len(chunk_ids)
    nch = int(chunk_ids.max()) + 1 if T else 0
    h = len(recs)
    out = np.zeros((nch, h, 32, 4), dtype=np.uint32)
    out[:, 0, :, 0] = INVALID
    if T:
        order = np.argsort(chunk_ids, kind="stable")
        starts = np.searchsorted(chunk_ids[order], np.arange(nch))
        slot = np.empty(T, dtype=np.int64)
        slot[order] = np.arange(T) - starts[chunk_ids[order]]
        for q in range(h):
            out[chunk_ids, q, slot] = recs[q]
    return out.reshape(-1, 4), nch


def _f2u(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32)


def _pack16(a, b) -> np.ndarray:
    return (np.asarray(a, dtype=np.uint32) & 0xFFFF) | (np.asarray(b, dtype=np.uint32) << 16)


def _bonded_records(p):
    """(chunked records, chunk count) per term type, in the kernel's order.

    Terms may be stored reversed (bond j-i, angle k-j-i, stretch-bend k-j-i with
    its two sides swapped, out-of-plane with i and k swapped, torsion l-k-j-i):
    each reversed form has the same energy and the same per-atom gradient.
    """
    z = lambda n: np.zeros(n, dtype=np.uint32)
    a32 = lambda a: np.asarray(a, dtype=np.int64)
    out = []

    def sel(flip, a, b):
        return np.where(flip, b, a)

    # bonds
    bi, bj = a32(p.bond_idx1), a32(p.bond_idx2)
    cid, fl = _chunk(np.stack([bi, bj], 1), (1, 0))
    rec = np.stack([_pack16(sel(fl, bi, bj), sel(fl, bj, bi)), _f2u(p.bond_kb), _f2u(p.bond_r0),
                    z(len(bi))], 1)
    out.append(_place(cid, [rec]))
    # angles
    ai, aj, ak = a32(p.angle_idx1), a32(p.angle_idx2), a32(p.angle_idx3)
    cid, fl = _chunk(np.stack([ai, aj, ak], 1), (2, 1, 0))
    lin = (np.asarray(p.angle_is_linear) != 0).astype(np.uint32)
    rec = np.stack([_pack16(sel(fl, ai, ak), aj), _pack16(sel(fl, ak, ai), lin),
                    _f2u(p.angle_ka), _f2u(p.angle_theta0)], 1) if len(ai) else np.zeros((0, 4), np.uint32)
    out.append(_place(cid, [rec]))
    # stretch-bend
    si, sj, sk = a32(p.strbend_idx1), a32(p.strbend_idx2), a32(p.strbend_idx3)
    cid, fl = _chunk(np.stack([si, sj, sk], 1), (2, 1, 0))
    f32 = lambda a: np.asarray(a, dtype=np.float32)
    r0 = np.stack([_pack16(sel(fl, si, sk), sj), sel(fl, sk, si).astype(np.uint32),
                   _f2u(sel(fl, f32(p.strbend_r0_ij), f32(p.strbend_r0_kj))),
                   _f2u(sel(fl, f32(p.strbend_r0_kj), f32(p.strbend_r0_ij)))], 1) \
        if len(si) else np.zeros((0, 4), np.uint32)
    r1 = np.stack([_f2u(p.strbend_theta0),
                   _f2u(sel(fl, f32(p.strbend_kba_ijk), f32(p.strbend_kba_kji))),
                   _f2u(sel(fl, f32(p.strbend_kba_kji), f32(p.strbend_kba_ijk))), z(len(si))], 1) \
        if len(si) else np.zeros((0, 4), np.uint32)
    out.append(_place(cid, [r0, r1]))
    # out-of-plane
    oi, oj, ok_, ol = a32(p.oop_idx1), a32(p.oop_idx2), a32(p.oop_idx3), a32(p.oop_idx4)
    cid, fl = _chunk(np.stack([oi, oj, ok_, ol], 1), (2, 1, 0, 3))
    rec = np.stack([_pack16(sel(fl, oi, ok_), oj), _pack16(sel(fl, ok_, oi), ol),
                    _f2u(p.oop_koop), z(len(oi))], 1) if len(oi) else np.zeros((0, 4), np.uint32)
    out.append(_place(cid, [rec]))
    # torsions
    ti, tj, tk, tl = (a32(p.torsion_idx1), a32(p.torsion_idx2), a32(p.torsion_idx3),
                      a32(p.torsion_idx4))
    cid, fl = _chunk(np.stack([ti, tj, tk, tl], 1), (3, 2, 1, 0))
    r0 = np.stack([_pack16(sel(fl, ti, tl), sel(fl, tj, tk)), _pack16(sel(fl, tk, tj), sel(fl, tl, ti)),
                   _f2u(p.torsion_V1), _f2u(p.torsion_V2)], 1) if len(ti) else np.zeros((0, 4), np.uint32)
    r1 = np.stack([_f2u(p.torsion_V3), z(len(ti)), z(len(ti)), z(len(ti))], 1) \
        if len(ti) else np.zeros((0, 4), np.uint32)
    out.append(_place(cid, [r0, r1]))
    return out


def _nonbonded(p):
    """Verified class table, per-atom class/charge and the two bit-row masks of one molecule."""
    n = int(p.n_atoms)
    if p.atom_type is None or p.partial_charge is None:
        raise ValueError("non-bonded packing needs per-atom MMFF types and partial charges "
                         "(MMFFParams.atom_type / partial_charge, filled by extract_mmff_params)")
    types = np.asarray(p.atom_type, dtype=np.int64)
    q = np.asarray(p.partial_charge, dtype=np.float64).copy()
    q[np.abs(q) <= 1e-10] = 0.0
    uniq, cls = np.unique(types, return_inverse=True)
    ncls = len(uniq)
    vi = np.asarray(p.vdw_idx1, dtype=np.int64)
    vj = np.asarray(p.vdw_idx2, dtype=np.int64)
    ei = np.asarray(p.ele_idx1, dtype=np.int64)
    ej = np.asarray(p.ele_idx2, dtype=np.int64)
    R = np.asarray(p.vdw_R_star, dtype=np.float32)
    E = np.asarray(p.vdw_eps, dtype=np.float32)
    tab = np.zeros((ncls, ncls, 2), dtype=np.float32)
    tab[..., 0] = 1.0
    seen = np.zeros((ncls, ncls), dtype=bool)
    ci, cj = cls[vi], cls[vj]
    for a, b in ((ci, cj), (cj, ci)):
        key = a * ncls + b
        order = np.argsort(key, kind="stable")
        ks = key[order]
        first = np.ones(len(ks), dtype=bool)
        first[1:] = ks[1:] != ks[:-1]
        fa, fb = a[order][first], b[order][first]
        tab[fa, fb, 0] = R[order][first]
        tab[fa, fb, 1] = E[order][first]
        seen[fa, fb] = True
    got_r, got_e = tab[ci, cj, 0], tab[ci, cj, 1]
    if not (np.array_equal(got_r.view(np.uint32), R.view(np.uint32))
            and np.array_equal(got_e.view(np.uint32), E.view(np.uint32))):
        raise ValueError("vdW pair parameters are not a function of the atom types")
    if not np.array_equal(tab[ci, cj].view(np.uint32), tab[cj, ci].view(np.uint32)):
        raise ValueError("vdW pair parameters are not symmetric in the atom types")
    W = (n + 31) // 32
    pair = np.zeros((n, W * 32), dtype=bool)
    p14 = np.zeros((n, W * 32), dtype=bool)
    lo = np.minimum(vi, vj); hi = np.maximum(vi, vj)
    if np.any(lo == hi):
        raise ValueError("self pair in the vdW list")
    pair[lo, hi] = True
    elo = np.minimum(ei, ej); ehi = np.maximum(ei, ej)
    if len(ei) and not pair[elo, ehi].all():
        raise ValueError("electrostatic pair without a vdW pair")
    ct = np.asarray(p.ele_charge_term, dtype=np.float32)
    if not np.array_equal((q[ei] * q[ej]).astype(np.float32).view(np.uint32), ct.view(np.uint32)):
        raise ValueError("electrostatic charge terms are not float32(q_i * q_j)")
    is_ele = np.zeros((n, W * 32), dtype=bool)
    is_ele[elo, ehi] = True
    vd_only = pair & ~is_ele
    oi, oj = np.nonzero(vd_only)
    if len(oi) and np.any(q[oi] * q[oj] != 0.0):
        raise ValueError("vdW-only pair with a non-zero charge product")
    p14[elo, ehi] = np.asarray(p.ele_is_1_4, dtype=bool)
    words = lambda m: np.packbits(m.reshape(n, W, 32), axis=-1,
                                  bitorder="little").view("<u4").astype(np.uint32).reshape(-1)
    mask = np.concatenate([words(pair), words(p14)]) if n else np.zeros(0, np.uint32)
    return tab.reshape(-1, 2), cls.astype(np.int32), q, mask, ncls


_TERM_COUNT_FIELDS = ("bond_idx1", "angle_idx1", "strbend_idx1", "oop_idx1", "torsion_idx1", "vdw_idx1",
                      "ele_idx1")


def pack_molecules(params_list, n_threads: int = 0) -> PackedBatch:
    """Device layout of a list of MMFFParams (one entry per molecule).

    Built by the native packer of libmmffb200.so (``mmffb_pack_begin`` /
    ``mmffb_pack_finish``) on ``n_threads`` host threads (0: all cores); the result
    equals ``pack_molecules_py``'s bit for bit.  Raises ``ValueError`` where that
    would.
    """
    import ctypes

    from . import _lib
    params_list = list(params_list)
    M = len(params_list)
    for p in params_list:
        if p.atom_type is None or p.partial_charge is None:
            raise ValueError("non-bonded packing needs per-atom MMFF types and partial charges "
                             "(MMFFParams.atom_type / partial_charge, filled by extract_mmff_params)")
    L = _lib.load()
    keep = []

    def arr(xs, dt):
        a = np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(1), dtype=dt)
        if a.size == 0:
            a = np.zeros(1, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    counts = np.array([[len(getattr(p, f)) for f in _TERM_COUNT_FIELDS] for p in params_list],
                      dtype=np.int64).reshape(M, 7)
    starts = np.zeros((M + 1, 7), dtype=np.int64)
    np.cumsum(counts, axis=0, out=starts[1:])
    t = _lib.MMFFTermsHost()
    t.n_mols = M
    t.n_atoms = arr([np.array([int(p.n_atoms) for p in params_list])], np.int32)
    t.diel = arr([np.array([int(p.ele_diel_model) for p in params_list])], np.int32)
    t.term_start = arr([starts.reshape(-1)], np.int64)
    for cf, pf, ct in _lib.TERMS_HOST_FIELDS:
        setattr(t, cf, arr([getattr(p, pf) for p in params_list], np.int32 if ct is ctypes.c_int32 else np.float32))
    t.atom_type = arr([p.atom_type for p in params_list], np.int64)
    t.atom_charge = arr([p.partial_charge for p in params_list], np.float64)
    sizes = _lib.MMFFPackSizes()
    h = L.mmffb_pack_begin(ctypes.byref(t), int(n_threads), ctypes.byref(sizes))
    if not h:
        raise ValueError(L.mmffb_last_error().decode(errors="replace"))
    out = PackedBatch(mol_desc=np.empty((M, MOL_DESC_INTS), np.int32),
                      bonded=np.empty((sizes.bonded_rows, 4), np.uint32),
                      atom_cls=np.empty(sizes.atoms, np.int32), atom_q=np.empty(sizes.atoms, np.float64),
                      cls_tab=np.empty((sizes.cls_pairs, 2), np.float32),
                      pair_mask=np.empty(sizes.mask_words, np.uint32),
                      n_atoms=np.asarray([int(p.n_atoms) for p in params_list], dtype=np.int32))
    rc = L.mmffb_pack_finish(h, out.mol_desc.ctypes.data, out.bonded.ctypes.data, out.atom_cls.ctypes.data,
                             out.atom_q.ctypes.data, out.cls_tab.ctypes.data, out.pair_mask.ctypes.data)
    if rc != 0:
        raise ValueError(L.mmffb_last_error().decode(errors="replace"))
    return out


def pack_molecules_py(params_list) -> PackedBatch:
    """Device layout of a list of MMFFParams (one entry per molecule): the packing rule in
    numpy, molecule by molecule (the native packer's specification)."""
    descs, bonded, clss, qs, tabs, masks, natoms = [], [], [], [], [], [], []
    rec_off = atom_off = tab_off = mask_off = 0
    for p in params_list:
        n = int(p.n_atoms)
        if n > MAX_ATOMS:
            raise ValueError(f"molecule of {n} atoms exceeds {MAX_ATOMS}")
        tab, cls, q, mask, ncls = _nonbonded(p)
        if ncls > 64:
            raise ValueError(f"molecule with {ncls} non-bonded classes exceeds 64")
        recs = _bonded_records(p)
        d = np.zeros(MOL_DESC_INTS, dtype=np.int32)
        d[MD_N] = n
        d[MD_ATOM_OFF] = atom_off
        d[MD_NCLS] = ncls
        d[MD_CLS_OFF] = tab_off
        d[MD_MASK_OFF] = mask_off
        d[MD_DIEL] = 2 if int(p.ele_diel_model) == 2 else 1
        for t, (arr, nch) in enumerate(recs):
            d[MD_B_OFF + 2 * t] = rec_off
            d[MD_B_NCH + 2 * t] = nch
            bonded.append(arr)
            rec_off += len(arr)
        descs.append(d)
        clss.append(cls)
        qs.append(q)
        tabs.append(tab)
        masks.append(mask)
        natoms.append(n)
        atom_off += n
        tab_off += len(tab)
        mask_off += len(mask)
    cat = lambda xs, dt, w=None: (np.concatenate(xs).astype(dt) if xs else
                                  np.zeros((0,) if w is None else (0, w), dt))
    bonded_arr = np.concatenate(bonded) if bonded else np.zeros((0, 4), np.uint32)
    if len(bonded_arr) == 0:
        bonded_arr = np.full((1, 4), INVALID, dtype=np.uint32)
    return PackedBatch(
        mol_desc=np.stack(descs).astype(np.int32) if descs else np.zeros((0, 16), np.int32),
        bonded=np.ascontiguousarray(bonded_arr, dtype=np.uint32),
        atom_cls=cat(clss, np.int32), atom_q=cat(qs, np.float64),
        cls_tab=np.ascontiguousarray(np.concatenate(tabs) if tabs else np.zeros((1, 2)), dtype=np.float32),
        pair_mask=np.ascontiguousarray(np.concatenate(masks) if masks else np.zeros(1), dtype=np.uint32),
        n_atoms=np.asarray(natoms, dtype=np.int32))


def merge_packed(batches) -> PackedBatch:
    """One PackedBatch holding the molecules of several, in order.

    The tables are concatenated and every molecule descriptor's offsets shifted
    by the sizes of the tables before it, so a batch packed molecule by molecule
    (e.g. as requests arrive) merges without repacking.
    """
    batches = list(batches)
    if not batches:
        return pack_molecules([])
    descs, bonded, clss, qs, tabs, masks, natoms = [], [], [], [], [], [], []
    rec_off = atom_off = tab_off = mask_off = 0
    for b in batches:
        d = b.mol_desc.copy()
        d[:, MD_ATOM_OFF] += atom_off
        d[:, MD_CLS_OFF] += tab_off
        d[:, MD_MASK_OFF] += mask_off
        for t in range(5):
            d[:, MD_B_OFF + 2 * t] += rec_off
        descs.append(d)
        bonded.append(b.bonded)
        clss.append(b.atom_cls)
        qs.append(b.atom_q)
        tabs.append(b.cls_tab)
        masks.append(b.pair_mask)
        natoms.append(b.n_atoms)
        rec_off += len(b.bonded)
        atom_off += len(b.atom_cls)
        tab_off += len(b.cls_tab)
        mask_off += len(b.pair_mask)
    return PackedBatch(
        mol_desc=np.ascontiguousarray(np.concatenate(descs), dtype=np.int32),
        bonded=np.ascontiguousarray(np.concatenate(bonded), dtype=np.uint32),
        atom_cls=np.concatenate(clss).astype(np.int32), atom_q=np.concatenate(qs).astype(np.float64),
        cls_tab=np.ascontiguousarray(np.concatenate(tabs), dtype=np.float32),
        pair_mask=np.ascontiguousarray(np.concatenate(masks), dtype=np.uint32),
        n_atoms=np.concatenate(natoms).astype(np.int32))


def conformer_index(n_atoms_per_mol, conf_counts):
    """conf_mol (int32), conf_coord (int64 float offsets, molecule-major order) and total floats."""
    n_atoms_per_mol = np.asarray(n_atoms_per_mol, dtype=np.int64)
    conf_mol = np.repeat(np.arange(len(conf_counts), dtype=np.int32), conf_counts)
    sizes = 3 * n_atoms_per_mol[conf_mol]
    coord = np.zeros(len(conf_mol), dtype=np.int64)
    if len(sizes):
        coord[1:] = np.cumsum(sizes)[:-1]
    return conf_mol, coord, int(sizes.sum())


def lpt_order(n_atoms_per_mol, conf_mol) -> np.ndarray:
    """Largest molecules first (longest-processing-time order), a molecule's conformers together."""
    n = np.asarray(n_atoms_per_mol, dtype=np.int64)[conf_mol]
    return np.lexsort((np.arange(len(conf_mol)), conf_mol, -n)).astype(np.int32)
