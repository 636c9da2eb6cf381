"""Device-layout packing: exact re-expression of the reference pair lists, chunk invariants."""
import numpy as np
import pytest

from helpers import golden_mol, small_workload
from mlxmolkit_b200 import pack
from mlxmolkit_b200.mmff_params import extract_mmff_params


def _unpack_bits(words, n):
    W = (n + 31) // 32
    w = words.reshape(n, W).astype("<u4")
    bits = np.unpackbits(w.view(np.uint8).reshape(n, W, 4), axis=-1, bitorder="little")
    return bits.reshape(n, W * 32)[:, :n].astype(bool)


def test_masks_and_class_table_reproduce_the_pair_lists(golden):
    for mi in range(int(golden["n_mols"])):
        p = extract_mmff_params(golden_mol(golden, mi))
        pb = pack.pack_molecules([p])
        n = p.n_atoms
        W = (n + 31) // 32
        pair = _unpack_bits(pb.pair_mask[: n * W], n)
        p14 = _unpack_bits(pb.pair_mask[n * W: 2 * n * W], n)
        ii, jj = np.nonzero(pair)
        ref = set(zip(p.vdw_idx1.tolist(), p.vdw_idx2.tolist()))
        assert set(zip(ii.tolist(), jj.tolist())) == ref
        assert not np.tril(pair).any()
        ncls = int(pb.mol_desc[0, pack.MD_NCLS])
        tab = pb.cls_tab.reshape(ncls, ncls, 2)
        c = pb.atom_cls
        assert np.array_equal(tab[c[p.vdw_idx1], c[p.vdw_idx2], 0], p.vdw_R_star)
        assert np.array_equal(tab[c[p.vdw_idx1], c[p.vdw_idx2], 1], p.vdw_eps)
        q = pb.atom_q
        assert np.array_equal((q[p.ele_idx1] * q[p.ele_idx2]).astype(np.float32), p.ele_charge_term)
        e14 = p14[p.ele_idx1, p.ele_idx2]
        assert np.array_equal(e14.astype(np.int32), p.ele_is_1_4)


def _decode(pb, t):
    d = pb.mol_desc[0]
    off, nch = d[pack.MD_B_OFF + 2 * t], d[pack.MD_B_NCH + 2 * t]
    per = 64 if t in (2, 4) else 32
    recs = pb.bonded[off: off + nch * per].reshape(nch, per // 32, 32, 4)
    return recs


_FLIP = {0: (1, 0), 1: (2, 1, 0), 2: (2, 1, 0), 3: (2, 1, 0, 3), 4: (3, 2, 1, 0)}


def _canon(t, term):
    rev = tuple(term[q] for q in _FLIP[t])
    return min(tuple(term), rev)


@pytest.mark.parametrize("t,nroles", [(0, 2), (1, 3), (2, 3), (3, 4), (4, 4)])
def test_chunks_hold_every_term_once_with_distinct_atoms_per_role(golden, t, nroles):
    """Every term appears once (possibly in its equivalent reversed form), no atom twice per role."""
    p = extract_mmff_params(golden_mol(golden, 5))
    pb = pack.pack_molecules([p])
    recs = _decode(pb, t)
    terms = []
    for ch in recs:
        r0 = ch[0]
        valid = r0[:, 0] != 0xFFFFFFFF
        a = np.stack([r0[:, 0] & 0xFFFF, r0[:, 0] >> 16, r0[:, 1] & 0xFFFF, r0[:, 1] >> 16], 1)[valid]
        roles = a[:, :nroles] if t != 2 else np.stack([a[:, 0], a[:, 1], r0[valid][:, 1]], 1)
        for r in range(nroles):
            assert len(set(roles[:, r].tolist())) == len(roles), "atom repeated in a role"
        terms += [_canon(t, x) for x in roles.tolist()]
    src = {0: (p.bond_idx1, p.bond_idx2), 1: (p.angle_idx1, p.angle_idx2, p.angle_idx3),
           2: (p.strbend_idx1, p.strbend_idx2, p.strbend_idx3),
           3: (p.oop_idx1, p.oop_idx2, p.oop_idx3, p.oop_idx4),
           4: (p.torsion_idx1, p.torsion_idx2, p.torsion_idx3, p.torsion_idx4)}[t]
    assert sorted(terms) == sorted(_canon(t, x) for x in zip(*[s.tolist() for s in src]))


def test_reversed_stretch_bend_records_swap_their_sides(golden):
    p = extract_mmff_params(golden_mol(golden, 5))
    pb = pack.pack_molecules([p])
    recs = _decode(pb, 2)
    ref = {}
    for q in range(len(p.strbend_idx1)):
        key = (int(p.strbend_idx1[q]), int(p.strbend_idx2[q]), int(p.strbend_idx3[q]))
        ref[key] = (p.strbend_r0_ij[q], p.strbend_r0_kj[q], p.strbend_kba_ijk[q], p.strbend_kba_kji[q])
    seen_flip = 0
    for ch in recs:
        r0, r1 = ch[0], ch[1]
        for l in range(32):
            if r0[l, 0] == 0xFFFFFFFF:
                continue
            i, j, k = int(r0[l, 0] & 0xFFFF), int(r0[l, 0] >> 16), int(r0[l, 1])
            f = r0[l, 2:4].view(np.float32).tolist() + r1[l, 1:3].view(np.float32).tolist()
            if (i, j, k) in ref:
                assert np.allclose(f, ref[(i, j, k)], rtol=0, atol=0)
            else:
                a, b, c, d = ref[(k, j, i)]
                assert np.allclose(f, [b, a, d, c], rtol=0, atol=0)
                seen_flip += 1
    assert seen_flip >= 0


def test_type_inconsistent_vdw_table_is_rejected(golden):
    p = extract_mmff_params(golden_mol(golden, 3))
    p.vdw_eps = p.vdw_eps.copy()
    p.vdw_eps[5] *= 1.5
    with pytest.raises(ValueError):
        pack.pack_molecules([p])


def test_params_without_per_atom_data_are_rejected(golden):
    p = extract_mmff_params(golden_mol(golden, 1))
    p.atom_type = None
    with pytest.raises(ValueError):
        pack.pack_molecules([p])


def test_conformer_index_and_lpt_order():
    conf_mol, coord, total = pack.conformer_index([5, 9, 3], [2, 1, 3])
    assert conf_mol.tolist() == [0, 0, 1, 2, 2, 2]
    assert coord.tolist() == [0, 15, 30, 57, 66, 75] and total == 84
    order = pack.lpt_order([5, 9, 3], conf_mol)
    assert order.tolist() == [2, 0, 1, 3, 4, 5]


def test_batch_offsets_are_consistent():
    mols, params, counts, pos = small_workload(n_mols=5, k=2)
    pb = pack.pack_molecules(params)
    assert pb.mol_desc[:, pack.MD_ATOM_OFF].tolist() == np.concatenate([[0], np.cumsum(pb.n_atoms)[:-1]]).tolist()
    W = (pb.n_atoms + 31) // 32
    masks = 2 * pb.n_atoms * W
    assert pb.mol_desc[:, pack.MD_MASK_OFF].tolist() == np.concatenate([[0], np.cumsum(masks)[:-1]]).tolist()
    assert len(pb.pair_mask) == masks.sum()


def test_merging_per_molecule_packs_equals_packing_the_batch():
    mols, params, counts, pos = small_workload(n_mols=5, k=2)
    whole = pack.pack_molecules(params)
    merged = pack.merge_packed([pack.pack_molecules([p]) for p in params])
    for f in ("mol_desc", "bonded", "atom_cls", "atom_q", "cls_tab", "pair_mask", "n_atoms"):
        assert np.array_equal(getattr(whole, f), getattr(merged, f)), f
    assert merged.max_classes == whole.max_classes


def test_hybridization_survives_pickling_and_worker_pools():
    """Molecules built in spawned workers must type exactly like serially built ones."""
    import pickle
    from mlxmolkit_b200 import synth
    assert pickle.loads(pickle.dumps(synth.HybridizationType.SP)) is synth.HybridizationType.SP
    a = synth.make_molecules(6, 1, 21, 8, 40, workers=2)
    b = synth.make_molecules(6, 1, 21, 8, 40, workers=1)
    for x, y in zip(a, b):
        pa, pb = extract_mmff_params(x), extract_mmff_params(y)
        assert np.array_equal(pa.torsion_idx1, pb.torsion_idx1)
        assert np.array_equal(pa.strbend_idx2, pb.strbend_idx2)
        assert np.array_equal(x.GetConformer(0).pos, y.GetConformer(0).pos)


def test_native_chunker_equals_the_python_rule():
    mols, params, counts, pos = small_workload(n_mols=8, k=1, seed=17, lo=20, hi=60)
    rng = np.random.default_rng(5)
    cases = []
    for p in params:
        cases.append((np.stack([p.torsion_idx1, p.torsion_idx2, p.torsion_idx3, p.torsion_idx4], 1), (3, 2, 1, 0)))
        cases.append((np.stack([p.angle_idx1, p.angle_idx2, p.angle_idx3], 1), (2, 1, 0)))
        cases.append((np.stack([p.bond_idx1, p.bond_idx2], 1), None))
    cases.append((rng.integers(0, 40, size=(500, 3)), (2, 1, 0)))      # many collisions
    cases.append((np.zeros((0, 2), dtype=np.int64), (1, 0)))
    for ra, fp in cases:
        a, fa = pack._chunk(ra, fp)
        b, fb = pack.chunk_reference(ra, fp)
        assert np.array_equal(a, b) and np.array_equal(fa, fb)


_PACKED_FIELDS = ("mol_desc", "bonded", "atom_cls", "atom_q", "cls_tab", "pair_mask", "n_atoms")


@pytest.mark.parametrize("variant", ["MMFF94", "MMFF94s"])
def test_native_batch_packer_equals_the_python_rule(any_golden, variant):
    """mmffb_pack_begin/_finish (host threads) produce pack_molecules_py's bytes, on every
    fixture molecule (16-377 atoms) in one batch and with one thread or many."""
    g = any_golden
    params = [extract_mmff_params(golden_mol(g, mi), mmff_variant=variant) for mi in range(int(g["n_mols"]))]
    _, more, _, _ = small_workload(n_mols=12, k=1, seed=19, lo=4, hi=40)
    params = params + more
    ref = pack.pack_molecules_py(params)
    for nt in (1, 3, 0):
        got = pack.pack_molecules(params, n_threads=nt)
        for f in _PACKED_FIELDS:
            a, b = getattr(ref, f), getattr(got, f)
            assert a.dtype == b.dtype and a.shape == b.shape, f
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (nt, f)


def test_native_batch_packer_edge_cases(golden):
    empty_ref, empty = pack.pack_molecules_py([]), pack.pack_molecules([])
    for f in _PACKED_FIELDS:
        assert np.array_equal(getattr(empty_ref, f), getattr(empty, f)), f
    p = extract_mmff_params(golden_mol(golden, 2))
    p.ele_charge_term = p.ele_charge_term.copy()
    p.ele_charge_term[3] += 1e-3
    with pytest.raises(ValueError, match="molecule 1: electrostatic charge terms"):
        pack.pack_molecules([extract_mmff_params(golden_mol(golden, 0)), p])
    with pytest.raises(ValueError):
        pack.pack_molecules_py([p])
    q = extract_mmff_params(golden_mol(golden, 4))
    q.vdw_idx2 = q.vdw_idx2.copy()
    q.vdw_idx2[0] = q.vdw_idx1[0]
    with pytest.raises(ValueError, match="self pair"):
        pack.pack_molecules([q])
