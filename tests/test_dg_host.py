"""The distance-geometry stage without a GPU: host side against the reference, and the oracle.

* packing, extraction and the initial embeddings against the reference's own
  functions (tests/golden/ref_dg_batches.npz, written by make_golden_dg.py);
* the FP64 oracle (oracle/dg_oracle.c) against finite differences and the
  outcomes the reference's DG tests assert (tests/test_conformer_metal.py:108-260);
* the device layout (``dg_device_arrays``): a host emulation of the kernel's
  per-atom incidence gradient and flat-record energy reproduces the oracle.
"""
import numpy as np
import pytest

from helpers import all_pairs_dg, dg_golden_mol, dg_synth_params
from mlxmolkit_b200.dg_extract import (DGParams, extract_dg_params, metric_matrix_positions,
                                       synth_bounds_matrix, synth_chiral_tags)
from mlxmolkit_b200.shared_batch import dg_device_arrays, init_random_positions, pack_shared_dg_batch
from oracle import dg

BATCH_FIELDS = ("conf_atom_starts", "conf_to_mol", "mol_n_atoms", "dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2",
                "dist_weight", "dist_term_starts", "chiral_idx1", "chiral_idx2", "chiral_idx3", "chiral_idx4",
                "chiral_vol_lower", "chiral_vol_upper", "chiral_term_starts", "fourth_idx", "fourth_term_starts")
PARAM_FIELDS = ("dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2", "dist_weight", "chiral_idx1", "chiral_idx2",
                "chiral_idx3", "chiral_idx4", "chiral_vol_lower", "chiral_vol_upper", "fourth_idx")
ALLPAIRS, ALLPAIRS_K = [(5, 1.0, 4.0), (8, 1.0, 4.0), (6, 1.5, 3.0)], [3, 2, 2]
SYNTH_K = [2, 3, 1]


def _golden_synth_params(g):
    out = []
    for mi in range(3):
        pre = f"s{mi}_"
        out.append(DGParams(n_atoms=len(g[pre + "elements"]), **{f: g[pre + "ref_" + f] for f in PARAM_FIELDS}))
    return out


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b)


def test_pack_matches_the_reference(dg_golden):
    b = pack_shared_dg_batch([all_pairs_dg(*s) for s in ALLPAIRS], ALLPAIRS_K, dim=4)
    for f in BATCH_FIELDS:
        assert _same(getattr(b, f), dg_golden["ap_" + f]), f
    b = pack_shared_dg_batch(_golden_synth_params(dg_golden), SYNTH_K, dim=4)
    for f in BATCH_FIELDS:
        assert _same(getattr(b, f), dg_golden["sy_" + f]), f
    assert b.n_confs_total == 6 and b.n_atoms_total == int(dg_golden["sy_conf_atom_starts"][-1])


def test_init_random_positions_matches_the_reference(dg_golden):
    b = pack_shared_dg_batch([all_pairs_dg(*s) for s in ALLPAIRS], ALLPAIRS_K, dim=4)
    assert _same(init_random_positions(b, seed=7), dg_golden["ap_init_seed7"])


def test_extraction_from_a_bounds_matrix_matches_the_reference(dg_golden):
    for mi in range(3):
        mol = dg_golden_mol(dg_golden, mi)
        assert np.array_equal(synth_bounds_matrix(mol), dg_golden[f"s{mi}_bounds_mat"])
        assert synth_chiral_tags(mol) == mol.chiral_tags
        p = extract_dg_params(mol, dg_golden[f"s{mi}_bounds_mat"])
        for f in PARAM_FIELDS:
            assert _same(getattr(p, f), dg_golden[f"s{mi}_ref_{f}"]), (mi, f)
    assert sum(len(dg_golden[f"s{mi}_ref_chiral_idx1"]) for mi in range(3)) > 0   # chiral terms are covered


def test_metric_matrix_positions_match_the_reference(dg_golden):
    params = _golden_synth_params(dg_golden)
    bms = [dg_golden[f"s{mi}_bounds_mat"] for mi in range(3)]
    got = metric_matrix_positions(pack_shared_dg_batch(params, SYNTH_K, dim=4), bms, seed=42, dim=4)
    np.testing.assert_allclose(got, dg_golden["sy_metric_seed42"], rtol=0, atol=1e-5)
    got = metric_matrix_positions(pack_shared_dg_batch(params, SYNTH_K, dim=3), bms, seed=5, dim=3)
    np.testing.assert_allclose(got, dg_golden["sy_metric_seed5_dim3"], rtol=0, atol=1e-5)


def test_oracle_gradient_matches_finite_differences(dg_golden):
    b = pack_shared_dg_batch(_golden_synth_params(dg_golden), SYNTH_K, dim=4)
    x = init_random_positions(b, seed=3).astype(np.float64) * 2.0
    for conf in (0, 3):
        a0, a1 = int(b.conf_atom_starts[conf]) * 4, int(b.conf_atom_starts[conf + 1]) * 4
        e0, g = dg.energy_grad(b, x, conf, chiral_weight=1.0, fourth_dim_weight=0.1)
        assert e0 > 0
        rng = np.random.default_rng(conf)
        for k in rng.choice(a1 - a0, 12, replace=False):
            xp, xm = x.copy(), x.copy()
            xp[a0 + k] += 1e-6
            xm[a0 + k] -= 1e-6
            fd = (dg.energy_grad(b, xp, conf)[0] - dg.energy_grad(b, xm, conf)[0]) / 2e-6
            assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (conf, k, fd, g[k])


def test_oracle_reproduces_the_reference_test_outcomes():
    """What tests/test_conformer_metal.py:115-239 asserts of the reference kernel holds for the oracle."""
    b = pack_shared_dg_batch([all_pairs_dg(10)], [5], dim=4)
    _, e, s, _ = dg.minimize(b, init_random_positions(b, 42), max_iters=200)
    assert np.all(s == 0)
    b = pack_shared_dg_batch([all_pairs_dg(8)], [3], dim=4)
    _, e, _, _ = dg.minimize(b, init_random_positions(b, 99), max_iters=200)
    assert np.all(e < 1.0)
    b = pack_shared_dg_batch([all_pairs_dg(6)], [2], dim=4)
    x, _, _, _ = dg.minimize(b, init_random_positions(b, 55), max_iters=300, fourth_dim_weight=1.0)
    assert np.abs(x.reshape(-1, 4)[:, 3]).max() < 2.0
    b = pack_shared_dg_batch([all_pairs_dg(8), all_pairs_dg(6), all_pairs_dg(10)], [20, 20, 20], dim=4)
    _, _, s, _ = dg.minimize(b, init_random_positions(b, 42), max_iters=200)
    assert np.sum(s == 0) >= 55
    empty = DGParams(3, *[np.zeros(0, np.int32)] * 2, *[np.zeros(0, np.float32)] * 3, *[np.zeros(0, np.int32)] * 4,
                     np.zeros(0, np.float32), np.zeros(0, np.float32), np.arange(3, dtype=np.int32))
    b = pack_shared_dg_batch([empty], [2], dim=4)
    _, e, s, _ = dg.minimize(b, init_random_positions(b, 1), max_iters=50)
    assert len(e) == 2 and np.all(np.isfinite(e))


def _emulate_device_layout(arrs, x, dim, conf_mol, conf_start, cw, fw):
    """Energy and gradient of one conformer computed the kernel's way from the device arrays."""
    m = conf_mol
    n = int(arrs["mol_n_atoms"][m])
    base = int(arrs["mol_atom_base"][m])
    X = np.zeros((n, 4))
    X[:, :dim] = x[conf_start * dim:(conf_start + n) * dim].reshape(n, dim)
    e = 0.0
    rec = arrs["dist_rec"]
    for t in range(arrs["dist_starts"][m], arrs["dist_starts"][m + 1]):
        ij = rec[t:t + 1, 0].view(np.int32)[0]
        i, j = ij & 0xFFFF, ij >> 16
        lb2, ub2, w = (float(v) for v in rec[t, 1:])
        d2 = float(((X[i] - X[j]) ** 2).sum())
        if d2 > ub2:
            e += w * (d2 / ub2 - 1) ** 2
        elif d2 < lb2:
            e += w * (2 * lb2 / (lb2 + d2) - 1) ** 2
    quads, bnds = arrs["chiral_quads"], arrs["chiral_bounds"]

    def geom(q):
        v1, v2, v3 = (X[q[k], :3] - X[q[3], :3] for k in range(3))
        return np.cross(v2, v3), np.cross(v3, v1), np.cross(v1, v2), float(np.dot(v1, np.cross(v2, v3)))

    for t in range(arrs["chiral_starts"][m], arrs["chiral_starts"][m + 1]):
        vol = geom(quads[t])[3]
        lo, hi = (float(v) for v in bnds[t])
        if vol < lo:
            e += cw * (vol - lo) ** 2
        elif vol > hi:
            e += cw * (vol - hi) ** 2
    G = np.zeros((n, 4))
    inc, cinc = arrs["dinc_rec"], arrs["cinc_rec"]
    for a in range(n):
        r = base + a
        for k in range(arrs["dinc_starts"][r], arrs["dinc_starts"][r + 1]):
            o = inc[k:k + 1, 0].view(np.int32)[0]
            lb2, ub2, w = (float(v) for v in inc[k, 1:])
            df = X[a] - X[o]
            d2 = float((df ** 2).sum())
            pf = 0.0
            if d2 > ub2:
                pf = w * 4 * (d2 / ub2 - 1) / ub2
            elif d2 < lb2:
                ll = d2 + lb2
                pf = w * 8 * lb2 * (1 - 2 * lb2 / ll) / (ll * ll)
            G[a] += pf * df
        for k in range(arrs["cinc_starts"][r], arrs["cinc_starts"][r + 1]):
            t, role = cinc[k]
            c23, c31, c12, vol = geom(quads[t])
            lo, hi = (float(v) for v in bnds[t])
            pf = 2 * cw * (vol - lo) if vol < lo else 2 * cw * (vol - hi) if vol > hi else 0.0
            G[a, :3] += pf * (c23, c31, c12, -(c23 + c31 + c12))[role]
        if dim == 4:
            cnt = int(arrs["fourth_count"][r])
            G[a, 3] += cnt * 2 * fw * X[a, 3]
            e += cnt * fw * float(X[a, 3]) ** 2
    return e, G[:, :dim].reshape(-1)


@pytest.mark.parametrize("dim", [4, 3])
def test_device_layout_reproduces_the_oracle(dim):
    params = dg_synth_params(3, seed=17, lo=8, hi=18) + [all_pairs_dg(7)]
    b = pack_shared_dg_batch(params, [2, 1, 1, 2], dim=dim)
    arrs = dg_device_arrays(b)
    # every distance term appears twice in the incidence rows, chiral terms four times
    assert len(arrs["dinc_rec"]) == 2 * len(b.dist_idx1) and len(arrs["cinc_rec"]) == 4 * len(b.chiral_idx1)
    assert np.all(np.diff(b.mol_n_atoms[b.conf_to_mol[arrs["conf_order"]]]) <= 0)   # largest molecules first
    x = init_random_positions(b, seed=11).astype(np.float64) * 1.5
    for conf in range(b.n_confs_total):
        e_ref, g_ref = dg.energy_grad(b, x, conf, chiral_weight=0.7, fourth_dim_weight=0.2)
        e, g = _emulate_device_layout(arrs, x, dim, int(b.conf_to_mol[conf]), int(b.conf_atom_starts[conf]), 0.7, 0.2)
        assert abs(e - e_ref) <= 1e-9 * max(1.0, e_ref)
        np.testing.assert_allclose(g, g_ref, rtol=1e-9, atol=1e-9)


def test_device_layout_rejects_bad_indices():
    p = all_pairs_dg(4)
    p.dist_idx2 = p.dist_idx2.copy()
    p.dist_idx2[0] = 4
    with pytest.raises(ValueError):
        dg_device_arrays(pack_shared_dg_batch([p], [1]))
    with pytest.raises(ValueError):
        dg_device_arrays(pack_shared_dg_batch([all_pairs_dg(4)], [1], dim=5))


def test_tetrahedral_centres_match_the_reference(dg_golden):
    from mlxmolkit_b200.stereo_checks import extract_tetrahedral_data, tetrahedral_quads
    for mi in range(3):
        mol = dg_golden_mol(dg_golden, mi)
        ref = dg_golden[f"s{mi}_ref_tetrahedral"]
        got = np.array(extract_tetrahedral_data(mol)[:5], dtype=np.int32).reshape(5, -1)
        assert np.array_equal(got, ref), mi
        q = tetrahedral_quads(mol)
        assert np.array_equal(q, ref[1:5].T)


def _sequential_starts(b, bms, seed, dim):
    from mlxmolkit_b200.dg_extract import _metric_embed_sequential
    out = np.zeros(int(b.conf_atom_starts[-1]) * dim, np.float32)
    _metric_embed_sequential(b, bms, np.random.default_rng(seed), dim, out, 0)
    return out


def test_metric_starts_batched_equal_sequential_with_extra_draws(dg_golden):
    """The batched start generator equals the one-conformer-at-a-time one, also when a conformer
    needs the extra uniform columns: a 3-atom molecule has fewer eigenvalues than 4 dimensions, and
    a molecule of two atoms at zero distance has no positive one."""
    from mlxmolkit_b200.dg_extract import metric_matrix_positions
    params = _golden_synth_params(dg_golden)
    bms = [dg_golden[f"s{mi}_bounds_mat"] for mi in range(3)]
    tiny = np.array([[0, 1.5, 2.5], [1.4, 0, 1.5], [2.4, 1.4, 0]])           # 3 atoms
    flat = np.zeros((2, 2))                                                 # 2 atoms, zero bounds
    extra = [all_pairs_dg(3), all_pairs_dg(2)]
    b = pack_shared_dg_batch(params + extra, [2, 2, 1, 2, 2], dim=4)
    allb = bms + [tiny, flat]
    got = metric_matrix_positions(b, allb, seed=11, dim=4)
    ref = _sequential_starts(b, allb, 11, 4)
    assert np.array_equal(got, ref)
    assert np.isfinite(got).all()


def test_per_molecule_starts_assemble_to_the_batch_sequence(dg_golden):
    """The pipeline computes each molecule's starts apart (its terms and its slice of the draw
    sequence, on the process pool); assembled, they equal ``metric_matrix_positions``, also when a
    conformer needs extra uniform columns and the rest of the batch is redone in sequence."""
    from mlxmolkit_b200 import conformer_pipeline_v2 as cp
    from mlxmolkit_b200.dg_extract import (embed_conformers, metric_matrix_positions, pair_draw_offsets,
                                           uniform_draws)
    params = _golden_synth_params(dg_golden)
    for p, mi in zip(params, range(3)):
        p.bounds_mat = dg_golden[f"s{mi}_bounds_mat"]
    tiny, flat = all_pairs_dg(3), all_pairs_dg(2)
    tiny.bounds_mat = np.array([[0, 1.5, 2.5], [1.4, 0, 1.5], [2.4, 1.4, 0]])
    flat.bounds_mat = np.zeros((2, 2))
    for mols, ks in ((params, [2, 3, 1]), (params + [tiny] + params[:2], [2, 1, 2, 2, 3, 1]),
                     (params[:1] + [flat] + params[1:], [1, 2, 0, 2])):
        b = pack_shared_dg_batch(mols, ks, dim=4)
        offs = pair_draw_offsets(np.repeat([p.n_atoms for p in mols], ks))
        first = np.concatenate([[0], np.cumsum(ks)])
        res = []
        for i, (p, k) in enumerate(zip(mols, ks)):
            n = p.n_atoms
            u = uniform_draws(5, int(offs[first[i]]), k * n * (n - 1) // 2)
            res.append((p, *embed_conformers(p.bounds_mat, u, k, 4)) if k else (p, None, 0))
        got = cp._assemble_starts(res, ks, b, 5, 4)
        ref = metric_matrix_positions(b, [p.bounds_mat for p in mols], seed=5, dim=4)
        assert np.array_equal(got, ref)
        # the tiny and the zero-bounds molecule each need the extra columns at their first conformer
        assert any(r[1] is not None and r[2] < k for r, k in zip(res, ks)) == (len(mols) > 3)


def test_dg_layout_does_not_depend_on_the_thread_split(dg_golden):
    """Large batches build the DG tables as runs of molecules on host threads and merge them;
    every split gives the bytes of the one-run build (distance, chiral and fourth-dimension
    terms, molecules without chiral terms included)."""
    from mlxmolkit_b200.shared_batch import _runs_by_terms
    params = _golden_synth_params(dg_golden) + dg_synth_params(12, 21) + [all_pairs_dg(3), all_pairs_dg(5)]
    ks = [1 + i % 3 for i in range(len(params))]
    for dim in (4, 3):
        b = pack_shared_dg_batch(params, ks, dim=dim)
        one = dg_device_arrays(b, workers=1)
        for w in (2, 3, 6):
            assert len(_runs_by_terms(np.diff(np.asarray(b.dist_term_starts)), w)) > 1
            got = dg_device_arrays(b, workers=w)
            assert set(got) == set(one)
            for f in one:
                if isinstance(one[f], np.ndarray):
                    assert got[f].dtype == one[f].dtype and np.array_equal(got[f].view(np.uint8),
                                                                            one[f].view(np.uint8)), (dim, w, f)
                else:
                    assert got[f] == one[f], (dim, w, f)


def test_recentred_bounds_take_the_last_conformer(dg_golden):
    """conformer_pipeline_v2.py:224-258: the 1-2 / 1-3 bounds move to the measured distances of the
    molecule's last conformer, keeping their half-widths."""
    from mlxmolkit_b200.conformer_pipeline_v2 import _recenter_bounds
    from mlxmolkit_b200.etk_extract import synth_etk_params
    from mlxmolkit_b200.shared_batch import add_etk_to_batch
    params = _golden_synth_params(dg_golden)
    mols = [dg_golden_mol(dg_golden, mi) for mi in range(3)]
    b3 = pack_shared_dg_batch(params, [2, 3, 1], dim=3)
    add_etk_to_batch(b3, [synth_etk_params(m, dg_golden[f"s{mi}_bounds_mat"]) for mi, m in enumerate(mols)])
    hw = (b3.etk_dist12_ub - b3.etk_dist12_lb).copy() / 2
    rng = np.random.default_rng(2)
    pos = rng.normal(0, 2.0, int(b3.conf_atom_starts[-1]) * 3).astype(np.float32)
    _recenter_bounds(b3, pos)
    for m, last in ((0, 1), (1, 4), (2, 5)):
        t0, t1 = b3.etk_dist12_term_starts[m], b3.etk_dist12_term_starts[m + 1]
        a0 = int(b3.conf_atom_starts[last]) * 3
        x = pos[a0:a0 + 3 * int(b3.mol_n_atoms[m])].reshape(-1, 3).astype(np.float64)
        d = np.linalg.norm(x[b3.etk_dist12_idx1[t0:t1]] - x[b3.etk_dist12_idx2[t0:t1]], axis=1)
        np.testing.assert_allclose(b3.etk_dist12_lb[t0:t1], d - hw[t0:t1], atol=1e-5)
        np.testing.assert_allclose(b3.etk_dist12_ub[t0:t1], d + hw[t0:t1], atol=1e-5)


def test_recentring_is_the_per_molecule_computation_bit_for_bit(dg_golden):
    """The vectorised re-centring gives the bytes of the reference's per-molecule loop: FP64
    distances of the molecule's last conformer, FP64 half-widths, rounded once to FP32; a
    molecule without conformers keeps its bounds."""
    from mlxmolkit_b200.conformer_pipeline_v2 import _recenter_bounds
    from mlxmolkit_b200.etk_extract import synth_etk_params
    from mlxmolkit_b200.shared_batch import add_etk_to_batch
    params = _golden_synth_params(dg_golden)
    mols = [dg_golden_mol(dg_golden, mi) for mi in range(3)]
    ks = [3, 0, 2]
    b3 = pack_shared_dg_batch(params, ks, dim=3)
    add_etk_to_batch(b3, [synth_etk_params(m, dg_golden[f"s{mi}_bounds_mat"]) for mi, m in enumerate(mols)])
    pos = np.random.default_rng(4).normal(0, 2.0, int(b3.conf_atom_starts[-1]) * 3).astype(np.float32)
    want = {}
    for tag in ("12", "13"):
        st = getattr(b3, f"etk_dist{tag}_term_starts")
        lb = getattr(b3, f"etk_dist{tag}_lb").copy()
        ub = getattr(b3, f"etk_dist{tag}_ub").copy()
        for m, last in ((0, 2), (2, 4)):
            t0, t1 = int(st[m]), int(st[m + 1])
            n, a0 = int(b3.mol_n_atoms[m]), int(b3.conf_atom_starts[last]) * 3
            x = pos[a0:a0 + 3 * n].reshape(n, 3).astype(np.float64)
            i1, i2 = getattr(b3, f"etk_dist{tag}_idx1")[t0:t1], getattr(b3, f"etk_dist{tag}_idx2")[t0:t1]
            d = np.linalg.norm(x[i1] - x[i2], axis=1)
            hw = (ub[t0:t1].astype(np.float64) - lb[t0:t1]) / 2.0
            lb[t0:t1], ub[t0:t1] = (d - hw).astype(np.float32), (d + hw).astype(np.float32)
        want[tag] = lb, ub
    before13 = b3.etk_dist13_lb[b3.etk_dist13_term_starts[1]:b3.etk_dist13_term_starts[2]].copy()
    _recenter_bounds(b3, pos)
    for tag, (lb, ub) in want.items():
        assert np.array_equal(getattr(b3, f"etk_dist{tag}_lb").view(np.uint32), lb.view(np.uint32)), tag
        assert np.array_equal(getattr(b3, f"etk_dist{tag}_ub").view(np.uint32), ub.view(np.uint32)), tag
    assert np.array_equal(b3.etk_dist13_lb[b3.etk_dist13_term_starts[1]:b3.etk_dist13_term_starts[2]], before13)


def test_pooled_extraction_equals_in_process():
    """generate_conformers_nk maps the per-molecule term extraction over spawned host processes for
    large batches; the terms are the same as in-process."""
    from dataclasses import fields

    from mlxmolkit_b200 import conformer_pipeline_v2 as cp
    from mlxmolkit_b200 import synth
    from mlxmolkit_b200.dg_extract import metric_matrix_positions
    from mlxmolkit_b200.shared_batch import pack_shared_dg_batch
    mols = synth.make_molecules(cp._POOL_MIN, 1, 9, 8, 16, workers=1)
    serial = [cp._dg_terms(m) for m in mols]
    ks = [1 + i % 4 for i in range(len(mols))]
    pooled, b4, x4 = cp._dg_terms_and_positions(mols, ks, 42)    # terms and starts in one task
    for a, b in zip(serial, pooled):
        for f in fields(a):
            assert np.array_equal(np.asarray(getattr(a, f.name)), np.asarray(getattr(b, f.name))), f.name
    ref = metric_matrix_positions(pack_shared_dg_batch(serial, ks, dim=4), [p.bounds_mat for p in serial], seed=42)
    assert np.array_equal(x4, ref)
    from mlxmolkit_b200.mmff_params import extract_mmff_params
    from mlxmolkit_b200.pack import merge_packed, pack_molecules
    items = [(m, "MMFF94s") for m in mols]
    serial = [cp._mmff_pack(x) for x in items]
    pooled = cp._pmap(cp._mmff_pack, items)
    for ka, kb in zip(serial, pooled):
        for f in fields(ka):
            assert np.array_equal(np.asarray(getattr(ka, f.name)), np.asarray(getattr(kb, f.name))), f.name
    # the per-molecule packs merge into exactly the tables of packing the parameter list at once
    params = [extract_mmff_params(m, conf_id=m.GetConformers()[0].GetId(), mmff_variant="MMFF94s") for m in mols]
    whole, merged = pack_molecules(params), merge_packed(pooled)
    for f in fields(whole):
        assert np.array_equal(np.asarray(getattr(whole, f.name)), np.asarray(getattr(merged, f.name))), f.name
