"""The ETK stage without a GPU: packing against the reference, the oracle, the device layout.

* ``add_etk_to_batch`` against the reference's own (tests/golden/ref_dg_batches.npz);
* the FP64 oracle's ETK energy and gradient (oracle/dg_oracle.c) against finite
  differences, and the reference's ETK consistency test
  (tests/test_etk_metal_consistency.py:90-105) restated on the oracle;
* ``etk_device_arrays``: a host emulation of the kernel's two-phase gradient
  (Fourier-term rows, then per-atom sums) reproduces the oracle.
"""
import numpy as np
import pytest

from helpers import all_pairs_dg, dg_golden_mol
from mlxmolkit_b200.dg_extract import DGParams, synth_bounds_matrix, synth_dg_params
from mlxmolkit_b200.etk_extract import ETKParams, synth_etk_params
from mlxmolkit_b200.shared_batch import add_etk_to_batch, etk_device_arrays, pack_shared_dg_batch
from oracle import dg

ETK_FIELDS = ("torsion_idx", "torsion_V", "torsion_signs", "improper_idx", "improper_weight", "dist12_idx1",
              "dist12_idx2", "dist12_lb", "dist12_ub", "dist12_weight", "dist13_idx1", "dist13_idx2", "dist13_lb",
              "dist13_ub", "dist13_weight", "dist14_idx1", "dist14_idx2", "dist14_lb", "dist14_ub", "dist14_weight")
ETK_BATCH = ["etk_torsion_idx", "etk_torsion_V", "etk_torsion_signs", "etk_torsion_term_starts", "etk_improper_idx",
             "etk_improper_weight", "etk_improper_term_starts"] + [
    f"etk_dist{t}_{f}" for t in ("12", "13", "14") for f in ("idx1", "idx2", "lb", "ub", "weight", "term_starts")]
PARAM_FIELDS = ("dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2", "dist_weight", "chiral_idx1", "chiral_idx2",
                "chiral_idx3", "chiral_idx4", "chiral_vol_lower", "chiral_vol_upper", "fourth_idx")
SYNTH_K = [2, 3, 1]


def _golden_batch3(g):
    dgp = [DGParams(n_atoms=len(g[f"s{mi}_elements"]), **{f: g[f"s{mi}_ref_{f}"] for f in PARAM_FIELDS})
           for mi in range(3)]
    etk = [ETKParams(n_atoms=len(g[f"s{mi}_elements"]), **{f: g[f"s{mi}_etk_{f}"] for f in ETK_FIELDS})
           for mi in range(3)]
    b = pack_shared_dg_batch(dgp, SYNTH_K, dim=3)
    add_etk_to_batch(b, etk)
    return b


def _etk_from_mols(g):
    """The fixture molecules' ETK terms recomputed by this package's stand-in."""
    return [synth_etk_params(dg_golden_mol(g, mi), g[f"s{mi}_bounds_mat"]) for mi in range(3)]


def test_synthetic_etk_terms_are_reproducible(dg_golden):
    for mi, p in enumerate(_etk_from_mols(dg_golden)):
        for f in ETK_FIELDS:
            assert np.array_equal(getattr(p, f), dg_golden[f"s{mi}_etk_{f}"]), (mi, f)
        assert np.array_equal(synth_bounds_matrix(dg_golden_mol(dg_golden, mi)), dg_golden[f"s{mi}_bounds_mat"])


def test_add_etk_to_batch_matches_the_reference(dg_golden):
    b = _golden_batch3(dg_golden)
    for f in ETK_BATCH:
        got, ref = np.asarray(getattr(b, f)), dg_golden["sy3_" + f]
        assert got.dtype == ref.dtype and np.array_equal(got.reshape(ref.shape), ref), f
    assert len(b.etk_torsion_idx) > 0 and len(b.etk_improper_idx) > 0 and len(b.etk_dist14_idx1) > 0


def _positions(b, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(int(b.conf_atom_starts[-1]) * 3) * scale


def test_oracle_etk_gradient_matches_finite_differences(dg_golden):
    b = _golden_batch3(dg_golden)
    x = _positions(b, 5, 1.5)
    for conf in (0, 2, 5):
        a0, a1 = int(b.conf_atom_starts[conf]) * 3, int(b.conf_atom_starts[conf + 1]) * 3
        e0, g = dg.energy_grad(b, x, conf, stage="etk")
        assert e0 > 0
        rng = np.random.default_rng(conf)
        for k in rng.choice(a1 - a0, 15, replace=False):
            xp, xm = x.copy(), x.copy()
            xp[a0 + k] += 1e-6
            xm[a0 + k] -= 1e-6
            fd = (dg.energy_grad(b, xp, conf, stage="etk")[0] - dg.energy_grad(b, xm, conf, stage="etk")[0]) / 2e-6
            assert abs(fd - g[k]) <= 2e-5 * max(1.0, abs(g[k])), (conf, k, fd, g[k])


def _distance_only_batch():
    """The reference's distance-only ETK case (tests/test_etk_metal_consistency.py:13-87)."""
    e = np.zeros(0, np.float32)
    p = ETKParams(3, np.zeros((0, 4), np.int32), np.zeros((0, 6), np.float32), np.zeros((0, 6), np.int32),
                  np.zeros((0, 4), np.int32), e,
                  np.array([0], np.int32), np.array([1], np.int32), np.array([0.95], np.float32),
                  np.array([1.05], np.float32), np.array([100.0], np.float32),
                  np.array([0], np.int32), np.array([2], np.int32), np.array([1.45], np.float32),
                  np.array([1.55], np.float32), np.array([100.0], np.float32),
                  np.zeros(0, np.int32), np.zeros(0, np.int32), e, e, e)
    dgp = DGParams(3, *[np.zeros(0, np.int32)] * 2, *[np.zeros(0, np.float32)] * 3, *[np.zeros(0, np.int32)] * 4,
                   np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.int32))
    b = pack_shared_dg_batch([dgp], [1], dim=3)
    add_etk_to_batch(b, [p])
    return b, np.array([0, 0, 0, 2, 0, 0, 3, 0, 0], np.float32)


def test_oracle_reproduces_the_reference_etk_consistency_case():
    b, x = _distance_only_batch()
    out, e, _, _ = dg.minimize(b, x, max_iters=1, stage="etk")
    _, e0, _, _ = dg.minimize(b, out.astype(np.float32), max_iters=0, stage="etk")
    np.testing.assert_allclose(e, e0, atol=1e-4)
    e_start = dg.energy_grad(b, x, 0, stage="etk")[0]
    assert e[0] < e_start


def _emulate_etk(arrs, x, conf_mol, conf_start):
    m = conf_mol
    n = int(arrs["mol_n_atoms"][m])
    base = int(arrs["mol_atom_base"][m])
    X = x[conf_start * 3:(conf_start + n) * 3].reshape(n, 3).astype(np.float64)
    e = 0.0
    for t in range(arrs["fb_starts"][m], arrs["fb_starts"][m + 1]):
        ij = arrs["fb_rec"][t:t + 1, 0].view(np.int32)[0]
        i, j = ij & 0xFFFF, ij >> 16
        lb, ub, w = (float(v) for v in arrs["fb_rec"][t, 1:])
        d = float(np.sqrt(((X[i] - X[j]) ** 2).sum() + 1e-12))
        e += w * (d - lb) ** 2 if d < lb else (w * (d - ub) ** 2 if d > ub else 0.0)
    ts, te = int(arrs["tor_starts"][m]), int(arrs["tor_starts"][m + 1])
    rows = np.zeros((max(te - ts, 0), 4, 3))
    for t in range(ts, te):
        q = [int(v) for v in arrs["tor_quads"][t]]
        V, S = arrs["tor_coef"][t, :6].astype(np.float64), arrs["tor_coef"][t, 6:].astype(np.float64)
        # an isolated one-conformer system per Fourier term: the oracle's torsion as a Fourier term
        r1, r2, r4 = X[q[0]] - X[q[1]], X[q[2]] - X[q[1]], X[q[3]] - X[q[2]]
        t0, t1 = np.cross(r1, r2), np.cross(-r2, r4)
        comb = float(t0 @ t0) * float(t1 @ t1)
        c = 0.0 if comb < 1e-16 else float(np.clip((t0 @ t1) / np.sqrt(comb), -1, 1))
        e += sum(V[k] * (1 + S[k] * np.cos((k + 1) * np.arccos(c))) for k in range(6))
        h = 1e-6
        for r in range(4):
            for d in range(3):
                Xp, Xm = X.copy(), X.copy()
                Xp[q[r], d] += h
                Xm[q[r], d] -= h

                def E(Y):
                    a1, a2, a4 = Y[q[0]] - Y[q[1]], Y[q[2]] - Y[q[1]], Y[q[3]] - Y[q[2]]
                    u0, u1 = np.cross(a1, a2), np.cross(-a2, a4)
                    cc = float(np.clip((u0 @ u1) / np.sqrt(float(u0 @ u0) * float(u1 @ u1)), -1, 1))
                    return sum(V[k] * (1 + S[k] * np.cos((k + 1) * np.arccos(cc))) for k in range(6))
                rows[t - ts, r, d] = (E(Xp) - E(Xm)) / (2 * h)
    G = np.zeros((n, 3))
    for a in range(n):
        r = base + a
        for k in range(arrs["fbinc_starts"][r], arrs["fbinc_starts"][r + 1]):
            o = arrs["fbinc_rec"][k:k + 1, 0].view(np.int32)[0]
            lb, ub, w = (float(v) for v in arrs["fbinc_rec"][k, 1:])
            df = X[a] - X[o]
            d = float(np.sqrt((df ** 2).sum() + 1e-12))
            pf = w * 2 * (d - lb) / d if d < lb else (w * 2 * (d - ub) / d if d > ub else 0.0)
            G[a] += pf * df
        for k in range(arrs["tinc_starts"][r], arrs["tinc_starts"][r + 1]):
            term, role = (int(v) for v in arrs["tinc_rec"][k])
            G[a] += rows[term - ts, role]
    return e, G.reshape(-1)


def test_device_layout_reproduces_the_oracle(dg_golden):
    b = _golden_batch3(dg_golden)
    arrs = etk_device_arrays(b)
    n_tor = len(b.etk_torsion_idx) + len(b.etk_improper_idx)
    assert len(arrs["tinc_rec"]) == 4 * n_tor and len(arrs["fbinc_rec"]) == 2 * len(arrs["fb_rec"])
    assert arrs["max_tor"] == max(np.diff(arrs["tor_starts"]))
    x = _positions(b, 9, 1.2)
    for conf in (0, 2, 5):
        e_ref, g_ref = dg.energy_grad(b, x, conf, stage="etk")
        e, g = _emulate_etk(arrs, x, int(b.conf_to_mol[conf]), int(b.conf_atom_starts[conf]))
        assert abs(e - e_ref) <= 1e-8 * max(1.0, abs(e_ref))
        np.testing.assert_allclose(g, g_ref, rtol=1e-5, atol=1e-5 * max(1.0, np.abs(g_ref).max()))


def test_patched_bounds_equal_a_fresh_layout(dg_golden):
    """The pipeline builds the ETK tables while the GPU runs DG and patches the re-centred 1-2 /
    1-3 bounds in afterwards; the patched tables equal tables built from the re-centred batch."""
    from mlxmolkit_b200.conformer_pipeline_v2 import _recenter_bounds
    from mlxmolkit_b200.shared_batch import patch_fb_bounds
    b = _golden_batch3(dg_golden)
    early = etk_device_arrays(b)
    _recenter_bounds(b, _positions(b, 12, 1.5).astype(np.float32))
    fresh = etk_device_arrays(b)
    assert not np.array_equal(early["fb_rec"], fresh["fb_rec"])
    patch_fb_bounds(early, b)
    for f in fresh:
        if isinstance(fresh[f], np.ndarray):
            assert np.array_equal(early[f].view(np.uint8), fresh[f].view(np.uint8)), f
        else:
            assert early[f] == fresh[f], f


def _empty_etk(n):
    z4, z6 = np.zeros((0, 4), np.int32), np.zeros((0, 6), np.float32)
    e, i = np.zeros(0, np.float32), np.zeros(0, np.int32)
    return ETKParams(n, z4, z6, np.zeros((0, 6), np.int32), z4, e, *([i, i, e, e, e] * 3))


def test_etk_layout_does_not_depend_on_the_thread_split(dg_golden):
    """Large batches build their tables as runs of molecules on host threads and merge them;
    every split gives the bytes of the one-run build, patch indices included."""
    from mlxmolkit_b200 import synth
    g = dg_golden
    dgp = [DGParams(n_atoms=len(g[f"s{mi}_elements"]), **{f: g[f"s{mi}_ref_{f}"] for f in PARAM_FIELDS})
           for mi in range(3)]
    etk = [ETKParams(n_atoms=len(g[f"s{mi}_elements"]), **{f: g[f"s{mi}_etk_{f}"] for f in ETK_FIELDS})
           for mi in range(3)]
    dist_b, _ = _distance_only_batch()
    mols = synth.make_molecules(20, 1, 13, 6, 14, workers=1)
    sp = [synth_dg_params(m) for m in mols]
    dgp = dgp[:2] + [all_pairs_dg(3), all_pairs_dg(4)] + dgp[2:] + sp
    etk = etk[:2] + [_one_etk(dist_b), _empty_etk(4)] + etk[2:] + [synth_etk_params(m, p.bounds_mat)
                                                                   for m, p in zip(mols, sp)]
    b = pack_shared_dg_batch(dgp, [1 + i % 3 for i in range(len(dgp))], dim=3)
    add_etk_to_batch(b, etk)
    one = etk_device_arrays(b, workers=1)
    from mlxmolkit_b200.shared_batch import _etk_runs
    for w in (2, 3, 5, 7):
        assert len(_etk_runs(b, w)) > 1
        got = etk_device_arrays(b, workers=w)
        assert set(got) == set(one)
        for f in one:
            if isinstance(one[f], np.ndarray):
                assert got[f].dtype == one[f].dtype, (w, f)
                assert np.array_equal(got[f].view(np.uint8), one[f].view(np.uint8)), (w, f)
            else:
                assert got[f] == one[f], (w, f)


def _one_etk(b):
    """The ETKParams of a one-molecule batch's etk_* fields."""
    return ETKParams(int(b.mol_n_atoms[0]), *[np.asarray(getattr(b, "etk_" + f)) for f in ETK_FIELDS])


def test_etk_device_layout_rejects_a_4d_batch(dg_golden):
    b = _golden_batch3(dg_golden)
    b.dim = 4
    with pytest.raises(ValueError):
        etk_device_arrays(b)
