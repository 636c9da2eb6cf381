"""The DG stage on the GPU (csrc/dg_kernels.cu through include/mmffb200_dg.h) against the FP64 oracle.

* energy and gradient of the kernel against oracle/dg_oracle.c (FP32 vs FP64,
  relative 1e-5 of the largest gradient component);
* the first L-BFGS iterations against the oracle's trajectory;
* full runs: the outcomes the reference's DG tests assert of its own kernel
  (tests/test_conformer_metal.py:108-260), and agreement with the oracle's
  statuses and energies;
* bit-identical results from run to run; thread counts change nothing but rounding.
"""
import numpy as np
import pytest

from helpers import all_pairs_dg, dg_synth_params
from mlxmolkit_b200.conformer_metal import dg_energy_grad, dg_minimize_shared
from mlxmolkit_b200.dg_extract import DGParams, metric_matrix_positions
from mlxmolkit_b200.shared_batch import init_random_positions, pack_shared_dg_batch
from oracle import dg

pytestmark = pytest.mark.gpu


def _synth_batch(dim=4, n_mols=4, k=3, seed=23, lo=8, hi=40):
    params = dg_synth_params(n_mols, seed, lo, hi)
    return pack_shared_dg_batch(params, [k] * n_mols, dim=dim), params


@pytest.mark.parametrize("dim", [4, 3])
def test_energy_and_gradient_match_the_oracle(dim):
    b, _ = _synth_batch(dim=dim)
    x = init_random_positions(b, seed=4) * np.float32(2.0)
    e, g = dg_energy_grad(b, x, chiral_weight=0.8, fourth_dim_weight=0.3)
    for c in range(b.n_confs_total):
        a0, a1 = int(b.conf_atom_starts[c]) * dim, int(b.conf_atom_starts[c + 1]) * dim
        e_ref, g_ref = dg.energy_grad(b, x.astype(np.float64), c, chiral_weight=0.8, fourth_dim_weight=0.3)
        assert abs(e[c] - e_ref) <= 1e-5 * max(1.0, abs(e_ref)), (c, e[c], e_ref)
        assert np.abs(g[a0:a1] - g_ref).max() <= 1e-5 * max(1.0, np.abs(g_ref).max()), c


def test_first_iterations_follow_the_oracle():
    b, _ = _synth_batch(k=2)
    x0 = init_random_positions(b, seed=9)
    for iters in (1, 3):
        xg, eg, sg = dg_minimize_shared(b, x0, max_iters=iters)
        xo, eo, so, _ = dg.minimize(b, x0, max_iters=iters)
        assert np.array_equal(sg, so)
        np.testing.assert_allclose(eg, eo, rtol=2e-4, atol=1e-4)
        np.testing.assert_allclose(xg, xo, rtol=0, atol=2e-3 * max(1.0, np.abs(xo).max()))


def test_reference_test_outcomes():
    """What tests/test_conformer_metal.py:115-239 asserts of the reference kernel."""
    b = pack_shared_dg_batch([all_pairs_dg(10)], [5], dim=4)
    _, e, s = dg_minimize_shared(b, init_random_positions(b, seed=42), max_iters=200)
    assert np.all(s == 0), s
    b = pack_shared_dg_batch([all_pairs_dg(8)], [3], dim=4)
    _, e, _ = dg_minimize_shared(b, init_random_positions(b, seed=99), max_iters=200)
    assert np.all(e < 1.0)
    b = pack_shared_dg_batch([all_pairs_dg(10)], [3], dim=4)
    x, _, _ = dg_minimize_shared(b, init_random_positions(b, seed=42), max_iters=200)
    c0, c1 = x[0:40], x[40:80]
    assert np.abs(c0 - c1).max() > 0.01
    b = pack_shared_dg_batch([all_pairs_dg(5), all_pairs_dg(8)], [3, 2], dim=4)
    _, e, s = dg_minimize_shared(b, init_random_positions(b, seed=7), max_iters=200)
    assert np.all(s == 0) and len(e) == 5
    b = pack_shared_dg_batch([all_pairs_dg(6)], [2], dim=4)
    x, _, _ = dg_minimize_shared(b, init_random_positions(b, seed=55), max_iters=300, fourth_dim_weight=1.0)
    assert np.abs(x.reshape(-1, 4)[:, 3]).max() < 2.0
    empty = DGParams(3, *[np.zeros(0, np.int32)] * 2, *[np.zeros(0, np.float32)] * 3, *[np.zeros(0, np.int32)] * 4,
                     np.zeros(0, np.float32), np.zeros(0, np.float32), np.arange(3, dtype=np.int32))
    b = pack_shared_dg_batch([empty], [2], dim=4)
    _, e, s = dg_minimize_shared(b, init_random_positions(b, seed=1), max_iters=50)
    assert len(e) == 2 and np.all(np.isfinite(e))
    b = pack_shared_dg_batch([all_pairs_dg(8), all_pairs_dg(6), all_pairs_dg(10)], [20, 20, 20], dim=4)
    _, e, s = dg_minimize_shared(b, init_random_positions(b, seed=42), max_iters=200)
    assert np.sum(s == 0) >= 55
    dgl = [all_pairs_dg(n) for n in [5, 8, 10, 6, 12, 7, 9, 4, 11, 8]]
    b = pack_shared_dg_batch(dgl, [10] * 10, dim=4)
    _, e, s = dg_minimize_shared(b, init_random_positions(b, seed=42), max_iters=200)
    assert np.sum(s == 0) >= 90


def test_full_runs_agree_with_the_oracle():
    """Synthetic molecules from metric-matrix starts, as the pipeline runs them: the same
    statuses for nearly all conformers, and energies that agree where both converged."""
    b, params = _synth_batch(n_mols=8, k=4, seed=31, lo=10, hi=45)
    bms = [p.bounds_mat for p in params]
    x0 = metric_matrix_positions(b, bms, seed=42, dim=4)
    cap = max(300, 300 + 20 * int(b.mol_n_atoms.max()))      # the pipeline's budget (conformer_pipeline_v2.py:123-166)
    _, eg, sg, ig = dg_minimize_shared(b, x0, max_iters=cap, return_iters=True)
    _, eo, so, io = dg.minimize(b, x0, max_iters=cap)
    assert np.mean(sg == so) >= 0.9
    both = (sg == 0) & (so == 0)
    assert both.mean() >= 0.8
    # DG minima are flat and FP32 / FP64 trajectories may settle in neighbouring basins:
    # a large majority agree closely, none by much
    d = np.abs(eg[both].astype(np.float64) - eo[both])
    assert np.median(d) <= 1e-4 and np.mean(d <= 2e-3) >= 0.9 and d.max() <= 0.05, d
    assert np.all((ig >= 1) & (ig <= cap))


def test_runs_are_bit_identical_and_thread_counts_agree():
    b, _ = _synth_batch(n_mols=3, k=4, seed=41, lo=20, hi=60)
    x0 = init_random_positions(b, seed=8)
    r1 = dg_minimize_shared(b, x0, max_iters=150)
    r2 = dg_minimize_shared(b, x0, max_iters=150)
    for a, c in zip(r1, r2):
        assert np.array_equal(a, c)
    ref = dg_minimize_shared(b, x0, max_iters=5, tpm=32)
    for tpm in (64, 128, 256):
        r = dg_minimize_shared(b, x0, max_iters=5, tpm=tpm)
        np.testing.assert_allclose(r[1], ref[1], rtol=1e-3, atol=1e-3)
        assert np.array_equal(r[2], ref[2])


def test_stereo_checks_match_the_reference(dg_golden):
    """The reference's own run_stereo_checks verdicts (stereo_checks_metal.py:102-141) on conformers
    as embedded, mirrored and flattened (tests/golden/ref_dg_batches.npz)."""
    from helpers import dg_golden_mol
    from mlxmolkit_b200.stereo_checks import run_stereo_checks
    fields = ("dist_idx1", "dist_idx2", "dist_lb2", "dist_ub2", "dist_weight", "chiral_idx1", "chiral_idx2",
              "chiral_idx3", "chiral_idx4", "chiral_vol_lower", "chiral_vol_upper", "fourth_idx")
    params = [DGParams(n_atoms=len(dg_golden[f"s{mi}_elements"]), **{f: dg_golden[f"s{mi}_ref_{f}"] for f in fields})
              for mi in range(3)]
    mols = [dg_golden_mol(dg_golden, mi) for mi in range(3)]
    b = pack_shared_dg_batch(params, [2, 3, 1], dim=4)
    got = run_stereo_checks(dg_golden["sy_stereo_pos4"], params, mols, b.conf_atom_starts, b.conf_to_mol,
                            [0, 1, 2], b.n_confs_total, dim=4)
    ref = dg_golden["sy_stereo_passed"]
    assert np.array_equal(got, ref) and (~ref).any() and ref.any()


def test_history_placement_changes_nothing():
    """The L-BFGS history in shared memory or in a device slot: the same arithmetic, bit-identical."""
    import torch
    from mlxmolkit_b200.conformer_metal import DGDeviceBatch
    b, _ = _synth_batch(n_mols=3, k=3, seed=43, lo=10, hi=30)
    x0 = init_random_positions(b, seed=12)
    out = []
    for hm in (1, 2):
        dev = DGDeviceBatch(b)
        pos = torch.from_numpy(x0.copy()).cuda()
        e, s = dev.minimize_device(pos, dev.params(300, 1e-4, 1.0, 0.1, hist_mode=hm))
        torch.cuda.synchronize()
        out.append((pos.cpu().numpy(), e.cpu().numpy(), s.cpu().numpy()))
    for a, c in zip(*out):
        assert np.array_equal(a, c)
