"""The ETK stage on the GPU (the ETK instance of csrc/dg_kernels.cu) against the FP64 oracle.

* energy and gradient against oracle/dg_oracle.c (FP32 vs FP64);
* the first iterations against the oracle's trajectory;
* the reference's consistency test: the returned energy is the objective at the
  returned positions (tests/test_etk_metal_consistency.py:90-105);
* the stages chained as the pipeline runs them (DG 4-D, collapse, 3-D ETK) on
  synthetic molecules, with the descent of the objective against the oracle's.
"""
import numpy as np
import pytest

from mlxmolkit_b200 import synth
from mlxmolkit_b200.conformer_metal import dg_minimize_shared
from mlxmolkit_b200.dg_extract import DGParams, metric_matrix_positions, synth_dg_params
from mlxmolkit_b200.etk_extract import ETKParams, synth_etk_params
from mlxmolkit_b200.etk_metal import etk_energy_grad, etk_minimize_shared
from mlxmolkit_b200.shared_batch import add_etk_to_batch, pack_shared_dg_batch
from oracle import dg

pytestmark = pytest.mark.gpu


def _etk_batch(n_mols=4, k=3, seed=29, lo=8, hi=35):
    mols = synth.make_molecules(n_mols, 1, seed, lo, hi, workers=1)
    dgp = [synth_dg_params(m) for m in mols]
    b3 = pack_shared_dg_batch(dgp, [k] * n_mols, dim=3)
    add_etk_to_batch(b3, [synth_etk_params(m, p.bounds_mat) for m, p in zip(mols, dgp)])
    x = np.concatenate([np.tile(m.GetConformers()[0].pos.reshape(-1), k) for m in mols]).astype(np.float32)
    return b3, dgp, x


def test_energy_and_gradient_match_the_oracle():
    b, _, x0 = _etk_batch()
    rng = np.random.default_rng(3)
    x = (x0 + rng.normal(0, 0.3, x0.shape)).astype(np.float32)
    e, g = etk_energy_grad(b, x)
    for c in range(b.n_confs_total):
        a0, a1 = int(b.conf_atom_starts[c]) * 3, int(b.conf_atom_starts[c + 1]) * 3
        e_ref, g_ref = dg.energy_grad(b, x.astype(np.float64), c, stage="etk")
        assert abs(e[c] - e_ref) <= 2e-5 * max(1.0, abs(e_ref)), (c, e[c], e_ref)
        assert np.abs(g[a0:a1] - g_ref).max() <= 1e-4 * max(1.0, np.abs(g_ref).max()), c


def test_first_iterations_follow_the_oracle():
    b, _, x0 = _etk_batch(k=2)
    rng = np.random.default_rng(4)
    x = (x0 + rng.normal(0, 0.2, x0.shape)).astype(np.float32)
    for iters in (1, 3):
        xg, eg, sg = etk_minimize_shared(b, x, max_iters=iters)
        xo, eo, so, _ = dg.minimize(b, x, max_iters=iters, stage="etk")
        assert np.array_equal(sg, so)
        np.testing.assert_allclose(eg, eo, rtol=1e-3, atol=1e-3)
        np.testing.assert_allclose(xg, xo, rtol=0, atol=2e-3 * max(1.0, np.abs(xo).max()))


def test_reference_consistency_case():
    """tests/test_etk_metal_consistency.py:13-105 of the reference, on the GPU."""
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
    x = np.array([0, 0, 0, 2, 0, 0, 3, 0, 0], np.float32)
    out, energy, _ = etk_minimize_shared(b, x, max_iters=1)
    _, recomputed, _ = etk_minimize_shared(b, out, max_iters=0)
    np.testing.assert_allclose(energy, recomputed, atol=1e-4)


def test_pipeline_stages_chain_and_agree_with_the_oracle():
    """DG 4-D -> collapse -> 3-D ETK, the budgets of conformer_pipeline_v2.py:162-170."""
    mols = synth.make_molecules(6, 1, 37, 10, 30, workers=1)
    dgp = [synth_dg_params(m) for m in mols]
    k = 4
    b4 = pack_shared_dg_batch(dgp, [k] * len(mols), dim=4)
    x4 = metric_matrix_positions(b4, [p.bounds_mat for p in dgp], seed=42, dim=4)
    n_max = int(b4.mol_n_atoms.max())
    x4, _, s4 = dg_minimize_shared(b4, x4, max_iters=max(300, 300 + 20 * n_max))
    x4, _, _ = dg_minimize_shared(b4, x4, max_iters=200, fourth_dim_weight=1.0, chiral_weight=0.2)
    assert np.mean(s4 == 0) >= 0.9
    x3 = x4.reshape(-1, 4)[:, :3].reshape(-1).copy()
    b3 = pack_shared_dg_batch(dgp, [k] * len(mols), dim=3)
    add_etk_to_batch(b3, [synth_etk_params(m, p.bounds_mat) for m, p in zip(mols, dgp)])
    cap = max(150, 150 + 10 * n_max)
    xg, eg, sg = etk_minimize_shared(b3, x3, max_iters=cap)
    xo, eo, so, _ = dg.minimize(b3, x3, max_iters=cap, stage="etk")
    e0 = np.array([dg.energy_grad(b3, x3.astype(np.float64), c, stage="etk")[0] for c in range(b3.n_confs_total)])
    assert np.all(eg <= e0 + 1e-3)                       # the refinement never raises the objective
    # stiff flat-bottom terms (force constant 100) leave many conformers at the reference's
    # iteration budget in both runs; what both must show is the same descent
    assert np.all(eg <= 0.1 * e0) and np.all(eo <= 0.1 * e0)
    ratio = (eg.astype(np.float64) + 1e-3) / (eo + 1e-3)
    assert 0.5 <= np.median(ratio) <= 2.0, ratio
    # statuses are not compared: on these stiff terms an FP32 run reaches the relative-step
    # (TOLX) exit where the FP64 run keeps descending to the budget
    assert set(np.unique(sg)) <= {0, 1}


def test_refreshed_bounds_equal_a_fresh_upload():
    """The pipeline uploads the ETK tables while DG runs and writes the re-centred 1-2 / 1-3
    bounds in afterwards (ETKDeviceBatch.refresh_bounds): the device tables then equal those of
    a batch uploaded after the re-centring."""
    import torch
    from mlxmolkit_b200.conformer_pipeline_v2 import _recenter_bounds
    from mlxmolkit_b200.etk_metal import ETKDeviceBatch
    b, _, x = _etk_batch(n_mols=5, k=2)
    early = ETKDeviceBatch(b)
    _recenter_bounds(b, (x + np.random.default_rng(8).normal(0, 0.2, x.shape)).astype(np.float32))
    early.refresh_bounds()
    fresh = ETKDeviceBatch(b)
    torch.cuda.synchronize()
    for f in ("fb_rec", "fbinc_rec"):
        assert torch.equal(early.dev[f].view(torch.int32), fresh.dev[f].view(torch.int32)), f
    eg, _ = early.energy_grad_device(torch.from_numpy(x).cuda(), early.params(0, 0.0, 0.0, 0.0))
    ef, _ = fresh.energy_grad_device(torch.from_numpy(x).cuda(), fresh.params(0, 0.0, 0.0, 0.0))
    assert torch.equal(eg, ef)
