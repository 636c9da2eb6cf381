"""The reference-facing Python surface on the GPU: multi_mol, fused, mmff_minimize_nk, the pipeline.

multi_mol is checked against the FP64 restatement of the reference's own loop
(oracle/multimol.py): step by step on a short run, at the minima on a full
run; and for the behaviours the reference's tests pin
(tests/test_metal_multi_mol_convergence.py in the reference).
"""
import numpy as np
import pytest

from helpers import golden_mol
from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200 import synth
from mlxmolkit_b200.mmff_metal_optimizer import (mmff_optimize_metal_fused_multi_mol,
                                                 mmff_optimize_metal_multi_mol)
from mlxmolkit_b200.mmff_params import extract_mmff_params
from oracle import multimol, oracle

pytestmark = pytest.mark.gpu


def _golden_specs(golden, n=3):
    return [(golden_mol(golden, mi), None) for mi in range(n)]


def _flat(specs):
    return np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m, _ in specs])


def _run_both(specs, **kw):
    params = [extract_mmff_params(m) for m, _ in specs]
    counts = [m.GetNumConformers() for m, _ in specs]
    x0 = _flat(specs).astype(np.float32).astype(np.float64)
    ref = multimol.multi_mol(params, counts, x0, **kw)
    got = mmff_optimize_metal_multi_mol(specs, **kw)
    return ref, got, params, counts


def test_multi_mol_follows_the_restated_reference_step_by_step(golden):
    specs = _golden_specs(golden)
    ref, got, params, counts = _run_both(specs, max_iters=8, eval_freq=4)
    c = 0
    for mr, p in zip(got.mol_results, params):
        for k in range(mr.n_conformers):
            d = ref["dims"][c]
            assert np.abs(mr.positions[k].reshape(-1) - ref["positions"][c, :d]).max() < 2e-3
            assert abs(mr.energies[k] - ref["energies"][c]) <= 1e-3 * max(1.0, abs(ref["energies"][c]))
            assert abs(mr.grad_norms[k] - ref["grad_norms"][c]) <= 1e-3 * max(1.0, ref["grad_norms"][c])
            c += 1
        assert mr.n_iters == ref["n_iters"]


def test_multi_mol_full_run_reaches_the_restatement_minima(golden):
    """Run to convergence: most conformers end on the restatement's minimum to rounding.  Without
    a line search, FP32 and FP64 trajectories of a flexible conformer can settle in different
    basins (lower or higher), so the bar is a large majority, not all."""
    specs = _golden_specs(golden, 6)
    ref, got, params, counts = _run_both(specs, max_iters=1000, grad_tol=1e-3)
    e_got = np.concatenate([r.energies for r in got.mol_results]).astype(np.float64)
    d = np.abs(e_got - ref["energies"])
    assert np.mean(d <= 1e-2) >= 0.7, d
    conv = np.concatenate([r.converged for r in got.mol_results])
    assert abs(conv.mean() - ref["converged"].mean()) <= 0.2
    x0 = _flat(specs).astype(np.float64)
    e0, o = [], 0
    for p, k in zip(params, counts):
        for _ in range(k):
            e0.append(oracle.energy_grad(p, x0[o: o + 3 * p.n_atoms], mode=oracle.MODE_MEGA)[0])
            o += 3 * p.n_atoms
    assert np.all(e_got <= np.array(e0) + 1e-3)     # the best-seen guard never returns a worse point


def _small_specs(n=4, k=3, seed=61):
    mols = synth.make_molecules(n, k, seed, 6, 14, workers=1)
    return [(m, None) for m in mols]


def test_multi_mol_reference_behaviours():
    specs = _small_specs()
    r1 = mmff_optimize_metal_multi_mol(specs, max_iters=1000, grad_tol=1e-3)
    for mr, (mol, _) in zip(r1.mol_results, specs):
        assert mr.converged.all()
        assert np.array_equal(mr.converged, mr.grad_norms <= 1e-3)
        assert np.all(mr.per_conf_iters <= mr.n_iters) and mr.n_iters % 10 == 0
        assert mr.energies.dtype == np.float32 and mr.positions.shape == (mr.n_conformers, mol.GetNumAtoms(), 3)
        # written back into the molecule's conformers
        assert np.allclose(np.stack([c.pos for c in mol.GetConformers()]), mr.positions)
    # raising the cap past convergence does not change the answer
    specs2 = _small_specs()
    r2 = mmff_optimize_metal_multi_mol(specs2, max_iters=2000, grad_tol=1e-3)
    for a, b in zip(r1.mol_results, r2.mol_results):
        assert np.array_equal(a.energies, b.energies) and np.array_equal(a.positions, b.positions)
    # grad_tol = 0: never converged, per-conformer iterations = max_iters
    r0 = mmff_optimize_metal_multi_mol(_small_specs(), max_iters=40, grad_tol=0.0)
    for mr in r0.mol_results:
        assert not mr.converged.any() and np.all(mr.per_conf_iters == 40) and mr.n_iters == 40


def test_multi_mol_conf_ids_select_conformers():
    mol = _small_specs(1, 4)[0][0]
    before = np.stack([c.pos.copy() for c in mol.GetConformers()])
    r = mmff_optimize_metal_multi_mol([(mol, [1, 3])], max_iters=200)
    after = np.stack([c.pos for c in mol.GetConformers()])
    assert r.mol_results[0].n_conformers == 2
    assert np.array_equal(after[[0, 2]], before[[0, 2]]) and not np.array_equal(after[1], before[1])


def test_fused_multi_mol_reports_like_the_reference():
    specs = _small_specs(3, 2, seed=67)
    params = [extract_mmff_params(m) for m, _ in specs]
    e0 = [oracle.energy_grad(p, c.pos.reshape(-1), mode=oracle.MODE_MEGA)[0]
          for p, (m, _) in zip(params, specs) for c in m.GetConformers()]
    r = mmff_optimize_metal_fused_multi_mol(specs, max_iters=300)
    e = np.concatenate([mr.energies for mr in r.mol_results])
    for mr in r.mol_results:
        assert np.all(mr.grad_norms == 0) and mr.n_iters == 300
    assert np.all(e <= np.array(e0) + 1.0)          # the +1 kcal/mol guard


def test_mmff_minimize_nk_drop_in():
    mols = synth.make_molecules(3, 2, 71, 8, 20, workers=1)
    params = [extract_mmff_params(m) for m in mols]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m in mols]).astype(np.float32)
    x, e, conv = mm.mmff_minimize_nk(params, [2, 2, 2], pos, max_iters=500)
    assert x.dtype == np.float32 and x.shape == pos.shape
    assert e.dtype == np.float32 and e.shape == (6,) and conv.dtype == bool and conv.all()
    r = mm.Minimizer(params, [2, 2, 2]).minimize(pos, max_iters=500)
    assert np.allclose(e, r.energies.astype(np.float32), rtol=0, atol=1e-3)
    x2, e2, conv2 = mm.mmff_minimize_nk(params, [2, 2, 2], pos, max_iters=500, use_lbfgs=True)
    assert np.isfinite(e2).all() and conv2.mean() >= 0.5


def test_pipelined_call_equals_one_launch_per_size_class():
    """mmff_minimize_nk packs and launches chunk by chunk (the largest molecules first, their
    class split in two); every conformer's result is bit-identical to BinnedMinimizer's one
    launch per size class, in the caller's conformer order, zero-conformer molecules included."""
    mols = synth.make_molecules(130, 2, 75, 6, 50, workers=1, max_atoms=150)
    params = [extract_mmff_params(m) for m in mols]
    counts = [0 if i == 7 else 2 for i in range(len(mols))]
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()][:k]).reshape(-1)
                          for m, k in zip(mols, counts) if k]).astype(np.float32)
    n = np.array([p.n_atoms for p in params])
    chunks = mm.launch_chunks(n, counts)
    assert len(chunks) == 4 and 7 not in np.concatenate(chunks)     # 49-150 atoms split in two
    x, e, conv, r = mm.mmff_minimize_nk(params, counts, pos, max_iters=300, return_result=True)
    assert r.timings["launch_chunks"] == len(chunks)
    b = mm.BinnedMinimizer(params, counts).minimize(pos, max_iters=300)
    assert np.array_equal(x, b.positions)
    assert np.array_equal(r.energies, b.energies)
    assert np.array_equal(r.status, b.status) and np.array_equal(r.iters, b.iters)
    assert np.array_equal(r.energies_fp64, b.energies_fp64)
    assert np.array_equal(conv, b.converged)
    # L-BFGS: the planner picks its instance (history in shared memory or not, register-capped
    # or not) from the class's atom bound, so the chunk of smaller molecules runs the same one
    x, e, conv, r = mm.mmff_minimize_nk(params, counts, pos, max_iters=300, use_lbfgs=True, return_result=True)
    b = mm.BinnedMinimizer(params, counts).minimize(pos, max_iters=300, history_m=mm.LBFGS_M)
    assert np.array_equal(x, b.positions) and np.array_equal(r.energies, b.energies)
    assert np.array_equal(r.status, b.status) and np.array_equal(r.iters, b.iters)


def test_generate_conformers_nk_runs_the_mmff_stage():
    from mlxmolkit_b200.conformer_pipeline_v2 import generate_conformers_nk
    mols = synth.make_molecules(3, 3, 73, 8, 20, workers=1)
    bad = mols[0].copy()
    bad.types[0] = "XX"                               # untypable: marked unconverged, batch goes on
    res = generate_conformers_nk(mols + [bad], 3, run_mmff=True, mmff_max_iters=500, embed="host")
    assert res.total_conformers == 12
    for r, m in zip(res.molecules[:3], mols):
        assert all(r.converged) and np.isfinite(r.energies).all()
        assert not np.allclose(r.positions_3d[0], m.GetConformers()[0].pos)
    assert not any(res.molecules[3].converged)


def test_generate_conformers_nk_embeds_on_the_device():
    """DG -> collapse -> ETK -> MMFF, all on the GPU: distinct conformers with sane geometry, the
    reference's convergence rule (every stage converged, conformer_pipeline_v2.py:337-341)."""
    from mlxmolkit_b200.conformer_pipeline_v2 import generate_conformers_nk
    mols = synth.make_molecules(4, 1, 79, 8, 22, workers=1)
    res = generate_conformers_nk(mols, 5, run_mmff=True)
    assert res.total_conformers == 20
    conv = np.concatenate([r.converged for r in res.molecules])
    assert conv.mean() >= 0.75
    for r, m in zip(res.molecules, mols):
        assert len(r.positions_3d) == 5 and np.isfinite(r.energies).all()
        x = np.stack(r.positions_3d)
        assert np.abs(x[0] - x[1]).max() > 0.05                      # independent conformers
        for b in m.GetBonds():                                       # MMFF bond lengths, not the generator's
            i, j = b.GetBeginAtomIdx(), b.GetEndAtomIdx()
            d = np.linalg.norm(x[:, i] - x[:, j], axis=1)
            assert np.all((d > 0.9) & (d < 2.0)) and np.ptp(d) < 0.05, (i, j, d)
    # embedding alone: DG + ETK energies, no MMFF
    res0 = generate_conformers_nk(mols, 5, run_mmff=False)
    e0 = np.concatenate([r.energies for r in res0.molecules])
    e1 = np.concatenate([r.energies for r in res.molecules])
    assert np.isfinite(e0).all() and not np.allclose(e0, e1)
