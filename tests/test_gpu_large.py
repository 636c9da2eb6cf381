"""CUDA kernels against the FP64 oracle at the large workload's sizes.

The large fixture (``tests/golden/ref_mmff_large.npz``, made by running the
reference's own extraction and numpy energy) holds molecules of 131 and 148
atoms -- the upper end of the 49-170-atom dense class, run by the
register-lean streamed instance in mixed precision -- and of 162, 178, 282
and 377 atoms, the L-BFGS sizes of the large workload (macrocycles and up to
20 rotatable bonds).  Every check goes through the C ABI.
"""
import numpy as np
import pytest

from helpers import golden_mol
from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200.mmff_params import extract_mmff_params
from oracle import oracle

pytestmark = pytest.mark.gpu

DENSE = [0, 1]            # 131, 148 atoms
LBFGS = [2, 3, 4, 5]      # 162, 178, 282, 377 atoms


def _batch(g, sel):
    mols = [golden_mol(g, mi) for mi in sel]
    params = [extract_mmff_params(m) for m in mols]
    pos = np.concatenate([g[f"m{mi}_pos"].reshape(-1) for mi in sel]).astype(np.float32)
    counts = [g[f"m{mi}_pos"].shape[0] for mi in sel]
    return params, counts, pos


def _split(params, counts, flat):
    out, o = [], 0
    for p, k in zip(params, counts):
        for _ in range(k):
            out.append(flat[o: o + 3 * p.n_atoms])
            o += 3 * p.n_atoms
    return out


def test_fixture_sizes(golden_large):
    params, _, _ = _batch(golden_large, DENSE + LBFGS)
    n = [p.n_atoms for p in params]
    assert all(111 < a <= 170 for a in n[:2]) and all(a >= 150 for a in n[2:]) and max(n) >= 350, n


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("fp32", 1e-4), ("fp64", 1e-11)])
def test_energy_and_gradient_match_the_oracle_at_large_sizes(golden_large, precision, tol):
    params, counts, pos = _batch(golden_large, DENSE + LBFGS)
    m = mm.Minimizer(params, counts)
    e, g = m.energy_grad(pos, precision=precision)
    pidx = np.repeat(np.arange(len(params)), counts)
    for c, (x, gg) in enumerate(zip(_split(params, counts, pos), _split(params, counts, g))):
        eo, go, _ = oracle.energy_grad(params[pidx[c]], x.astype(np.float64))
        assert abs(e[c] - eo) <= tol * max(1.0, abs(eo)), (c, e[c], eo)
        gt = 1e-6 if precision == "fp64" else 1e-4
        assert np.abs(gg - go).max() <= gt * max(1.0, np.abs(go).max()), c


@pytest.mark.parametrize("hist,sel", [(0, DENSE), (8, LBFGS), (8, [2, 3]), (8, [3, 4])])
def test_first_iterations_follow_the_oracle(golden_large, hist, sel):
    """Step by step: after 25 iterations the FP64 kernel's energies equal the FP64 oracle's to
    rounding and the mixed kernel's to FP32 accuracy.  Dense: the streamed global-slot
    instances.  Mixed L-BFGS, by the launch's atom bound: 377 atoms, 512 threads with the
    history in a global slot (one CTA of 16 warps per SM); 178, the register-capped instance
    with the history in shared memory; 282, the register-capped instance with the history in a
    global slot (two CTAs per SM)."""
    params, counts, pos = _batch(golden_large, sel)
    m = mm.Minimizer(params, counts)
    _, eo, _, io = oracle.minimize(params, counts, pos.astype(np.float64), max_iters=25, history_m=hist,
                                   consts=oracle.TG_CONSTS)
    r64 = m.minimize(pos, max_iters=25, history_m=hist, precision="fp64")
    np.testing.assert_allclose(r64.energies, eo, rtol=1e-7)
    assert np.array_equal(r64.iters, io)
    rmx = m.minimize(pos, max_iters=25, history_m=hist)
    np.testing.assert_allclose(rmx.energies, eo, rtol=2e-4)


def test_dense_lean_instance_reaches_the_fp64_minimum(golden_large):
    params, counts, pos = _batch(golden_large, DENSE)
    m = mm.Minimizer(params, counts)
    _, eo, so, _ = oracle.minimize(params, counts, pos.astype(np.float64), max_iters=4000,
                                   consts=oracle.RDKIT_CONSTS)
    assert np.isin(so, mm.CONVERGED_STATUSES).all()
    r64 = m.minimize(pos, max_iters=4000, precision="fp64", consts=mm.RDKIT_CONSTS)
    assert np.isin(r64.status, mm.CONVERGED_STATUSES).all()
    assert np.all(np.abs(r64.energies - eo) < 1e-3), r64.energies - eo
    r = m.minimize(pos, max_iters=1000)
    assert r.converged.all(), r.status
    assert np.all(np.abs(r.energies - eo) <= 0.1), r.energies - eo
    assert np.all(r.grad_rms_fp64 < 0.05), r.grad_rms_fp64

