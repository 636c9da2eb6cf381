"""The FP64 oracle optimizer (TG-kernel semantics) behaves like an optimizer."""
import numpy as np

from helpers import golden_params
from oracle import oracle


def test_bfgs_lowers_energy_and_converges(golden):
    for mi in (0, 1, 2, 6):
        p = golden_params(golden, mi)
        pos = golden[f"m{mi}_pos"]
        x0 = pos.reshape(-1)
        e0 = [oracle.energy_grad(p, c)[0] for c in pos]
        x, e, st, it = oracle.minimize([p], [pos.shape[0]], x0, max_iters=2000, consts=oracle.RDKIT_CONSTS)
        assert np.all(e < np.array(e0))
        assert np.all(st != 1), st             # converged before the cap
        # the returned energy is the energy of the returned coordinates
        for c in range(pos.shape[0]):
            xc = x.reshape(pos.shape)[c]
            assert abs(oracle.energy_grad(p, xc, want_grad=False)[0] - e[c]) < 1e-9 * max(1, abs(e[c]))


def test_lbfgs_reaches_the_bfgs_minimum_on_rigid_molecules(golden):
    p = golden_params(golden, 0)
    pos = golden["m0_pos"]
    _, eb, _, _ = oracle.minimize([p], [3], pos.reshape(-1), max_iters=3000, consts=oracle.RDKIT_CONSTS)
    _, el, _, _ = oracle.minimize([p], [3], pos.reshape(-1), max_iters=3000, history_m=8,
                                  consts=oracle.RDKIT_CONSTS)
    assert np.all(np.abs(eb - el) < 0.1), (eb, el)


def test_max_iters_zero_returns_initial_energy(golden):
    p = golden_params(golden, 1)
    pos = golden["m1_pos"]
    x, e, st, it = oracle.minimize([p], [3], pos.reshape(-1), max_iters=0)
    for c in range(3):
        assert e[c] == oracle.energy_grad(p, pos[c], want_grad=False)[0]
    assert np.all(st == 1) and np.all(it == 0)
    assert np.array_equal(x, pos.reshape(-1))


def test_threads_do_not_change_results(golden):
    p = [golden_params(golden, mi) for mi in (0, 1, 6)]
    pos = np.concatenate([golden[f"m{mi}_pos"].reshape(-1) for mi in (0, 1, 6)])
    a = oracle.minimize(p, [3, 3, 3], pos, max_iters=300, n_threads=1)
    b = oracle.minimize(p, [3, 3, 3], pos, max_iters=300, n_threads=4)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_multimol_restatement_descends_and_records_convergence(golden):
    from helpers import golden_mol
    from mlxmolkit_b200.mmff_params import extract_mmff_params
    from oracle import multimol
    mols = [golden_mol(golden, mi) for mi in range(2)]
    params = [extract_mmff_params(m) for m in mols]
    counts = [m.GetNumConformers() for m in mols]
    x0 = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m in mols])
    r = multimol.multi_mol(params, counts, x0, max_iters=300, grad_tol=1e-3)
    e0, o = [], 0
    for p, k in zip(params, counts):
        for _ in range(k):
            e0.append(oracle.energy_grad(p, x0[o: o + 3 * p.n_atoms], mode=oracle.MODE_MEGA)[0])
            o += 3 * p.n_atoms
    assert np.all(r["energies"] <= np.array(e0) + 1e-9)
    assert np.all(r["per_conf_iters"][r["converged"]] <= r["n_iters"])
    assert r["n_iters"] % 10 == 0 or r["n_iters"] == 300
