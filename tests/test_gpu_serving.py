"""Continuous-batching server: slot-level admission into running launches, the same result alone
and in a mix for every size class (the L-BFGS ones included), admission by budget, errors."""
import time

import numpy as np
import pytest

from mlxmolkit_b200 import synth

pytestmark = pytest.mark.gpu


def _mols(n=6, k=3, seed=31, lo=8, hi=40, max_atoms=None):
    return synth.make_molecules(n, k, seed, lo, hi, workers=1, max_atoms=max_atoms)


def _mixed_classes():
    """Molecules of every size class: <= 24, 25-48, 49-149 atoms (dense BFGS), 150-170 and
    171-288 (L-BFGS)."""
    small = _mols(n=3, k=3, seed=31, lo=4, hi=7)
    mid = _mols(n=3, k=3, seed=32, lo=10, hi=16)
    dense = _mols(n=3, k=2, seed=33, lo=30, hi=55, max_atoms=149)
    large = synth.make_molecules(2, 2, 34, 64, 76, workers=1, max_atoms=260)
    larger = synth.make_molecules(1, 2, 37, 80, 95, workers=1, max_atoms=300)
    return small + mid + dense + large + larger


def test_each_result_is_the_same_alone_and_in_the_mix_in_every_size_class():
    from mlxmolkit_b200.serve import MMFFServer, size_class
    from mlxmolkit_b200.mmff_params import extract_mmff_params
    mols = _mixed_classes()
    n = [extract_mmff_params(m).n_atoms for m in mols]
    classes = {size_class(a, 10).key[:2] for a in n}
    assert {("dense", 24), ("dense", 48), ("dense", 149), ("lbfgs", 170), ("lbfgs", 288)} <= classes, n
    alone = []
    srv = MMFFServer(hbm_budget_bytes=2 << 30)
    for m in mols:
        alone.append(srv.submit(m, max_iters=400).result(timeout=300))
    srv.close()
    srv = MMFFServer(hbm_budget_bytes=2 << 30)
    futs = [srv.submit(m, max_iters=400) for m in reversed(mols)]
    mixed = [f.result(timeout=300) for f in futs][::-1]
    srv.close()
    for a, b in zip(alone, mixed):
        assert np.array_equal(a.energies, b.energies)
        assert np.array_equal(a.positions, b.positions)
        assert np.array_equal(a.status, b.status)
    assert all(np.isfinite(r.energies).all() for r in alone)


def test_requests_join_the_running_launch():
    """Requests submitted while a long one runs are admitted into the same worker launch: its
    free CTAs take their slots while the first request is still on the GPU."""
    from mlxmolkit_b200.serve import MMFFServer
    big, other = synth.make_molecules(2, [8, 2], 34, 64, 76, workers=1, max_atoms=260)   # L-BFGS class
    # the first launch keeps 56 spare CTAs polling (64 CTAs for 8 conformers) for up to 3 s
    srv = MMFFServer(hbm_budget_bytes=2 << 30, worker_idle_ms=3000.0, min_worker_ctas=64)
    f_big = srv.submit(big, max_iters=3000)
    time.sleep(0.01)
    f_other = srv.submit(other, max_iters=3000)
    r_other = f_other.result(timeout=300)
    r_big = f_big.result(timeout=300)
    launches = {cs.key: cs.launches for cs in srv.classes.values()}
    srv.close()
    assert r_big.t_admit < r_other.t_admit < r_big.t_done      # admitted while the first one ran
    assert launches == {k: 1 for k in launches} and len(launches) == 1, launches
    # and its result is the one it gets alone
    srv = MMFFServer(hbm_budget_bytes=2 << 30)
    alone = srv.submit(other, max_iters=3000).result(timeout=300)
    srv.close()
    assert np.array_equal(alone.energies, r_other.energies) and np.array_equal(alone.positions, r_other.positions)


def test_requests_overlap_on_the_device():
    from mlxmolkit_b200.serve import MMFFServer
    mols = _mols(n=8, k=4, seed=33)
    srv = MMFFServer(hbm_budget_bytes=1 << 30)
    futs = [srv.submit(m) for m in mols]
    res = [f.result(timeout=120) for f in futs]
    srv.close()
    spans = sorted((r.t_admit, r.t_done) for r in res)
    overlapping = sum(1 for (a0, a1), (b0, b1) in zip(spans, spans[1:]) if b0 < a1)
    assert overlapping >= 1
    assert all(r.converged.mean() > 0.5 for r in res)


def test_request_over_the_budget_is_refused():
    from mlxmolkit_b200.serve import MMFFServer
    m = _mols(n=1, k=2)[0]
    srv = MMFFServer(hbm_budget_bytes=1 << 12)
    with pytest.raises(MemoryError):
        srv.submit(m).result(timeout=60)
    srv.close()


def test_untypable_molecule_fails_only_its_request():
    from mlxmolkit_b200.serve import MMFFServer
    good = _mols(n=1, k=2)[0]
    bad = good.copy()
    bad.types[0] = "XX"                      # no parameters for this type
    srv = MMFFServer(hbm_budget_bytes=1 << 30)
    fb, fg = srv.submit(bad), srv.submit(good)
    with pytest.raises(Exception):
        fb.result(timeout=60)
    assert fg.result(timeout=120).converged.all()
    srv.close()


def test_generations_switch_halves_when_the_arena_is_full():
    """A small arena forces the class onto its other half and back; results stay identical to
    a server with room to spare."""
    from mlxmolkit_b200.serve import MMFFServer
    mols = _mols(n=10, k=3, seed=51, lo=8, hi=14)
    srv = MMFFServer(hbm_budget_bytes=1 << 30, max_slots_per_half=8)
    small = [f.result(timeout=120) for f in [srv.submit(m, max_iters=300) for m in mols]]
    srv.close()
    srv = MMFFServer(hbm_budget_bytes=1 << 30)
    roomy = [f.result(timeout=120) for f in [srv.submit(m, max_iters=300) for m in mols]]
    srv.close()
    for a, b in zip(small, roomy):
        assert np.array_equal(a.energies, b.energies) and np.array_equal(a.positions, b.positions)
