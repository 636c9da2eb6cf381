"""Continuous-batching server: same result alone and in a mix, admission by budget, errors."""
import numpy as np
import pytest

from mlxmolkit_b200 import synth

pytestmark = pytest.mark.gpu


def _mols(n=6, k=3, seed=31):
    return synth.make_molecules(n, k, seed, 8, 40, workers=1)


def test_each_result_is_the_same_alone_and_in_the_mix():
    from mlxmolkit_b200.serve import MMFFServer
    mols = _mols()
    alone = []
    srv = MMFFServer(hbm_budget_bytes=1 << 30)
    for m in mols:
        alone.append(srv.submit(m).result(timeout=120))
    srv.close()
    srv = MMFFServer(hbm_budget_bytes=1 << 30)
    futs = [srv.submit(m, variant="MMFF94") for m in mols]
    mixed = [f.result(timeout=120) for f in futs]
    srv.close()
    for a, b in zip(alone, mixed):
        assert np.array_equal(a.energies, b.energies)
        assert np.array_equal(a.positions, b.positions)


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
