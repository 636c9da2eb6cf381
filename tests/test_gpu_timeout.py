"""The bounded waits of the streamed inverse-Hessian pass, made to give up.

With ``give_up_waits=True`` every wait on a row copy gives up before testing,
as if its copy never completed.  No copy is broken: the copies in flight finish
normally and the kernel drains them before the CTA leaves.  The test checks
that the call returns, that every conformer has a defined result, that the
error word is set, and that the context stays usable for a normal run
afterwards.
"""
import numpy as np
import pytest

from mlxmolkit_b200 import _lib
from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200 import synth
from mlxmolkit_b200.mmff_params import extract_mmff_params

pytestmark = pytest.mark.gpu


def _streamed_batch(seed=31, n_mols=4, k=6):
    """Molecules of 60-110 atoms: the inverse Hessian sits in a global slot and is streamed
    (mixed precision above 48 atoms; FP64 when it exceeds shared memory)."""
    mols = synth.make_molecules(n_mols, k, seed, 28, 40, workers=1, max_atoms=120)
    params = [extract_mmff_params(m) for m in mols]
    assert min(p.n_atoms for p in params) > 58
    pos = np.concatenate([np.stack([c.pos for c in m.GetConformers()]).reshape(-1) for m in mols])
    return params, [k] * n_mols, pos.astype(np.float32)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_a_wait_that_gives_up_ends_the_call_cleanly(precision):
    import torch
    params, counts, pos = _streamed_batch()
    m = mm.Minimizer(params, counts)
    C = m.confs.n_conf
    start = torch.from_numpy(pos).cuda()
    kw = dict(max_iters=200, precision=precision)

    ref_x = start.clone()
    ref = m.minimize_device(ref_x, **kw)
    torch.cuda.synchronize()
    ref = [t.cpu().numpy() for t in ref]

    x = start.clone()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = (torch.full((C,), -1.0, dtype=torch.float64, device="cuda"),
           torch.full((C,), -7, dtype=torch.int32, device="cuda"),
           torch.full((C,), -7, dtype=torch.int32, device="cuda"))
    e, st, it = m.minimize_device(x, out=out, err=err, give_up_waits=True, **kw)
    torch.cuda.synchronize()
    e, st, it = e.cpu().numpy(), st.cpu().numpy(), it.cpu().numpy()
    assert int(err.item()) == 1
    # every conformer has a status of the documented set; the waits gave up at the
    # first streamed pass of every CTA, so none finished
    assert np.all(st == _lib.ST_TIMEOUT), np.bincount(st + 7)
    reached = ~np.isnan(e)
    assert np.all(it[~reached] == 0)
    # a conformer whose CTA gave up reports the iterate it reached and its energy
    xs = x.cpu().numpy()
    assert np.isfinite(xs).all()
    if reached.any():
        e2, _ = m.energy_grad(xs)
        np.testing.assert_allclose(e2[reached], e[reached], rtol=1e-6, atol=1e-4)

    # the context is still usable: a normal run gives the reference results bit for bit
    y = start.clone()
    again = m.minimize_device(y, err=err, **kw)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for a, b in zip([t.cpu().numpy() for t in again], ref):
        assert np.array_equal(a, b)
    assert np.array_equal(y.cpu().numpy(), ref_x.cpu().numpy())


def test_the_synchronous_call_raises_on_a_timeout():
    params, counts, pos = _streamed_batch(seed=33, n_mols=2, k=2)
    m = mm.Minimizer(params, counts)
    with pytest.raises(_lib.MMFFBError, match="bounded wait"):
        m.minimize(pos, max_iters=50, give_up_waits=True)
    r = m.minimize(pos, max_iters=50)
    assert np.isfinite(r.energies).all()


def test_binned_launches_report_the_error_word():
    import torch
    params, counts, pos = _streamed_batch(seed=35, n_mols=3, k=2)
    m = mm.BinnedMinimizer(params, counts)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.from_numpy(pos).cuda()
    _, st, _ = m.minimize_device(x, max_iters=50, err=err, give_up_waits=True)
    torch.cuda.synchronize()
    assert int(err.item()) == 1 and bool((st == _lib.ST_TIMEOUT).all())
    x = torch.from_numpy(pos).cuda()
    m.minimize_device(x, max_iters=50, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
