"""mmffb_minimize_noalloc (fixed device scratch, no allocation) against mmffb_minimize.

The fixed array keeps whatever the previous call left in it, so each parity
check first leaves it dirty itself -- a call on another batch ends with a
non-zero work counter, and a call whose bounded waits give up sets the error
word -- and the entry point must start both at zero again.  The file name also
sorts last, so in a full run it comes after every other GPU test.  (The
MMFFB_ESCRATCH branch, one inverse-Hessian slot larger than the array, cannot
be reached: the largest dense slot, 170 atoms in FP64, is 2 MiB of the 64.)
"""
import ctypes

import numpy as np
import pytest

from helpers import small_workload
from mlxmolkit_b200 import _lib
from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200 import synth
from mlxmolkit_b200.mmff_params import extract_mmff_params

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 64 << 20      # MMFFB_NOALLOC_SCRATCH_BYTES


def _large_batch(n_conf=160, seed=11):
    """One ~140-atom molecule, n_conf seeded perturbations of its embedded conformer."""
    mol = synth.make_molecules(1, 1, seed, 60, 66, workers=1, max_atoms=150)[0]
    p = extract_mmff_params(mol)
    base = mol.GetConformers()[0].pos.reshape(-1).astype(np.float32)
    rng = np.random.default_rng(seed)
    pos = np.concatenate([base + rng.normal(0, 0.05, base.size).astype(np.float32) for _ in range(n_conf)])
    return [p], [n_conf], pos


def _noalloc(m, pos_dev, opt):
    """One mmffb_minimize_noalloc call; returns (energy, status, iters, ls_evals)."""
    import torch
    L = _lib.load()
    C = m.confs.n_conf
    e = torch.empty(C, dtype=torch.float64, device="cuda")
    st = torch.empty(C, dtype=torch.int32, device="cuda")
    it = torch.empty(C, dtype=torch.int32, device="cuda")
    ev = torch.empty(C, dtype=torch.int32, device="cuda")
    bd, cd = m.batch.desc(), m.confs.desc()
    rc = L.mmffb_minimize_noalloc(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(opt), pos_dev.data_ptr(),
                                  e.data_ptr(), st.data_ptr(), it.data_ptr(), ev.data_ptr(),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, "mmffb_minimize_noalloc")
    return e, st, it, ev


def _scratch_bytes(m, opt):
    L = _lib.load()
    bd, cd = m.batch.desc(), m.confs.desc()
    return L.mmffb_minimize_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(opt))


def _dirty_the_array():
    """Leave the fixed array as an earlier caller might: a finished call on another batch
    (work counter at its conformer count plus its grid) and a call whose bounded waits gave
    up (error word set)."""
    import torch
    _, params, counts, pos = small_workload(n_mols=3, k=5, seed=41)
    m = mm.Minimizer(params, counts)
    x = torch.from_numpy(pos.astype(np.float32)).cuda()
    _noalloc(m, x, mm.opt_params(max_iters=20, grad_tol=1e-4))
    params, counts, pos = _large_batch(n_conf=8, seed=13)
    m = mm.Minimizer(params, counts)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.from_numpy(pos.astype(np.float32)).cuda()
    _, st, _, _ = _noalloc(m, x, mm.opt_params(max_iters=20, grad_tol=1e-4, give_up_waits=True,
                                               err_word=err.data_ptr()))
    torch.cuda.synchronize()
    assert int(err.item()) == 1 and bool((st == _lib.ST_TIMEOUT).all())


@pytest.mark.parametrize("case,precision", [("large", "mixed"), ("large", "fp64"), ("large", "fp32"),
                                            ("small", "mixed"), ("small", "fp32")])
def test_noalloc_matches_mmffb_minimize_over_two_calls_in_a_row(case, precision):
    import torch
    if case == "large":
        params, counts, pos = _large_batch()
    else:
        _, params, counts, pos = small_workload(n_mols=6, k=4, seed=21)
    m = mm.Minimizer(params, counts)
    kw = dict(max_iters=300, grad_tol=1e-4, precision=precision)
    if case == "large":
        # the planned grid's slots exceed the fixed array, so the grid shrinks
        assert _scratch_bytes(m, mm.opt_params(**kw)) > NOALLOC_BYTES
    start = torch.from_numpy(pos.astype(np.float32)).cuda()

    x_ref = start.clone()
    ev_ref = torch.empty(m.confs.n_conf, dtype=torch.int32, device="cuda")
    e_ref, st_ref, it_ref = m.minimize_device(x_ref, evals=ev_ref, **kw)

    _dirty_the_array()
    err = torch.full((1,), 5, dtype=torch.int32, device="cuda")
    opt = mm.opt_params(**kw, err_word=err.data_ptr())
    x1, x2 = start.clone(), start.clone()
    r1 = _noalloc(m, x1, opt)
    r2 = _noalloc(m, x2, opt)          # queued right behind the first on the same stream
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = [t.cpu().numpy() for t in (x_ref, e_ref, st_ref, it_ref, ev_ref)]
    for x, r in ((x1, r1), (x2, r2)):
        got = [t.cpu().numpy() for t in (x, *r)]
        for name, a, b in zip(("positions", "energy", "status", "iters", "ls_evals"), got, ref):
            assert np.array_equal(a, b), name
    assert np.isfinite(ref[1]).all()


def test_noalloc_empty_batch_is_a_no_op():
    import torch
    _, params, counts, _ = small_workload(n_mols=2, k=1, seed=3)
    m = mm.Minimizer(params, counts)
    L = _lib.load()
    bd = m.batch.desc()
    cd = _lib.MMFFConfDev(0, m.confs.max_atoms, m.confs.conf_mol.data_ptr(), m.confs.conf_coord.data_ptr(), 0)
    opt = mm.opt_params(max_iters=10, grad_tol=1e-4)
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = L.mmffb_minimize_noalloc(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(opt), dummy.data_ptr(),
                                  dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), None,
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.MMFFB_OK
    assert torch.count_nonzero(dummy).item() == 0
