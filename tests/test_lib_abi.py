"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = "".join(open(p).read() for p in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    return sorted(set(re.findall(r"\b(mmffb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = _declared()
    for n in ("mmffb_minimize", "mmffb_energy_grad", "mmffb_plain_minimize", "mmffb_fused_sd",
              "mmffb_dg_minimize", "mmffb_dg_energy_grad", "mmffb_dg_scratch_bytes"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from mlxmolkit_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmmffb200.so not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    for n in _declared():
        assert hasattr(L, n), n
    assert set(_declared()) == set(_lib.EXPORTS)
    lib = _lib.load()
    assert lib.mmffb_version() >= 1


def test_bad_arguments_are_reported_without_a_gpu():
    from mlxmolkit_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmmffb200.so not built")
    L = _lib.load()
    rc = L.mmffb_minimize(None, None, None, None, None, None, None, None, None, 0, None)
    assert rc == _lib.MMFFB_EINVAL
    assert b"null" in L.mmffb_last_error()


def test_dg_bad_arguments_are_reported_without_a_gpu():
    from mlxmolkit_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmmffb200.so not built")
    L = _lib.load()
    b = _lib.MMFFDGBatchDev()
    p = _lib.MMFFDGParams(max_iters=10, lbfgs_m=8, threads=0, grad_tol=1e-4, chiral_weight=1.0,
                          fourth_dim_weight=0.1)
    b.n_conf, b.dim, b.max_atoms = 1, 5, 10
    assert L.mmffb_dg_minimize(ctypes.byref(b), ctypes.byref(p), None, None, None, None, None, 0, None) \
        == _lib.MMFFB_EINVAL
    assert b"dim" in L.mmffb_last_error()
    b.dim, p.lbfgs_m = 4, 17
    assert L.mmffb_dg_energy_grad(ctypes.byref(b), ctypes.byref(p), None, None, None, None) == _lib.MMFFB_EINVAL
    assert b"lbfgs_m" in L.mmffb_last_error()
    p.lbfgs_m, b.max_atoms = 8, 2000
    assert L.mmffb_dg_scratch_bytes(ctypes.byref(b), ctypes.byref(p)) == 0
    assert b"max_atoms" in L.mmffb_last_error()
