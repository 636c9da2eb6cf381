"""The C-ABI library loads and exports every entry point include/mmffb200.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "mmffb200.h")).read()
    return sorted(set(re.findall(r"\b(mmffb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = _declared()
    for n in ("mmffb_minimize", "mmffb_energy_grad", "mmffb_plain_minimize", "mmffb_fused_sd"):
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
