import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "mlxmolkit-archive_b200"), ROOT, os.path.join(ROOT, "tests", "golden"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmmffb200.so")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_mmff_synth.npz"))


@pytest.fixture(scope="session")
def golden_large():
    """Molecules of 130-380 atoms: the dense class above 111 atoms and the L-BFGS sizes."""
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_mmff_large.npz"))


@pytest.fixture(scope="session", params=["drug", "large"])
def any_golden(request):
    """Each golden MMFF fixture in turn."""
    return request.getfixturevalue("golden" if request.param == "drug" else "golden_large")


@pytest.fixture(scope="session")
def dg_golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_dg_batches.npz"))


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """Build libmmffb200.so (nvcc, sm_100a) once if a fresh checkout has none: the packer's
    chunker and every GPU test load it."""
    so = os.path.join(ROOT, "mlxmolkit-archive_b200", "mlxmolkit_b200", "libmmffb200.so")
    if not os.path.exists(so) and shutil.which("nvcc"):
        subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(ROOT, "mlxmolkit-archive_b200", "csrc")])
