import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import ORACLE_SO, Oracle
    if not ORACLE_SO.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True,
                       stdout=subprocess.DEVNULL)
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle_lib import Reference
    if not Reference.available():
        pytest.skip("TBTK reference subset not built (make -C oracle ref)")
    return Reference()


@pytest.fixture(scope="session")
def kpm():
    from tbtk_b200 import kpm as k
    if not k.LIB_PATH.exists():
        subprocess.run(["make", "-C", str(ROOT / "tbtk_b200" / "csrc")], check=True,
                       stdout=subprocess.DEVNULL)
    k.load_library()
    return k


@pytest.fixture(scope="session")
def gpu(kpm):
    if kpm.device_count() == 0:
        pytest.fail("GPU test without a CUDA device")
    return kpm


def golden(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def scaled_values(val, scale):
    """(v * complex(1/s, 0)) * complex(2, 0) with the reference's operation
    order (ChebyshevExpander.cpp:147,168), as numpy float64 operations."""
    a, b = val.real, val.imag
    inv = 1 / scale
    re = a * inv - b * 0.0
    im = a * 0.0 + b * inv
    re2 = re * 2.0 - im * 0.0
    im2 = re * 0.0 + im * 2.0
    return re2 + 1j * im2


def rel_err(x, ref):
    """Normwise error max|x - ref| / max|ref|."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    return float(np.abs(x - ref).max() / np.abs(ref).max())
