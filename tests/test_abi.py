"""CPU tests of the C ABI: the library loads, exports every entry point the
header declares, and rejects bad arguments with a status (never exits)."""
import re

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    text = (ROOT / "include" / "tbtkkpm.h").read_text()
    return sorted(set(re.findall(r"TBTKKPM_API\s+[\w\s\*]*?\b(tbtkkpm_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "tbtkkpm_moments" in syms and "tbtkkpm_ldos_sites" in syms
    assert len(syms) >= 17


def test_library_exports_every_header_symbol(kpm):
    lib = kpm.load_library()
    for name in header_symbols():
        assert hasattr(lib, name), name
    bound = {n for n, _, _ in kpm.SIGNATURES}
    assert set(header_symbols()) <= bound


def test_version_and_no_device_on_cpu(kpm):
    lib = kpm.load_library()
    assert lib.tbtkkpm_version() == 10000
    assert isinstance(kpm.device_count(), int)


def test_argument_errors_return_status(kpm):
    """Checks that run before any device work: bad scale, bad CSR."""
    rowptr = np.array([0, 1, 2], dtype=np.uint32)
    col = np.array([1, 0], dtype=np.uint32)
    val = np.array([1.0, 1.0], dtype=np.complex128)
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Matrix.from_csr(rowptr, col, val, 0.0)
    assert e.value.status == kpm.ERR_ARGUMENT
    assert "scaleFactor" in str(e.value)
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Matrix.from_csr(rowptr, np.array([1, 5], dtype=np.uint32), val, 10.0)
    assert e.value.status == kpm.ERR_ARGUMENT
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Matrix.from_csr(np.array([0, 2, 2], dtype=np.uint32),
                            np.array([1, 0], dtype=np.uint32), val, 10.0)
    assert e.value.status == kpm.ERR_ARGUMENT and "ascending" in str(e.value)
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Table.create(10, np.array([-10.0, 0.0]), 10.0)
    assert e.value.status == kpm.ERR_ARGUMENT
    for bad in (np.nan, np.inf):
        with pytest.raises(kpm.TBTKError) as e:
            kpm.Matrix.from_csr(rowptr, col, np.array([1.0, complex(0.5, bad)]), 10.0)
        assert e.value.status == kpm.ERR_ARGUMENT and "not finite" in str(e.value)
        with pytest.raises(kpm.TBTKError) as e:
            kpm.Matrix.from_triplets(np.array([0, 1]), np.array([1, 0]),
                                     np.array([bad, 1.0], dtype=np.complex128), 2, 10.0)
        assert e.value.status == kpm.ERR_ARGUMENT and "not finite" in str(e.value)
    for M, E, s in ((0, 64, 10.0), (10, 0, 10.0), (10, 48, 10.0), (10, 8192, 10.0),
                    (10, 64, 0.0), (10, 64, -1.0)):
        with pytest.raises(kpm.TBTKError) as e:
            kpm.Table.create_chebyshev(M, E, s)
        assert e.value.status == kpm.ERR_ARGUMENT, (M, E, s)
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Table.create_chebyshev(10, 6, 10.0)
    assert "power of two" in str(e.value)
    lib = kpm.load_library()
    assert lib.tbtkkpm_matrix_set_batch_width(None, kpm.MIXED, 64) == kpm.ERR_ARGUMENT
    assert lib.tbtkkpm_matrix_set_batch_width(None, 7, 64) == kpm.ERR_ARGUMENT
    assert "precision" in lib.tbtkkpm_last_error().decode()


def test_solver_setters_mirror_reference(kpm):
    """Defaults and setter checks of Solver::ChebyshevExpander
    (Test/include/TBTK/Test/Solver/ChebyshevExpander.h:35-137)."""
    s = kpm.ChebyshevExpander()
    assert s.getScaleFactor() == 1.1
    assert s.getNumCoefficients() == 1000
    assert s.getBroadening() == 1e-6
    assert np.array_equal(s.getEnergyWindow(), kpm.tbtk_range(-1, 1, 1000))
    for bad in (0, -1):
        with pytest.raises(kpm.TBTKError):
            s.setScaleFactor(bad)
    s.setScaleFactor(10)
    s.setEnergyWindow(kpm.tbtk_range(-9.999, 9.999, 10))
    with pytest.raises(kpm.TBTKError):
        s.setEnergyWindow(kpm.tbtk_range(-10, 9.999, 10))
    with pytest.raises(kpm.TBTKError):
        s.setEnergyWindow(kpm.tbtk_range(-9.999, 10, 10))
    s.setNumCoefficients(2000)
    assert s.getNumCoefficients() == 2000
    s.setBroadening(0.01)
    assert s.getBroadening() == 0.01
