"""Spin-polarized LDOS, density, magnetization and expectation values through
the C ABI (tbtkkpm_spin_polarized_ldos, _density, _magnetization,
_expectation_values) against TBTK's PropertyExtractor results
(tests/golden/props.npz, generated by the reference).

Tolerances: FP64 with the lookup table built on the host (the oracle's,
which equals the reference's) is compared bit for bit; with the table built
on the device (CUDA acos/sincos) normwise, max|x - ref| / max|ref| <= 1e-12;
the MIXED precision (complex64 vectors) normwise <= 1e-6, the path's
stated target.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


def _setup(gpu, oracle, host_table):
    g = golden("props")
    s, M = float(g["scale"]), int(g["M"])
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    if host_table:
        t = gpu.Table.upload(oracle.lookup_table(M, g["energies"], s))
    else:
        t = gpu.Table.create(M, g["energies"], s)
    return g, m, t


@pytest.mark.parametrize("host_table", [True, False])
def test_properties_fp64(gpu, oracle, host_table):
    g, m, t = _setup(gpu, oracle, host_table)
    bro, occ, dE = float(g["broadening"]), g["occupation"], float(g["dE"])
    sp = m.spin_polarized_ldos(t, g["sp_up"], g["sp_down"], bro)
    mag = m.magnetization(t, g["sp_up"], g["sp_down"], bro, occ, dE)
    dens = m.density(t, g["density_sites"], bro, occ, dE)
    ev = m.expectation_values(t, g["exp_to"], g["exp_from"], bro, occ, dE)
    if host_table:
        assert np.array_equal(sp, g["sp_ldos"])
        assert np.array_equal(mag, g["magnetization"])
        assert np.array_equal(dens, g["density"])
        assert np.array_equal(ev, g["expectation"])
    else:
        assert rel_err(sp, g["sp_ldos"]) <= 1e-12
        assert rel_err(mag, g["magnetization"]) <= 1e-12
        assert rel_err(dens, g["density"]) <= 1e-12
        assert rel_err(ev, g["expectation"]) <= 1e-12


def test_properties_mixed(gpu, oracle):
    g, m, t = _setup(gpu, oracle, False)
    bro, occ, dE = float(g["broadening"]), g["occupation"], float(g["dE"])
    sp = m.spin_polarized_ldos(t, g["sp_up"], g["sp_down"], bro, gpu.MIXED)
    for k in range(sp.shape[0]):
        assert rel_err(sp[k], g["sp_ldos"][k]) <= 1e-6
    dens = m.density(t, g["density_sites"], bro, occ, dE, gpu.MIXED)
    assert rel_err(dens, g["density"]) <= 1e-6
    mag = m.magnetization(t, g["sp_up"], g["sp_down"], bro, occ, dE, gpu.MIXED)
    assert rel_err(mag, g["magnetization"]) <= 1e-6


def test_properties_consistent(gpu, oracle):
    """The density of a spin row is the diagonal of the magnetization, the
    LDOS integrated with the occupation; the expectation value of (up, down)
    is the conjugate of the magnetization's (up, down) entry; argument errors
    are caught."""
    g, m, t = _setup(gpu, oracle, True)
    bro, occ, dE = float(g["broadening"]), g["occupation"], float(g["dE"])
    mag = m.magnetization(t, g["sp_up"], g["sp_down"], bro, occ, dE)
    dens = m.density(t, np.concatenate([g["sp_up"], g["sp_down"]]), bro, occ, dE)
    S = g["sp_up"].size
    assert rel_err(mag[:, 0, 0].real, dens[:S]) <= 1e-14
    assert rel_err(mag[:, 1, 1].real, dens[S:]) <= 1e-14
    ev = m.expectation_values(t, g["sp_up"], g["sp_down"], bro, occ, dE)
    assert rel_err(ev, np.conj(mag[:, 0, 1])) <= 1e-14
    with pytest.raises(ValueError):
        m.density(t, [0], bro, occ[:-1], dE)
    with pytest.raises(gpu.TBTKError):
        m.density(t, [10 ** 6], bro, occ, dE)


def test_property_extractor_mirror(gpu, oracle):
    """kpm.PropertyExtractor's property methods on the golden window give
    the golden values (device table, FP64)."""
    g = golden("props")
    lo, hi, res = g["window"]
    solver = gpu.ChebyshevExpander()
    solver.setModel((g["rowptr"], g["col"], g["val"]))
    solver.setScaleFactor(float(g["scale"]))
    solver.setNumCoefficients(int(g["M"]))
    solver.setBroadening(float(g["broadening"]))
    pe = gpu.PropertyExtractor(solver)
    pe.setEnergyWindow(float(lo), float(hi), int(res))
    occ = g["occupation"]
    assert rel_err(pe.calculateSpinPolarizedLDOS(g["sp_up"], g["sp_down"]), g["sp_ldos"]) <= 1e-12
    assert rel_err(pe.calculateDensity(g["density_sites"], occ), g["density"]) <= 1e-12
    assert rel_err(pe.calculateMagnetization(g["sp_up"], g["sp_down"], occ),
                   g["magnetization"]) <= 1e-12
    ev = pe.calculateExpectationValue(int(g["exp_to"][0]), int(g["exp_from"][0]), occ)
    assert abs(ev - g["expectation"][0]) <= 1e-12 * abs(g["expectation"][0])
