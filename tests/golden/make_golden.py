"""Generates the golden vectors of the KPM path from the TBTK reference.

Runs the reference classes compiled from the reference sources
(oracle/_ref/libtbtkref.so, ``make -C oracle ref``) through
tests/oracle_lib.py and writes tests/golden/*.npz.  Every array comes from a
reference call: Model -> HoppingAmplitudeSet::getSparseMatrix (CSR),
Solver::ChebyshevExpander::calculateCoefficients (moments),
generateGreensFunction (G, table and closed form), and
PropertyExtractor::ChebyshevExpander::calculateLDOS /
calculateGreensFunctions, and the JSON text of Property::LDOS,
GreensFunction and Density (serialize(Serializable::Mode::JSON)).

    python tests/golden/make_golden.py [case ...]    (default: every case)
"""
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from oracle_lib import Reference  # noqa: E402
from tbtk_b200 import lattice as L  # noqa: E402


def pe_window(s, res):
    """Open grid (-s, s) with res points, as the PropertyExtractor's inclusive
    Range(lo, hi, res) with lo = -s + 2s/(res+1), hi = lo + (res-1)*dx."""
    dx = 2 * s / (res + 1)
    lo = -s + dx
    hi = lo + (res - 1) * dx
    return lo, hi


def model_case(ref, lat, s, M, bro, to, frm, ldos_sites, E, types=(0, 1, 2, 3)):
    m = ref.model(lat)
    rowptr, col, val = m.csr()
    out = dict(rowptr=rowptr, col=col, val=val, shape=np.array(lat.shape),
               scale=s, M=M, broadening=bro,
               to=np.array([lat.basis(t) for t in to], dtype=np.uint32),
               frm=np.uint32(lat.basis(frm)),
               to_index=np.array(to, dtype=np.int32),
               from_index=np.array(frm, dtype=np.int32))
    out["moments"] = m.coefficients(s, M, bro, to, frm)
    lo, hi = pe_window(s, E)
    out["window"] = np.array([lo, hi, E])
    out["ldos_sites"] = np.array([lat.basis(t) for t in ldos_sites], dtype=np.uint32)
    out["ldos"] = m.ldos(s, M, bro, lo, hi, E, ldos_sites)
    for ty in types:
        out[f"greens_{ty}"] = m.greens_pe(s, M, bro, lo, hi, E, ty, to, frm)
    return out


def export_case(ref):
    """Serialized properties: the reference's JSON text next to the same
    property's values per index in argument order (from the calls the other
    fixtures use), on a disordered Rashba lattice (complex Green's
    functions) and a honeycomb lattice (four subindices)."""
    out = {}
    lat = L.square(6, 5, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    m = ref.model(lat)
    s, M, bro, lo, hi, res, T, mu = 8.0, 256, 1e-3, -3.9, 3.9, 40, 300.0, 0.1
    out["window"] = np.array([lo, hi, res])
    sites = [(2, 3, 0), (0, 4, 1), (5, 1, 0), (1, 1, 1)]
    out["ldos_sites"] = np.array(sites, dtype=np.int32)
    out["ldos_text"] = np.array(m.property_json(0, s, M, bro, lo, hi, res, sites)[0])
    out["ldos"] = m.ldos(s, M, bro, lo, hi, res, sites)
    to, frm = [(2, 3, 0), (2, 3, 1), (4, 0, 1)], (2, 3, 0)
    out["gf_to"] = np.array(to, dtype=np.int32)
    out["gf_from"] = np.array(frm, dtype=np.int32)
    for ty in (1, 3):
        out[f"gf_text_{ty}"] = np.array(
            m.property_json(1, s, M, bro, lo, hi, res, to, frm=frm, type_=ty)[0])
        out[f"gf_{ty}"] = m.greens_pe(s, M, bro, lo, hi, res, ty, to, frm)
    dsites = [(2, 3, 0), (2, 3, 1), (4, 0, 1)]
    out["density_sites"] = np.array(dsites, dtype=np.int32)
    out["density_text"] = np.array(
        m.property_json(2, s, M, bro, lo, hi, res, dsites, T=T, mu=mu)[0])
    out["density"] = np.array([m.prop(1, s, M, bro, lo, hi, res, T, mu, list(d))
                               for d in dsites])
    # wildcard patterns of calculateLDOS(patterns) (IDX_ALL expands,
    # IDX_SUM_ALL sums), with the LDOS of every model index for the sums
    from tbtk_b200 import export as X
    S, A = X.IDX_SUM_ALL, X.IDX_ALL
    every = [tuple(int(v) for v in np.unravel_index(b, lat.shape)) for b in range(lat.num_states)]
    out["pat_ldos_all"] = m.ldos(s, 128, bro, lo, 3.9, 20, every)
    out["pat_window"] = np.array([lo, 3.9, 20])
    pattern_sets = [[(2, 3, S)], [(A, 1, 0)], [(2, 3, S), (A, 1, 0)], [(4, S, S)], [(S, S, 1)]]
    out["pat_count"] = np.array(len(pattern_sets))
    for k, pats in enumerate(pattern_sets):
        out[f"pat_patterns_{k}"] = np.array(pats, dtype=np.int32)
        out[f"pat_text_{k}"] = np.array(m.property_json(0, s, 128, bro, lo, 3.9, 20, pats)[0])
    lat = L.honeycomb(6, 5, t=1.0, J=0.3, W=1.5, periodic=True, seed=5)
    m = ref.model(lat)
    hsites = [(2, 2, 0, 0), (5, 4, 1, 1), (0, 1, 1, 0)]
    out["hc_window"] = np.array([-11.5, 11.5, 64])
    out["hc_sites"] = np.array(hsites, dtype=np.int32)
    out["hc_text"] = np.array(m.property_json(0, 12.0, 200, 1e-3, -11.5, 11.5, 64, hsites)[0])
    out["hc_ldos"] = m.ldos(12.0, 200, 1e-3, -11.5, 11.5, 64, hsites)
    return out


def main(only=()):
    ref = Reference()
    cases = {}

    # Reference coefficient test: 5x5 periodic spinless, mu=-2, t=1, s=10,
    # M=100, broadening 0 (Test/include/TBTK/Test/Solver/ChebyshevExpander.h:184-278).
    lat = L.test_square()
    m = ref.model(lat)
    rowptr, col, val = m.csr()
    cases["kat5x5"] = dict(
        rowptr=rowptr, col=col, val=val, scale=10.0, M=100, broadening=0.0,
        to=np.array([lat.basis((0, 0)), lat.basis((1, 0))], dtype=np.uint32),
        frm=np.uint32(lat.basis((0, 0))),
        moments=m.coefficients(10.0, 100, 0.0, [[0, 0], [1, 0]], [0, 0]))

    # The CPU-runnable configuration: 30x30 with spin, open, t=1, J=0.5,
    # s=10, M=1000, broadening 1e-3, site (15,15,0), 1000 open-grid energies.
    lat = L.square(30, 30, t=1.0, J=0.5, periodic=False)
    cases["cfg1"] = model_case(ref, lat, 10.0, 1000, 1e-3,
                               [(15, 15, 0), (16, 15, 0), (15, 15, 1)],
                               (15, 15, 0), [(15, 15, 0), (0, 0, 1)], 1000)

    # Rashba + disorder, periodic (complex off-diagonal amplitudes).
    lat = L.square(8, 6, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    cases["rashba"] = model_case(ref, lat, 12.0, 256, 1e-3,
                                 [(3, 2, 0), (3, 2, 1), (4, 2, 1), (0, 5, 0)],
                                 (3, 2, 0), [(3, 2, 0), (7, 5, 1), (1, 1, 0)], 300)

    # Honeycomb + disorder, periodic.
    lat = L.honeycomb(6, 5, t=1.0, J=0.3, W=1.5, periodic=True, seed=5)
    cases["honeycomb"] = model_case(ref, lat, 12.0, 200, 1e-3,
                                    [(2, 2, 0, 0), (2, 2, 1, 0), (1, 2, 1, 0)],
                                    (2, 2, 0, 0), [(2, 2, 0, 0), (5, 4, 1, 1)], 128)

    # Duplicate amplitudes: a 2x2 periodic lattice repeats each hopping, and
    # mu, Zeeman and disorder stack three on-site terms.
    lat = L.square(2, 2, t=1.0, J=0.5, mu=0.7, W=1.0, periodic=True, seed=2)
    cases["duplicates"] = model_case(ref, lat, 10.0, 64, 1e-3,
                                     [(0, 0, 0), (1, 1, 1)], (0, 0, 0),
                                     [(0, 0, 0)], 50)

    # Reference LDOS test ring: 10 sites, s=10, default M=1000 and
    # broadening 1e-6, windows +-9 and +-7 of 1000 points
    # (Test/include/TBTK/Test/PropertyExtractor/ChebyshevExpander.h:19-45).
    lat = L.ring(10)
    m = ref.model(lat)
    rowptr, col, val = m.csr()
    ring = dict(rowptr=rowptr, col=col, val=val, scale=10.0, M=1000, broadening=1e-6)
    for f in (0.9, 0.7):
        ring[f"ldos_{int(f * 10)}"] = m.ldos(10.0, 1000, 1e-6, -10 * f, 10 * f, 1000, [[0]])
    cases["ring"] = ring

    # Closed-form Green's functions, c = {1, 2, 3}, s = 10, Range(-5, 5, 10)
    # (ChebyshevExpander.h:371-564), and complex coefficients on a half-open
    # window.
    g = {}
    for ty in range(4):
        for tab in (0, 1):
            g[f"real_{ty}_{tab}"] = ref.greens(10.0, [1, 2, 3], -5, 5, 10, ty, tab)
    cc = np.array([1 + 0.5j, 2 - 1j, 3 + 2j, -0.3 + 0.1j])
    g["cc"] = cc
    for ty in range(4):
        for tab in (0, 1):
            g[f"cplx_{ty}_{tab}"] = ref.greens(10.0, cc, -9.5, 9.5, 37, ty, tab, False, True)
    cases["greens"] = g

    # The PropertyExtractor's other properties (spin-polarized LDOS, density,
    # magnetization, expectation values) on a disordered Rashba lattice at
    # T = 300 and chemical potential 0.1, with the inclusive window
    # Range(-3.9, 3.9, 120); one reference call per site.
    lat = L.square(6, 5, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    m = ref.model(lat)
    rowptr, col, val = m.csr()
    s, M, bro, lo, hi, res, T, mu = 8.0, 256, 1e-3, -3.9, 3.9, 120, 300.0, 0.1
    energies = np.array([ref.range_value(lo, hi, res, True, True, k) for k in range(res)])
    sp_sites = [(2, 3), (0, 4), (5, 1)]
    dens_sites = [(2, 3, 0), (2, 3, 1), (4, 0, 1)]
    pairs = [((2, 3, 0), (2, 3, 1)), ((4, 4, 1), (4, 4, 1)), ((1, 2, 0), (2, 2, 1))]
    cases["props"] = dict(
        rowptr=rowptr, col=col, val=val, scale=s, M=M, broadening=bro,
        window=np.array([lo, hi, res]), energies=energies, dE=energies[1] - energies[0],
        T=T, mu=mu, occupation=ref.fermi_dirac(energies, mu, T),
        sp_up=np.array([lat.basis((x, y, 0)) for x, y in sp_sites], dtype=np.uint32),
        sp_down=np.array([lat.basis((x, y, 1)) for x, y in sp_sites], dtype=np.uint32),
        sp_ldos=np.array([m.prop(0, s, M, bro, lo, hi, res, T, mu, [x, y, -1])
                          for x, y in sp_sites]),
        magnetization=np.array([m.prop(2, s, M, bro, lo, hi, res, T, mu, [x, y, -1])
                                for x, y in sp_sites]),
        density_sites=np.array([lat.basis(d) for d in dens_sites], dtype=np.uint32),
        density=np.array([m.prop(1, s, M, bro, lo, hi, res, T, mu, list(d))
                          for d in dens_sites]),
        exp_to=np.array([lat.basis(a) for a, _ in pairs], dtype=np.uint32),
        exp_from=np.array([lat.basis(b) for _, b in pairs], dtype=np.uint32),
        expectation=np.array([m.expectation(s, M, bro, lo, hi, res, T, mu, list(a), list(b))
                              for a, b in pairs]))

    cases["export"] = export_case(ref)

    for name, arrays in cases.items():
        if only and name not in only:
            continue
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, sum(np.asarray(v).nbytes for v in arrays.values()), "bytes")


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
