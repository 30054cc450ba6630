"""CPU tests: the oracle restatement and the lattice generators against the
reference's golden vectors and known answers (no GPU)."""
import numpy as np
import pytest

from conftest import golden
from tbtk_b200 import lattice as L
from tbtk_b200.kpm import tbtk_range

EPS100 = 100 * np.finfo(np.float64).eps
MODEL_CASES = ["cfg1", "rashba", "honeycomb", "duplicates"]


def _lattice(name):
    if name == "cfg1":
        return L.square(30, 30, t=1.0, J=0.5, periodic=False)
    if name == "rashba":
        return L.square(8, 6, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    if name == "honeycomb":
        return L.honeycomb(6, 5, t=1.0, J=0.3, W=1.5, periodic=True, seed=5)
    if name == "duplicates":
        return L.square(2, 2, t=1.0, J=0.5, mu=0.7, W=1.0, periodic=True, seed=2)
    raise KeyError(name)


@pytest.mark.parametrize("name", MODEL_CASES)
def test_lattice_csr_matches_reference(name):
    """Direct CSR generation == HoppingAmplitudeSet::getSparseMatrix()."""
    g = golden(name)
    rowptr, col, val = _lattice(name).csr()
    assert np.array_equal(rowptr, g["rowptr"])
    assert np.array_equal(col, g["col"])
    assert np.array_equal(val, g["val"])


@pytest.mark.parametrize("name", MODEL_CASES)
def test_oracle_csr_from_triplets(oracle, name):
    g = golden(name)
    lat = _lattice(name)
    rowptr, col, val = oracle.csr_from_triplets(lat.to_basis, lat.from_basis, lat.amp)
    assert np.array_equal(rowptr, g["rowptr"])
    assert np.array_equal(col, g["col"])
    assert np.array_equal(val, g["val"])


def test_sparse_matrix_known_answer(oracle):
    """HoppingAmplitudeSet.getSparseMatrix (Test/include/Core/TBTK/Test/
    HoppingAmplitudeSet.h:494-541): amplitudes 1..5 from {0},{1},{2},{3},{4}
    to {1},{0},{2},{4},{3} give one entry per column, row = to and column =
    from; the same matrix as CSR, the layout this path reads."""
    to = np.array([1, 0, 2, 4, 3], dtype=np.uint32)
    frm = np.array([0, 1, 2, 3, 4], dtype=np.uint32)
    amp = np.array([1, 2, 3, 4, 5], dtype=np.complex128)
    rowptr, col, val = oracle.csr_from_triplets(to, frm, amp)
    assert rowptr.tolist() == [0, 1, 2, 3, 4, 5]
    assert col.tolist() == [1, 0, 2, 4, 3]
    assert val.tolist() == [2, 1, 3, 5, 4]


@pytest.mark.parametrize("name", MODEL_CASES)
def test_oracle_moments_bit_exact(oracle, name):
    g = golden(name)
    mu = oracle.moments(g["rowptr"], g["col"], g["val"], float(g["scale"]), int(g["M"]),
                        int(g["frm"]), g["to"])
    mu = oracle.damp(mu, float(g["broadening"]))
    assert np.array_equal(mu, g["moments"])


@pytest.mark.parametrize("name", MODEL_CASES)
def test_oracle_ldos_and_greens_bit_exact(oracle, name):
    g = golden(name)
    lo, hi, E = g["window"]
    energies = tbtk_range(lo, hi, int(E))
    s, M = float(g["scale"]), int(g["M"])
    table = oracle.lookup_table(M, energies, s)
    for k, site in enumerate(g["ldos_sites"]):
        mu = oracle.damp(oracle.moments(g["rowptr"], g["col"], g["val"], s, M, int(site),
                                        [int(site)]), float(g["broadening"]))
        assert np.array_equal(oracle.ldos_table(table, mu[0]), g["ldos"][k])
    for ty in range(4):
        for k in range(g["to"].size):
            gt = oracle.greens_table(table, ty, g["moments"][k])
            assert np.array_equal(gt, g[f"greens_{ty}"][k]), (ty, k)


def test_kat_5x5(oracle):
    """Closed-form moments of the reference test
    (Test/include/TBTK/Test/Solver/ChebyshevExpander.h:184-277)."""
    g = golden("kat5x5")
    mu_, t, s = -2.0, 1.0, 10.0
    mu = oracle.moments(g["rowptr"], g["col"], g["val"], s, 100, int(g["frm"]), g["to"])
    assert np.array_equal(mu, g["moments"])
    d, o = mu
    assert abs(d[0] - 1) < EPS100 and abs(d[1] - (-mu_ / s)) < EPS100
    assert abs(d[2] - (2 * (mu_ * mu_ + 4 * t * t) / (s * s) - 1)) < EPS100
    assert abs(o[0]) < EPS100 and abs(o[1] - (-t / s)) < EPS100
    assert abs(o[2] - 4 * mu_ * t / (s * s)) < EPS100


def test_greens_closed_forms(oracle):
    """generateGreensFunction0..4 (ChebyshevExpander.h:371-564) and complex
    coefficients against the reference."""
    g = golden("greens")
    E = tbtk_range(-5, 5, 10)
    c = np.array([1, 2, 3], dtype=np.complex128)
    th = np.arccos(E / 10)
    closed = {
        1: -(c[0] / 2 + c[1] * np.exp(-1j * th) + c[2] * np.exp(-2j * th)) * 2j / np.sqrt(100 - E * E),
        0: (c[0] / 2 + c[1] * np.exp(1j * th) + c[2] * np.exp(2j * th)) * 2j / np.sqrt(100 - E * E),
        2: (c[1] * np.sin(th) + c[2] * np.sin(2 * th)) * 2 / np.sqrt(100 - E * E),
        3: (c[0] / 2 + c[1] * np.cos(th) + c[2] * np.cos(2 * th)) * 2j / np.sqrt(100 - E * E),
    }
    table = oracle.lookup_table(3, E, 10.0)
    for ty in range(4):
        gc = oracle.greens_closed(E, 10.0, ty, c)
        gt = oracle.greens_table(table, ty, c)
        assert np.array_equal(gc, g[f"real_{ty}_0"])
        assert np.array_equal(gt, g[f"real_{ty}_1"])
        assert np.abs(gc - closed[ty]).max() < EPS100
        assert np.abs(gt - gc).max() < EPS100
    E2 = tbtk_range(-9.5, 9.5, 37, False, True)
    t2 = oracle.lookup_table(4, E2, 10.0)
    for ty in range(4):
        assert np.array_equal(oracle.greens_closed(E2, 10.0, ty, g["cc"]), g[f"cplx_{ty}_0"])
        assert np.array_equal(oracle.greens_table(t2, ty, g["cc"]), g[f"cplx_{ty}_1"])


def test_ring_ldos_integrates_to_one(oracle):
    """calculateLDOS0 (Test/include/TBTK/Test/PropertyExtractor/ChebyshevExpander.h:19-45)."""
    g = golden("ring")
    for f in (9, 7):
        E = tbtk_range(-f, f, 1000)
        mu = oracle.damp(oracle.moments(g["rowptr"], g["col"], g["val"], 10.0, 1000, 0, [0]), 1e-6)
        ldos = oracle.ldos_table(oracle.lookup_table(1000, E, 10.0), mu[0])
        assert np.array_equal(ldos, g[f"ldos_{f}"][0])
        assert abs(ldos.sum() * (E[1] - E[0]) - 1) < 1e-3


def _smooth_gaussian(data, sigma, window, lower, upper):
    """Smooth::gaussian of an LDOS block: sigma in energy units scaled to
    bins, weights normalised over the whole window, truncated at the edges
    (Lib/include/Utilities/TBTK/Smooth.h:86-134,237-269)."""
    R = data.size
    s = sigma / (upper - lower) * R
    half = window // 2
    norm = 1.0 / sum(np.exp(-n * n / (2 * s * s)) for n in range(-half, half + 1))
    out = np.zeros(R)
    for n in range(R):
        c = np.arange(max(0, n - half), min(n + half + 1, R))
        out[n] = (data[c] * np.exp(-(c - n) ** 2 / (2 * s * s))).sum() * norm
    return out


def test_ring_ldos_matches_exact_diagonalization(oracle):
    """calculateLDOS1 (Test/include/TBTK/Test/PropertyExtractor/
    ChebyshevExpander.h:47-104): on the 10-site ring the KPM LDOS at site 0
    (s = 10, the Solver's default M = 1000 and broadening 1e-6, window
    Range(-2.5, 2.5, 1000)) and the exact one agree within 10 % after both
    pass Smooth::gaussian(sigma 0.3, window 1001).  The exact LDOS puts
    |u_n(0)|^2 / dE of every eigenvalue strictly inside the window into bin
    round((E_n - E_0)/dE), as the Diagonalizer's LDOS callback does
    (Lib/src/PropertyExtractor/Diagonalizer.cpp:594-619); numpy's eigh
    stands in for its LAPACK solver."""
    g = golden("ring")
    lo, hi, R = -2.5, 2.5, 1000
    E = tbtk_range(lo, hi, R)
    mu = oracle.damp(oracle.moments(g["rowptr"], g["col"], g["val"], 10.0, 1000, 0, [0]), 1e-6)
    kpm = oracle.ldos_table(oracle.lookup_table(1000, E, 10.0), mu[0])
    N = g["rowptr"].size - 1
    H = np.zeros((N, N), dtype=np.complex128)
    for r in range(N):
        for k in range(g["rowptr"][r], g["rowptr"][r + 1]):
            H[r, g["col"][k]] += g["val"][k]
    w, v = np.linalg.eigh(H)
    dE = E[1] - E[0]
    exact = np.zeros(R)
    for n in range(N):
        if E[0] < w[n] < E[-1]:
            e = int(np.floor((w[n] - E[0]) / dE + 0.5))  # C round(), argument >= 0
            if 0 <= e < R:
                exact[e] += abs(v[0, n]) ** 2 / dE
    a = _smooth_gaussian(kpm, 0.3, 1001, lo, hi)
    b = _smooth_gaussian(exact, 0.3, 1001, lo, hi)
    assert np.all(np.abs(a - b) <= 0.1 * (a + b)), np.max(np.abs(a - b) / (a + b))
    assert abs(exact.sum() * dE - 1) < 1e-9  # every eigenvalue of the ring lies in the window


def test_range_matches_reference(reference):
    for args in [(-1, 1, 1000, True, True), (-10, 10, 1000, False, False),
                 (-9.5, 9.5, 37, False, True), (-0.1, 0.2, 10, True, False)]:
        ours = tbtk_range(*args)
        ref = [reference.range_value(*args, k) for k in range(args[2])]
        assert np.array_equal(ours, np.array(ref))


def test_oracle_vs_reference_random_models(oracle, reference):
    """Fresh seeds, not in the golden set: restatement == reference."""
    rng = np.random.default_rng(7)
    for seed in range(3):
        Lx, Ly = rng.integers(3, 9, size=2)
        lat = L.square(int(Lx), int(Ly), t=1.0, J=float(rng.uniform(0, 1)),
                       W=float(rng.uniform(0, 3)), alpha=0.2 * seed,
                       periodic=bool(seed % 2), seed=seed)
        m = reference.model(lat)
        rowptr, col, val = lat.csr()
        r2, c2, v2 = m.csr()
        assert np.array_equal(rowptr, r2) and np.array_equal(col, c2) and np.array_equal(val, v2)
        site = (1, 1, 0)
        to = [(1, 1, 0), (1, 2, 1), (0, 0, 0)]
        ref = m.coefficients(12.0, 150, 1e-3, to, site)
        ours = oracle.damp(oracle.moments(rowptr, col, val, 12.0, 150, lat.basis(site),
                                          [lat.basis(t) for t in to]), 1e-3)
        assert np.array_equal(ours, ref)


def test_basis_order_matches_reference(reference):
    lat = L.honeycomb(3, 4, W=0.5, seed=1)
    m = reference.model(lat)
    assert m.basis_size() == lat.num_states
    for idx in [(0, 0, 0, 0), (2, 3, 1, 1), (1, 2, 0, 1)]:
        assert m.basis_index(idx) == lat.basis(idx)


def _props_greens(oracle, g, pairs):
    """Damped NonPrincipal G of (to, from) basis pairs on the golden window."""
    M, s = int(g["M"]), float(g["scale"])
    table = oracle.lookup_table(M, g["energies"], s)
    out = []
    for to, frm in pairs:
        mu = oracle.damp(oracle.moments(g["rowptr"], g["col"], g["val"], s, M, int(frm), [int(to)]),
                         float(g["broadening"]))
        out.append(oracle.greens_table(table, 3, mu[0]))
    return np.array(out)


def test_properties_restatement_matches_reference(oracle):
    """Spin-polarized LDOS, density, magnetization and expectation values from
    the oracle's moments and Green's functions, formed as the reference's
    PropertyExtractor forms them, equal TBTK's own results bit for bit."""
    from oracle_lib import (density_from_greens, expectation_from_greens,
                            magnetization_from_greens, sp_ldos_from_greens)
    g = golden("props")
    occ, dE = g["occupation"], float(g["dE"])
    for k, (u, d) in enumerate(zip(g["sp_up"], g["sp_down"])):
        G4 = _props_greens(oracle, g, [(u, u), (u, d), (d, u), (d, d)])
        assert np.array_equal(sp_ldos_from_greens(G4), g["sp_ldos"][k])
        assert np.array_equal(magnetization_from_greens(G4, occ, dE), g["magnetization"][k])
    for k, site in enumerate(g["density_sites"]):
        G = _props_greens(oracle, g, [(site, site)])[0]
        assert density_from_greens(G, occ, dE) == g["density"][k]
    for k, (to, frm) in enumerate(zip(g["exp_to"], g["exp_from"])):
        G = _props_greens(oracle, g, [(to, frm)])[0]
        assert expectation_from_greens(G, occ, dE) == g["expectation"][k]
