"""Table-free energy sums (tbtkkpm_table_create_clenshaw): the same Green's
functions and LDOS as the lookup-table sums, evaluated by Clenshaw
recurrences.  Compared normwise (max|x - ref| / max|ref|) with the
reference's own Green's functions (golden vectors: with its lookup table and
with its closed form) at 1e-11, and with the device table sums at 1e-12."""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["real", "cplx"])
def test_clenshaw_matches_reference_greens(gpu, oracle, kind):
    g = golden("greens")
    if kind == "real":
        coeff = np.array([1, 2, 3], dtype=np.complex128)
        energies = oracle.range(-5, 5, 10)
    else:
        coeff = g["cc"]
        energies = oracle.range(-9.5, 9.5, 37, False, True)
    t = gpu.Table.create_clenshaw(coeff.size, energies, 10.0)
    for ty in range(4):
        G = t.greens(coeff[None, :], ty)[0]
        # the reference's closed form (tab 0) and its table (tab 1) agree for
        # real coefficients; for complex ones its table form is the one the
        # library follows (Advanced: c_n conj(T) against conj(c_n e^{-in theta}),
        # Lib/src/Solver/ChebyshevExpander.cpp:334-340,395-401)
        for tab in ((0, 1) if kind == "real" else (1,)):
            assert rel_err(G, g[f"{kind}_{ty}_{tab}"]) <= 1e-11, (ty, tab)


@pytest.mark.parametrize("name", ["cfg1", "rashba", "honeycomb"])
def test_clenshaw_matches_table_sums(gpu, name):
    g = golden(name)
    s, M, bro = float(g["scale"]), int(g["M"]), float(g["broadening"])
    lo, hi, E = g["window"]
    energies = gpu.tbtk_range(float(lo), float(hi), int(E))
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    tab = gpu.Table.create(M, energies, s)
    cl = gpu.Table.create_clenshaw(M, energies, s)
    sites = g["ldos_sites"]
    ref, _ = m.ldos_sites(tab, sites, bro, gpu.FP64)
    got, _ = m.ldos_sites(cl, sites, bro, gpu.FP64)
    assert rel_err(got, ref) <= 1e-12
    assert rel_err(got, g["ldos"]) <= 1e-11
    mu = m.moments(int(g["frm"]), g["to"], M, bro)
    for ty in range(4):
        assert rel_err(cl.greens(mu, ty), tab.greens(mu, ty)) <= 1e-12, ty
    mixed, _ = m.ldos_sites(cl, sites, bro, gpu.MIXED)
    assert rel_err(mixed, ref) <= 1e-6


def test_server_table_free(gpu):
    """A server with table-free energy sums returns the table server's LDOS
    up to rounding (same lanes, same moments)."""
    from tbtk_b200 import workloads
    S = 12.0
    energies = workloads.open_grid(S, 300)
    csr = workloads.square_csr(20, 20, J=0.5, W=2.0, alpha=0.3, seed=2)
    sites = [3, 77, 400]
    out = []
    for free in (False, True):
        srv = gpu.Server(512, energies, hbm_budget=1 << 30, tick_steps=16, tolerance=0)
        srv.set_table_free(free)
        mid = srv.add_model(*csr, S, 4)
        ldos, _, _ = srv.wait(srv.submit(mid, sites, 512, 1e-3), timeout=300)
        out.append(ldos)
        srv.close()
    assert rel_err(out[1], out[0]) <= 1e-12


def _random_coefficients(K, M, seed):
    rng = np.random.default_rng(seed)
    decay = np.exp(-np.arange(M) / max(M / 4, 1))
    return (rng.standard_normal((K, M)) + 1j * rng.standard_normal((K, M))) * decay


def _node_sums(mu, E, s, ty):
    """The five sums on the Chebyshev nodes with exactly reduced phases:
    n theta_k = pi m / (2E), m = n (2k + 1) mod 4E (numpy, FP64)."""
    K, M = mu.shape
    k = np.arange(E)
    ph = np.exp(1j * np.pi * ((np.arange(M)[:, None] * (2 * k + 1)) % (4 * E)) / (2 * E))
    a = mu.copy()
    a[:, 0] *= 0.5
    C = (a @ ph + a @ np.conj(ph)) / 2
    S = (a @ ph - a @ np.conj(ph)) / 2j
    A = 2 / (s * np.sin(np.pi * (2 * k + 1) / (2 * E)))
    g = {0: -A * (S - 1j * C), 1: -A * (S + 1j * C), 2: A * S, 3: 1j * A * C,
         4: A * C.real / np.pi}[ty]
    return g[:, ::-1]


@pytest.mark.parametrize("M,E", [(1, 1), (7, 2), (300, 64), (1000, 1024), (3000, 512),
                                 (2048, 2048), (4096, 4096)])
def test_chebyshev_grid_matches_table_sums(gpu, M, E):
    """Energy sums on the Chebyshev-node grid by one FFT per vector
    (tbtkkpm_table_create_chebyshev), every type: against the same sums with
    exactly reduced phases at 1e-13, and against the lookup-table sums on the
    same energies.  The table evaluates e^{-i n acos x} at the energies as
    stored; near the band edge acos turns their last-bit rounding into a
    phase error of about eps / q (q = sqrt(1 - x^2)), times n.  So the table
    agrees at 1e-11 on the nodes with q >= 1/2, and within 16 M eps / q_min
    on all of them.  M > 2E folds terms onto the transform."""
    s = 12.0
    cheb = gpu.Table.create_chebyshev(M, E, s)
    e = np.arange(E)
    assert np.allclose(cheb.energies, -s * np.cos(np.pi * (2 * e + 1) / (2 * E)), rtol=0,
                       atol=1e-14 * s)
    assert np.all(np.diff(cheb.energies) > 0) and np.all(np.abs(cheb.energies) < s)
    tab = gpu.Table.create(M, cheb.energies, s)
    mu = _random_coefficients(5, M, M + E)
    # errors against the largest Retarded value (it holds both the cosine
    # and the sine sums; a single type can vanish, e.g. Principal at M = 1)
    scale = np.abs(_node_sums(mu, E, s, 1)).max()

    q = np.sqrt(1 - (cheb.energies / s) ** 2)
    inner = q >= 0.5
    edge_tol = 1e-11 + 16 * M * np.finfo(np.float64).eps / q.min()

    def err(x, ref, where=slice(None)):
        return float(np.abs(x[:, where] - ref[:, where]).max() / scale)

    for ty in range(4):
        G = cheb.greens(mu, ty)
        assert err(G, _node_sums(mu, E, s, ty)) <= 1e-13, ty
        T = tab.greens(mu, ty)
        if inner.any():
            assert err(G, T, inner) <= 1e-11, ty
        assert err(G, T) <= edge_tol, ty
    rho = cheb.ldos(mu)
    assert err(rho, _node_sums(mu, E, s, 4)) <= 1e-13
    T = tab.ldos(mu)
    if inner.any():
        assert err(rho, T, inner) <= 1e-11
    assert err(rho, T) <= edge_tol
    one = cheb.greens(mu[2:3], 1)
    assert np.array_equal(one[0], cheb.greens(mu, 1)[2])  # one block per vector


def test_chebyshev_grid_ldos_sites(gpu):
    """ldos_sites through a Chebyshev-grid handle on the 30x30 spin lattice
    (M = 1000) equals the table-handle result on the same energies."""
    g = golden("cfg1")
    s, M, bro = float(g["scale"]), int(g["M"]), float(g["broadening"])
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    cheb = gpu.Table.create_chebyshev(M, 1024, s)
    tab = gpu.Table.create(M, cheb.energies, s)
    sites = g["ldos_sites"]
    ref, _ = m.ldos_sites(tab, sites, bro, gpu.FP64)
    got, _ = m.ldos_sites(cheb, sites, bro, gpu.FP64)
    # the table's acos of the stored energies is ill-conditioned at the edge
    # nodes (see test_chebyshev_grid_matches_table_sums)
    q = np.sqrt(1 - (cheb.energies / s) ** 2)
    inner = q >= 0.5
    assert np.abs(got - ref)[:, inner].max() <= 1e-12 * np.abs(ref).max()
    assert rel_err(got, ref) <= 1e-9
    # the grid's outer nodes lie within q = 1.5e-3 of the band edge, where
    # the 2/(s q) weight of the sum scales a mixed-precision moment error up
    # ~650x: the inner nodes meet the mixed bar, and the per-site estimate
    # (whose weight is the grid's largest) covers the error on all of them
    mixed, est = m.ldos_sites(cheb, sites, bro, gpu.MIXED)
    assert np.abs(mixed - ref)[:, inner].max() <= 1e-6 * np.abs(ref).max()
    for k in range(len(sites)):
        assert rel_err(mixed[k], ref[k]) <= est[k], k
    # Gauss-Chebyshev quadrature: the integral of the LDOS (mu_0 = 1) is
    # sum_e rho(E_e) (pi s / E) q_e
    total = got @ (np.pi * s / 1024 * q)
    assert np.allclose(total, 1.0, rtol=0, atol=1e-10)  # exact for degree < 2E
