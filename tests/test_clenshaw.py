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
