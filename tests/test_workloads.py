"""CPU tests: the fast full-size CSR builders equal the generic lattice
generators (which equal the reference's getSparseMatrix)."""
import numpy as np
import pytest

from tbtk_b200 import lattice as L
from tbtk_b200 import workloads as W


@pytest.mark.parametrize("Lx,Ly,alpha", [(3, 3, 0.0), (5, 4, 0.0), (4, 6, 0.3), (7, 3, 0.25)])
def test_square_csr_matches_lattice(Lx, Ly, alpha):
    a = W.square_csr(Lx, Ly, t=1.0, J=0.4, W=2.0, alpha=alpha, seed=9)
    b = L.square(Lx, Ly, t=1.0, J=0.4, W=2.0, alpha=alpha, periodic=True, seed=9).csr()
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("Lx,Ly", [(2, 2), (3, 4), (5, 3)])
def test_honeycomb_csr_matches_lattice(Lx, Ly):
    a = W.honeycomb_csr(Lx, Ly, t=1.0, J=0.7, W=1.5, seed=4)
    b = L.honeycomb(Lx, Ly, t=1.0, J=0.7, W=1.5, periodic=True, seed=4).csr()
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_sample_sites_matches_lattice():
    lat = L.square(10, 10)
    assert np.array_equal(W.sample_sites(100, 2, 7, 5), L.random_sites(lat, 7, 5))


def test_open_grid_is_reference_range():
    from tbtk_b200.kpm import tbtk_range
    assert np.array_equal(W.open_grid(12.0, 2000), tbtk_range(-12.0, 12.0, 2000, False, False))


def test_cfg4_specs_ranges():
    specs = W.cfg4_specs()
    assert len(specs) == 1000
    kinds = {s[0] for s in specs}
    assert kinds == {"square", "honeycomb"}
    assert all(16 <= s[1] <= 256 and 1 <= s[4] <= 32 and s[5] in (512, 1024, 2048, 4096)
               for s in specs)
