"""Synthetic workloads of the KPM path at full size.

Fast CSR builders for periodic lattices (one vectorised pass over rows, the
columns of each row sorted in place) that produce exactly the matrices of
``tbtk_b200.lattice`` (checked in tests/test_workloads.py), and the five
benchmark configurations:

1. ``cfg1``  30x30 square with spin, open, t=1, J=0.5, s=10, M=1000,
   broadening 1e-3, site (15,15,0), 1000 energies on the open grid (-10, 10).
2. ``cfg2``  2048x2048 periodic square with spin (N = 8,388,608), t=1,
   J=0.5, disorder U[-1, 1], s=12, M=4096, broadening 1e-3, 64 seeded sites,
   2000 energies on the open grid (-12, 12).
3. ``cfg3``  1024x1024 periodic square with spin + Rashba alpha=0.3, J=0.5,
   disorder U[-1, 1] (N = 2,097,152, 9 entries per row), s=12, M=2048,
   256 seeded sites in one tbtkkpm_ldos_sites call, 1000 energies (the
   library runs doubling calls as SpMM batches of 128 sources; a batch width
   of 256 runs them as one).
4. ``cfg4``  uneven batch of seeded models (square or honeycomb, L in
   [16, 256], J in [0, 1], W in [0, 3]) with 1-32 sites and M in
   {512, 1024, 2048, 4096}, s=12, 1000 energies.
5. ``cfg5``  serving pool: seeded square / honeycomb / Rashba models with N
   log-uniform in [1e3, 4e6], requests of 1-16 sites and M in [512, 4096].

The energy grids are open at +-s (``Range(-s, s, E, false, false)``)
because the reference rejects windows that touch +-scaleFactor
(Lib/include/TBTK/Solver/ChebyshevExpander.h:434-445).
"""
from __future__ import annotations

import dataclasses

import numpy as np


def _disorder(n_sites, W, seed):
    if W == 0.0:
        return np.zeros(n_sites)
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(-W / 2, W / 2, size=n_sites)


def _assemble(cols, vals):
    """Rows of equal length: sort each row's columns, keep values aligned."""
    order = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    vals = np.take_along_axis(vals, order, axis=1)
    N, k = cols.shape
    rowptr = (np.arange(N + 1, dtype=np.int64) * k).astype(np.uint32)
    return rowptr, cols.reshape(-1).astype(np.uint32), np.ascontiguousarray(vals.reshape(-1))


def square_csr(Lx, Ly, *, t=1.0, J=0.5, W=0.0, alpha=0.0, seed=0):
    """Periodic square lattice with spin (Lx, Ly >= 3): CSR in TBTK basis
    order, equal to ``lattice.square(..., periodic=True).csr()``."""
    assert Lx >= 3 and Ly >= 3
    N = Lx * Ly * 2
    b = np.arange(N, dtype=np.int64)
    s = b & 1
    site = b >> 1
    x, y = site // Ly, site % Ly
    v = _disorder(Lx * Ly, W, seed)
    diag = (-J * 2.0 * (0.5 - s)) + v[site]
    def idx(xx, yy, ss):
        return ((xx % Lx) * Ly + (yy % Ly)) * 2 + ss
    cols = [idx(x - 1, y, s), idx(x, y - 1, s), b, idx(x, y + 1, s), idx(x + 1, y, s)]
    vals = [np.full(N, -t, dtype=np.complex128)] * 2 + [diag.astype(np.complex128)] + \
           [np.full(N, -t, dtype=np.complex128)] * 2
    if alpha != 0.0:
        f = 1 - s
        up = s == 0  # row spin up: <up|H|down>
        # hop from (x-1) to x (d=+x, row is `to`): <to,up|H|from,down> = -alpha
        a_px = np.where(up, -alpha, alpha).astype(np.complex128)
        a_mx = np.conj(np.where(f == 0, -alpha, alpha)).astype(np.complex128)
        a_py = np.full(N, 1j * alpha, dtype=np.complex128)
        a_my = np.full(N, -1j * alpha, dtype=np.complex128)
        cols += [idx(x - 1, y, f), idx(x + 1, y, f), idx(x, y - 1, f), idx(x, y + 1, f)]
        vals += [a_px, a_mx, a_py, a_my]
    return _assemble(np.stack(cols, axis=1), np.stack(vals, axis=1))


def honeycomb_csr(Lx, Ly, *, t=1.0, J=0.5, W=0.0, seed=0):
    """Periodic brick-wall honeycomb with spin (Lx, Ly >= 2): equal to
    ``lattice.honeycomb(..., periodic=True).csr()``."""
    assert Lx >= 2 and Ly >= 2
    N = Lx * Ly * 4
    b = np.arange(N, dtype=np.int64)
    s = b & 1
    a = (b >> 1) & 1
    cell = b >> 2
    x, y = cell // Ly, cell % Ly
    v = _disorder(Lx * Ly * 2, W, seed)
    diag = (-J * 2.0 * (0.5 - s)) + v[(b >> 1)]
    def idx(xx, yy, aa, ss):
        return (((xx % Lx) * Ly + (yy % Ly)) * 2 + aa) * 2 + ss
    # A (a=0) at (x, y) couples to B at (x, y), (x-1, y), (x, y-1);
    # B at (x, y) couples to A at (x, y), (x+1, y), (x, y+1).
    dxs = np.where(a == 0, -1, 1)
    cols = [b, idx(x, y, 1 - a, s), idx(x + dxs, y, 1 - a, s), idx(x, y + dxs, 1 - a, s)]
    hop = np.full(N, -t, dtype=np.complex128)
    vals = [diag.astype(np.complex128), hop, hop, hop]
    return _assemble(np.stack(cols, axis=1), np.stack(vals, axis=1))


def sample_sites(n_sites, spin_count, count, seed, spin=0):
    """``count`` seeded lattice sites (spin component ``spin``) as basis
    numbers (same stream as ``lattice.random_sites``)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pick = rng.choice(n_sites, size=count, replace=count > n_sites)
    return (pick * spin_count + spin).astype(np.uint32)


def open_grid(scale, E):
    """Energies of Range(-s, s, E, false, false)."""
    dx = (scale - (-scale)) / (E + 1)
    start = -scale + dx
    return np.array([start + k * dx for k in range(E)])


@dataclasses.dataclass
class Problem:
    """One model with its expansion parameters and LDOS sites."""

    name: str
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    scale: float
    M: int
    broadening: float
    energies: np.ndarray
    sites: np.ndarray

    @property
    def N(self):
        return self.rowptr.size - 1

    @property
    def nnz(self):
        return int(self.rowptr[-1])


def cfg2(n_sites=64, L=2048, seed=2048):
    rowptr, col, val = square_csr(L, L, t=1.0, J=0.5, W=2.0, seed=seed)
    sites = sample_sites(L * L, 2, n_sites, seed + 1)
    return Problem("square 2048x2048 spin periodic, W=2, s=12, M=4096", rowptr, col, val,
                   12.0, 4096, 1e-3, open_grid(12.0, 2000), sites)


def cfg3(n_sites=256, L=1024, seed=1024):
    rowptr, col, val = square_csr(L, L, t=1.0, J=0.5, W=2.0, alpha=0.3, seed=seed)
    sites = sample_sites(L * L, 2, n_sites, seed + 1)
    return Problem("rashba 1024x1024 spin periodic, alpha=0.3, W=2, s=12, M=2048", rowptr,
                   col, val, 12.0, 2048, 1e-3, open_grid(12.0, 1000), sites)


def cfg4_specs(n_models=1000, seed=4):
    """Specs of the uneven batch: (kind, L, J, W, n_sites, M, model seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for i in range(n_models):
        kind = "square" if rng.uniform() < 0.5 else "honeycomb"
        L = int(rng.integers(16, 257))
        J = float(rng.uniform(0, 1))
        W = float(rng.uniform(0, 3))
        ns = int(rng.integers(1, 33))
        M = int(rng.choice([512, 1024, 2048, 4096]))
        specs.append((kind, L, J, W, ns, M, seed * 100000 + i))
    return specs


def cfg5_pool(n_models=64, seed=5):
    """Serving pool: (kind, L, J, W, alpha, model seed) with the basis size
    log-uniform in [1e3, 4e6] over square, honeycomb and Rashba lattices."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pool = []
    for i in range(n_models):
        kind = ("square", "honeycomb", "rashba")[i % 3]
        N = float(np.exp(rng.uniform(np.log(1e3), np.log(4e6))))
        per_cell = 4 if kind == "honeycomb" else 2
        L = max(8, int(round((N / per_cell) ** 0.5)))
        J = float(rng.uniform(0, 1))
        W = float(rng.uniform(0, 3))
        pool.append((kind, L, J, W, 0.3 if kind == "rashba" else 0.0, seed * 100000 + i))
    return pool


def cfg5_requests(pool_sizes, rate, duration, seed=55, max_sites=16, m_range=(512, 4096)):
    """Poisson arrivals at `rate` per second for `duration` seconds: (time,
    model, sites, M) with 1..max_sites distinct sites and M uniform in
    m_range."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            return out
        m = int(rng.integers(len(pool_sizes)))
        k = int(rng.integers(1, max_sites + 1))
        sites = rng.choice(pool_sizes[m], size=k, replace=False).astype(np.uint32)
        M = int(rng.integers(m_range[0], m_range[1] + 1))
        out.append((t, m, sites, M))


def build_model(kind, L, J, W, seed, alpha=0.0):
    if kind == "square":
        return square_csr(L, L, t=1.0, J=J, W=W, seed=seed)
    if kind == "rashba":
        return square_csr(L, L, t=1.0, J=J, W=W, alpha=alpha or 0.3, seed=seed)
    return honeycomb_csr(L, L, t=1.0, J=J, W=W, seed=seed)
