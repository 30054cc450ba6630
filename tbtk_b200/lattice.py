"""Seeded synthetic tight-binding lattices in TBTK's basis order.

Every generator returns a :class:`Lattice` holding the hopping amplitudes as
TBTK would receive them (``model << HoppingAmplitude(a, to, from) + HC``) and
can emit the Hamiltonian directly as CSR in TBTK's basis order, with columns
ascending in each row and duplicate entries summed, which is the matrix
``HoppingAmplitudeSet::getSparseMatrix()`` followed by
``setStorageFormat(CSR)`` produces
(Lib/include/Core/TBTK/HoppingAmplitudeSet.h:397-424,
Lib/include/Utilities/TBTK/SparseMatrix.h:1375-1551).

Basis order.  TBTK numbers the leaves of its index tree depth first in
ascending subindex order (Lib/src/Core/HoppingAmplitudeTree.cpp:596-617).
On a full lattice that is lexicographic order over the index, so
``basis(x, y, s) = (x*Ly + y)*2 + s`` for the square lattice and
``basis(x, y, a, s) = ((x*Ly + y)*2 + a)*2 + s`` for the honeycomb lattice.

Conventions (a HoppingAmplitude(a, to, from) is <to|H|from> = a):

* square: nearest-neighbour hopping ``-t`` along +x and +y plus HC, Zeeman
  ``-J*2*(1/2 - s)`` and on-site disorder ``V(x, y)`` drawn once per site
  (shared by both spins) from U[-W/2, W/2]; ``-mu`` on site when mu != 0;
* rashba: the square lattice plus the spin flip ``i*alpha*(sigma x d)_z`` to
  the +x and +y neighbours plus HC, i.e. for d = +x the block
  ``[[0, -alpha], [alpha, 0]]`` and for d = +y ``[[0, i alpha], [i alpha, 0]]``
  (rows: spin of ``to``, columns: spin of ``from``);
* honeycomb: brick-wall honeycomb, sublattice a=0 (A) at cell (x, y) hops to
  B at (x, y), (x-1, y) and (x, y-1) with ``-t`` plus HC; Zeeman and disorder
  per site (cell and sublattice) as above.

The disorder stream is numpy's PCG64 seeded with ``seed``; one value per
lattice site in basis order of the sites.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Lattice:
    """A tight-binding model: amplitude triplets in insertion order.

    ``to_index``/``from_index`` are ``[n, idx_len]`` int32 TBTK indices,
    ``to_basis``/``from_basis`` their basis numbers and ``amp`` the complex
    amplitudes.  ``shape`` is the index extent per subindex.
    """

    name: str
    shape: tuple
    to_index: np.ndarray
    from_index: np.ndarray
    amp: np.ndarray
    to_basis: np.ndarray
    from_basis: np.ndarray

    @property
    def num_states(self) -> int:
        return int(np.prod(self.shape))

    @property
    def idx_len(self) -> int:
        return len(self.shape)

    def basis(self, index) -> int:
        """TBTK basis number of a full index (lexicographic order)."""
        b = 0
        for i, extent in zip(index, self.shape):
            b = b * extent + int(i)
        return b

    def csr(self):
        """(rowptr uint32[N+1], col uint32[nnz], val complex128[nnz])."""
        return triplets_to_csr(self.to_basis, self.from_basis, self.amp,
                               self.num_states)


def triplets_to_csr(rows, cols, vals, num_rows):
    """Sort triplets by (row, col) keeping insertion order among duplicates,
    then sum duplicates, as SparseMatrix::constructCSX does for short lists.

    Duplicates are folded from the back (``d0 + (d1 + d2)``), the order of
    SparseMatrix::mergeLIL (SparseMatrix.h:1393-1414).
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.complex128)
    order = np.lexsort((np.arange(rows.size), cols, rows))
    r = rows[order]
    c = cols[order]
    v = vals[order]
    if r.size:
        new = np.ones(r.size, dtype=bool)
        new[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
        starts = np.flatnonzero(new)
        if starts.size == r.size:
            merged = v
        else:
            merged = v[starts].copy()
            counts = np.diff(np.append(starts, r.size))
            for g in np.flatnonzero(counts > 1):
                s0, n = starts[g], counts[g]
                acc = v[s0 + n - 1]
                for y in range(s0 + n - 2, s0 - 1, -1):
                    acc = v[y] + acc
                merged[g] = acc
        r = r[starts]
        c = c[starts]
        v = merged
    rowptr = np.zeros(num_rows + 1, dtype=np.int64)
    np.add.at(rowptr, r + 1, 1)
    rowptr = np.cumsum(rowptr)
    return (rowptr.astype(np.uint32), c.astype(np.uint32),
            np.ascontiguousarray(v))


def _finish(name, shape, to_idx, from_idx, amp):
    to_idx = np.ascontiguousarray(np.stack(to_idx, axis=-1).reshape(-1, len(shape)), dtype=np.int32)
    from_idx = np.ascontiguousarray(np.stack(from_idx, axis=-1).reshape(-1, len(shape)), dtype=np.int32)
    amp = np.ascontiguousarray(np.asarray(amp, dtype=np.complex128).reshape(-1))
    mult = np.ones(len(shape), dtype=np.int64)
    for k in range(len(shape) - 2, -1, -1):
        mult[k] = mult[k + 1] * shape[k + 1]
    to_b = to_idx.astype(np.int64) @ mult
    from_b = from_idx.astype(np.int64) @ mult
    return Lattice(name, tuple(shape), to_idx, from_idx, amp, to_b, from_b)


def _hc(to_idx, from_idx, amp):
    """Interleave each amplitude with its Hermitian conjugate, the order
    ``model << HoppingAmplitude(...) + HC`` inserts them in."""
    t = [np.stack([a, b], axis=-1).reshape(-1) for a, b in zip(to_idx, from_idx)]
    f = [np.stack([b, a], axis=-1).reshape(-1) for a, b in zip(to_idx, from_idx)]
    amps = np.stack([amp, np.conj(amp)], axis=-1).reshape(-1)
    return t, f, amps


def _concat(parts):
    ts, fs, amps = zip(*parts)
    t = [np.concatenate([p[k] for p in ts]) for k in range(len(ts[0]))]
    f = [np.concatenate([p[k] for p in fs]) for k in range(len(fs[0]))]
    return t, f, np.concatenate(amps)


def square(Lx, Ly, *, t=1.0, J=0.5, mu=0.0, W=0.0, alpha=0.0,
           periodic=False, seed=0, name=None):
    """Square lattice with spin; Rashba spin-orbit when alpha != 0."""
    x, y, s = np.meshgrid(np.arange(Lx), np.arange(Ly), np.arange(2),
                          indexing="ij")
    x, y, s = x.reshape(-1), y.reshape(-1), s.reshape(-1)
    parts = []
    # on-site: Zeeman, chemical potential, disorder (shared by both spins)
    onsite = -J * 2.0 * (0.5 - s)
    parts.append(((x, y, s), (x, y, s), onsite.astype(np.complex128)))
    if mu != 0.0:
        parts.append(((x, y, s), (x, y, s),
                      np.full(x.size, -mu, dtype=np.complex128)))
    if W != 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        v = rng.uniform(-W / 2, W / 2, size=Lx * Ly)
        parts.append(((x, y, s), (x, y, s),
                      v[x * Ly + y].astype(np.complex128)))
    # nearest-neighbour hopping +x, +y with HC
    for dx, dy, extent in ((1, 0, Lx), (0, 1, Ly)):
        xs, ys = x + dx, y + dy
        if periodic:
            keep = np.ones(x.size, dtype=bool)
            xs, ys = xs % Lx, ys % Ly
        else:
            keep = (xs < Lx) & (ys < Ly)
        if extent == 1 and periodic:
            keep[:] = False
        tt = (xs[keep], ys[keep], s[keep])
        ff = (x[keep], y[keep], s[keep])
        parts.append(_hc(tt, ff, np.full(keep.sum(), -t, dtype=np.complex128)))
    if alpha != 0.0:
        for dx, dy, extent in ((1, 0, Lx), (0, 1, Ly)):
            for s_to, s_from in ((0, 1), (1, 0)):
                if dx == 1:
                    a = -alpha if s_to == 0 else alpha
                else:
                    a = 1j * alpha
                sel = s == s_from
                xs, ys = x[sel] + dx, y[sel] + dy
                if periodic:
                    keep = np.ones(xs.size, dtype=bool)
                    xs, ys = xs % Lx, ys % Ly
                else:
                    keep = (xs < Lx) & (ys < Ly)
                if extent == 1 and periodic:
                    keep[:] = False
                tt = (xs[keep], ys[keep], np.full(keep.sum(), s_to))
                ff = (x[sel][keep], y[sel][keep], np.full(keep.sum(), s_from))
                parts.append(_hc(tt, ff, np.full(keep.sum(), a,
                                                 dtype=np.complex128)))
    t_idx, f_idx, amp = _concat(parts)
    nm = name or ("rashba" if alpha else "square")
    return _finish(nm, (Lx, Ly, 2), t_idx, f_idx, amp)


def honeycomb(Lx, Ly, *, t=1.0, J=0.5, W=0.0, periodic=True, seed=0,
              name="honeycomb"):
    """Brick-wall honeycomb lattice with spin (index {x, y, a, s})."""
    x, y, a, s = np.meshgrid(np.arange(Lx), np.arange(Ly), np.arange(2),
                             np.arange(2), indexing="ij")
    x, y, a, s = (v.reshape(-1) for v in (x, y, a, s))
    parts = []
    onsite = -J * 2.0 * (0.5 - s)
    parts.append(((x, y, a, s), (x, y, a, s), onsite.astype(np.complex128)))
    if W != 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        v = rng.uniform(-W / 2, W / 2, size=Lx * Ly * 2)
        parts.append(((x, y, a, s), (x, y, a, s),
                      v[(x * Ly + y) * 2 + a].astype(np.complex128)))
    selA = a == 0
    xa, ya, sa = x[selA], y[selA], s[selA]
    for dx, dy in ((0, 0), (-1, 0), (0, -1)):
        xb, yb = xa + dx, ya + dy
        if periodic:
            keep = np.ones(xa.size, dtype=bool)
            if (dx and Lx == 1) or (dy and Ly == 1):
                keep[:] = False
            xb, yb = xb % Lx, yb % Ly
        else:
            keep = (xb >= 0) & (yb >= 0)
        tt = (xb[keep], yb[keep], np.ones(keep.sum(), dtype=np.int64), sa[keep])
        ff = (xa[keep], ya[keep], np.zeros(keep.sum(), dtype=np.int64), sa[keep])
        parts.append(_hc(tt, ff, np.full(keep.sum(), -t, dtype=np.complex128)))
    t_idx, f_idx, amp = _concat(parts)
    return _finish(name, (Lx, Ly, 2, 2), t_idx, f_idx, amp)


def ring(size, *, t=1.0):
    """The 10-site ring of the reference LDOS tests
    (Test/include/TBTK/Test/PropertyExtractor/ChebyshevExpander.h:19-24):
    ``HoppingAmplitude(-t, {n}, {(n+1)%size}) + HC``."""
    n = np.arange(size)
    tt = (n,)
    ff = ((n + 1) % size,)
    t_idx, f_idx, amp = _hc(tt, ff, np.full(size, -t, dtype=np.complex128))
    return _finish("ring", (size,), t_idx, f_idx, amp)


def test_square(size=5, *, mu=-2.0, t=1.0):
    """The 5x5 periodic spinless lattice of the reference coefficient test
    (Test/include/TBTK/Test/Solver/ChebyshevExpander.h:184-197)."""
    x, y = np.meshgrid(np.arange(size), np.arange(size), indexing="ij")
    x, y = x.reshape(-1), y.reshape(-1)
    # insertion order per site: on-site, +x (+HC), +y (+HC)
    to_x, to_y, fr_x, fr_y, amps = [], [], [], [], []
    for xi, yi in zip(x, y):
        to_x.append(xi); to_y.append(yi); fr_x.append(xi); fr_y.append(yi)
        amps.append(-mu)
        for tx, ty in (((xi + 1) % size, yi), (xi, (yi + 1) % size)):
            to_x += [tx, xi]; to_y += [ty, yi]
            fr_x += [xi, tx]; fr_y += [yi, ty]
            amps += [-t, -t]
    return _finish("test_square", (size, size),
                   (np.array(to_x), np.array(to_y)),
                   (np.array(fr_x), np.array(fr_y)), np.array(amps))


def random_sites(lat: Lattice, count: int, seed: int, spin=0):
    """``count`` seeded random lattice sites (spin component ``spin``) as
    basis numbers; distinct when the lattice is large enough."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_sites = lat.num_states // lat.shape[-1]
    pick = rng.choice(n_sites, size=count, replace=count > n_sites)
    return (pick * lat.shape[-1] + spin).astype(np.uint32)
