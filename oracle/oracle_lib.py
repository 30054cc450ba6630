"""ctypes access to the two CPU checkers of the KPM path (test infrastructure).

* :class:`Oracle` — the C restatement in oracle/kpm_oracle.c
  (oracle/_build/libkpm_oracle.so, built by ``make -C oracle``).
* :class:`Reference` — the TBTK reference classes compiled from the reference
  sources with oracle/ref_driver.cpp (oracle/_ref/libtbtkref.so, built by
  ``make -C oracle ref``).  Absent when the reference was never compiled.

Complex arrays cross the boundary as interleaved (re, im) doubles.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent.parent
# Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
# this module.
ORACLE_SO = ROOT / "oracle" / "_build" / "libkpm_oracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libtbtkref.so"

_p = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_u32 = ctypes.c_uint32


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _cx(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


class Oracle:
    def __init__(self, path=ORACLE_SO):
        self.lib = lib = ctypes.CDLL(str(path))
        lib.kpm_csr_from_triplets.restype = _i64
        lib.kpm_csr_from_triplets.argtypes = [_i64, _p, _p, _p, _p, _p, _p, _p]
        lib.kpm_moments.restype = _i
        lib.kpm_moments.argtypes = [_u32, _p, _p, _p, _d, _i, _u32, _i, _p, _p]
        lib.kpm_damp.argtypes = [_i, _i, _d, _p]
        lib.kpm_lookup_table.argtypes = [_i, _i, _p, _d, _p]
        lib.kpm_greens_table.argtypes = [_i, _i, _p, _i, _p, _p]
        lib.kpm_greens_closed.argtypes = [_i, _i, _p, _d, _i, _p, _p]
        lib.kpm_ldos_table.argtypes = [_i, _i, _p, _p, _p]
        lib.kpm_range.argtypes = [_d, _d, _i, _i, _i, _p]

    def csr_from_triplets(self, rows, cols, vals):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        vals = _cx(vals)
        n = rows.size
        nr = int(rows.max()) + 1 if n else 0
        rowptr = np.zeros(nr + 1, dtype=np.uint32)
        col = np.zeros(max(n, 1), dtype=np.uint32)
        val = np.zeros(max(n, 1), dtype=np.complex128)
        num_rows = ctypes.c_uint32(0)
        nnz = self.lib.kpm_csr_from_triplets(
            n, _ptr(rows), _ptr(cols), _ptr(vals), _ptr(rowptr), _ptr(col),
            _ptr(val), ctypes.byref(num_rows))
        return rowptr, col[:nnz].copy(), val[:nnz].copy()

    def moments(self, rowptr, col, val, scale, M, frm, to):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
        col = np.ascontiguousarray(col, dtype=np.uint32)
        val = _cx(val)
        to = np.ascontiguousarray(np.atleast_1d(to), dtype=np.uint32)
        out = np.zeros((to.size, M), dtype=np.complex128)
        rc = self.lib.kpm_moments(rowptr.size - 1, _ptr(rowptr), _ptr(col),
                                  _ptr(val), scale, M, int(frm), to.size,
                                  _ptr(to), _ptr(out))
        if rc != 0:
            raise ValueError("kpm_moments rejected its arguments")
        return out

    def damp(self, mu, broadening):
        mu = _cx(mu).copy()
        K, M = mu.shape
        self.lib.kpm_damp(K, M, broadening, _ptr(mu))
        return mu

    def lookup_table(self, M, energies, scale):
        energies = np.ascontiguousarray(energies, dtype=np.float64)
        table = np.zeros((M, energies.size), dtype=np.complex128)
        self.lib.kpm_lookup_table(M, energies.size, _ptr(energies), scale,
                                  _ptr(table))
        return table

    def greens_table(self, table, type_, coeff):
        coeff = _cx(coeff)
        M, E = table.shape
        out = np.zeros(E, dtype=np.complex128)
        self.lib.kpm_greens_table(M, E, _ptr(np.ascontiguousarray(table)),
                                  type_, _ptr(coeff), _ptr(out))
        return out

    def greens_closed(self, energies, scale, type_, coeff):
        coeff = _cx(coeff)
        energies = np.ascontiguousarray(energies, dtype=np.float64)
        out = np.zeros(energies.size, dtype=np.complex128)
        self.lib.kpm_greens_closed(coeff.size, energies.size, _ptr(energies),
                                   scale, type_, _ptr(coeff), _ptr(out))
        return out

    def ldos_table(self, table, coeff):
        coeff = _cx(coeff)
        M, E = table.shape
        out = np.zeros(E, dtype=np.float64)
        self.lib.kpm_ldos_table(M, E, _ptr(np.ascontiguousarray(table)),
                                _ptr(coeff), _ptr(out))
        return out

    def range(self, lower, upper, res, incl_lo=True, incl_hi=True):
        out = np.zeros(res, dtype=np.float64)
        self.lib.kpm_range(lower, upper, res, int(incl_lo), int(incl_hi),
                           _ptr(out))
        return out


class Reference:
    """The compiled TBTK reference, driven through its public classes."""

    def __init__(self, path=REF_SO):
        self.lib = lib = ctypes.CDLL(str(path))
        lib.ref_model_create.restype = _p
        lib.ref_model_create.argtypes = [_i64, _i, _p, _p, _p]
        lib.ref_model_destroy.argtypes = [_p]
        lib.ref_model_basis_size.restype = _i
        lib.ref_model_basis_size.argtypes = [_p]
        lib.ref_model_basis_index.restype = _i
        lib.ref_model_basis_index.argtypes = [_p, _p, _i]
        lib.ref_model_csr.restype = _i64
        lib.ref_model_csr.argtypes = [_p, _p, _p, _p, _i64, _p]
        lib.ref_coefficients.restype = _i
        lib.ref_coefficients.argtypes = [_p, _d, _i, _d, _i, _i, _p, _p, _p]
        lib.ref_range_value.restype = _d
        lib.ref_range_value.argtypes = [_d, _d, _i, _i, _i, _i]
        lib.ref_greens.restype = _i
        lib.ref_greens.argtypes = [_d, _i, _d, _d, _i, _i, _i, _i, _i, _p, _p]
        lib.ref_ldos.restype = _i
        lib.ref_ldos.argtypes = [_p, _d, _i, _d, _d, _d, _i, _i, _i, _i, _p, _p]
        lib.ref_greens_pe.restype = _i
        lib.ref_greens_pe.argtypes = [_p, _d, _i, _d, _d, _d, _i, _i, _i, _i,
                                      _i, _p, _p, _p]
        lib.ref_property.restype = _i
        lib.ref_property.argtypes = [_p, _d, _i, _d, _d, _d, _i, _i, _d, _d, _i,
                                     _i, _p, _p]
        lib.ref_expectation.restype = _i
        lib.ref_expectation.argtypes = [_p, _d, _i, _d, _d, _d, _i, _i, _d, _d,
                                        _i, _p, _p, _p]
        lib.ref_fermi_dirac.restype = _d
        lib.ref_fermi_dirac.argtypes = [_d, _d, _d]
        lib.ref_property_json.restype = _i64
        lib.ref_property_json.argtypes = [_p, _d, _i, _d, _d, _d, _i, _i, _d, _d, _i,
                                          _i, _i, _i, _p, _p, _p, _i64, _p, _i64]
        lib.ref_json_reserialize.restype = _i64
        lib.ref_json_reserialize.argtypes = [_i, ctypes.c_char_p, _p, _i64, _p, _i64]

    @staticmethod
    def available(path=REF_SO) -> bool:
        return os.path.exists(path)

    def model(self, lat):
        return RefModel(self, lat)

    def range_value(self, lower, upper, res, incl_lo, incl_hi, k):
        return self.lib.ref_range_value(lower, upper, res, int(incl_lo),
                                        int(incl_hi), k)

    def fermi_dirac(self, energies, mu, T):
        """Functions::fermiDiracDistribution at each energy."""
        return np.array([self.lib.ref_fermi_dirac(float(e), mu, T) for e in energies])

    def reserialize(self, kind, text, n_values):
        """TBTK's deserializing constructor on `text` (kind 0 Property::LDOS,
        1 EnergyResolvedProperty<complex<double>>, 2 Property::Density), then
        serialize() again.  Returns (new JSON text, the data array read, as
        n_values doubles)."""
        values = np.zeros(max(n_values, 1), dtype=np.float64)
        raw = text.encode()
        n = self.lib.ref_json_reserialize(kind, raw, None, 0, _ptr(values), n_values)
        buf = ctypes.create_string_buffer(n + 1)
        self.lib.ref_json_reserialize(kind, raw, buf, n + 1, _ptr(values), n_values)
        return buf.value.decode(), values[:n_values]

    def greens(self, scale, coeff, lower, upper, res, type_, use_table,
               incl_lo=True, incl_hi=True):
        coeff = _cx(coeff)
        out = np.zeros(res, dtype=np.complex128)
        self.lib.ref_greens(scale, coeff.size, lower, upper, res, int(incl_lo),
                            int(incl_hi), int(use_table), type_, _ptr(coeff),
                            _ptr(out))
        return out


class RefModel:
    """A TBTK Model built from a :class:`tbtk_b200.lattice.Lattice`."""

    def __init__(self, ref, lat):
        self.ref = ref
        self.lat = lat
        amp = np.ascontiguousarray(lat.amp.view(np.float64))
        self.h = ref.lib.ref_model_create(
            lat.amp.size, lat.idx_len, _ptr(lat.to_index),
            _ptr(lat.from_index), _ptr(amp))

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.lib.ref_model_destroy(self.h)
            self.h = None

    def _idx(self, idx):
        return np.ascontiguousarray(np.asarray(idx, dtype=np.int32).reshape(-1, self.lat.idx_len))

    def basis_size(self):
        return self.ref.lib.ref_model_basis_size(self.h)

    def basis_index(self, idx):
        a = self._idx(idx)
        return self.ref.lib.ref_model_basis_index(self.h, _ptr(a), a.shape[1])

    def csr(self):
        cap = self.lat.amp.size
        rowptr = np.zeros(self.lat.num_states + 1, dtype=np.uint32)
        col = np.zeros(cap, dtype=np.uint32)
        val = np.zeros(cap, dtype=np.complex128)
        nr = ctypes.c_int(0)
        nnz = self.ref.lib.ref_model_csr(self.h, _ptr(rowptr), _ptr(col),
                                         _ptr(val), cap, ctypes.byref(nr))
        assert nnz >= 0
        return rowptr[: nr.value + 1].copy(), col[:nnz].copy(), val[:nnz].copy()

    def coefficients(self, scale, M, broadening, to, frm):
        to = self._idx(to)
        frm = self._idx(frm)
        out = np.zeros((to.shape[0], M), dtype=np.complex128)
        self.ref.lib.ref_coefficients(self.h, scale, M, broadening,
                                      to.shape[0], to.shape[1], _ptr(to),
                                      _ptr(frm), _ptr(out))
        return out

    def ldos(self, scale, M, broadening, lower, upper, res, sites,
             use_table=True):
        sites = self._idx(sites)
        out = np.zeros((sites.shape[0], res), dtype=np.float64)
        self.ref.lib.ref_ldos(self.h, scale, M, broadening, lower, upper, res,
                              int(use_table), sites.shape[0], sites.shape[1],
                              _ptr(sites), _ptr(out))
        return out

    def greens_pe(self, scale, M, broadening, lower, upper, res, type_, to,
                  frm, use_table=True):
        to = self._idx(to)
        frm = self._idx(frm)
        out = np.zeros((to.shape[0], res), dtype=np.complex128)
        self.ref.lib.ref_greens_pe(self.h, scale, M, broadening, lower, upper,
                                   res, int(use_table), type_, to.shape[0],
                                   to.shape[1], _ptr(to), _ptr(frm), _ptr(out))
        return out

    def prop(self, kind, scale, M, broadening, lower, upper, res, T, mu, index,
             use_table=True):
        """One site of calculateSpinPolarizedLDOS (kind 0, [res][2][2]
        complex), calculateDensity (kind 1, scalar) or calculateMagnetization
        (kind 2, [2][2] complex); -1 in `index` marks the spin subindex."""
        idx = np.ascontiguousarray(np.asarray(index, dtype=np.int32))
        n = {0: res * 8, 1: 1, 2: 8}[kind]
        out = np.zeros(n, dtype=np.float64)
        got = self.ref.lib.ref_property(self.h, scale, M, broadening, lower, upper,
                                        res, int(use_table), T, mu, kind, idx.size,
                                        _ptr(idx), _ptr(out))
        assert got == (res if kind == 0 else 1), got
        if kind == 1:
            return out[0]
        c = out.view(np.complex128)
        return c.reshape(res, 2, 2) if kind == 0 else c.reshape(2, 2)

    def property_json(self, kind, scale, M, broadening, lower, upper, res, sites,
                      frm=None, type_=3, T=300.0, mu=0.0, use_table=True):
        """A property from the reference's PropertyExtractor and its JSON
        serialization: kind 0 calculateLDOS(sites), 1
        calculateGreensFunctions(sites, frm, type_), 2 calculateDensity(sites).
        Returns (JSON text, data array; complex for kind 1)."""
        sites = self._idx(sites)
        frm_a = self._idx(frm if frm is not None else sites[0])
        n_values = sites.shape[0] * (res if kind == 0 else 2 * res if kind == 1 else 1)
        values = np.zeros(n_values, dtype=np.float64)
        args = (self.h, scale, M, broadening, lower, upper, res, int(use_table), T, mu,
                kind, type_, sites.shape[0], sites.shape[1], _ptr(sites), _ptr(frm_a))
        n = self.ref.lib.ref_property_json(*args, None, 0, _ptr(values), n_values)
        buf = ctypes.create_string_buffer(n + 1)
        self.ref.lib.ref_property_json(*args, buf, n + 1, _ptr(values), n_values)
        data = values.view(np.complex128) if kind == 1 else values
        return buf.value.decode(), data

    def expectation(self, scale, M, broadening, lower, upper, res, T, mu, to, frm,
                    use_table=True):
        """calculateExpectationValue(to, from)."""
        to = np.ascontiguousarray(np.asarray(to, dtype=np.int32))
        frm = np.ascontiguousarray(np.asarray(frm, dtype=np.int32))
        out = np.zeros(2, dtype=np.float64)
        self.ref.lib.ref_expectation(self.h, scale, M, broadening, lower, upper, res,
                                     int(use_table), T, mu, to.size, _ptr(to), _ptr(frm),
                                     _ptr(out))
        return complex(out[0], out[1])


# ---------------------------------------------------------------------------
# The PropertyExtractor's other properties from NonPrincipal Green's
# functions, restated with the reference's expressions and operation order
# (Lib/src/PropertyExtractor/ChebyshevExpander.cpp:297-327,584-720): scalar
# IEEE arithmetic as std::complex<double> evaluates it (products
# (ac - bd, ad + bc), division and scaling by a real number per component),
# sums over the energies in order.

_PI = float(np.pi)


def _cmul(a, b):
    return complex(a.real * b.real - a.imag * b.imag, a.real * b.imag + a.imag * b.real)


def _scale(z, x):
    return complex(z.real * x, z.imag * x)


def _div(z, x):
    return complex(z.real / x, z.imag / x)


def sp_ldos_from_greens(G4):
    """G4 [4][E]: G_NP of (to spin n/2, from spin n%2).  Returns [E][2][2]:
    data.at(n/2, n%2) += -i*G/M_PI (calculateSP_LDOSCallback, :686-720)."""
    G4 = np.asarray(G4)
    out = np.zeros((G4.shape[1], 2, 2), dtype=np.complex128)
    mi = complex(-0.0, -1.0)
    for n in range(4):
        for e in range(G4.shape[1]):
            v = _div(_cmul(mi, complex(G4[n, e])), _PI)
            out[e, n // 2, n % 2] = complex(0.0 + v.real, 0.0 + v.imag)
    return out


def density_from_greens(G, occupation, dE):
    """data += weight*imag(G)/M_PI*dE over the energies (:584-616)."""
    d = 0.0
    for e in range(len(G)):
        d += occupation[e] * complex(G[e]).imag / _PI * dE
    return d


def magnetization_from_greens(G4, occupation, dE):
    """data.at(n/2, n%2) += weight*(-i)*G/M_PI*dE (:618-659)."""
    out = np.zeros((2, 2), dtype=np.complex128)
    mi = complex(-0.0, -1.0)
    for n in range(4):
        v = complex(0.0, 0.0)
        for e in range(G4.shape[1]):
            t = _scale(_div(_cmul(_scale(mi, occupation[e]), complex(G4[n, e])), _PI), dE)
            v = complex(v.real + t.real, v.imag + t.imag)
        out[n // 2, n % 2] = v
    return out


def expectation_from_greens(G, occupation, dE):
    """expectationValue -= weight*conj(i*G)*dE/M_PI (:297-327)."""
    v = complex(0.0, 0.0)
    for e in range(len(G)):
        ig = _cmul(complex(0.0, 1.0), complex(G[e]))
        t = _div(_scale(_scale(ig.conjugate(), occupation[e]), dE), _PI)
        v = complex(v.real - t.real, v.imag - t.imag)
    return v
