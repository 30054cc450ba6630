"""Python host layer over the C ABI of include/tbtkkpm.h (libtbtkkpm.so).

The classes mirror the TBTK interface of the KPM path so that calling code
reads like TBTK's own:

* :class:`ChebyshevExpander` — ``Solver::ChebyshevExpander``
  (Lib/include/TBTK/Solver/ChebyshevExpander.h:72-223): the same setters,
  defaults (scale 1.1, 1000 coefficients, broadening 1e-6, window
  Range(-1, 1, 1000)) and argument checks, ``calculateCoefficients`` and
  ``generateGreensFunction``.  The model is a CSR matrix in TBTK basis
  order (what ``HoppingAmplitudeSet::getSparseMatrix`` returns).
* :class:`PropertyExtractor` — ``PropertyExtractor::ChebyshevExpander``
  (Lib/include/TBTK/PropertyExtractor/ChebyshevExpander.h:51-178):
  ``setEnergyWindow``, ``calculateLDOS``, ``calculateGreensFunctions``,
  ``calculateSpinPolarizedLDOS``, ``calculateDensity``,
  ``calculateMagnetization`` and ``calculateExpectationValue`` over basis
  indices (occupation weights at the window energies as an argument).

Where the reference exits through TBTKAssert/TBTKExit
(Lib/include/Utilities/TBTK/TBTKMacros.h:55-94) these classes raise
:class:`TBTKError`.  There is no CPU fallback: importing this module on a
machine without the built library raises, and every compute call needs a
CUDA device.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "lib" / "libtbtkkpm.so"

OK = 0
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_MEMORY = -3
ERR_TIMEOUT = -4
ERR_UNSUPPORTED = -5
ERR_STATE = -6
ERR_CANCELLED = -7

ADVANCED, RETARDED, PRINCIPAL, NONPRINCIPAL = 0, 1, 2, 3
FP64, MIXED, MIXED_DIRECT = 0, 1, 2

_TYPES = {"Advanced": ADVANCED, "Retarded": RETARDED, "Principal": PRINCIPAL,
          "NonPrincipal": NONPRINCIPAL}


class TBTKError(RuntimeError):
    """A failed call of the C ABI (status, message)."""

    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


_p = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64

# (name, restype, argtypes) for every entry point of include/tbtkkpm.h
SIGNATURES = [
    ("tbtkkpm_last_error", ctypes.c_char_p, []),
    ("tbtkkpm_version", _i, []),
    ("tbtkkpm_device_count", _i, [_p]),
    ("tbtkkpm_set_device", _i, [_i]),
    ("tbtkkpm_kernel_launches", _u64, []),
    ("tbtkkpm_matrix_set_profiling", _i, [_p, _i]),
    ("tbtkkpm_matrix_profile", _i, [_p, _p, _p, _p]),
    ("tbtkkpm_matrix_create_csr", _i, [_p, _p, _p, _u32, _d, _p]),
    ("tbtkkpm_matrix_create_triplets", _i, [_p, _p, _p, _u64, _u32, _d, _p]),
    ("tbtkkpm_matrix_destroy", _i, [_p]),
    ("tbtkkpm_matrix_set_stream", _i, [_p, _p]),
    ("tbtkkpm_matrix_shape", _i, [_p, _p, _p]),
    ("tbtkkpm_matrix_download_csr", _i, [_p, _p, _p, _p]),
    ("tbtkkpm_moments", _i, [_p, _u32, _p, _u32, _u32, _d, _p]),
    ("tbtkkpm_moments_noalloc", _i, [_p, _p, _p, _u32, _u64, _d, _u32, _p, _u32, _u32, _d, _p, _p]),
    ("tbtkkpm_moments_batched", _i, [_p, _p, _u32, _p, _p, _u32, _u32, _d, _i, _p, _p]),
    ("tbtkkpm_table_create", _i, [_u32, _p, _u32, _d, _p]),
    ("tbtkkpm_table_upload", _i, [_u32, _u32, _p, _p]),
    ("tbtkkpm_table_create_clenshaw", _i, [_u32, _p, _u32, _d, _p]),
    ("tbtkkpm_table_create_chebyshev", _i, [_u32, _u32, _d, _p, _p]),
    ("tbtkkpm_table_destroy", _i, [_p]),
    ("tbtkkpm_greens", _i, [_p, _p, _u32, _i, _p]),
    ("tbtkkpm_ldos", _i, [_p, _p, _u32, _p]),
    ("tbtkkpm_ldos_sites", _i, [_p, _p, _p, _u32, _d, _i, _p, _p]),
    ("tbtkkpm_matrix_autotune", _i, [_p, _u32, _i, _i, _u32, _p, _p, _p, _p]),
    ("tbtkkpm_matrix_set_config", _i, [_p, _u32, _i, _i, _i, _i, _i]),
    ("tbtkkpm_step_configs", _i, [_i, _i, _p, _i]),
    ("tbtkkpm_matrix_set_real", _i, [_p, _i]),
    ("tbtkkpm_matrix_real", _i, [_p, _p, _p]),
    ("tbtkkpm_matrix_step_configs", _i, [_p, _i, _i, _p, _i]),
    ("tbtkkpm_matrix_set_fp64_head", _i, [_p, _u32]),
    ("tbtkkpm_matrix_set_wait_limit", _i, [_p, _u32]),
    ("tbtkkpm_matrix_fp64_head", _i, [_p, _p, _p]),
    ("tbtkkpm_matrix_set_batch_width", _i, [_p, _i, _u32]),
    ("tbtkkpm_matrix_batch_width", _i, [_p, _i, _i, _p]),
    ("tbtkkpm_spin_polarized_ldos", _i, [_p, _p, _p, _p, _u32, _d, _i, _p]),
    ("tbtkkpm_density", _i, [_p, _p, _p, _u32, _d, _i, _p, _d, _p]),
    ("tbtkkpm_magnetization", _i, [_p, _p, _p, _p, _u32, _d, _i, _p, _d, _p]),
    ("tbtkkpm_expectation_values", _i, [_p, _p, _p, _p, _u32, _d, _i, _p, _d, _p]),
    ("tbtkkpm_server_create", _i, [_u32, _p, _u32, _u64, _u32, _d, _p]),
    ("tbtkkpm_server_add_model", _i, [_p, _p, _p, _p, _u32, _d, _u32, _p]),
    ("tbtkkpm_server_submit", _i, [_p, _u32, _p, _u32, _u32, _d, _p]),
    ("tbtkkpm_server_submit_greens", _i, [_p, _u32, _p, _p, _u32, _u32, _d, _i, _p]),
    ("tbtkkpm_server_wait", _i, [_p, _u64, _d, _p, _p, _p]),
    ("tbtkkpm_server_wait_greens", _i, [_p, _u64, _d, _p, _p, _p]),
    ("tbtkkpm_server_cancel", _i, [_p, _u64]),
    ("tbtkkpm_server_stats", _i, [_p, _p, _u32]),
    ("tbtkkpm_server_autotune", _i, [_p, _u32, _u32, _p, _p, _p, _p]),
    ("tbtkkpm_server_set_config", _i, [_p, _u32, _i, _i, _i]),
    ("tbtkkpm_server_step_configs", _i, [_i, _u32, _p, _i]),
    ("tbtkkpm_server_set_wait_limit", _i, [_p, _u32]),
    ("tbtkkpm_server_set_graphs", _i, [_p, _i]),
    ("tbtkkpm_server_set_adaptive_width", _i, [_p, _i]),
    ("tbtkkpm_server_set_real", _i, [_p, _i]),
    ("tbtkkpm_server_set_fp64_head", _i, [_p, _u32]),
    ("tbtkkpm_server_set_table_free", _i, [_p, _i]),
    ("tbtkkpm_server_destroy", _i, [_p]),
]

PENDING = 1
STAT_NAMES = ["completed", "p50_ms", "p99_ms", "mean_ms", "reruns", "ticks", "steps",
              "lane_steps", "resident_bytes", "evictions", "waited", "busy_s", "step_s",
              "step_bytes", "finish_s", "rerun_s", "join_s", "plan_s", "tick_s", "graph_ticks",
              "relayouts"]


def step_configs(precision, ldos=True):
    """Compiled step configurations (tpr, vpt, variant) of the kernels a call
    at this precision uses; variant 2-4 is a register cap, 100 + 10*S + W a
    bulk-copy kernel with S stages per warp and W warps per block."""
    lib = load_library()
    n = lib.tbtkkpm_step_configs(int(precision), int(bool(ldos)), None, 0)
    if n < 0:
        raise TBTKError(ERR_ARGUMENT, f"unknown precision {precision}")
    out = np.zeros(3 * n, dtype=np.int32)
    lib.tbtkkpm_step_configs(int(precision), int(bool(ldos)), _ptr(out), n)
    return [tuple(int(v) for v in out[3 * i:3 * i + 3]) for i in range(n)]


def padded_width(B, precision):
    """Batch columns the library allocates for B sources."""
    widths = [1, 2, 4, 8, 16, 32, 64, 128] + ([256] if precision != FP64 else [])
    for w in widths:
        if B <= w:
            return w
    raise TBTKError(ERR_ARGUMENT, f"batch of {B} exceeds one launch")


def configs_for(B, precision, ldos=True):
    """All compiled (tpr, vpt, variant) serving batches of B sources."""
    w = padded_width(B, precision)
    return [c for c in step_configs(precision, ldos) if c[0] * c[1] == w]

_lib = None


def load_library(path=LIB_PATH):
    """Loads libtbtkkpm.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not pathlib.Path(path).exists():
            raise ImportError(
                f"{path} is missing: build it with __graft_entry__.build() "
                "(make -C tbtk_b200/csrc); there is no CPU fallback")
        lib = ctypes.CDLL(str(path))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _check(rc):
    if rc != OK:
        msg = load_library().tbtkkpm_last_error().decode(errors="replace")
        raise TBTKError(rc, msg)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _u32a(a):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(a)), dtype=np.uint32)


def _cxa(a):
    return np.ascontiguousarray(np.asarray(a), dtype=np.complex128)


def kernel_launches() -> int:
    """Kernels launched by this process through the library."""
    return int(load_library().tbtkkpm_kernel_launches())


def device_count() -> int:
    n = ctypes.c_int(0)
    _check(load_library().tbtkkpm_device_count(ctypes.byref(n)))
    return n.value


def tbtk_range(lower, upper, resolution, include_lower=True,
               include_upper=True):
    """Energies of TBTK's ``Range`` (Lib/src/Utilities/Range.cpp:30-57):
    ``start + k*dx`` with the reference's dx/start rules."""
    if resolution <= 1:
        raise TBTKError(ERR_ARGUMENT, "'resolution' must be larger than 1.")
    if include_lower and include_upper:
        dx = (upper - lower) / (resolution - 1)
    elif include_lower or include_upper:
        dx = (upper - lower) / resolution
    else:
        dx = (upper - lower) / (resolution + 1)
    start = lower if include_lower else lower + dx
    return np.array([start + k * dx for k in range(resolution)])


class Matrix:
    """Device copy of H/s (the C ABI's ``tbtkkpm_matrix``)."""

    def __init__(self, handle, N):
        self._h = handle
        self.N = N

    @classmethod
    def from_csr(cls, rowptr, col, val, scale):
        lib = load_library()
        rowptr = _u32a(rowptr)
        col = _u32a(col)
        val = _cxa(val)
        h = ctypes.c_void_p()
        _check(lib.tbtkkpm_matrix_create_csr(_ptr(rowptr), _ptr(col), _ptr(val),
                                             rowptr.size - 1, float(scale),
                                             ctypes.byref(h)))
        return cls(h, rowptr.size - 1)

    @classmethod
    def from_triplets(cls, rows, cols, vals, N, scale):
        lib = load_library()
        rows = _u32a(rows)
        cols = _u32a(cols)
        vals = _cxa(vals)
        h = ctypes.c_void_p()
        _check(lib.tbtkkpm_matrix_create_triplets(_ptr(rows), _ptr(cols), _ptr(vals),
                                                  rows.size, N, float(scale),
                                                  ctypes.byref(h)))
        return cls(h, N)

    def shape(self):
        n = ctypes.c_uint32()
        nnz = ctypes.c_uint64()
        _check(load_library().tbtkkpm_matrix_shape(self._h, ctypes.byref(n),
                                                   ctypes.byref(nnz)))
        return n.value, nnz.value

    def set_stream(self, cuda_stream):
        """Issue this handle's work on ``cuda_stream`` (an int cudaStream_t,
        e.g. ``torch.cuda.current_stream().cuda_stream``; 0/None restores
        the handle's own stream)."""
        _check(load_library().tbtkkpm_matrix_set_stream(self._h, cuda_stream or None))

    def autotune(self, B, precision, ldos=True, probe_steps=8):
        """Times the compiled step configurations for batches of B sources
        and keeps the fastest on this handle; returns (tpr, vpt, minb,
        ms per step)."""
        t = ctypes.c_int()
        v = ctypes.c_int()
        mb = ctypes.c_int()
        ms = ctypes.c_double()
        _check(load_library().tbtkkpm_matrix_autotune(
            self._h, int(B), int(precision), int(bool(ldos)), int(probe_steps),
            ctypes.byref(t), ctypes.byref(v), ctypes.byref(mb), ctypes.byref(ms)))
        return t.value, v.value, mb.value, ms.value

    def set_real(self, enable=True):
        """Allow (default) or forbid real float vectors at mixed precision."""
        _check(load_library().tbtkkpm_matrix_set_real(self._h, int(bool(enable))))

    def real(self):
        """(values are real, real vectors in use at mixed precision)."""
        vr, use = ctypes.c_int(), ctypes.c_int()
        _check(load_library().tbtkkpm_matrix_real(self._h, ctypes.byref(vr), ctypes.byref(use)))
        return bool(vr.value), bool(use.value)

    def set_wait_limit(self, polls=0xFFFFFFFF):
        """Polls per staged-row wait of the tile-staged steps
        (tbtkkpm_matrix_set_wait_limit; the default restores the library's
        bound, 0 makes every such wait give up at once)."""
        _check(load_library().tbtkkpm_matrix_set_wait_limit(self._h, int(polls)))

    def set_fp64_head(self, steps=32):
        """FP64 steps at the head of MIXED doubling runs (0 turns it off)."""
        _check(load_library().tbtkkpm_matrix_set_fp64_head(self._h, int(steps)))

    def fp64_head(self):
        """(head steps setting, pattern allows a head)."""
        st, sym = ctypes.c_uint32(), ctypes.c_int()
        _check(load_library().tbtkkpm_matrix_fp64_head(self._h, ctypes.byref(st), ctypes.byref(sym)))
        return st.value, bool(sym.value)

    def set_batch_width(self, precision, width=0):
        """Sources per recursion batch at this precision (0: the library's
        choice)."""
        _check(load_library().tbtkkpm_matrix_set_batch_width(self._h, int(precision),
                                                              int(width)))

    def batch_width(self, precision, ldos=True):
        """Sources per batch that ldos_sites (ldos=True) or the moment calls
        use at this precision."""
        w = ctypes.c_uint32()
        _check(load_library().tbtkkpm_matrix_batch_width(self._h, int(precision), int(ldos),
                                                         ctypes.byref(w)))
        return w.value

    def configs_for(self, B, precision, ldos=True):
        """The compiled (tpr, vpt, variant) this matrix's calls for B sources
        choose from (real-vector kernels for a real matrix at mixed
        precision)."""
        lib = load_library()
        n = lib.tbtkkpm_matrix_step_configs(self._h, int(precision), int(bool(ldos)), None, 0)
        out = np.zeros(3 * max(n, 0), dtype=np.int32)
        lib.tbtkkpm_matrix_step_configs(self._h, int(precision), int(bool(ldos)), _ptr(out), n)
        w = padded_width(B, precision)
        return [tuple(int(v) for v in out[3 * i:3 * i + 3]) for i in range(n)
                if out[3 * i] * out[3 * i + 1] == w]

    def set_config(self, B, precision, tpr, vpt, minb, ldos=True):
        _check(load_library().tbtkkpm_matrix_set_config(
            self._h, int(B), int(precision), int(bool(ldos)), int(tpr), int(vpt), int(minb)))

    def set_profiling(self, enable=True):
        _check(load_library().tbtkkpm_matrix_set_profiling(self._h, int(enable)))

    def profile(self):
        """(recursion ms, energy-sum ms, recursion-step launches) accumulated
        since the last read, from CUDA events on the handle's stream."""
        r = ctypes.c_double()
        e = ctypes.c_double()
        n = ctypes.c_uint64()
        _check(load_library().tbtkkpm_matrix_profile(self._h, ctypes.byref(r),
                                                     ctypes.byref(e), ctypes.byref(n)))
        return r.value, e.value, n.value

    def download_csr(self):
        N, nnz = self.shape()
        rowptr = np.zeros(N + 1, dtype=np.uint32)
        col = np.zeros(max(nnz, 1), dtype=np.uint32)
        val = np.zeros(max(nnz, 1), dtype=np.complex128)
        _check(load_library().tbtkkpm_matrix_download_csr(self._h, _ptr(rowptr),
                                                          _ptr(col), _ptr(val)))
        return rowptr, col[:nnz], val[:nnz]

    def moments(self, frm, to, M, broadening):
        to = _u32a(to)
        out = np.zeros((to.size, M), dtype=np.complex128)
        _check(load_library().tbtkkpm_moments(self._h, int(frm), _ptr(to), to.size,
                                              M, float(broadening), _ptr(out)))
        return out

    def moments_batched(self, frm, to, owner, M, broadening, precision=FP64):
        frm = _u32a(frm)
        to = _u32a(to)
        owner = _u32a(owner)
        out = np.zeros((to.size, M), dtype=np.complex128)
        err = np.zeros(to.size, dtype=np.float64)
        _check(load_library().tbtkkpm_moments_batched(
            self._h, _ptr(frm), frm.size, _ptr(to), _ptr(owner), to.size, M,
            float(broadening), int(precision), _ptr(out), _ptr(err)))
        return out, err

    def ldos_sites(self, table, sites, broadening, precision=FP64):
        sites = _u32a(sites)
        out = np.zeros((sites.size, table.E), dtype=np.float64)
        err = np.zeros(sites.size, dtype=np.float64)
        _check(load_library().tbtkkpm_ldos_sites(self._h, table._h, _ptr(sites),
                                                 sites.size, float(broadening),
                                                 int(precision), _ptr(out), _ptr(err)))
        return out, err

    def spin_polarized_ldos(self, table, up, down, broadening, precision=FP64):
        """[S][E][2][2] complex: -i G_NP(spin a, spin b) / pi per site
        (PropertyExtractor::ChebyshevExpander::calculateSpinPolarizedLDOS)."""
        up, down = _u32a(up), _u32a(down)
        if up.size != down.size:
            raise ValueError("up and down need one row per site")
        out = np.zeros((up.size, table.E, 2, 2), dtype=np.complex128)
        _check(load_library().tbtkkpm_spin_polarized_ldos(
            self._h, table._h, _ptr(up), _ptr(down), up.size, float(broadening),
            int(precision), _ptr(out)))
        return out

    def density(self, table, sites, broadening, occupation, dE, precision=FP64):
        """[S]: sum_e occupation[e] Im G_NP / pi dE (calculateDensity)."""
        sites = _u32a(sites)
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        if occ.size != table.E:
            raise ValueError("occupation needs one value per table energy")
        out = np.zeros(sites.size, dtype=np.float64)
        _check(load_library().tbtkkpm_density(
            self._h, table._h, _ptr(sites), sites.size, float(broadening), int(precision),
            _ptr(occ), float(dE), _ptr(out)))
        return out

    def magnetization(self, table, up, down, broadening, occupation, dE, precision=FP64):
        """[S][2][2] complex: sum_e occupation[e] (-i) G_NP(a, b) / pi dE
        (calculateMagnetization)."""
        up, down = _u32a(up), _u32a(down)
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        if up.size != down.size or occ.size != table.E:
            raise ValueError("one up and one down row per site, one occupation per energy")
        out = np.zeros((up.size, 2, 2), dtype=np.complex128)
        _check(load_library().tbtkkpm_magnetization(
            self._h, table._h, _ptr(up), _ptr(down), up.size, float(broadening),
            int(precision), _ptr(occ), float(dE), _ptr(out)))
        return out

    def expectation_values(self, table, to, frm, broadening, occupation, dE,
                           precision=FP64):
        """[P] complex <c_to^dagger c_from> (calculateExpectationValue)."""
        to, frm = _u32a(to), _u32a(frm)
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        if to.size != frm.size or occ.size != table.E:
            raise ValueError("one from per to, one occupation per energy")
        out = np.zeros(to.size, dtype=np.complex128)
        _check(load_library().tbtkkpm_expectation_values(
            self._h, table._h, _ptr(to), _ptr(frm), to.size, float(broadening),
            int(precision), _ptr(occ), float(dE), _ptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            load_library().tbtkkpm_matrix_destroy(self._h)
            self._h = None

    __del__ = close


class Table:
    """Device lookup table T[n][e] (the C ABI's ``tbtkkpm_table``)."""

    def __init__(self, handle, M, E):
        self._h = handle
        self.M = M
        self.E = E

    @classmethod
    def create(cls, M, energies, scale):
        energies = np.ascontiguousarray(energies, dtype=np.float64)
        h = ctypes.c_void_p()
        _check(load_library().tbtkkpm_table_create(M, _ptr(energies), energies.size,
                                                   float(scale), ctypes.byref(h)))
        return cls(h, M, energies.size)

    @classmethod
    def create_clenshaw(cls, M, energies, scale):
        """A table handle without the M x E table: energy sums by Clenshaw
        recurrences (tbtkkpm_table_create_clenshaw)."""
        energies = np.ascontiguousarray(energies, dtype=np.float64)
        h = ctypes.c_void_p()
        _check(load_library().tbtkkpm_table_create_clenshaw(M, _ptr(energies), energies.size,
                                                            float(scale), ctypes.byref(h)))
        return cls(h, M, energies.size)

    @classmethod
    def create_chebyshev(cls, M, E, scale):
        """A table handle on the grid of E Chebyshev nodes (E a power of two,
        at most 4096): energy sums by one FFT per vector
        (tbtkkpm_table_create_chebyshev).  The ascending grid is in
        ``.energies``."""
        energies = np.zeros(int(E), dtype=np.float64)
        h = ctypes.c_void_p()
        _check(load_library().tbtkkpm_table_create_chebyshev(int(M), int(E), float(scale),
                                                             _ptr(energies), ctypes.byref(h)))
        t = cls(h, M, int(E))
        t.energies = energies
        return t

    @classmethod
    def upload(cls, table):
        table = _cxa(table)
        M, E = table.shape
        h = ctypes.c_void_p()
        _check(load_library().tbtkkpm_table_upload(M, E, _ptr(table), ctypes.byref(h)))
        return cls(h, M, E)

    def greens(self, mu, type_):
        mu = _cxa(np.atleast_2d(mu))
        out = np.zeros((mu.shape[0], self.E), dtype=np.complex128)
        _check(load_library().tbtkkpm_greens(self._h, _ptr(mu), mu.shape[0],
                                             int(type_), _ptr(out)))
        return out

    def ldos(self, mu):
        mu = _cxa(np.atleast_2d(mu))
        out = np.zeros((mu.shape[0], self.E), dtype=np.float64)
        _check(load_library().tbtkkpm_ldos(self._h, _ptr(mu), mu.shape[0], _ptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            load_library().tbtkkpm_table_destroy(self._h)
            self._h = None

    __del__ = close


class Server:
    """Continuous-batching LDOS and Green's-function service over many
    device-resident models (the C ABI's ``tbtkkpm_server``).  ``submit``
    queues the LDOS of up to ``width`` sites of a registered model and
    ``submit_greens`` the Green's functions of up to ``width`` (to, from)
    pairs; both return a request id.  ``wait`` returns ``(ldos [K][E], err
    [K], rerun [K])``, or ``(G [K][E] complex, err, rerun)`` for a
    Green's-function request, once it is done (``None`` on timeout);
    ``cancel`` stops a queued or running request (its ``wait`` then raises
    ``TBTKError`` with ``ERR_CANCELLED``).  Any thread may submit and
    wait."""

    def __init__(self, max_moments, energies, hbm_budget, tick_steps=64, tolerance=1e-6):
        self.energies = np.ascontiguousarray(energies, dtype=np.float64)
        self.E = self.energies.size
        h = ctypes.c_void_p()
        _check(load_library().tbtkkpm_server_create(
            int(max_moments), _ptr(self.energies), self.E, int(hbm_budget), int(tick_steps),
            float(tolerance), ctypes.byref(h)))
        self._h = h
        self._sites = {}

    def add_model(self, rowptr, col, val, scale, width):
        rowptr, col, val = _u32a(rowptr), _u32a(col), _cxa(val)
        mid = ctypes.c_uint32()
        _check(load_library().tbtkkpm_server_add_model(
            self._h, _ptr(rowptr), _ptr(col), _ptr(val), rowptr.size - 1, float(scale),
            int(width), ctypes.byref(mid)))
        return mid.value

    def submit(self, model, sites, M, broadening):
        sites = _u32a(sites)
        rid = ctypes.c_uint64()
        _check(load_library().tbtkkpm_server_submit(self._h, int(model), _ptr(sites), sites.size,
                                                    int(M), float(broadening), ctypes.byref(rid)))
        self._sites[rid.value] = (sites.size, False)
        return rid.value

    def submit_greens(self, model, to, from_, M, broadening, type=NONPRINCIPAL):
        """Green's functions G(to[k], from_[k]) of ``type`` (a type code or
        its name, as ``ChebyshevExpander.Type``)."""
        to, from_ = _u32a(to), _u32a(from_)
        if to.size != from_.size:
            raise TBTKError(ERR_ARGUMENT, "submit_greens: to and from differ in length")
        type = _TYPES.get(type, type)
        rid = ctypes.c_uint64()
        _check(load_library().tbtkkpm_server_submit_greens(
            self._h, int(model), _ptr(to), _ptr(from_), to.size, int(M), float(broadening),
            int(type), ctypes.byref(rid)))
        self._sites[rid.value] = (to.size, True)
        return rid.value

    def wait(self, request, timeout=600.0):
        K, greens = self._sites[request]
        out = np.zeros((K, self.E), dtype=np.complex128 if greens else np.float64)
        err = np.zeros(K, dtype=np.float64)
        rerun = np.zeros(K, dtype=np.int32)
        fn = (load_library().tbtkkpm_server_wait_greens if greens
              else load_library().tbtkkpm_server_wait)
        rc = fn(self._h, ctypes.c_uint64(request), float(timeout), _ptr(out), _ptr(err),
                _ptr(rerun))
        if rc == PENDING:
            return None
        del self._sites[request]
        _check(rc)
        return out, err, rerun

    def cancel(self, request):
        _check(load_library().tbtkkpm_server_cancel(self._h, ctypes.c_uint64(request)))

    def stats(self):
        out = np.zeros(len(STAT_NAMES), dtype=np.float64)
        _check(load_library().tbtkkpm_server_stats(self._h, _ptr(out), out.size))
        return dict(zip(STAT_NAMES, out.tolist()))

    def autotune(self, width, probe_steps=8):
        t, v, m, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(load_library().tbtkkpm_server_autotune(
            self._h, int(width), int(probe_steps), ctypes.byref(t), ctypes.byref(v),
            ctypes.byref(m), ctypes.byref(ms)))
        return {"tpr": t.value, "vpt": v.value, "minb": m.value, "ms_per_step": ms.value}

    @staticmethod
    def step_configs(width, real):
        """Compiled step configurations (tpr, vpt, variant) of a lane width
        for real float lanes or complex64 lanes."""
        lib = load_library()
        n = lib.tbtkkpm_server_step_configs(int(bool(real)), int(width), None, 0)
        out = np.zeros(3 * max(n, 1), dtype=np.int32)
        lib.tbtkkpm_server_step_configs(int(bool(real)), int(width), _ptr(out), n)
        return [tuple(int(v) for v in out[3 * i:3 * i + 3]) for i in range(n)]

    def set_config(self, width, tpr, vpt, minb):
        _check(load_library().tbtkkpm_server_set_config(self._h, int(width), int(tpr), int(vpt),
                                                        int(minb)))

    def set_graphs(self, enable=True):
        """Replay a captured CUDA graph per tick (default) or launch directly."""
        _check(load_library().tbtkkpm_server_set_graphs(self._h, int(bool(enable))))

    def set_adaptive_width(self, enable=True):
        """Step each model at the narrowest width that covers its busy lanes
        (default) or always at its full lane count."""
        _check(load_library().tbtkkpm_server_set_adaptive_width(self._h, int(bool(enable))))

    def set_wait_limit(self, polls=0xFFFFFFFF):
        """Polls per staged-row wait of the tile-staged steps (default: the
        library's bound; 0 makes every wait give up at once)."""
        _check(load_library().tbtkkpm_server_set_wait_limit(self._h, int(polls)))

    def set_real(self, enable=True):
        """Real float lanes for real models added from now on (default)."""
        _check(load_library().tbtkkpm_server_set_real(self._h, int(bool(enable))))

    def set_fp64_head(self, steps=32):
        """FP64 head steps of the lanes of models added from now on."""
        _check(load_library().tbtkkpm_server_set_fp64_head(self._h, int(steps)))

    def set_table_free(self, enable=True):
        """Clenshaw energy sums (no lookup table) for scales first used from now on."""
        _check(load_library().tbtkkpm_server_set_table_free(self._h, int(bool(enable))))

    def close(self):
        if getattr(self, "_h", None):
            load_library().tbtkkpm_server_destroy(self._h)
            self._h = None

    __del__ = close


class ChebyshevExpander:
    """``Solver::ChebyshevExpander`` over the B200 kernels.

    Coefficients and Green's functions always run on the GPU here; the
    ``set...OnGPU`` flags are kept for interface compatibility and
    ``setUseLookupTable(False)`` with GPU Green's functions is rejected as in
    ``ensureLookupTableIsReady`` (ChebyshevExpander.h:548-566).
    """

    Type = _TYPES

    def __init__(self):
        self.scaleFactor = 1.1
        self.numCoefficients = 1000
        self.broadening = 1e-6
        self.energyWindow = tbtk_range(-1, 1, 1000)
        self.calculateCoefficientsOnGPU = True
        self.generateGreensFunctionsOnGPU = True
        self.useLookupTable = True
        self.precision = FP64
        self._csr = None
        self._matrix = None
        self._table = None

    # -- model -------------------------------------------------------------
    def setModel(self, csr):
        """csr = (rowptr, col, val) of H in TBTK basis order."""
        self._csr = csr
        self._matrix = None

    def _get_matrix(self):
        if self._csr is None:
            raise TBTKError(ERR_STATE, "Solver::ChebyshevExpander: no model set")
        if self._matrix is None:
            self._matrix = Matrix.from_csr(*self._csr, self.scaleFactor)
        return self._matrix

    # -- setters (ChebyshevExpander.h:394-489) ------------------------------
    def setScaleFactor(self, scaleFactor):
        if not scaleFactor > 0:
            raise TBTKError(ERR_ARGUMENT, f"The 'scaleFactor={scaleFactor}' has to be larger than '0'.")
        self.scaleFactor = float(scaleFactor)
        self._matrix = None
        self._table = None

    def getScaleFactor(self):
        return self.scaleFactor

    def setNumCoefficients(self, numCoefficients):
        self.numCoefficients = int(numCoefficients)
        self._table = None

    def getNumCoefficients(self):
        return self.numCoefficients

    def setBroadening(self, broadening):
        self.broadening = float(broadening)

    def getBroadening(self):
        return self.broadening

    def setEnergyWindow(self, energies):
        energies = np.asarray(energies, dtype=np.float64)
        eps = np.finfo(np.float64).eps
        s = self.scaleFactor
        if not (energies[0] > -s * (1 - 16 * eps) and energies[-1] < s * (1 - 16 * eps)):
            raise TBTKError(
                ERR_ARGUMENT,
                f"Invalid energy window. The 'energyWindow=[{energies[0]}, {energies[-1]}]' is"
                f" not contained in the interval (-scaleFactor, scaleFactor)=({-s}, {s}).")
        self.energyWindow = energies
        self._table = None

    def getEnergyWindow(self):
        return self.energyWindow

    def setCalculateCoefficientsOnGPU(self, flag):
        self.calculateCoefficientsOnGPU = bool(flag)

    def setGenerateGreensFunctionsOnGPU(self, flag):
        self.generateGreensFunctionsOnGPU = bool(flag)

    def setUseLookupTable(self, flag):
        self.useLookupTable = bool(flag)
        if not flag:
            self._table = None

    def setPrecision(self, precision):
        if precision not in (FP64, MIXED, MIXED_DIRECT):
            raise TBTKError(ERR_ARGUMENT, f"unknown precision {precision}")
        self.precision = precision

    # -- compute -----------------------------------------------------------
    def calculateCoefficients(self, to, frm):
        """``calculateCoefficients(to, from)``: [K][M] damped moments for a
        list of to basis indices (or one index -> [M])."""
        if self.numCoefficients <= 0:
            raise TBTKError(ERR_ARGUMENT, "numCoefficients has to be larger than 0.")
        single = np.ndim(to) == 0
        mu = self._get_matrix().moments(frm, to, self.numCoefficients, self.broadening)
        return mu[0] if single else mu

    def _get_table(self):
        if not self.useLookupTable:
            raise TBTKError(ERR_STATE, "Green's functions can only be generated on GPU using lookup tables.")
        if self._table is None:
            e = self.energyWindow
            s = self.scaleFactor
            if not (e[0] > -s and e[-1] < s):
                raise TBTKError(ERR_ARGUMENT, "The energy windows bounds have to lie in (-scaleFactor, scaleFactor).")
            self._table = Table.create(self.numCoefficients, e, s)
        return self._table

    def generateGreensFunction(self, coefficients, type_="Retarded"):
        t = _TYPES[type_] if isinstance(type_, str) else int(type_)
        g = self._get_table().greens(coefficients, t)
        return g[0] if np.ndim(coefficients) == 1 else g


class PropertyExtractor:
    """``PropertyExtractor::ChebyshevExpander`` over basis indices."""

    def __init__(self, solver: ChebyshevExpander):
        self.solver = solver
        e = solver.getEnergyWindow()
        self.setEnergyWindow(e[0], e[-1], e.size)

    def setEnergyWindow(self, lowerBound, upperBound, energyResolution):
        """Inclusive ``Range(lower, upper, res)`` pushed to the solver
        (PropertyExtractor ChebyshevExpander.cpp:79-94)."""
        self.solver.setEnergyWindow(tbtk_range(lowerBound, upperBound, energyResolution))

    def getEnergyWindow(self):
        return self.solver.getEnergyWindow()

    def calculateLDOS(self, sites):
        """LDOS [len(sites)][E] at basis indices, all sites in one batched
        recursion (the reference loops over sites one recursion each)."""
        s = self.solver
        out, _ = s._get_matrix().ldos_sites(s._get_table(), sites, s.broadening,
                                            s.precision)
        return out

    def _occupation(self, occupation):
        """The occupation weights at the window energies and the spacing dE
        (the reference's energyWindow[1] - energyWindow[0])."""
        e = self.getEnergyWindow()
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        if occ.shape != e.shape:
            raise ValueError("occupation needs one weight per window energy")
        return occ, float(e[1] - e[0])

    def calculateSpinPolarizedLDOS(self, up, down):
        """[S][E][2][2] complex at spin sites given by their spin-up and
        spin-down basis indices (calculateSpinPolarizedLDOS)."""
        s = self.solver
        return s._get_matrix().spin_polarized_ldos(s._get_table(), up, down, s.broadening,
                                                   s.precision)

    def calculateDensity(self, sites, occupation):
        """[S] densities; occupation = the equilibrium occupation at each
        window energy (the reference takes it from the model's statistics,
        temperature and chemical potential)."""
        s = self.solver
        occ, dE = self._occupation(occupation)
        return s._get_matrix().density(s._get_table(), sites, s.broadening, occ, dE, s.precision)

    def calculateMagnetization(self, up, down, occupation):
        """[S][2][2] complex (calculateMagnetization)."""
        s = self.solver
        occ, dE = self._occupation(occupation)
        return s._get_matrix().magnetization(s._get_table(), up, down, s.broadening, occ, dE,
                                             s.precision)

    def calculateExpectationValue(self, to, frm, occupation):
        """<c_to^dagger c_from> (calculateExpectationValue)."""
        s = self.solver
        occ, dE = self._occupation(occupation)
        return complex(s._get_matrix().expectation_values(
            s._get_table(), [to], [frm], s.broadening, occ, dE, s.precision)[0])

    def calculateGreensFunctions(self, to, frm, type_="Retarded"):
        s = self.solver
        mu = s.calculateCoefficients(np.atleast_1d(to), frm)
        return s.generateGreensFunction(mu, type_)
