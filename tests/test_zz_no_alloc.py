"""GPU test of tbtkkpm_moments_noalloc, the entry point for callers that
cannot allocate device memory (code inside another framework's memory pool
or under a fixed device budget).  It keeps its scratch in a fixed array
inside the library; the caller passes the matrix and the output as device
buffers.

The test calls it through the C ABI on two calls in a row and checks each
against tbtkkpm_moments, bit for bit (the FP64 moments tolerance of these
tests), that the second call leaves free device memory unchanged, and that
sizes past the fixed scratch are rejected.  Malformed caller buffers (a
row pointer that decreases, does not start at 0 or does not end at nnz, a
column or to index >= N) are found on the device without an out-of-range
access and return TBTKKPM_ERR_ARGUMENT.  This file is collected last so a
stop at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from tbtk_b200 import lattice as L

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _call(kpm, torch, csr, N, scale, frm, to, M, broadening):
    rowptr, col, val = csr
    d_rowptr = _dev(torch, rowptr.astype(np.int32).view(np.int32))
    d_col = _dev(torch, col.astype(np.int32).view(np.int32))
    d_val = _dev(torch, np.ascontiguousarray(val, dtype=np.complex128).view(np.float64))
    d_to = _dev(torch, np.asarray(to, dtype=np.int32))
    d_mu = torch.zeros((len(to), M, 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    return (d_rowptr, d_col, d_val, d_to, d_mu)


def _run(kpm, bufs, N, scale, frm, K, M, broadening, nnz=None):
    d_rowptr, d_col, d_val, d_to, d_mu = bufs
    if nnz is None:
        nnz = d_col.numel()
    p = ctypes.c_void_p
    return kpm.load_library().tbtkkpm_moments_noalloc(
        p(d_rowptr.data_ptr()), p(d_col.data_ptr()), p(d_val.data_ptr()), N, nnz, scale, frm,
        p(d_to.data_ptr()), K, M, broadening, p(d_mu.data_ptr()), None)


def test_noalloc_matches_moments_twice(gpu):
    torch = pytest.importorskip("torch")
    kpm = gpu
    lat = L.square(40, 36, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=17)
    csr = lat.csr()
    N = lat.num_states
    mat = kpm.Matrix.from_csr(*csr, 12.0)
    cases = [(lat.basis((3, 4, 0)), [lat.basis((3, 4, 0)), lat.basis((3, 5, 1)), 7], 300, 1e-3),
             (lat.basis((20, 11, 1)), [lat.basis((20, 11, 1)), 0], 129, 0.0)]
    bufs = [_call(kpm, torch, csr, N, 12.0, frm, to, M, b) for frm, to, M, b in cases]
    for i, ((frm, to, M, b), buf) in enumerate(zip(cases, bufs)):
        free_before = torch.cuda.mem_get_info()[0]
        rc = _run(kpm, buf, N, 12.0, frm, len(to), M, b)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert rc == 0, kpm.load_library().tbtkkpm_last_error()
        got = buf[4].cpu().numpy().view(np.complex128)[..., 0]
        ref = mat.moments(frm, to, M, b)
        assert np.array_equal(got, ref), (i, np.abs(got - ref).max())
        if i == 1:
            # the scratch was set up by the first call: nothing is allocated now
            assert free_after == free_before


def test_noalloc_rejects_oversized(gpu):
    torch = pytest.importorskip("torch")
    kpm = gpu
    lat = L.square(4, 4)
    csr = lat.csr()
    bufs = _call(kpm, torch, csr, lat.num_states, 10.0, 0, [0], 8, 0.0)
    # 32*N + 8*M + 256 must fit the fixed 32 MiB scratch
    rc = _run(kpm, bufs, 1 << 20, 10.0, 0, 1, 8, 0.0)
    assert rc == kpm.ERR_ARGUMENT
    assert "32 MiB" in kpm.load_library().tbtkkpm_last_error().decode()


def test_noalloc_rejects_malformed_device_buffers(gpu):
    """Bad caller-owned device buffers end in TBTKKPM_ERR_ARGUMENT: the row
    pointer is checked on the device before any step reads through it, and
    out-of-range column and to indices are skipped and reported."""
    torch = pytest.importorskip("torch")
    kpm = gpu
    lat = L.square(6, 5, t=1.0, J=0.5, W=1.0, periodic=True, seed=2)
    rowptr, col, val = lat.csr()
    N, nnz = lat.num_states, int(rowptr[-1])
    err = lambda: kpm.load_library().tbtkkpm_last_error().decode()

    def run(rp, cl, to, nnz_arg=nnz):
        bufs = _call(kpm, torch, (rp, cl, val), N, 10.0, 0, to, 16, 0.0)
        rc = _run(kpm, bufs, N, 10.0, 0, len(to), 16, 0.0, nnz=nnz_arg)
        torch.cuda.synchronize()
        return rc

    assert run(rowptr, col, [0, 3]) == 0
    bad = rowptr.copy()
    bad[4], bad[5] = bad[5], bad[4]  # decreasing between rows 4 and 5
    assert run(bad, col, [0]) == kpm.ERR_ARGUMENT and "rowptr" in err()
    assert run(rowptr, col, [0], nnz_arg=nnz - 1) == kpm.ERR_ARGUMENT and "rowptr" in err()
    shifted = rowptr + 1  # does not start at 0
    assert run(shifted, col, [0], nnz_arg=nnz + 1) == kpm.ERR_ARGUMENT and "rowptr" in err()
    wide = col.copy()
    wide[7] = N + 3
    assert run(rowptr, wide, [0]) == kpm.ERR_ARGUMENT and "column" in err()
    assert run(rowptr, col, [0, N]) == kpm.ERR_ARGUMENT and "to index" in err()
    # a good call afterwards still matches tbtkkpm_moments
    mat = kpm.Matrix.from_csr(rowptr, col, val, 10.0)
    bufs = _call(kpm, torch, (rowptr, col, val), N, 10.0, 0, [0, 5], 16, 0.0)
    assert _run(kpm, bufs, N, 10.0, 0, 2, 16, 0.0) == 0
    got = bufs[4].cpu().numpy().view(np.complex128)[..., 0]
    assert np.array_equal(got, mat.moments(0, [0, 5], 16, 0.0))
