"""GPU parity of the KPM path through the C ABI against the CPU oracle and
the reference's golden vectors.

Tolerances: the FP64 recursion follows the reference's operation order and
is compared bit for bit; Green's functions and LDOS from the device-built
table (CUDA acos/sincos) are compared normwise, max|x - ref| / max|ref|
<= 1e-12; from a table built on the host they are bit-exact; the MIXED
(complex64-vector) path is compared normwise on moments (<= 2e-6) and LDOS
(<= 1e-6, the path's stated target).
"""
import numpy as np
import pytest

from conftest import golden, rel_err, scaled_values
from tbtk_b200 import lattice as L

pytestmark = pytest.mark.gpu

EPS100 = 100 * np.finfo(np.float64).eps
MODEL_CASES = ["cfg1", "rashba", "honeycomb", "duplicates"]


def _lattice(name):
    from test_oracle import _lattice as lat
    return lat(name)


@pytest.mark.parametrize("name", MODEL_CASES + ["kat5x5"])
def test_matrix_scaling_bit_exact(gpu, name):
    g = golden(name)
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], float(g["scale"]))
    rowptr, col, val = m.download_csr()
    assert np.array_equal(rowptr, g["rowptr"])
    assert np.array_equal(col, g["col"])
    assert np.array_equal(val, scaled_values(g["val"], float(g["scale"])))


@pytest.mark.parametrize("name", MODEL_CASES)
def test_triplet_builder_matches_getSparseMatrix(gpu, name):
    """Device sort + duplicate fold == HoppingAmplitudeSet::getSparseMatrix."""
    g = golden(name)
    lat = _lattice(name)
    m = gpu.Matrix.from_triplets(lat.to_basis, lat.from_basis, lat.amp, lat.num_states,
                                 float(g["scale"]))
    rowptr, col, val = m.download_csr()
    assert np.array_equal(rowptr, g["rowptr"])
    assert np.array_equal(col, g["col"])
    assert np.array_equal(val, scaled_values(g["val"], float(g["scale"])))


@pytest.mark.parametrize("name", MODEL_CASES)
def test_moments_bit_exact(gpu, name):
    g = golden(name)
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], float(g["scale"]))
    mu = m.moments(int(g["frm"]), g["to"], int(g["M"]), float(g["broadening"]))
    assert np.array_equal(mu, g["moments"])
    # one to-index at a time equals the multi-to call (the reference test's
    # "multiple to-Indices at once")
    for k, t in enumerate(g["to"]):
        single = m.moments(int(g["frm"]), [int(t)], int(g["M"]), float(g["broadening"]))
        assert np.array_equal(single[0], g["moments"][k])


def test_kat_5x5_closed_forms(gpu):
    g = golden("kat5x5")
    mu_, t, s = -2.0, 1.0, 10.0
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    d, o = m.moments(int(g["frm"]), g["to"], 100, 0.0)
    assert abs(d[0] - 1) < EPS100 and abs(d[1] - (-mu_ / s)) < EPS100
    assert abs(d[2] - (2 * (mu_ * mu_ + 4 * t * t) / (s * s) - 1)) < EPS100
    assert abs(o[1] - (-t / s)) < EPS100 and abs(o[2] - 4 * mu_ * t / (s * s)) < EPS100
    assert np.array_equal(np.stack([d, o]), g["moments"])


def test_batched_fp64_bit_exact(gpu, oracle):
    """B sources in one SpMM recursion give each source's single-vector
    moments bit for bit."""
    lat = L.square(9, 7, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=4)
    rowptr, col, val = lat.csr()
    s, M, bro = 12.0, 120, 1e-3
    rng = np.random.default_rng(1)
    for B in (1, 3, 8, 33, 70):
        frm = rng.integers(0, lat.num_states, size=B).astype(np.uint32)
        to, owner = [], []
        for b in range(B):
            for t in {int(frm[b]), int(rng.integers(0, lat.num_states))}:
                to.append(t)
                owner.append(b)
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        mu, err = m.moments_batched(frm, to, owner, M, bro, gpu.FP64)
        assert np.all(err == 0)
        for k in range(len(to)):
            ref = oracle.damp(oracle.moments(rowptr, col, val, s, M, int(frm[owner[k]]), [to[k]]), bro)
            assert np.array_equal(mu[k], ref[0]), (B, k)


def test_batched_more_than_one_chunk(gpu, oracle):
    """More sources than one batch holds (FP64 batches hold 128)."""
    lat = L.square(6, 6, t=1.0, J=0.5, W=1.0, periodic=True, seed=8)
    rowptr, col, val = lat.csr()
    B = 130
    frm = (np.arange(B) % lat.num_states).astype(np.uint32)
    m = gpu.Matrix.from_csr(rowptr, col, val, 10.0)
    mu, _ = m.moments_batched(frm, frm, np.arange(B), 40, 0.0, gpu.FP64)
    for b in (0, 64, 127, 128, 129):
        ref = oracle.moments(rowptr, col, val, 10.0, 40, int(frm[b]), [int(frm[b])])
        assert np.array_equal(mu[b], ref[0])


def test_mixed_precision_moments(gpu, oracle):
    lat = L.square(16, 16, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=6)
    rowptr, col, val = lat.csr()
    s, M, bro = 12.0, 512, 1e-3
    for B in (1, 5, 16, 64, 200):
        frm = L.random_sites(lat, B, seed=B)
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, bro, gpu.MIXED)
        for b in (0, B // 2, B - 1):
            ref = oracle.damp(oracle.moments(rowptr, col, val, s, M, int(frm[b]), [int(frm[b])]), bro)
            assert rel_err(mu[b], ref[0]) <= 2e-6, (B, b, rel_err(mu[b], ref[0]))


@pytest.mark.parametrize("name", MODEL_CASES)
def test_greens_all_types(gpu, oracle, name):
    """All four types on the GPU (the reference GPU path had Retarded only)."""
    g = golden(name)
    lo, hi, E = g["window"]
    energies = gpu.tbtk_range(lo, hi, int(E))
    s, M = float(g["scale"]), int(g["M"])
    dev = gpu.Table.create(M, energies, s)
    host = gpu.Table.upload(oracle.lookup_table(M, energies, s))
    for ty in range(4):
        ref = g[f"greens_{ty}"]
        assert rel_err(dev.greens(g["moments"], ty), ref) <= 1e-12
        assert np.array_equal(host.greens(g["moments"], ty), ref)


def test_device_table_close_to_host_table(gpu, oracle):
    energies = gpu.tbtk_range(-12, 12, 2000, False, False)
    M = 4096
    dev = gpu.Table.create(M, energies, 12.0)
    host = oracle.lookup_table(M, energies, 12.0)
    # read the device table back through the Retarded sum of unit vectors
    eye = np.zeros((3, M), dtype=np.complex128)
    for j, n in enumerate((0, 1, M - 1)):
        eye[j, n] = 1
    got = dev.greens(eye, gpu.RETARDED)
    # CUDA's acos and glibc's may differ by an ulp; exp(-i n acos x) carries
    # that difference times n, so the bound grows with the coefficient index.
    eps = np.finfo(np.float64).eps
    for j, n in enumerate((0, 1, M - 1)):
        assert rel_err(got[j], host[n]) <= 4 * max(n, 1) * eps + 4 * eps


@pytest.mark.parametrize("name", MODEL_CASES)
def test_ldos_sites_fp64(gpu, oracle, name):
    g = golden(name)
    lo, hi, E = g["window"]
    energies = gpu.tbtk_range(lo, hi, int(E))
    s, M = float(g["scale"]), int(g["M"])
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    host = gpu.Table.upload(oracle.lookup_table(M, energies, s))
    ldos, err = m.ldos_sites(host, g["ldos_sites"], float(g["broadening"]), gpu.FP64)
    assert np.array_equal(ldos, g["ldos"])
    dev = gpu.Table.create(M, energies, s)
    ldos2, _ = m.ldos_sites(dev, g["ldos_sites"], float(g["broadening"]), gpu.FP64)
    assert rel_err(ldos2, g["ldos"]) <= 1e-12


@pytest.mark.parametrize("name", MODEL_CASES)
def test_ldos_sites_mixed(gpu, name):
    g = golden(name)
    lo, hi, E = g["window"]
    energies = gpu.tbtk_range(lo, hi, int(E))
    s, M = float(g["scale"]), int(g["M"])
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    dev = gpu.Table.create(M, energies, s)
    ldos, _ = m.ldos_sites(dev, g["ldos_sites"], float(g["broadening"]), gpu.MIXED)
    for k in range(ldos.shape[0]):
        assert rel_err(ldos[k], g["ldos"][k]) <= 1e-6, rel_err(ldos[k], g["ldos"][k])


@pytest.mark.parametrize("name", MODEL_CASES)
def test_ldos_sites_mixed_direct(gpu, name):
    """complex64 vectors with every moment gathered directly (no doubling)."""
    g = golden(name)
    lo, hi, E = g["window"]
    energies = gpu.tbtk_range(lo, hi, int(E))
    s, M = float(g["scale"]), int(g["M"])
    m = gpu.Matrix.from_csr(g["rowptr"], g["col"], g["val"], s)
    dev = gpu.Table.create(M, energies, s)
    ldos, err = m.ldos_sites(dev, g["ldos_sites"], float(g["broadening"]), gpu.MIXED_DIRECT)
    assert np.all(err == -1.0)
    for k in range(ldos.shape[0]):
        assert rel_err(ldos[k], g["ldos"][k]) <= 1e-6, rel_err(ldos[k], g["ldos"][k])


@pytest.mark.parametrize("M", [1, 2, 3, 4, 5, 64, 257])
def test_doubling_moment_counts(gpu, M):
    """The doubling schedule covers every moment for odd and even M."""
    lat = L.square(7, 6, t=1.0, J=0.5, W=1.5, alpha=0.2, periodic=True, seed=12)
    rowptr, col, val = lat.csr()
    s = 12.0
    sites = L.random_sites(lat, 5, seed=M)
    energies = gpu.tbtk_range(-11.0, 11.0, 64)
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    t = gpu.Table.create(M, energies, s)
    ref, _ = m.ldos_sites(t, sites, 1e-3, gpu.FP64)
    got, err = m.ldos_sites(t, sites, 1e-3, gpu.MIXED)
    for k in range(sites.size):
        assert rel_err(got[k], ref[k]) <= 1e-6, (M, k, rel_err(got[k], ref[k]))
    assert np.all(err >= 0)


def test_doubling_error_estimate(gpu):
    """On a disordered Rashba lattice at M=2048 the doubling LDOS stays within
    1e-6 of the FP64 recursion and the per-site estimate is small and at
    least the site's actual error."""
    lat = L.square(40, 40, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=21)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 2048
    sites = L.random_sites(lat, 24, seed=5)
    energies = gpu.tbtk_range(-12.0, 12.0, 500, False, False)
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    t = gpu.Table.create(M, energies, s)
    ref, _ = m.ldos_sites(t, sites, 1e-3, gpu.FP64)
    got, err = m.ldos_sites(t, sites, 1e-3, gpu.MIXED)
    errs = [rel_err(got[k], ref[k]) for k in range(sites.size)]
    assert max(errs) <= 1e-6, max(errs)
    assert np.all(err >= 0) and np.all(err < 1e-4), err
    assert all(err[k] >= errs[k] for k in range(sites.size)), list(zip(err, errs))


def test_every_config_same_result(gpu, oracle):
    """Every compiled step configuration of a batch width gives the same
    FP64 moments (bit for bit) and the autotuner picks one of them."""
    lat = L.square(11, 9, t=1.0, J=0.5, W=2.0, alpha=0.25, periodic=True, seed=31)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 40
    frm = L.random_sites(lat, 40, seed=2)
    ref = None
    for (t, v, mb) in gpu.configs_for(40, gpu.FP64):
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(40, gpu.FP64, t, v, mb, ldos=False)
        mu, _ = m.moments_batched(frm, frm, np.arange(40), M, 0.0, gpu.FP64)
        if ref is None:
            ref = mu
            o = oracle.moments(rowptr, col, val, s, M, int(frm[7]), [int(frm[7])])
            assert np.array_equal(mu[7], o[0])
        assert np.array_equal(mu, ref), (t, v, mb)
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    t, v, mb, ms = m.autotune(40, gpu.MIXED, ldos=True, probe_steps=4)
    assert (t, v, mb) in gpu.configs_for(40, gpu.MIXED) and ms > 0
    with pytest.raises(gpu.TBTKError):
        m.set_config(40, gpu.MIXED, 32, 1, 2)


@pytest.mark.parametrize("B", [1, 2, 4, 8, 16, 32])
def test_every_fp64_config_small_batches(gpu, oracle, B):
    """Every compiled FP64 configuration of small batches (register-staged,
    per-warp rings, tile-staged) gives the reference's moments bit for bit,
    on a lattice whose row count is not a multiple of any tile height."""
    lat = L.square(13, 7, t=1.0, J=0.5, W=2.0, alpha=0.25, periodic=True, seed=B)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 32
    frm = L.random_sites(lat, B, seed=5)
    refs = [oracle.moments(rowptr, col, val, s, M, int(f), [int(f)])[0] for f in frm]
    configs = gpu.configs_for(B, gpu.FP64)
    assert any(mb >= 100000 for (_, _, mb) in configs)
    for (t, v, mb) in configs:
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(B, gpu.FP64, t, v, mb, ldos=False)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, 0.0, gpu.FP64)
        for b in range(B):
            assert np.array_equal(mu[b], refs[b]), (t, v, mb, b)


@pytest.mark.gpu
@pytest.mark.parametrize("B", [4, 8, 20, 40, 100])
def test_every_mixed_config_same_result(gpu, B):
    """Every compiled complex64 step configuration (register-staged, bulk
    ring, cp.async ring) takes the same per-element arithmetic in the same
    entry order: directly gathered moments bit for bit.  Doubling LDOS agree
    to 1e-7: the partial sums of the dot products are grouped by the grid,
    and the bulk-ring kernels form them from the FP64 values before the
    complex64 rounding (the others from the stored values).  Rows of 9
    entries exceed the 6-entry rings, so their tail takes the global path."""
    lat = L.square(11, 9, t=1.0, J=0.5, W=2.0, alpha=0.25, periodic=True, seed=31)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 48
    frm = L.random_sites(lat, B, seed=3)
    energies = gpu.tbtk_range(-12.0, 12.0, 64, False, False)
    ref_mu = ref_ldos = None
    for (t, v, mb) in gpu.configs_for(B, gpu.MIXED, ldos=False):
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=False)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
        if ref_mu is None:
            ref_mu = mu
        assert np.array_equal(mu, ref_mu), (t, v, mb)
    tab = gpu.Table.create(M, energies, s)
    fp64, _ = gpu.Matrix.from_csr(rowptr, col, val, s).ldos_sites(tab, frm, 1e-3, gpu.FP64)
    for (t, v, mb) in gpu.configs_for(B, gpu.MIXED, ldos=True):
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=True)
        out, _ = m.ldos_sites(tab, frm, 1e-3, gpu.MIXED)
        if ref_ldos is None:
            ref_ldos = out
        assert rel_err(out, ref_ldos) <= 1e-7, (t, v, mb)
        assert rel_err(out, fp64) <= 1e-6, (t, v, mb)


@pytest.mark.gpu
@pytest.mark.parametrize("B", [32, 64, 128])
def test_row_pair_steps_on_ragged_rows(gpu, B):
    """The row-pair form of the tile-staged complex step (two adjacent rows
    per thread group over the merge of their column lists) on a random
    complex Hermitian matrix with an odd row count (the last pair has one
    row), empty rows, rows of up to 13 entries and columns shared by some
    pairs only:
    directly gathered moments bit for bit against the library's default
    step, and the same doubling LDOS up to the grouping of the dot-product
    sums."""
    rng = np.random.default_rng(B)
    N = 301
    A = {}
    for i in range(N):
        for j in rng.choice(N, size=int(rng.integers(0, 6)), replace=False):
            v = complex(rng.standard_normal(), rng.standard_normal())
            A[(i, int(j))] = A.get((i, int(j)), 0) + v
            A[(int(j), i)] = A.get((int(j), i), 0) + v.conjugate()
    for i in range(0, N, 3):
        A[(i, i)] = A.get((i, i), 0) + rng.standard_normal()
    rows = sorted(A)
    rowptr = np.zeros(N + 1, dtype=np.uint32)
    for (i, _) in rows:
        rowptr[i + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.uint32)
    col = np.array([j for (_, j) in rows], dtype=np.uint32)
    val = np.array([A[k] for k in rows], dtype=np.complex128)
    s = 2.0 * np.abs(np.linalg.eigvalsh(_dense(rowptr, col, val, N))).max() + 1.0
    M = 48
    frm = rng.choice(N, size=B, replace=False).astype(np.uint32)
    ref, _ = gpu.Matrix.from_csr(rowptr, col, val, s).moments_batched(
        frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
    pair = [c for c in gpu.configs_for(B, gpu.MIXED, ldos=False)
            if c[2] >= 100000 and (c[2] - 100000) // 1000000 >= 100]
    assert pair
    for (t, v, mb) in pair:
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=False)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
        assert np.array_equal(mu, ref), (t, v, mb)
    tab = gpu.Table.create(M, gpu.tbtk_range(-s, s, 64, False, False), s)
    dref, _ = gpu.Matrix.from_csr(rowptr, col, val, s).ldos_sites(tab, frm, 1e-3, gpu.MIXED)
    for (t, v, mb) in [c for c in gpu.configs_for(B, gpu.MIXED, ldos=True)
                       if c[2] >= 100000 and (c[2] - 100000) // 1000000 >= 100]:
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=True)
        out, _ = m.ldos_sites(tab, frm, 1e-3, gpu.MIXED)
        assert rel_err(out, dref) <= 1e-7, (t, v, mb)


def _dense(rowptr, col, val, N):
    d = np.zeros((N, N), dtype=np.complex128)
    for i in range(N):
        for k in range(int(rowptr[i]), int(rowptr[i + 1])):
            d[i, int(col[k])] += val[k]
    return d


def test_real_matrix_detected(gpu):
    """A real Hamiltonian runs the mixed precisions on real vectors; a
    complex one (Rashba spin-orbit) and a forbidding caller keep complex64."""
    real = L.square(8, 6, t=1.0, J=0.5, W=2.0, periodic=True, seed=7)
    cplx = L.square(8, 6, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=7)
    m = gpu.Matrix.from_csr(*real.csr(), 12.0)
    assert m.real() == (True, True)
    m.set_real(False)
    assert m.real() == (True, False)
    assert gpu.Matrix.from_csr(*cplx.csr(), 12.0).real() == (False, False)


@pytest.mark.parametrize("B", [1, 4, 8, 16, 20, 64, 200])
def test_real_vectors_match_complex_vectors(gpu, B):
    """Real float vectors give the complex64 path's values: directly gathered
    moments bit for bit for every compiled real configuration; doubling LDOS
    up to the grouping of the dot-product sums; and within the mixed bar of
    the FP64 path."""
    lat = L.square(13, 11, t=1.0, J=0.5, W=2.0, periodic=True, seed=41)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 64
    frm = L.random_sites(lat, min(B, 286), seed=4)[:B]
    B = frm.size
    cm = gpu.Matrix.from_csr(rowptr, col, val, s)
    cm.set_real(False)
    ref, _ = cm.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
    configs = gpu.Matrix.from_csr(rowptr, col, val, s).configs_for(B, gpu.MIXED, ldos=False)
    assert configs
    for (t, v, mb) in configs:
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        assert m.real()[1]
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=False)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
        assert np.array_equal(mu, ref), (t, v, mb)
    energies = gpu.tbtk_range(-12.0, 12.0, 80, False, False)
    tab = gpu.Table.create(M, energies, s)
    direct_c, _ = cm.ldos_sites(tab, frm, 1e-3, gpu.MIXED_DIRECT)
    dbl_c, _ = cm.ldos_sites(tab, frm, 1e-3, gpu.MIXED)
    rm = gpu.Matrix.from_csr(rowptr, col, val, s)
    direct_r, _ = rm.ldos_sites(tab, frm, 1e-3, gpu.MIXED_DIRECT)
    dbl_r, _ = rm.ldos_sites(tab, frm, 1e-3, gpu.MIXED)
    fp64, _ = rm.ldos_sites(tab, frm, 1e-3, gpu.FP64)
    assert np.array_equal(direct_r, direct_c)
    assert rel_err(dbl_r, dbl_c) <= 1e-10
    assert rel_err(dbl_r, fp64) <= 1e-6
    assert rel_err(direct_r, fp64) <= 1e-6
    # every compiled doubling configuration of the real vectors: the same
    # LDOS up to the grouping of the dot-product sums by the grid
    for (t, v, mb) in rm.configs_for(B, gpu.MIXED, ldos=True):
        m = gpu.Matrix.from_csr(rowptr, col, val, s)
        m.set_batch_width(gpu.MIXED, 256)  # all B sources in one batch of this shape
        m.set_config(B, gpu.MIXED, t, v, mb, ldos=True)
        out, _ = m.ldos_sites(tab, frm, 1e-3, gpu.MIXED)
        assert rel_err(out, dbl_r) <= 1e-7, (t, v, mb)
        assert rel_err(out, fp64) <= 1e-6, (t, v, mb)


def test_batch_width_splits_without_changing_results(gpu):
    """tbtkkpm_matrix_set_batch_width splits a call's sources into batches:
    FP64 LDOS, directly gathered moments and the MIXED_DIRECT LDOS are bit
    for bit the same at every width, doubling LDOS agree to the 1e-7 of the
    dot-sum grouping; doubling LDOS default to batches of 128 on real and
    complex matrices."""
    lat = L.square(13, 11, t=1.0, J=0.5, W=2.0, periodic=True, seed=41)
    rowptr, col, val = lat.csr()
    s, M = 12.0, 64
    frm = L.random_sites(lat, 200, seed=9)
    B = frm.size
    tab = gpu.Table.create(M, gpu.tbtk_range(-12.0, 12.0, 80, False, False), s)
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    assert m.real()[1]
    assert m.batch_width(gpu.MIXED, ldos=True) == 128
    assert m.batch_width(gpu.MIXED, ldos=False) == 256
    assert m.batch_width(gpu.MIXED_DIRECT) == 256 and m.batch_width(gpu.FP64) == 128
    precs = (gpu.FP64, gpu.MIXED_DIRECT, gpu.MIXED)
    base = {p: m.ldos_sites(tab, frm, 1e-3, p)[0] for p in precs}
    mu_base, _ = m.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
    assert rel_err(base[gpu.MIXED], base[gpu.FP64]) <= 1e-6
    for w in (1, 7, 64, 128, 256):
        for p in precs:
            if p == gpu.FP64 and w > 128:
                with pytest.raises(gpu.TBTKError) as e:
                    m.set_batch_width(p, w)
                assert e.value.status == gpu.ERR_ARGUMENT
                continue
            m.set_batch_width(p, w)
            assert m.batch_width(p) == w
            out, _ = m.ldos_sites(tab, frm, 1e-3, p)
            if p == gpu.MIXED:
                assert rel_err(out, base[p]) <= 1e-7, w
                assert rel_err(out, base[gpu.FP64]) <= 1e-6, w
            else:
                assert np.array_equal(out, base[p]), (w, p)
        mu, _ = m.moments_batched(frm, frm, np.arange(B), M, 1e-3, gpu.MIXED)
        assert np.array_equal(mu, mu_base), w
    m.set_batch_width(gpu.MIXED, 0)
    assert m.batch_width(gpu.MIXED, ldos=True) == 128
    cm = gpu.Matrix.from_csr(*L.square(5, 4, t=1.0, J=0.5, alpha=0.3, periodic=True).csr(), s)
    assert not cm.real()[1]
    assert cm.batch_width(gpu.MIXED, ldos=True) == 128 and cm.batch_width(gpu.MIXED, False) == 256


def test_ring_ldos_integral(gpu):
    g = golden("ring")
    solver = gpu.ChebyshevExpander()
    solver.setModel((g["rowptr"], g["col"], g["val"]))
    solver.setScaleFactor(10)
    pe = gpu.PropertyExtractor(solver)
    for f in (9, 7):
        pe.setEnergyWindow(-f, f, 1000)
        ldos = pe.calculateLDOS([0])
        E = pe.getEnergyWindow()
        assert abs(ldos[0].sum() * (E[1] - E[0]) - 1) < 1e-3
        assert rel_err(ldos[0], g[f"ldos_{f}"][0]) <= 1e-12


def test_solver_interface_calculate_coefficients(gpu):
    """The reference test's call sequence through the Solver mirror."""
    g = golden("kat5x5")
    solver = gpu.ChebyshevExpander()
    solver.setModel((g["rowptr"], g["col"], g["val"]))
    solver.setScaleFactor(10)
    solver.setUseLookupTable(True)
    solver.setNumCoefficients(100)
    solver.setBroadening(0)
    c0 = solver.calculateCoefficients(int(g["to"][0]), int(g["frm"]))
    c1 = solver.calculateCoefficients(int(g["to"][1]), int(g["frm"]))
    c2 = solver.calculateCoefficients(g["to"], int(g["frm"]))
    assert c0.shape == (100,)
    assert np.array_equal(c2[0], c0) and np.array_equal(c2[1], c1)
    assert np.array_equal(c2, g["moments"])


def test_edge_cases(gpu, oracle):
    lat = L.square(5, 4, t=1.0, J=0.5, W=1.0, periodic=False, seed=3)
    rowptr, col, val = lat.csr()
    m = gpu.Matrix.from_csr(rowptr, col, val, 10.0)
    for M in (1, 2, 3):
        mu = m.moments(3, [3, 4], M, 1e-3)
        ref = oracle.damp(oracle.moments(rowptr, col, val, 10.0, M, 3, [3, 4]), 1e-3)
        assert np.array_equal(mu, ref)
    assert m.moments(3, [], 10, 0.0).shape == (0, 10)
    with pytest.raises(gpu.TBTKError) as e:
        m.moments(lat.num_states, [0], 10, 0.0)
    assert e.value.status == gpu.ERR_ARGUMENT
    with pytest.raises(gpu.TBTKError):
        m.moments(0, [lat.num_states + 3], 10, 0.0)
    with pytest.raises(gpu.TBTKError):
        m.moments(0, [0], 0, 0.0)
    with pytest.raises(gpu.TBTKError):
        m.moments_batched([0, 1], [0], [2], 10, 0.0, gpu.FP64)
    with pytest.raises(gpu.TBTKError):
        m.moments_batched([0], [0], [0], 10, 0.0, 7)


def test_empty_rows_and_isolated_states(gpu, oracle):
    """Rows without entries (a state with no amplitudes) stay zero."""
    rowptr = np.array([0, 2, 2, 4, 4], dtype=np.uint32)
    col = np.array([0, 2, 0, 2], dtype=np.uint32)
    val = np.array([0.5, -1.0, -1.0, 0.25 + 0.1j], dtype=np.complex128)
    m = gpu.Matrix.from_csr(rowptr, col, val, 3.0)
    mu = m.moments(0, [0, 1, 2, 3], 30, 0.0)
    ref = oracle.moments(rowptr, col, val, 3.0, 30, 0, [0, 1, 2, 3])
    assert np.array_equal(mu, ref)
    assert np.all(mu[1] == 0) and np.all(mu[3] == 0)


def test_full_size_properties(gpu):
    """At the 2048x2048 periodic lattice with spin (N = 8,388,608): the first
    moments follow from the matrix rows, batched FP64 equals single-vector
    FP64 bit for bit, and <i|j><j|i> symmetry holds."""
    from tbtk_b200 import workloads
    p = workloads.cfg2(n_sites=4)
    rowptr, col, val, sites = p.rowptr, p.col, p.val, p.sites
    s, M = p.scale, 24
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    single = [m.moments(int(i), [int(i)], M, 0.0)[0] for i in sites]
    batched, _ = m.moments_batched(sites, sites, np.arange(sites.size), M, 0.0, gpu.FP64)
    for b in range(sites.size):
        assert np.array_equal(batched[b], single[b])
        i = int(sites[b])
        row = slice(int(rowptr[i]), int(rowptr[i + 1]))
        cols, vals = col[row], val[row]
        diag = vals[cols == i]
        assert abs(single[b][0] - 1) == 0
        assert abs(single[b][1] - (diag[0] / s if diag.size else 0)) < EPS100
        assert abs(single[b][2] - (2 * np.sum(np.abs(vals) ** 2) / s ** 2 - 1)) < EPS100
    a, b_ = int(sites[0]), int(sites[1])
    ab = m.moments(b_, [a], M, 0.0)[0]
    ba = m.moments(a, [b_], M, 0.0)[0]
    assert np.abs(ab - np.conj(ba)).max() < 1e-13
