"""The LDOS server (tbtkkpm_server_*): continuous batching over many models.

Parity: every result against tbtkkpm_ldos_sites on the same model (FP64:
the reference-exact path, pinned against TBTK elsewhere) within the mixed
precision bar, and bit-identical whether a request runs alone or among
others, joins at step 1 or in the middle of other requests, and whatever
the step configuration.
"""
import threading

import numpy as np
import pytest

from conftest import rel_err
from tbtk_b200 import workloads

S = 12.0
E = 200
TOL_MIXED = 1e-6


def grid():
    return workloads.open_grid(S, E)


def models():
    """Square, Rashba and honeycomb models of different sizes."""
    return [
        ("square", workloads.square_csr(24, 24, J=0.5, W=2.0, seed=1)),
        ("rashba", workloads.square_csr(20, 20, J=0.5, W=2.0, alpha=0.3, seed=2)),
        ("honeycomb", workloads.honeycomb_csr(16, 16, J=0.3, W=1.0, seed=3)),
        ("small", workloads.square_csr(8, 8, J=0.2, W=1.0, seed=4)),
    ]


def fp64_ldos(kpm, csr, sites, M, broadening):
    m = kpm.Matrix.from_csr(*csr, S)
    t = kpm.Table.create(M, grid(), S)
    out, _ = m.ldos_sites(t, sites, broadening, kpm.FP64)
    return out


@pytest.mark.gpu
def test_server_matches_fp64_ldos(gpu):
    kpm = gpu
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=0)
    ms = models()
    ids = [srv.add_model(*csr, S, 8) for _, csr in ms]
    rng = np.random.default_rng(0)
    jobs = []
    for i, (_, csr) in enumerate(ms):
        N = csr[0].size - 1
        for M in (64, 257, 512):
            sites = rng.choice(N, size=int(rng.integers(1, 9)), replace=False).astype(np.uint32)
            jobs.append((i, csr, sites, M, srv.submit(ids[i], sites, M, 1e-3)))
    for i, csr, sites, M, rid in jobs:
        ldos, err, rerun = srv.wait(rid)
        ref = fp64_ldos(kpm, csr, sites, M, 1e-3)
        assert not rerun.any()
        for k in range(sites.size):
            assert rel_err(ldos[k], ref[k]) <= TOL_MIXED, (ms[i][0], M, k)
            assert 0 <= err[k] < 1e-4
    st = srv.stats()
    assert st["completed"] == len(jobs)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def _solo(kpm, csr, sites, M, broadening, width, config=None):
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=0)
    mid = srv.add_model(*csr, S, width)
    if config:
        # the model steps at `width` (not at the narrower width its busy
        # lanes would take), so the configuration applies
        srv.set_adaptive_width(False)
        srv.set_config(width, *config)
    out = srv.wait(srv.submit(mid, sites, M, broadening))
    srv.close()
    return out


@pytest.mark.gpu
def test_server_result_alone_equals_in_mix(gpu):
    kpm = gpu
    name, csr = models()[1]
    probe_sites = np.array([5, 77, 300], dtype=np.uint32)
    alone = _solo(kpm, csr, probe_sites, 384, 1e-3, 8)

    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=7, tolerance=0)
    ms = models()
    ids = [srv.add_model(*c, S, 8) for _, c in ms]
    rng = np.random.default_rng(1)
    # background traffic on every model, the probe request in the middle
    bg = []
    for r in range(12):
        i = r % len(ms)
        N = ms[i][1][0].size - 1
        sites = rng.choice(N, size=int(rng.integers(1, 6)), replace=False).astype(np.uint32)
        bg.append(srv.submit(ids[i], sites, int(rng.integers(16, 512)), 1e-3))
    import time
    time.sleep(0.05)
    rid = srv.submit(ids[1], probe_sites, 384, 1e-3)
    more = [srv.submit(ids[1], np.array([1, 2], dtype=np.uint32), 100, 1e-3)]
    mixed = srv.wait(rid)
    for b in bg + more:
        srv.wait(b)
    for a, b in zip(alone, mixed):
        assert np.array_equal(a, b)
    srv.close()


@pytest.mark.gpu
def test_server_result_independent_of_configuration(gpu):
    kpm = gpu
    _, csr = models()[0]
    sites = np.array([0, 33, 101, 400], dtype=np.uint32)
    ref = _solo(kpm, csr, sites, 200, 1e-3, 16)
    for cfg in [(8, 2, 1), (4, 4, 2), (2, 8, 1)]:
        got = _solo(kpm, csr, sites, 200, 1e-3, 16, cfg)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), cfg


def _mixed_traffic(kpm, srv, ids, ms, seed):
    """LDOS and Green's-function requests on every model; their results."""
    rng = np.random.default_rng(seed)
    reqs = []
    for r in range(8):
        i = r % len(ms)
        N = ms[i][1][0].size - 1
        sites = rng.choice(N, size=int(rng.integers(1, 3)), replace=False).astype(np.uint32)
        M = int(rng.integers(16, 200))
        reqs.append(srv.submit(ids[i], sites, M, 1e-3))
        reqs.append(srv.submit_greens(ids[i], sites + 1, sites, M, 1e-3, "Retarded"))
    return [srv.wait(q) for q in reqs]


@pytest.mark.gpu
@pytest.mark.parametrize("width", [2, 4, 8, 16, 32, 64])
def test_server_tiled_steps_equal_register_steps(gpu, width):
    """Every compiled step configuration of a lane width, the tile-staged
    ones (rows staged in shared memory by bulk copies) among them, gives
    the register-staged default's results bit for bit, on real and complex
    models, for LDOS and directly gathered Green's-function lanes."""
    kpm = gpu
    ms = models()
    outs = {}
    for real in (True, False):
        for cfg in [None] + kpm.Server.step_configs(width, real):
            srv = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=6, tolerance=0)
            ids = [srv.add_model(*c, S, width) for _, c in ms]
            if cfg is not None:
                srv.set_adaptive_width(False)  # every step at `width`, in this configuration
                srv.set_config(width, *cfg)
            outs[(real, cfg)] = _mixed_traffic(kpm, srv, ids, ms, 11)
            srv.close()
    ref = outs[(True, None)]
    tiled = 0
    for key, got in outs.items():
        tiled += key[1] is not None and key[1][2] >= 100000
        for a, b in zip(ref, got):
            for x, y in zip(a, b):
                assert np.array_equal(x, y), key
    assert tiled >= 1 or width < 4


@pytest.mark.gpu
def test_server_adaptive_width_equals_full_width(gpu):
    """Models that step at the narrowest width covering their busy lanes,
    restrided in place while requests are in flight (narrowed when short
    requests leave, widened when new ones join), give the results of models
    that always step at their full lane count bit for bit: real and complex
    lanes, LDOS and directly gathered Green's-function lanes.  They move
    fewer bytes."""
    kpm = gpu
    ms = models()[:2]
    outs, stats = [], []
    for adaptive in (True, False):
        srv = kpm.Server(2048, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
        srv.set_adaptive_width(adaptive)
        ids = [srv.add_model(*c, S, 32) for _, c in ms]

        def sites(i, k, off):
            N = ms[i][1][0].size - 1
            return (np.arange(off, off + k, dtype=np.uint32) * 7) % N

        first, late = [], []
        for i in range(len(ms)):
            first.append(srv.submit(ids[i], sites(i, 2, 1), 1600, 1e-3))
            first.append(srv.submit_greens(ids[i], sites(i, 3, 5) + 1, sites(i, 3, 5), 900, 1e-3,
                                           "Retarded"))
        short = [srv.submit(ids[i], sites(i, k, 20 + k), M, 1e-3)
                 for i in range(len(ms)) for k, M in ((10, 40), (16, 48))]
        res = [srv.wait(q) for q in short]
        for i in range(len(ms)):
            late.append(srv.submit(ids[i], sites(i, 12, 60), 64, 1e-3))
        res += [srv.wait(q) for q in first + late]
        outs.append(res)
        stats.append(srv.stats())
        srv.close()
    for a, b in zip(*outs):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert stats[0]["relayouts"] >= 2 and stats[1]["relayouts"] == 0
    assert stats[0]["step_bytes"] < stats[1]["step_bytes"]


@pytest.mark.gpu
def test_server_graph_replay_equals_direct_launches(gpu):
    """Ticks that replay a captured graph of one step give the results of
    direct launches bit for bit, and the graph path is the one taken."""
    kpm = gpu
    ms = models()
    outs = []
    for graphs in (True, False):
        srv = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=6, tolerance=0)
        srv.set_graphs(graphs)
        ids = [srv.add_model(*c, S, 8) for _, c in ms]
        outs.append(_mixed_traffic(kpm, srv, ids, ms, 17))
        st = srv.stats()
        assert (st["graph_ticks"] > 0) == graphs
        srv.close()
    for a, b in zip(*outs):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_server_real_lanes_equal_complex_lanes(gpu):
    """Real models on real float lanes give the complex64 lanes' results bit
    for bit (the fixed-point sums make them independent of the kernel)."""
    kpm = gpu
    outs = []
    for real in (True, False):
        srv = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=0)
        srv.set_real(real)
        ms = models()
        ids = [srv.add_model(*c, S, 8) for _, c in ms]
        reqs = [srv.submit(ids[i], np.array([3, 40 + i, 77], dtype=np.uint32), 200, 1e-3)
                for i in range(len(ms))]
        outs.append([srv.wait(r) for r in reqs])
        srv.close()
    for a, b in zip(*outs):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_server_widths(gpu):
    kpm = gpu
    _, csr = models()[3]
    sites = np.array([3], dtype=np.uint32)
    ref = _solo(kpm, csr, sites, 128, 1e-3, 1)
    for w in (2, 4, 8, 16, 32, 64):
        got = _solo(kpm, csr, sites, 128, 1e-3, w)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), w


@pytest.mark.gpu
def test_server_fp64_rerun_on_miss(gpu):
    kpm = gpu
    _, csr = models()[0]
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=1e-300)
    mid = srv.add_model(*csr, S, 4)
    sites = np.array([7, 8, 200], dtype=np.uint32)
    ldos, err, rerun = srv.wait(srv.submit(mid, sites, 256, 1e-3))
    assert rerun.all()
    assert np.array_equal(ldos, fp64_ldos(kpm, csr, sites, 256, 1e-3))
    assert srv.stats()["reruns"] == 3
    srv.close()


@pytest.mark.gpu
def test_server_error_estimate_bounds_error_on_uneven_batch(gpu):
    """The per-site error estimate is at least the actual LDOS error on
    every sampled solve of uneven-batch models (the uneven batch's
    distribution of lattices, disorder, site counts and coefficient counts,
    with sides up to 96), and with the FP64 rerun at tolerance 1e-6 every
    returned LDOS is within 1e-6 of the FP64 recursion."""
    kpm = gpu
    energies = workloads.open_grid(S, 1000)
    specs = [sp for sp in workloads.cfg4_specs(1000, seed=4) if sp[1] <= 96][:40]
    srv = kpm.Server(4096, energies, hbm_budget=8 << 30, tick_steps=64, tolerance=1e-6)
    jobs = []
    for kind, L, J, W, ns, M, seed in specs:
        csr = workloads.build_model(kind, L, J, W, seed)
        cells = 2 * L * L if kind == "honeycomb" else L * L
        sites = workloads.sample_sites(cells, 2, ns, seed + 1)
        w = 1 << max(ns - 1, 0).bit_length()
        jobs.append((csr, sites, M, srv.submit(srv.add_model(*csr, S, w), sites, M, 1e-3)))
    solves = reruns = 0
    ratios = []
    for csr, sites, M, rid in jobs:
        ldos, est, rerun = srv.wait(rid, timeout=600)
        m = kpm.Matrix.from_csr(*csr, S)
        t = kpm.Table.create(M, energies, S)
        ref, _ = m.ldos_sites(t, sites, 1e-3, kpm.FP64)
        for k in range(sites.size):
            e = rel_err(ldos[k], ref[k])
            assert e <= 1e-6, (M, k, e, est[k], rerun[k])
            if rerun[k]:
                assert e == 0.0
                reruns += 1
            else:
                assert est[k] >= e, (M, k, e, est[k])
                ratios.append(est[k] / e if e > 0 else np.inf)
            solves += 1
    assert solves >= 200
    assert srv.stats()["reruns"] == reruns
    srv.close()


@pytest.mark.gpu
def test_server_hbm_budget_admission(gpu):
    """A budget for one model's lanes: requests to two models alternate
    through eviction and still give the right answers."""
    kpm = gpu
    ms = models()[:2]
    probe = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    probe.add_model(*ms[0][1], S, 8)
    probe.close()
    N0 = ms[0][1][0].size - 1
    N1 = ms[1][1][0].size - 1
    need = max(2 * N * 8 * 8 + 8 * (2 * 256 + 129) * 16 + 1024 + N // 8 for N in (N0, N1))
    srv = kpm.Server(256, grid(), hbm_budget=need, tick_steps=8, tolerance=0)
    ids = [srv.add_model(*c, S, 8) for _, c in ms]
    jobs = []
    for r in range(6):
        i = r % 2
        sites = np.array([r, r + 10], dtype=np.uint32)
        jobs.append((i, sites, srv.submit(ids[i], sites, 128, 1e-3)))
    for i, sites, rid in jobs:
        ldos, _, _ = srv.wait(rid)
        ref = fp64_ldos(kpm, ms[i][1], sites, 128, 1e-3)
        assert rel_err(ldos, ref) <= TOL_MIXED
    st = srv.stats()
    assert st["evictions"] >= 1
    assert st["resident_bytes"] <= need
    srv.close()


@pytest.mark.gpu
def test_server_concurrent_submitters(gpu):
    kpm = gpu
    ms = models()
    srv = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    ids = [srv.add_model(*c, S, 16) for _, c in ms]
    results = {}
    lock = threading.Lock()

    def client(t):
        rng = np.random.default_rng(100 + t)
        for _ in range(5):
            i = int(rng.integers(len(ms)))
            N = ms[i][1][0].size - 1
            sites = rng.choice(N, size=int(rng.integers(1, 5)), replace=False).astype(np.uint32)
            M = int(rng.integers(8, 256))
            out = srv.wait(srv.submit(ids[i], sites, M, 1e-3))
            with lock:
                results[(t, len(results))] = (i, sites, M, out)

    th = [threading.Thread(target=client, args=(t,)) for t in range(4)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert len(results) == 20
    for i, sites, M, (ldos, _, _) in results.values():
        assert rel_err(ldos, fp64_ldos(kpm, ms[i][1], sites, M, 1e-3)) <= TOL_MIXED
    srv.close()


@pytest.mark.gpu
def test_server_argument_errors(gpu):
    kpm = gpu
    _, csr = models()[3]
    srv = kpm.Server(128, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    with pytest.raises(kpm.TBTKError):
        srv.add_model(*csr, S, 3)               # width not a power of two
    with pytest.raises(kpm.TBTKError):
        srv.add_model(*csr, 5.0, 4)             # energies outside (-s, s)
    mid = srv.add_model(*csr, S, 4)
    with pytest.raises(kpm.TBTKError):
        srv.submit(mid, np.arange(5), 64, 1e-3)  # more sites than lanes
    with pytest.raises(kpm.TBTKError):
        srv.submit(mid, [0], 129, 1e-3)          # M above max_moments
    with pytest.raises(kpm.TBTKError):
        srv.submit(mid, [0], 1, 1e-3)            # M < 2
    with pytest.raises(kpm.TBTKError):
        srv.submit(mid, [10 ** 6], 64, 1e-3)     # site outside the model
    with pytest.raises(kpm.TBTKError):
        srv.submit(mid + 1, [0], 64, 1e-3)       # no such model
    with pytest.raises(kpm.TBTKError):
        srv.set_config(4, 8, 8, 2)               # shape of another width
    srv.close()
    small = kpm.Server(128, grid(), hbm_budget=1000, tick_steps=8, tolerance=0)
    with pytest.raises(kpm.TBTKError):
        small.add_model(*csr, S, 4)              # lanes exceed the budget
    small.close()


@pytest.mark.gpu
def test_server_autotune(gpu):
    kpm = gpu
    _, csr = models()[0]
    srv = kpm.Server(256, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    mid = srv.add_model(*csr, S, 16)
    cfg = srv.autotune(16, probe_steps=4)
    assert cfg["tpr"] * cfg["vpt"] == 16 and cfg["ms_per_step"] > 0
    sites = np.array([1, 2, 3], dtype=np.uint32)
    ldos, _, _ = srv.wait(srv.submit(mid, sites, 128, 1e-3))
    assert rel_err(ldos, fp64_ldos(kpm, csr, sites, 128, 1e-3)) <= TOL_MIXED
    srv.close()


def fp64_greens(kpm, csr, to, frm, M, broadening, type_):
    """G(to[k], frm[k]) through the FP64 batched recursion and the lookup
    table (both pinned against the reference elsewhere)."""
    m = kpm.Matrix.from_csr(*csr, S)
    t = kpm.Table.create(M, grid(), S)
    src = list(dict.fromkeys(int(f) for f in frm))
    owner = [src.index(int(f)) for f in frm]
    mu, _ = m.moments_batched(src, to, owner, M, broadening, kpm.FP64)
    return t.greens(mu, type_)


GF_CASES = [
    # (model, to, from, M, type): diagonal pairs run the doubling lanes,
    # the others gather every moment directly
    (1, [5, 77, 300], [5, 77, 300], 384, "Retarded"),
    (1, [6, 7, 40, 5], [5, 5, 5, 300], 256, "NonPrincipal"),
    (0, [3, 5, 4, 51], [3, 3, 3, 3], 320, "Advanced"),
    (2, [10, 11, 12, 13], [10, 10, 12, 12], 200, "Principal"),
]


@pytest.mark.gpu
def test_server_greens_match_fp64(gpu):
    """Green's-function requests of every type, diagonal (doubling lanes)
    and off-diagonal (directly gathered pairs), on real and complex models,
    within the mixed-precision bar of the FP64 recursion's G(E)."""
    kpm = gpu
    ms = models()
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=0)
    ids = [srv.add_model(*c, S, 8) for _, c in ms]
    jobs = [(c, srv.submit_greens(ids[c[0]], c[1], c[2], c[3], 1e-3, c[4])) for c in GF_CASES]
    for (i, to, frm, M, ty), rid in jobs:
        G, err, rerun = srv.wait(rid)
        ref = fp64_greens(kpm, ms[i][1], to, frm, M, 1e-3, kpm.ChebyshevExpander.Type[ty])
        assert G.shape == (len(to), E) and not rerun.any()
        for k in range(len(to)):
            assert 0 <= err[k] < 1e-3
            if not ref[k].any():
                # to and from in sectors the Hamiltonian does not connect
                assert not G[k].any()
                continue
            e = rel_err(G[k], ref[k])
            assert e <= TOL_MIXED, (ms[i][0], ty, k, e)
            # the estimate bounds the error of Green's functions too
            assert err[k] >= e, (ms[i][0], ty, k, e, err[k])
    srv.close()


@pytest.mark.gpu
def test_server_greens_alone_equals_in_mix(gpu):
    """A Green's-function request gives the same bits alone and in a mix of
    LDOS and other Green's-function traffic."""
    kpm = gpu
    ms = models()
    alone = []
    for i, to, frm, M, ty in GF_CASES[:2]:
        srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=0)
        mid = srv.add_model(*ms[i][1], S, 8)
        alone.append(srv.wait(srv.submit_greens(mid, to, frm, M, 1e-3, ty)))
        srv.close()
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=5, tolerance=0)
    ids = [srv.add_model(*c, S, 8) for _, c in ms]
    rng = np.random.default_rng(7)
    bg = []
    for r in range(10):
        i = r % len(ms)
        N = ms[i][1][0].size - 1
        sites = rng.choice(N, size=int(rng.integers(1, 4)), replace=False).astype(np.uint32)
        bg.append(srv.submit(ids[i], sites, int(rng.integers(16, 400)), 1e-3))
        if r % 3 == 0:
            bg.append(srv.submit_greens(ids[i], sites, sites[::-1], int(rng.integers(16, 300)),
                                        1e-3, "Retarded"))
    import time
    time.sleep(0.05)
    probes = [srv.submit_greens(ids[i], to, frm, M, 1e-3, ty) for i, to, frm, M, ty in GF_CASES[:2]]
    mixed = [srv.wait(p) for p in probes]
    for b in bg:
        srv.wait(b)
    for a, b in zip(alone, mixed):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    srv.close()


@pytest.mark.gpu
def test_server_greens_fp64_rerun(gpu):
    kpm = gpu
    _, csr = models()[1]
    srv = kpm.Server(512, grid(), hbm_budget=1 << 30, tick_steps=16, tolerance=1e-300)
    mid = srv.add_model(*csr, S, 4)
    to, frm = [6, 7, 40], [5, 5, 300]
    G, err, rerun = srv.wait(srv.submit_greens(mid, to, frm, 256, 1e-3, "Retarded"))
    assert rerun.all()
    assert np.array_equal(G, fp64_greens(kpm, csr, to, frm, 256, 1e-3, kpm.RETARDED))
    srv.close()


@pytest.mark.gpu
def test_server_cancel(gpu):
    """A cancelled request in flight frees its lanes for the next one, a
    cancelled queued request never starts, and a finished one is not
    affected."""
    kpm = gpu
    _, csr = models()[0]
    srv = kpm.Server(4096, grid(), hbm_budget=1 << 30, tick_steps=4, tolerance=0)
    mid = srv.add_model(*csr, S, 2)
    long_a = srv.submit(mid, [1, 2], 4096, 1e-3)    # takes both lanes
    queued = srv.submit(mid, [3], 64, 1e-3)         # waits for a lane
    srv.cancel(queued)
    srv.cancel(queued)                               # twice is not an error
    with pytest.raises(kpm.TBTKError) as e:
        srv.wait(queued)
    assert e.value.status == kpm.ERR_CANCELLED
    srv.cancel(long_a)
    with pytest.raises(kpm.TBTKError) as e:
        srv.wait(long_a)
    assert e.value.status == kpm.ERR_CANCELLED
    # the lanes are free again: a new request runs and is right
    sites = np.array([5, 9], dtype=np.uint32)
    rid = srv.submit(mid, sites, 128, 1e-3)
    import time
    while srv.stats()["completed"] < 1:
        time.sleep(0.01)
    with pytest.raises(kpm.TBTKError) as e:
        srv.cancel(rid)
    assert e.value.status == kpm.ERR_STATE
    ldos, _, _ = srv.wait(rid)
    assert rel_err(ldos, fp64_ldos(kpm, csr, sites, 128, 1e-3)) <= TOL_MIXED
    with pytest.raises(kpm.TBTKError) as e:
        srv.cancel(rid)                              # released by wait
    assert e.value.status == kpm.ERR_ARGUMENT
    srv.close()


@pytest.mark.gpu
def test_server_greens_argument_errors(gpu):
    kpm = gpu
    _, csr = models()[3]
    srv = kpm.Server(128, grid(), hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    mid = srv.add_model(*csr, S, 4)
    with pytest.raises(kpm.TBTKError):
        srv.submit_greens(mid, [0, 1], [0], 64, 1e-3)          # lengths differ
    with pytest.raises(kpm.TBTKError):
        srv.submit_greens(mid, [0] * 5, [1] * 5, 64, 1e-3)     # more pairs than lanes
    with pytest.raises(kpm.TBTKError):
        srv.submit_greens(mid, [0], [10 ** 6], 64, 1e-3)       # from outside the model
    with pytest.raises(kpm.TBTKError):
        srv.submit_greens(mid, [10 ** 6], [0], 64, 1e-3)       # to outside the model
    with pytest.raises(kpm.TBTKError):
        srv.submit_greens(mid, [0], [0], 64, 1e-3, 7)          # unknown type
    srv.close()


def test_server_calls_check_their_handle(kpm):
    """Entry points of the server reject a NULL handle with a status."""
    lib = kpm.load_library()
    assert lib.tbtkkpm_server_cancel(None, 1) == kpm.ERR_ARGUMENT
    assert lib.tbtkkpm_server_wait_greens(None, 1, 0.0, None, None, None) == kpm.ERR_ARGUMENT
    assert lib.tbtkkpm_server_submit_greens(None, 0, None, None, 0, 64, 0.0, 1, None) \
        == kpm.ERR_ARGUMENT
    assert b"NULL server" in lib.tbtkkpm_last_error()


def test_server_needs_a_device(kpm):
    if kpm.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(kpm.TBTKError) as e:
        kpm.Server(128, grid(), hbm_budget=1 << 20)
    assert e.value.status == kpm.ERR_CUDA
