"""Uneven-batch and serving measurements of the LDOS server (tbtkkpm_server).

    python -m tbtk_b200.serve_bench --workload uneven [--models 1000]
    python -m tbtk_b200.serve_bench --workload serve --rate 100 --duration 10

uneven: 1000 seeded models, half square (N = 2L^2) and half honeycomb
(N = 4L^2), L uniform in [16, 256], t = 1, J ~ U[0, 1], disorder W ~ U[0, 3];
each asks for the LDOS of 1-32 sites at M in {512, 1024, 2048, 4096}
(s = 12, 1000 points of the open grid in (-12, 12)).  Every request is
submitted at once; the value is LDOS solves (sites) per second of wall time
until the last one is done.  Each model gets the lane width of its site
count rounded up to a power of two, and each width is autotuned first.

serve: a pool of 64 seeded models (square, honeycomb, Rashba; N
log-uniform in [1e3, 4e6]; 32 lanes each, stepped at the width their busy
lanes need) answering Poisson arrivals at --rate requests per second for
--duration seconds, each request 1-16 sites
with M uniform in [512, 4096].  Reports throughput and the latency
percentiles of the server's own clock (submit to result).

Both compare with the plain FP64 single-vector path (tbtkkpm_ldos_sites
with one site at TBTKKPM_FP64, the reference's arithmetic) on a seeded
sample of the same (model, site, M) solves, and check the server's LDOS of
those sites against it.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import threading
import time

import numpy as np

from tbtk_b200 import kpm, workloads

S = 12.0
E = 1000


def pow2(n):
    w = 1
    while w < n:
        w *= 2
    return w


def basis_sites(kind, L, count, seed):
    cells = 2 * L * L if kind == "honeycomb" else L * L
    return workloads.sample_sites(cells, 2, count, seed)


def plain_baseline(samples, energies, broadening):
    """Times the plain FP64 single-vector path on (csr, site, M) samples;
    returns (seconds per solve, [ldos]) ."""
    out, total = [], 0.0
    for csr, site, M in samples:
        m = kpm.Matrix.from_csr(*csr, S)
        t = kpm.Table.create(M, energies, S)
        m.ldos_sites(t, [site], broadening, kpm.FP64)  # warm
        t0 = time.perf_counter()
        ldos, _ = m.ldos_sites(t, [site], broadening, kpm.FP64)
        total += time.perf_counter() - t0
        out.append(ldos[0])
        m.close()
        t.close()
    return total / len(samples), out


def uneven(a):
    energies = workloads.open_grid(S, E)
    specs = workloads.cfg4_specs(a.models, seed=4)
    srv = kpm.Server(4096, energies, hbm_budget=int(a.budget_gb * 2**30), tick_steps=a.tick,
                     tolerance=a.tolerance)
    srv.set_fp64_head(a.fp64_head)
    t0 = time.perf_counter()
    reqs, csrs = [], {}
    rng = np.random.default_rng(a.sample_seed)
    sample_idx = set(rng.choice(len(specs), size=min(a.samples, len(specs)), replace=False).tolist())
    rows = nnz = 0
    for i, (kind, L, J, W, ns, M, seed) in enumerate(specs):
        csr = workloads.build_model(kind, L, J, W, seed)
        sites = basis_sites(kind, L, ns, seed + 1)
        mid = srv.add_model(*csr, S, pow2(ns))
        reqs.append((mid, sites, M))
        rows += csr[0].size - 1
        nnz += int(csr[0][-1])
        if i in sample_idx:
            csrs[i] = csr
    setup_s = time.perf_counter() - t0
    tuned = {w: srv.autotune(w, probe_steps=6) for w in sorted({pow2(s[4]) for s in specs})}
    t0 = time.perf_counter()
    ids = [srv.submit(mid, sites, M, 1e-3) for mid, sites, M in reqs]
    results = [srv.wait(r, timeout=3600) for r in ids]
    wall = time.perf_counter() - t0
    st = srv.stats()
    solves = sum(s.size for _, s, _ in reqs)
    lane_steps = sum(s.size * (M // 2) for _, s, M in reqs)
    # plain FP64 single-vector path on one site of each sampled model
    samples, where = [], []
    for i in sorted(csrs):
        samples.append((csrs[i], int(reqs[i][1][0]), reqs[i][2]))
        where.append(i)
    t_plain, ref = plain_baseline(samples, energies, 1e-3)
    errs = [float(np.abs(results[i][0][0] - r).max() / np.abs(r).max()) for i, r in zip(where, ref)]
    # the server's error estimate of each sampled site next to its error
    # against the FP64 path (a site recomputed in FP64 has error 0)
    est = [(float(results[i][1][0]), e, int(results[i][2][0])) for i, e in zip(where, errs)]
    srv.close()
    return {
        "estimate_vs_error": est,
        "workload": f"uneven batch: {a.models} models (square/honeycomb, L in [16,256]), "
                    f"1-32 sites, M in {{512..4096}}, s=12, E=1000",
        "metric": "LDOS solves/s", "value": solves / wall, "unit": "LDOS solves/s",
        "wall_s": wall, "solves": solves, "models": a.models, "basis_rows": rows, "nnz": nnz,
        "lane_steps_per_s": lane_steps / wall, "setup_s": setup_s, "autotuned": tuned,
        "plain_fp64": {"s_per_solve": t_plain, "solves_per_s": 1.0 / t_plain,
                       "sample": f"{len(samples)} seeded (model, site, M) solves, one at a time"},
        "speedup_vs_plain_fp64": (solves / wall) * t_plain,
        "ldos_rel_err_vs_fp64_max": max(errs), "server": st,
        "step_GBps": st["step_bytes"] / max(st["step_s"], 1e-12) / 1e9,
    }


def serve(a):
    energies = workloads.open_grid(S, E)
    pool = workloads.cfg5_pool(a.models, seed=5)
    srv = kpm.Server(4096, energies, hbm_budget=int(a.budget_gb * 2**30), tick_steps=a.tick,
                     tolerance=a.tolerance)
    srv.set_fp64_head(a.fp64_head)
    srv.set_adaptive_width(not a.full_width)
    sizes, csrs = [], []
    t0 = time.perf_counter()
    for kind, L, J, W, alpha, seed in pool:
        csr = workloads.build_model(kind, L, J, W, seed, alpha=alpha)
        srv.add_model(*csr, S, a.width)
        sizes.append(csr[0].size - 1)
        csrs.append(csr)
    setup_s = time.perf_counter() - t0
    tuned = srv.autotune(a.width, probe_steps=6)
    reqs = workloads.cfg5_requests(sizes, a.rate, a.duration, seed=55)
    ids = [None] * len(reqs)
    start = time.perf_counter()

    def submitter():
        for i, (t, m, sites, M) in enumerate(reqs):
            delay = start + t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids[i] = srv.submit(m, sites, M, 1e-3)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    results = [srv.wait(r, timeout=3600) for r in ids]
    wall = time.perf_counter() - start
    st = srv.stats()
    solves = sum(s.size for _, _, s, _ in reqs)
    rng = np.random.default_rng(56)
    pick = rng.choice(len(reqs), size=min(a.samples, len(reqs)), replace=False)
    samples = [(csrs[reqs[i][1]], int(reqs[i][2][0]), reqs[i][3]) for i in pick]
    t_plain, ref = plain_baseline(samples, energies, 1e-3)
    errs = [float(np.abs(results[i][0][0] - r).max() / np.abs(r).max()) for i, r in zip(pick, ref)]
    srv.close()
    return {
        "workload": f"serving: {a.models} models (N log-uniform 1e3-4e6, square/honeycomb/"
                    f"Rashba, {a.width} lanes{', full-width steps' if a.full_width else ''}), Poisson {a.rate}/s for {a.duration}s, 1-16 sites, "
                    f"M in [512,4096], s=12, E=1000",
        "metric": "LDOS solves/s", "value": solves / wall, "unit": "LDOS solves/s",
        "requests": len(reqs), "requests_per_s": len(reqs) / wall, "wall_s": wall,
        "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "setup_s": setup_s, "autotuned": tuned,
        "plain_fp64": {"s_per_solve": t_plain, "solves_per_s": 1.0 / t_plain,
                       "sample": f"{len(samples)} seeded requests' first site, one at a time"},
        "speedup_vs_plain_fp64": (solves / wall) * t_plain,
        "ldos_rel_err_vs_fp64_max": max(errs), "server": st,
        "step_GBps": st["step_bytes"] / max(st["step_s"], 1e-12) / 1e9,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["uneven", "serve"], default="uneven")
    ap.add_argument("--models", type=int, default=None)
    ap.add_argument("--rate", type=float, default=100.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--tick", type=int, default=64)
    ap.add_argument("--tolerance", type=float, default=1e-6)
    ap.add_argument("--samples", type=int, default=16)
    ap.add_argument("--sample-seed", type=int, default=44,
                    help="seed of the sampled solves checked against the FP64 path")
    ap.add_argument("--width", type=int, default=32,
                    help="lanes of every pool model (serve)")
    ap.add_argument("--full-width", action="store_true",
                    help="serve: step every model at its full lane count (no adaptive width)")
    ap.add_argument("--fp64-head", type=int, default=32,
                    help="FP64 head steps of every lane (0: none)")
    a = ap.parse_args()
    if a.models is None:
        a.models = 1000 if a.workload == "uneven" else 64
    print(json.dumps(uneven(a) if a.workload == "uneven" else serve(a)))


if __name__ == "__main__":
    main()
