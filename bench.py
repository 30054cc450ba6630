#!/usr/bin/env python
"""Benchmark of the KPM (Chebyshev) LDOS path on B200.

Workload (default): the 2048x2048 periodic square lattice with spin
(N = 8,388,608, nnz = 41,943,040), t=1, J=0.5, Anderson disorder U[-1, 1],
scaleFactor 12, 4096 Chebyshev moments, broadening 1e-3, 2000 energies on the
open grid (-12, 12), LDOS at 64 seeded sites per rank.

One step = the LDOS of the rank's 64 sites: the batched mixed-precision
recursion (float vectors [N][64] for this real model, complex64 ones for a
complex model; FP64 arithmetic and moments), FP64 damping and the FP64
energy sum through the lookup table, with the result copied to the host.
``value`` is LDOS solves/s over all ranks (sites per step x steps x ranks /
max over ranks of the device time).  Beside it the line carries the plain
FP64 single-vector path (one site per recursion, complex128, bit-exact with
the reference) on the same matrix, the LDOS error of the mixed result of
every site against the FP64 recursion (batched FP64, bit-identical per site
to the single-vector path, timed as ``fp64_batched``), the speed-up split
into its mechanisms, the roofline of the recursion step, the CPU baseline,
and three sub-results:
the 1024x1024 Rashba lattice (complex Hamiltonian, 256 sites, M = 2048),
the LDOS server on the 1000-model uneven batch at tolerance 1e-6, and the
server under Poisson arrivals (100 requests/s offered for 3 s, 32 lanes
per model).

Inputs are larger than L2 (13.8 GB of matrix and vectors per recursion step
against 126 MB of L2), so no flush is needed between steps.

    python bench.py [--steps K] [--warmup W] [--impl ours|reference]
    torchrun --nproc-per-node N bench.py --gpus N   (weak scaling: 64 sites per rank)
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sites", type=int, default=64)
    ap.add_argument("--lattice", type=int, default=2048, help="lattice side L (L x L x 2 states)")
    ap.add_argument("--moments", type=int, default=4096)
    ap.add_argument("--plain-sites", type=int, default=2,
                    help="sites timed one at a time on the plain FP64 single-vector path")
    ap.add_argument("--no-sub", action="store_true",
                    help="skip the Rashba and server sub-results")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (read + write) per row of one launch of the batched step, by
# (vectors, B, tpr, vpt, variant), from ncu captures on the 1024x1024
# lattice (N = 2,097,152 rows); the traffic grows with the rows, so a launch
# on N rows moves that figure times N.  complex64 (8, 8, 2): 3.427 GB there
# (algorithmic bytes 3.439 GB); real float vectors (8, 8, 2): 1.721 GB,
# (4, 16, 2): 1.808 GB, (4, 16, 802) (dot sums in shared memory): 1.713 GB
# (algorithmic bytes 1.744 GB).
# The tile-staged step (variant >= 100000) with 64-row tiles: real float
# vectors, (8, 8), 16 consumer warps: 1.686 GB (1.182 read + 0.504 write);
# keyed by (vectors, B, "tiled", rows per tile).
TRAFFIC_PER_ROW = {("real float", 64, "tiled", 64): 1.686e9 / 2097152,
                   ("complex64", 64, 8, 8, 2): 3.427e9 / 2097152,
                   ("real float", 64, 8, 8, 2): 1.721e9 / 2097152,
                   ("real float", 64, 4, 16, 2): 1.8075e9 / 2097152,
                   ("real float", 64, 4, 16, 802): 1.7130e9 / 2097152}


def traffic_per_row(vec_kind, B, tuned):
    tpr, vpt, variant = tuned[:3]
    if variant >= 100000:
        return TRAFFIC_PER_ROW.get((vec_kind, B, "tiled", ((variant - 100000) % 1000000) // 1000))
    return TRAFFIC_PER_ROW.get((vec_kind, B, tpr, vpt, variant))


def kernel_name(real_vectors, tuned):
    tpr, vpt, variant = tuned[:3]
    if variant >= 100000:
        v = variant - 100000
        cv = v // 1000000
        return (f"kpm_step_tiled<{'real' if real_vectors else 'complex64'}, tpr={tpr}, "
                f"vpt={vpt}, rows/tile={(v % 1000000) // 1000}, consumer warps={(v % 1000) // 10}, "
                f"blocks/SM={v % 10}, widening split={cv % 100}"
                f"{', row pairs' if cv >= 100 else ''}>")
    return f"{'kpm_step_real' if real_vectors else 'kpm_step<float2'}, tpr={tpr}, vpt={vpt}, minb={variant}"


def host_cpu():
    """Core count and model of this host (the CPU baselines' machine)."""
    model = None
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        lscpu = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        keep = ("Model name", "Socket(s)", "Core(s) per socket", "Thread(s) per core", "CPU(s)")
        info = {k.strip(): v.strip() for k, v in (ln.split(":", 1) for ln in lscpu.splitlines()
                                                  if ":" in ln) if k.strip() in keep}
    except (OSError, subprocess.SubprocessError):
        info = {}
    return {"nproc": os.cpu_count(), "model": model, "lscpu": info}


def peak_hbm():
    try:
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_problem(args, rank):
    from tbtk_b200 import workloads
    p = workloads.cfg2(n_sites=args.sites, L=args.lattice, seed=2048)
    # weak scaling: every rank solves its own seeded sites on the same model
    p.sites = workloads.sample_sites(args.lattice * args.lattice, 2, args.sites, 2049 + 7919 * rank)
    p.M = args.moments
    return p


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings; every rank gets it."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def step_bytes(p, B, s_vec, s_val=16):
    """Algorithmic bytes of one recursion step: the CSR matrix once (values,
    column indices, row pointers) and three vector passes per source
    (gather of j_n counted once, read of j_{n-1}, write of j_{n+1}).
    s_vec/s_val: bytes per vector element / stored value (complex128 16/16,
    complex64 8/16, real vectors of a real matrix 4/8)."""
    return p.nnz * (s_val + 4) + 4 * (p.N + 1) + 3 * p.N * B * s_vec


# ------------------------------------------------------------------ CPU baselines

def cpu_port_baseline(p, threads, sample_steps=(4, 36)):
    """The oracle restatement (bit-identical to the reference's CPU
    recursion), one site per thread, timed at two truncated coefficient
    counts; per-site time extrapolated linearly to the full M."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_lib import Oracle
    o = Oracle()
    sites = [int(x) for x in p.sites[:threads]]

    def run(M):
        ts = [0.0] * len(sites)

        def work(i):
            t0 = time.perf_counter()
            o.moments(p.rowptr, p.col, p.val, p.scale, M, sites[i], [sites[i]])
            ts[i] = time.perf_counter() - t0

        th = [threading.Thread(target=work, args=(i,)) for i in range(len(sites))]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        return time.perf_counter() - t0

    def fit(lo, hi):
        slope = (hi - lo) / (sample_steps[1] - sample_steps[0])
        if slope > 0:
            return slope, max(lo - slope * sample_steps[0], 0.0), "linear"
        return hi / sample_steps[1], 0.0, "degenerate (upper bound)"

    t_lo = run(sample_steps[0])
    t_hi = run(sample_steps[1])
    per_step, fixed, fit_kind = fit(t_lo, t_hi)
    t_site = fixed + per_step * p.M
    # one site alone on one core, the same fit
    all_sites, sites = sites, sites[:1]
    s1, f1, _ = fit(run(sample_steps[0]), run(sample_steps[1]))
    sites = all_sites
    t_one = f1 + s1 * p.M
    return {"value": len(sites) / t_site, "unit": "LDOS solves/s", "cores": len(sites),
            "kind": "port", "fit": fit_kind,
            "one_core": {"value": 1.0 / t_one, "unit": "LDOS solves/s", "s_per_solve": t_one},
            "sample": (f"{len(sites)} sites in parallel (one thread each) at M="
                       f"{sample_steps[0]} and M={sample_steps[1]} of the same matrix; "
                       f"per-site time {fixed:.2f} s + {per_step:.3f} s/step extrapolated to "
                       f"M={p.M} (energy sum excluded)")}


def reference_arm(args, world, rank):
    """The TBTK reference compiled from its sources (oracle/_ref): Model
    construction once, then per step P threads each running
    PropertyExtractor::ChebyshevExpander::calculateLDOS for one site with a
    truncated coefficient count; the per-site time is fitted linearly in M
    over the warm-up (M = 4) and timed (M = 68) samples and extrapolated to
    the full M."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_lib import Reference
    from tbtk_b200 import lattice as L
    from tbtk_b200 import workloads
    if not Reference.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libtbtkref.so was not built "
                "(the TBTK reference sources were absent at build time)"}
    ref = Reference()
    import psutil
    avail_gb = psutil.virtual_memory().available / 1e9
    lat = L.square(args.lattice, args.lattice, t=1.0, J=0.5, W=2.0, periodic=True, seed=2048)
    t0 = time.perf_counter()
    model = ref.model(lat)
    build_s = time.perf_counter() - t0
    del lat
    N = args.lattice * args.lattice * 2
    per_thread_gb = 5e-7 * N  # getSparseMatrix transient, measured at 512^2 and scaled
    threads = int(max(1, min(os.cpu_count() or 1, 32,
                             (psutil.virtual_memory().available / 1e9 - 4) // max(per_thread_gb, 0.1))))
    sites = workloads.sample_sites(args.lattice * args.lattice, 2, threads, 2049)
    s, E = 12.0, 2000
    dx = 2 * s / (E + 1)
    lo, hi = -s + dx, -s + dx + (E - 1) * dx

    def sample(M):
        def work(i):
            x, y = divmod(int(sites[i]) // 2, args.lattice)
            model.ldos(s, M, 1e-3, lo, hi, E, [[x, y, 0]])
        th = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        return time.perf_counter() - t0

    # Per site, the model's CSR build and setup cost tens of seconds before
    # the first step, and the recursion about 0.1-0.2 s a step, so the two
    # sample sizes lie 64 steps apart; the minimum of each set filters the
    # noise of threads contending for memory.
    m_lo, m_hi = 4, 68
    lo_t = [sample(m_lo) for _ in range(max(1, args.warmup))]
    hi_t = [sample(m_hi) for _ in range(max(1, args.steps))]
    t_lo, t_hi = min(lo_t), min(hi_t)
    slope = (t_hi - t_lo) / (m_hi - m_lo)
    if slope > 0:
        per_step, fixed, fit = slope, max(t_lo - slope * m_lo, 0.0), "linear"
    else:
        # no measurable step cost: bound it by the whole larger sample
        per_step, fixed, fit = t_hi / m_hi, 0.0, "degenerate (upper bound: no fixed cost)"
    t_site = fixed + per_step * args.moments
    value = threads / t_site
    return {
        "impl": "reference", "metric": "LDOS solves/s", "value": value, "unit": "LDOS solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        # the timed steps are the M=68 samples; the metric extrapolates them
        "ms_per_step": statistics.mean(hi_t) * 1e3,
        "extrapolated_ms_per_solve": t_site * 1e3 / threads,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded lattice)",
        "config": {"workload": f"square {args.lattice}x{args.lattice} spin periodic, W=2, s=12, "
                               f"M={args.moments}, E=2000, LDOS per site",
                   "model_build_s": round(build_s, 1)},
        "cpu_baseline": {"value": value, "unit": "LDOS solves/s", "cores": threads,
                         "kind": "reference", "host": host_cpu(),
                         "sample": (f"TBTK PropertyExtractor::calculateLDOS on {threads} threads "
                                    f"(one site each) at M={m_lo} ({len(lo_t)}x) and M={m_hi} "
                                    f"({len(hi_t)}x), minimum of each; per-site {fixed:.2f} s + "
                                    f"{per_step:.3f} s/step extrapolated to M={args.moments}"),
                         "fit": fit},
        "e2e": {"value": value, "unit": "LDOS solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ sub-results

def rashba_sub(args, stream):
    """The 1024x1024 Rashba lattice (complex Hamiltonian, 9 entries per row):
    256 sites in one tbtkkpm_ldos_sites call at M = 2048 (two 128-source
    complex64 SpMM recursions by default), against the plain FP64
    single-vector path on the same matrix, with the LDOS error of 16 sites
    spread over the batch against their FP64 recursion."""
    import torch
    from tbtk_b200 import kpm, workloads
    p = workloads.cfg3()
    mat = kpm.Matrix.from_csr(p.rowptr, p.col, p.val, p.scale)
    tab = kpm.Table.create(p.M, p.energies, p.scale)
    mat.set_stream(stream.cuda_stream)
    width = mat.batch_width(kpm.MIXED, ldos=True)
    tuned = mat.autotune(min(width, p.sites.size), kpm.MIXED, ldos=True, probe_steps=6)
    mat.set_profiling(True)
    with torch.cuda.stream(stream):
        mat.ldos_sites(tab, p.sites, p.broadening, kpm.MIXED)  # warm
        mat.profile()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        got, est = mat.ldos_sites(tab, p.sites, p.broadening, kpm.MIXED)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        rec, _, launches = mat.profile()
        mat.ldos_sites(tab, p.sites[:1], p.broadening, kpm.FP64)  # warm
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        mat.ldos_sites(tab, p.sites[1:2], p.broadening, kpm.FP64)
        f1.record(stream)
        torch.cuda.synchronize()
        plain_ms = f0.elapsed_time(f1)
        prec, _, plaunch = mat.profile()
        pick = np.linspace(0, p.sites.size - 1, 16).astype(int)
        ref, _ = mat.ldos_sites(tab, p.sites[pick], p.broadening, kpm.FP64)
    errs = [float(np.abs(got[i] - r).max() / np.abs(r).max()) for i, r in zip(pick, ref)]
    step_ms = rec / max(launches, 1)
    batches = [min(width, p.sites.size - b0) for b0 in range(0, p.sites.size, width)]
    bstep = sum(step_bytes(p, b, 8) for b in batches) / len(batches)
    peak, _ = peak_hbm()
    rate = p.sites.size / (ms / 1e3)
    return {
        "workload": (f"rashba 1024x1024 spin periodic alpha=0.3 (N={p.N}, nnz={p.nnz}), W=2, "
                     f"s=12, M={p.M}, E={p.energies.size}, {p.sites.size} sites in one call "
                     f"(batches of {width})"),
        "value": rate, "unit": "LDOS solves/s", "ms_per_call": ms,
        "step_ms": step_ms, "autotuned": dict(zip(("tpr", "vpt", "variant", "ms_per_step"), tuned)),
        "kernel": kernel_name(False, tuned),
        "roofline": {"achieved_GBps": bstep / (step_ms / 1e3) / 1e9,
                     "frac": bstep / (step_ms / 1e3) / 1e9 / peak, "bytes_per_launch": bstep},
        "plain_fp64": {"ms_per_solve": plain_ms, "value": 1e3 / plain_ms,
                       "step_ms": prec / max(plaunch, 1)},
        "speedup_vs_plain_fp64": rate * plain_ms / 1e3,
        "speedup_per_site_step": (prec / max(plaunch, 1)) / (step_ms / batches[0]),
        "ldos_rel_err_vs_fp64": max(errs), "ldos_err_sites": len(errs),
        "error_estimate_max": float(np.max(est)),
    }


def server_sub():
    """The LDOS server on the uneven batch (all 1000 models, every request
    submitted at once) at tolerance 1e-6 (FP64 rerun of a site whose error
    estimate exceeds it)."""
    from tbtk_b200 import serve_bench
    a = argparse.Namespace(models=1000, budget_gb=120.0, tick=64, tolerance=1e-6, samples=16,
                           sample_seed=44, fp64_head=32)
    r = serve_bench.uneven(a)
    st = r["server"]
    return {"workload": r["workload"], "value": r["value"], "unit": "LDOS solves/s",
            "p50_ms": st.get("p50_ms"), "p99_ms": st.get("p99_ms"), "reruns": st.get("reruns"),
            "rerun_rate": st.get("reruns", 0) / max(r["solves"], 1),
            "solves": r["solves"], "wall_s": r["wall_s"],
            "plain_fp64": r["plain_fp64"], "speedup_vs_plain_fp64": r["speedup_vs_plain_fp64"],
            "ldos_rel_err_vs_fp64_max": r["ldos_rel_err_vs_fp64_max"],
            "estimate_vs_error": r["estimate_vs_error"],
            "step_GBps": r["step_GBps"]}


def serving_sub():
    """The server answering Poisson arrivals at 100 requests/s for 3 s
    against the 64-model pool (LDOS requests of 1-16 sites, M in
    [512, 4096]): served throughput and the latency percentiles."""
    from tbtk_b200 import serve_bench
    a = argparse.Namespace(models=64, budget_gb=120.0, tick=64, tolerance=1e-6, samples=8,
                           sample_seed=44, fp64_head=32, rate=100.0, duration=3.0, width=32,
                           full_width=False)
    r = serve_bench.serve(a)
    st = r["server"]
    return {"workload": r["workload"], "value": r["value"], "unit": "LDOS solves/s",
            "requests": r["requests"], "requests_per_s_served": r["requests_per_s"],
            "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "reruns": st.get("reruns"),
            "wall_s": r["wall_s"], "plain_fp64": r["plain_fp64"],
            "speedup_vs_plain_fp64": r["speedup_vs_plain_fp64"],
            "ldos_rel_err_vs_fp64_max": r["ldos_rel_err_vs_fp64_max"],
            "step_GBps": r["step_GBps"]}


# ------------------------------------------------------------------ our arm

def ours(args, world, rank, local):
    import torch
    from tbtk_b200 import kpm
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    p = make_problem(args, rank)
    B = p.sites.size
    stream = torch.cuda.Stream()
    mat = kpm.Matrix.from_csr(p.rowptr, p.col, p.val, p.scale)
    tab = kpm.Table.create(p.M, p.energies, p.scale)
    mat.set_stream(stream.cuda_stream)
    # project autotuner: pick the step configuration of both batch shapes
    tuned_mixed = mat.autotune(B, kpm.MIXED, ldos=True, probe_steps=6)
    tuned_plain = mat.autotune(1, kpm.FP64, ldos=True, probe_steps=6)
    real_vectors = mat.real()[1]  # the model is real: the mixed path runs real vectors
    mat.set_profiling(True)

    def step(prec, sites):
        return mat.ldos_sites(tab, sites, p.broadening, prec)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(kpm.MIXED, p.sites)
        mat.profile()
        clocks = Clocks(local)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        launches0 = kpm.kernel_launches()
        # where a launch list of this command (ncu -k regex:'^(kpm_|k_)' -s N)
        # finds the timed region: the library's own kernels launched before it
        print(f"[bench] library kernel launches before the timed region: {launches0}",
              file=sys.stderr, flush=True)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev0.record(stream)
        marks[0].record(stream)
        results = None
        for i in range(args.steps):
            results, _ = step(kpm.MIXED, p.sites)
            marks[i + 1].record(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = kpm.kernel_launches() - launches0
        ck = clocks.stop()
        total_ms = ev0.elapsed_time(ev1)
        step_ms = sorted(marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps))
        rec_ms, energy_ms, rec_launches = mat.profile()

        # plain FP64 single-vector path (complex128, one site per recursion):
        # timing on the first sites
        plain, plain_out = [], []
        step(kpm.FP64, p.sites[:1])  # warm
        mat.profile()
        for i in range(args.plain_sites):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out1, _ = step(kpm.FP64, p.sites[i:i + 1])
            e1.record(stream)
            torch.cuda.synchronize()
            plain.append(e0.elapsed_time(e1))
            plain_out.append(out1[0])
        plain_rec, _, plain_launches = mat.profile()
        # FP64 LDOS of every site in one batched FP64 recursion (the
        # reference's arithmetic, what TBTK's own API gets by default): it
        # gives each site's single-vector result bit for bit
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        ref_all, _ = step(kpm.FP64, p.sites)
        f1.record(stream)
        torch.cuda.synchronize()
        fp64_ms = f0.elapsed_time(f1)
        fp64_rec, _, fp64_launches = mat.profile()
    errs = [float(np.abs(results[i] - ref_all[i]).max() / np.abs(ref_all[i]).max())
            for i in range(B)]

    # end to end through the C ABI from pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
               for k, v in (("rowptr", p.rowptr), ("col", p.col),
                            ("val", p.val.view(np.float64)), ("sites", p.sites),
                            ("energies", p.energies))}
        val = pin["val"].view(np.complex128)

        def e2e_step():
            m2 = kpm.Matrix.from_csr(pin["rowptr"], pin["col"], val, p.scale)
            t2 = kpm.Table.create(p.M, pin["energies"], p.scale)
            out, _ = m2.ldos_sites(t2, pin["sites"], p.broadening, kpm.MIXED)
            m2.close()
            t2.close()
            return out

        e2e_step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        h2d = (p.rowptr.nbytes + p.col.nbytes + p.val.nbytes + p.sites.nbytes
               + p.energies.nbytes)
        e2e = {"seconds": e2e_s, "h2d": h2d, "d2h": B * p.energies.size * 8}

    total_ms, e2e_max = max_over_ranks([total_ms, e2e["seconds"] if e2e else 0.0], dist, "cuda")

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return None

    solves = B * args.steps * world
    value = solves / (total_ms / 1e3)
    avg_step_ms = rec_ms / max(rec_launches, 1)
    bstep = step_bytes(p, B, 4, 8) if real_vectors else step_bytes(p, B, 8)
    achieved = bstep / (avg_step_ms / 1e3) / 1e9
    vec_kind = "real float" if real_vectors else "complex64"
    traffic_row = traffic_per_row(vec_kind, B, tuned_mixed)
    peak, peak_kind = peak_hbm()
    plain_ms = statistics.median(plain) if plain else None
    plain_rate = 1e3 / plain_ms if plain_ms else None
    out = {
        "metric": "LDOS solves/s", "value": value, "unit": "LDOS solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": (("f32 vectors (real model)" if real_vectors else "c64 vectors")
                  + " / f64 arithmetic+moments"),
        "data": "synthetic (seeded lattice, Anderson disorder)",
        "config": {"workload": (f"square {args.lattice}x{args.lattice} spin periodic (N={p.N}, "
                                f"nnz={p.nnz}), t=1 J=0.5 W=2, s=12, M={p.M}, broadening 1e-3, "
                                f"E={p.energies.size} open grid, {B} LDOS sites per rank as one "
                                f"batched mixed-precision recursion"),
                   "sites_per_step_per_rank": B, "l2": "inputs larger than L2 (no flush)",
                   "autotuned": {"mixed_ldos": dict(zip(("tpr", "vpt", "minb", "ms_per_step"),
                                                        tuned_mixed)),
                                 "plain_fp64": dict(zip(("tpr", "vpt", "minb", "ms_per_step"),
                                                        tuned_plain))},
                   "parallelism": f"replicas x{world} (sites sharded, no collective)"},
        "gpu_launches": int(launches),
        "vector_steps_per_s": {"value": solves * p.M / (total_ms / 1e3),
                               "note": "sum over solves of the M moments each returns, per "
                                       "second (doubling runs step to M/2)"},
        "plain_fp64": {"value": plain_rate, "unit": "LDOS solves/s", "ms_per_solve": plain_ms,
                       "sites": args.plain_sites},
        "fp64_batched": {
            "value": B / (fp64_ms / 1e3), "unit": "LDOS solves/s", "ms_per_call": fp64_ms,
            "sites": B,
            "step_ms": fp64_rec / max(fp64_launches, 1),
            "roofline": {"achieved_GBps": step_bytes(p, B, 16) / (fp64_rec / max(fp64_launches, 1)
                                                                  / 1e3) / 1e9,
                         "frac": step_bytes(p, B, 16) / (fp64_rec / max(fp64_launches, 1) / 1e3)
                                 / 1e9 / peak,
                         "bytes_per_launch": step_bytes(p, B, 16)},
            "bit_identical_to_single_vector": all(np.array_equal(ref_all[i], plain_out[i])
                                                  for i in range(len(plain_out))),
            "note": ("the same sites in one batched FP64 recursion on complex128 vectors, M-1 "
                     "steps in the reference's operation order (TBTK's default precision through "
                     "the seam); its LDOS is the reference for ldos_rel_err_vs_fp64")},
        "speedup_vs_plain_fp64": (value / world) / plain_rate if plain_rate else None,
        "speedup_mechanisms": {
            "doubling": (p.M - 1) / (p.M // 2),
            "batch_and_vectors_per_site_step": (plain_rec / max(plain_launches, 1))
                                               / (avg_step_ms / B),
            "plain_step_ms": plain_rec / max(plain_launches, 1),
            "batched_step_ms_per_site": avg_step_ms / B,
            "note": ("doubling: M-1 single-vector steps against M/2 doubling steps; the other "
                     "factor compares one complex128 single-vector step with one site's share of "
                     "the batched step (real float vectors for this real model); their product "
                     "is the speed-up before the energy sums and the FP64 head")},
        "ldos_rel_err_vs_fp64": max(errs) if errs else None,
        "ldos_err_sites": len(errs),
        "latency_ms": {"p50": statistics.median(step_ms),
                       "p99": step_ms[min(len(step_ms) - 1, int(0.99 * len(step_ms)))],
                       "note": (f"per {B}-site batch over the {args.steps} timed steps; "
                                "request-level latency is in the serving bench")},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": traffic_row * p.N if traffic_row else None,
                     "traffic_source": ("ncu dram__bytes_read+write of this kernel on the "
                                        "1024x1024 lattice (N=2097152), scaled by rows to N"),
                     "kernel": (f"{kernel_name(real_vectors, tuned_mixed)} (recursion step "
                                f"with the doubling dot products, B={B}, {vec_kind} vectors)"),
                     "bytes_per_launch": bstep, "avg_launch_ms": avg_step_ms,
                     "peak_kind": f"{peak_kind} (copy bandwidth)"},
        "recursion_share": rec_ms / total_ms if total_ms else None,
        "clocks": ck,
    }
    if e2e:
        out["e2e"] = {"value": solves / e2e_max * args.e2e_steps / args.steps,
                      "unit": "LDOS solves/s", "h2d_bytes_per_step": e2e["h2d"],
                      "d2h_bytes_per_step": e2e["d2h"], "steps": args.e2e_steps,
                      "includes": "CSR upload + device table + recursion + LDOS + download"}
    if world == 1 and not args.no_sub:
        out["rashba_cfg3"] = rashba_sub(args, stream)
        out["server_uneven"] = server_sub()
        out["server_serving"] = serving_sub()
    if world == 1 and not args.no_cpu:
        threads = int(min(os.cpu_count() or 1, B))
        out["cpu_baseline"] = cpu_port_baseline(p, threads)
        out["cpu_baseline"]["host"] = host_cpu()
    if dist:
        dist.destroy_process_group()
    return out


def main():
    args = parse()
    world, rank, local = dist_init()
    if args.impl == "reference":
        res = reference_arm(args, world, rank)
    else:
        res = ours(args, world, rank, local)
    if res is not None and rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
