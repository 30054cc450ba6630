"""One small LDOS batch of the KPM path, for profiler captures and sweeps (a
measurement tool beside bench.py; the commands in profiles/ run it).

    python profile_case.py --lattice 2048 --sites 1 --precision fp64 --moments 8
    python profile_case.py --lattice 2048 --sites 64 --sweep --moments 32

Builds the periodic square lattice with spin (L x L x 2 states, t=1, J=0.5,
disorder U[-1, 1]; Rashba spin-orbit with --rashba), a device lookup table
of --moments coefficients over --energies points, and runs
tbtkkpm_ldos_sites for --sites seeded sites.  Prints the device time of the
recursion (CUDA events on the handle's stream) and its bandwidth in
algorithmic bytes (matrix once per step plus three vector passes per
source).  --sweep times every compiled step configuration for the batch;
--autotune lets the library's autotuner choose first; --config T,V,MB forces
one; --batch-width splits the sites into batches of that many.  Without
--rashba the model is real and the mixed precisions run on real float
vectors; --complex-vectors keeps complex64 ones.  --grid picks the energy sums
(lookup table, Clenshaw recurrences, or FFTs on the Chebyshev-node grid); the
printed energy time is theirs.

    python profile_case.py --lattice 1024 --server 16 --moments 256 --config 4,4,164082

--server W runs the same lattice as one model of the LDOS server with W
lanes instead: one request of W sites at --moments moments, every step a
float step (no FP64 head), with --config T,V,VARIANT installed (a
configuration of tbtkkpm_server_step_configs), or each configuration of the
width in turn with --sweep.  Prints the server's step time and bandwidth
(algorithmic bytes, the server's own statistics).
"""
from __future__ import annotations

import argparse
import time

import pathlib
import sys

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent))
from tbtk_b200 import kpm, workloads  # noqa: E402


def step_bytes(N, nnz, B, s_vec, s_val=16):
    return nnz * (s_val + 4) + 4 * (N + 1) + 3 * N * B * s_vec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", type=int, default=1024)
    ap.add_argument("--sites", type=int, default=64)
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_direct"], default="mixed")
    ap.add_argument("--moments", type=int, default=8)
    ap.add_argument("--energies", type=int, default=256)
    ap.add_argument("--rashba", type=float, default=0.0)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--sweep", action="store_true")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--config", default=None)
    ap.add_argument("--complex-vectors", action="store_true",
                    help="keep complex64 vectors for a real model (no real-vector kernels)")
    ap.add_argument("--batch-width", type=int, default=0,
                    help="sources per recursion batch (default 0: the library's choice)")
    ap.add_argument("--fp64-head", type=int, default=0,
                    help="FP64 head steps of doubling runs (default 0: every step of a "
                         "doubling run is a timed FP32 step, as without a head)")
    ap.add_argument("--grid", choices=["table", "clenshaw", "chebyshev"], default="table",
                    help="energy sums: lookup table or Clenshaw recurrences on the open "
                         "grid, or FFTs on the Chebyshev-node grid (--energies a power of two)")
    ap.add_argument("--server", type=int, default=0,
                    help="run the lattice as one server model with this many lanes")
    a = ap.parse_args()
    if a.server:
        return server_case(a)
    prec = {"fp64": kpm.FP64, "mixed": kpm.MIXED, "mixed_direct": kpm.MIXED_DIRECT}[a.precision]
    rowptr, col, val = workloads.square_csr(a.lattice, a.lattice, t=1.0, J=0.5, W=2.0,
                                            alpha=a.rashba, seed=a.lattice)
    N, nnz = rowptr.size - 1, int(rowptr[-1])
    sites = workloads.sample_sites(a.lattice * a.lattice, 2, a.sites, 1 + a.lattice)
    mat = kpm.Matrix.from_csr(rowptr, col, val, 12.0)
    if a.grid == "chebyshev":
        tab = kpm.Table.create_chebyshev(a.moments, a.energies, 12.0)
    elif a.grid == "clenshaw":
        tab = kpm.Table.create_clenshaw(a.moments, workloads.open_grid(12.0, a.energies), 12.0)
    else:
        tab = kpm.Table.create(a.moments, workloads.open_grid(12.0, a.energies), 12.0)
    mat.set_profiling(True)
    mat.set_fp64_head(a.fp64_head)
    if a.complex_vectors:
        mat.set_real(False)
    if a.batch_width:
        mat.set_batch_width(prec, a.batch_width)
    real = prec != kpm.FP64 and mat.real()[1]
    s_vec = 16 if prec == kpm.FP64 else (4 if real else 8)
    # a call runs its sites in batches of the handle's width, each batch the
    # same number of steps: the mean algorithmic bytes of one launch
    width = mat.batch_width(prec, ldos=True)
    batches = [min(width, a.sites - b0) for b0 in range(0, a.sites, width)]
    bstep = sum(step_bytes(N, nnz, b, s_vec, 8 if real else 16) for b in batches) / len(batches)

    def run(label):
        for _ in range(a.repeat):
            t0 = time.perf_counter()
            mat.ldos_sites(tab, sites, 1e-3, prec)
            wall = time.perf_counter() - t0
            rec, en, steps = mat.profile()
            ms = rec / max(steps, 1)
            print(f"{label} N={N} nnz={nnz} B={a.sites} {a.precision} M={a.moments}: "
                  f"recursion {rec:.3f} ms / {steps} steps = {ms:.4f} ms/step "
                  f"({bstep / ms / 1e6:.0f} GB/s algorithmic), energy {en:.3f} ms, "
                  f"wall {wall * 1e3:.1f} ms", flush=True)

    if a.config:
        t, v, mb = (int(x) for x in a.config.split(","))
        mat.set_config(a.sites, prec, t, v, mb)
    if a.autotune:
        t, v, mb, ms = mat.autotune(a.sites, prec, ldos=True, probe_steps=8)
        print(f"autotune: tpr={t} vpt={v} minb={mb} {ms:.4f} ms/step", flush=True)
    if a.sweep:
        for (t, v, mb) in mat.configs_for(a.sites, prec):
            mat.set_config(a.sites, prec, t, v, mb)
            mat.ldos_sites(tab, sites, 1e-3, prec)  # warm
            mat.profile()
            run(f"[tpr={t} vpt={v} minb={mb}]")
    else:
        run("")


def server_case(a):
    rowptr, col, val = workloads.square_csr(a.lattice, a.lattice, t=1.0, J=0.5, W=2.0,
                                            alpha=a.rashba, seed=a.lattice)
    N = rowptr.size - 1
    W = a.server
    sites = workloads.sample_sites(a.lattice * a.lattice, 2, W, 1 + a.lattice)
    real = a.rashba == 0.0 and not a.complex_vectors
    cfgs = kpm.Server.step_configs(W, real) if a.sweep else [None]
    for cfg in cfgs:
        srv = kpm.Server(a.moments, workloads.open_grid(12.0, a.energies), hbm_budget=64 << 30,
                         tick_steps=64, tolerance=0)
        srv.set_fp64_head(0)
        srv.set_real(real)
        mid = srv.add_model(rowptr, col, val, 12.0, W)
        if cfg is None and a.config:
            cfg = tuple(int(x) for x in a.config.split(","))
        if cfg is not None:
            srv.set_config(W, *cfg)
        for _ in range(a.repeat):
            srv.wait(srv.submit(mid, sites, a.moments, 1e-3))
        st = srv.stats()
        ms = st["step_s"] / max(st["steps"], 1) * 1e3
        print(f"[server W={W} config={cfg}] N={N} M={a.moments}: {st['steps']:.0f} steps, "
              f"{ms:.4f} ms/step ({st['step_bytes'] / max(st['step_s'], 1e-12) / 1e9:.0f} GB/s "
              f"algorithmic)", flush=True)
        srv.close()


if __name__ == "__main__":
    main()
