"""Parity at the benchmark's own sizes against the CPU oracle.

The oracle restates calculateCoefficientsCPU
(Lib/src/Solver/ChebyshevExpander.cpp:103-199) and is bit-identical to the
reference on the golden models; here it runs on the full lattices at a
truncated coefficient count (M = 48), four sites at a time in threads.

* 2048x2048 periodic square lattice with spin (N = 8,388,608, the
  benchmark's workload): FP64 moments of the batched recursion equal the
  oracle's bit for bit; the mixed-precision moments (complex64 storage, FP64
  arithmetic; real float vectors for this real model) are within 2e-6
  (max|mu - mu_ref| / max|mu_ref|), for the library's default step and for
  the configuration the autotuner picks.
* 1024x1024 Rashba lattice (N = 2,097,152, complex Hamiltonian, 9 entries
  per row): the same, with 256 sources in batches of 128 (the default of
  doubling calls) and in one batch of 256.
* The doubling LDOS of both (the benchmark's MIXED path, FP64 head on) stay
  within 1e-6 of the FP64 recursion's LDOS of the same sites.
"""
import threading

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

M_TRUNC = 48


def _oracle_moments(oracle, p, sites, M):
    out = [None] * len(sites)

    def work(i):
        out[i] = oracle.moments(p.rowptr, p.col, p.val, p.scale, M, int(sites[i]),
                                [int(sites[i])])[0]

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(sites))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return out


def _check(gpu, oracle, p, B, widths):
    sites = p.sites[:B]
    check = np.linspace(0, B - 1, 4).astype(int)
    ref = _oracle_moments(oracle, p, sites[check], M_TRUNC)
    owner = np.arange(B)
    for width in widths:
        m = gpu.Matrix.from_csr(p.rowptr, p.col, p.val, p.scale)
        m.set_batch_width(gpu.MIXED, width)
        fp, _ = m.moments_batched(sites, sites, owner, M_TRUNC, 0.0, gpu.FP64)
        for j, k in enumerate(check):
            assert np.array_equal(fp[k], ref[j]), (width, k)
        mixed, _ = m.moments_batched(sites, sites, owner, M_TRUNC, 0.0, gpu.MIXED)
        for j, k in enumerate(check):
            assert rel_err(mixed[k], ref[j]) <= 2e-6, (width, k, rel_err(mixed[k], ref[j]))
        t, v, mb, _ = m.autotune(min(width, B), gpu.MIXED, ldos=False, probe_steps=4)
        tuned, _ = m.moments_batched(sites, sites, owner, M_TRUNC, 0.0, gpu.MIXED)
        for j, k in enumerate(check):
            assert rel_err(tuned[k], ref[j]) <= 2e-6, (width, t, v, mb, k)
        # the same arithmetic in every configuration: tuned == default
        assert np.array_equal(tuned, mixed), (width, t, v, mb)


def _check_ldos(gpu, p, B):
    sites = p.sites[:B]
    m = gpu.Matrix.from_csr(p.rowptr, p.col, p.val, p.scale)
    tab = gpu.Table.create(2 * M_TRUNC, p.energies, p.scale)
    fp64, _ = m.ldos_sites(tab, sites, p.broadening, gpu.FP64)
    mixed, est = m.ldos_sites(tab, sites, p.broadening, gpu.MIXED)
    errs = [rel_err(mixed[k], fp64[k]) for k in range(B)]
    assert max(errs) <= 1e-6, max(errs)
    assert np.all(est >= 0)


def test_cfg2_full_lattice_against_oracle(gpu, oracle):
    from tbtk_b200 import workloads
    p = workloads.cfg2(n_sites=64)
    _check(gpu, oracle, p, 64, [64])
    _check_ldos(gpu, p, 64)


def test_cfg3_full_lattice_against_oracle(gpu, oracle):
    from tbtk_b200 import workloads
    p = workloads.cfg3(n_sites=256)
    _check(gpu, oracle, p, 256, [128, 256])
    _check_ldos(gpu, p, 256)
