"""Failure paths of the device side, tested without faulting a GPU.

The tile-staged recursion steps wait on mbarriers for rows that bulk copies
stage in shared memory; every wait is bounded.  A handle whose wait bound is
0 gives up at the first wait: the step leaves its loops, waits (with the
library's own bound) for the copies it already issued, sets the device
status word, and the call returns TBTKKPM_ERR_TIMEOUT.  The context and the
handle stay usable: with the default bound restored the same call gives the
same LDOS as a fresh handle.
"""
import numpy as np
import pytest

from conftest import rel_err
from tbtk_b200 import lattice as L

pytestmark = pytest.mark.gpu


def _tiled_config(m, B, gpu):
    for (t, v, mb) in m.configs_for(B, gpu.MIXED, ldos=True):
        if mb >= 100000:
            return t, v, mb
    return None


@pytest.mark.parametrize("alpha", [0.0, 0.3])
def test_staged_row_wait_runs_out(gpu, alpha):
    lat = L.square(24, 20, t=1.0, J=0.5, W=2.0, alpha=alpha, periodic=True, seed=5)
    rowptr, col, val = lat.csr()
    s, M, B = 12.0, 64, 64
    sites = L.random_sites(lat, B, seed=2)
    tab = gpu.Table.create(M, gpu.tbtk_range(-11.9, 11.9, 100), s)
    ref, _ = gpu.Matrix.from_csr(rowptr, col, val, s).ldos_sites(tab, sites, 1e-3, gpu.MIXED)
    m = gpu.Matrix.from_csr(rowptr, col, val, s)
    cfg = _tiled_config(m, B, gpu)
    assert cfg is not None
    m.set_config(B, gpu.MIXED, *cfg, ldos=True)
    m.set_fp64_head(0)
    m.set_wait_limit(0)
    with pytest.raises(gpu.TBTKError) as e:
        m.ldos_sites(tab, sites, 1e-3, gpu.MIXED)
    assert e.value.status == gpu.ERR_TIMEOUT
    assert "bounded wait" in str(e.value)
    # the handle and the context still work
    m.set_wait_limit()
    m.set_fp64_head()
    again, _ = m.ldos_sites(tab, sites, 1e-3, gpu.MIXED)
    assert rel_err(again, ref) <= 1e-7


def test_server_staged_row_wait_runs_out(gpu):
    """A server whose tile-staged steps give up every staged-row wait at
    once fails its requests with ERR_TIMEOUT, and the device still serves a
    new server's requests correctly."""
    from tbtk_b200 import workloads
    csr = workloads.square_csr(24, 24, J=0.5, W=2.0, seed=1)
    grid = workloads.open_grid(12.0, 100)
    cfg = next(c for c in gpu.Server.step_configs(16, True) if c[2] >= 100000)
    srv = gpu.Server(256, grid, hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    mid = srv.add_model(*csr, 12.0, 16)
    srv.set_config(16, *cfg)
    srv.set_fp64_head(0)
    srv.set_wait_limit(0)
    sites = np.arange(0, 160, 10, dtype=np.uint32)
    with pytest.raises(gpu.TBTKError) as e:
        srv.wait(srv.submit(mid, sites, 128, 1e-3))
    assert e.value.status == gpu.ERR_TIMEOUT
    srv.close()
    good = gpu.Server(256, grid, hbm_budget=1 << 30, tick_steps=8, tolerance=0)
    mid = good.add_model(*csr, 12.0, 16)
    good.set_config(16, *cfg)
    ldos, _, _ = good.wait(good.submit(mid, sites, 128, 1e-3))
    ref, _ = gpu.Matrix.from_csr(*csr, 12.0).ldos_sites(gpu.Table.create(128, grid, 12.0), sites,
                                                        1e-3, gpu.FP64)
    assert rel_err(ldos, ref) <= 1e-6
    good.close()
