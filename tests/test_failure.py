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
