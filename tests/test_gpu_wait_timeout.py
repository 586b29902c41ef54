"""A bounded device wait that runs out returns GPK_ERR_TIMEOUT.

The ordered crossing sweep and the remap exchange loops are persistent
cooperative kernels whose blocks meet at grid barriers; every barrier wait
is bounded and, when the bound is reached, records GPK_ERR_TIMEOUT and
leaves the kernel.  gpk_grid_inject_wait_timeout makes the next such
barrier wait for a block that was never launched (a flag nothing sets) with
a short bound: the step must fail with the timeout status, promptly, and the
CUDA context must stay usable — a fresh grid afterwards steps bit for bit
like the oracle.  No GPU fault is involved: the wait simply gives up.
"""
import time

import numpy as np
import pytest

from gpk_b200 import GPKError, GPKGrid, thermo
from gpk_b200._lib import check, lib

from _cases import compare_all

pytestmark = pytest.mark.gpu


def test_injected_barrier_wait_times_out(oracle_mod):
    phi, g = oracle_mod.voronoi(1, 96, 96, 30, 7)
    grid = GPKGrid(1, 96, 96, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    grid.set("phi", phi)
    grid.set("g", g)
    grid.set("alpha", 1.0)
    check(lib().gpk_grid_inject_wait_timeout(grid._h, 1 << 14))
    err = None
    t0 = time.perf_counter()
    for _ in range(60):   # the knob is consumed by the first step with crossing candidates
        try:
            grid.step()
        except GPKError as e:
            err = e
            break
    elapsed = time.perf_counter() - t0
    assert err is not None and err.code == 6, err      # GPK_ERR_TIMEOUT
    assert "bounded device wait" in str(err)
    assert elapsed < 30.0
    with pytest.raises(GPKError):
        grid.step()          # the grid keeps reporting its failure
    grid.close()
    # the context is intact: a new grid matches the oracle step for step
    fresh = GPKGrid(1, 96, 96, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    ora = oracle_mod.OracleGrid(1, 96, 96, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    for G in (fresh, ora):
        G.set("phi", phi)
        G.set("g", g)
        G.set("alpha", 1.0)
    for s in range(20):
        assert fresh.step() == ora.step(), s
    assert not compare_all(fresh, ora, ["phi", "alpha", "phi_comp"])


def test_inject_wait_timeout_validates_its_limit():
    grid = GPKGrid(1, 16, 16, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    assert lib().gpk_grid_inject_wait_timeout(grid._h, 0) == 1
    assert lib().gpk_grid_inject_wait_timeout(grid._h, (1 << 24) + 1) == 1
