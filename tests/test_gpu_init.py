"""The device-built Voronoi polycrystal equals the host construction
(gpk_voronoi_init, itself following demos/gpk.cpp:51-189) cell for cell:
labels, orientations and the number of reattached tie cells."""
import ctypes as C

import numpy as np
import pytest

from gpk_b200 import GPKGrid, thermo
from gpk_b200._lib import lib

pytestmark = pytest.mark.gpu


def _host(nz, ny, nx, n, seed):
    phi = np.empty((nz, ny, nx), np.int32)
    g = np.empty((nz, ny, nx), np.float32)
    moved = C.c_int()
    assert lib().gpk_voronoi_init(nz, ny, nx, n, seed, phi.ctypes.data, g.ctypes.data, C.byref(moved)) == 0
    return phi, g, moved.value


@pytest.mark.parametrize("shape,n,seed", [
    ((1, 64, 64), 48, 3),
    ((1, 50, 70), 300, 4),        # small grains: many raster ties and fragments
    ((24, 24, 24), 500, 5),
    ((40, 32, 48), 60, 6),
    ((7, 9, 11), 40, 7),          # odd extents, grains of a few cells
])
def test_device_voronoi_equals_host(shape, n, seed):
    phi, g, moved = _host(*shape, n, seed)
    grid = GPKGrid(*shape, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    dmoved = grid.voronoi(n, seed)
    assert np.array_equal(grid.get("phi"), phi)
    assert np.array_equal(grid.get("g"), g)
    assert dmoved == moved
    assert grid.n_grains() == len(np.unique(phi))


def test_device_voronoi_f64_grid():
    phi, g, _ = _host(16, 20, 24, 30, 9)
    grid = GPKGrid(16, 20, 24, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5, precision="f64")
    grid.voronoi(30, 9)
    assert np.array_equal(grid.get("phi"), phi)
    assert np.array_equal(grid.get("g"), g.astype(np.float64))
