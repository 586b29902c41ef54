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


@pytest.mark.parametrize("shape,n,seed", [
    ((1, 64, 64), 48, 3),
    ((20, 22, 18), 40, 7),         # one raster tie cell reattached
    ((1, 37, 53), 9, 1),
    ((32, 32, 32), 60, 5),
    ((9, 11, 13), 120, 8),
])
def test_device_voronoi_equals_reference_voronoi_init(oracle_mod, shape, n, seed):
    """Given the seeds the reference's voronoi_init draws (std::mt19937 and
    the libstdc++ distributions, demos/gpk.cpp:56-71), the device
    construction equals that function's polycrystal, labels and orientations,
    cell for cell (demos/gpk.cpp:73-189, compiled from the reference's
    source into oracle/_ref)."""
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built")
    seeds, sg = oracle_mod.ref_voronoi_seeds(*shape, n, seed)
    ref_phi, ref_g = oracle_mod.ref_voronoi(*shape, n, seed)
    grid = GPKGrid(*shape, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    grid.voronoi_seeds(seeds, sg)
    assert np.array_equal(grid.get("phi"), ref_phi)
    assert np.array_equal(grid.get("g").view(np.uint32), ref_g.view(np.uint32))


def test_device_voronoi_seeds_rejects_bad_lists():
    from gpk_b200 import GPKError
    grid = GPKGrid(1, 16, 16, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    with pytest.raises(GPKError):
        grid.voronoi_seeds(np.array([[0, 0], [3, 3], [4, 4]]), np.zeros(2, np.float32))   # same cell twice
    with pytest.raises(GPKError):
        grid.voronoi_seeds(np.array([[0], [16], [4]]), np.zeros(1, np.float32))           # outside the grid
