"""The oracle's Voronoi construction (oracle/voronoi_oracle.c) pinned two
ways on the CPU: against the reference driver's own voronoi_init
(demos/gpk.cpp:51-189, compiled from its source into oracle/_ref) on the
seeds that function draws, and against the library's host construction
gpk_voronoi_init for the library's seed stream.  The benchmark's reference
arm builds its input with this oracle, so that it never loads the library."""
import numpy as np
import pytest

from gpk_b200.grid import voronoi as lib_voronoi


@pytest.mark.parametrize("shape,n,seed", [
    ((1, 64, 64), 12, 3), ((20, 22, 18), 40, 7), ((1, 37, 53), 9, 1), ((32, 32, 32), 60, 5),
    ((9, 11, 13), 120, 8), ((1, 5, 7), 35, 2),     # every cell a seed
])
def test_oracle_voronoi_equals_reference(oracle_mod, shape, n, seed):
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built")
    seeds, sg = oracle_mod.ref_voronoi_seeds(*shape, n, seed)
    phi, g, _ = oracle_mod.voronoi_from_seeds(shape, seeds, sg)
    ref_phi, ref_g = oracle_mod.ref_voronoi(*shape, n, seed)
    assert np.array_equal(phi, ref_phi)
    assert np.array_equal(g.view(np.uint32), ref_g.view(np.uint32))


@pytest.mark.parametrize("shape,n,seed", [
    ((1, 64, 64), 12, 3), ((20, 22, 18), 40, 7), ((16, 16, 16), 1, 5), ((7, 9, 11), 200, 2),
    ((64, 64, 64), 300, 11), ((1, 256, 256), 128, 42), ((1, 50, 70), 300, 4),
])
def test_oracle_voronoi_equals_library_host_construction(oracle_mod, shape, n, seed):
    phi, g = oracle_mod.voronoi(*shape, n, seed)
    lphi, lg = lib_voronoi(*shape, n, seed)
    assert np.array_equal(phi, lphi)
    assert np.array_equal(g.view(np.uint32), lg.view(np.uint32))


def test_oracle_voronoi_rejects_bad_arguments(oracle_mod):
    with pytest.raises(ValueError):
        oracle_mod.voronoi(1, 4, 4, 17, 1)
    with pytest.raises(ValueError):
        oracle_mod.voronoi_from_seeds((1, 4, 4), np.array([[0], [4], [0]]), np.zeros(1, np.float32))
