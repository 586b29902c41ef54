"""The CUDA spectral-elasticity solve (cuFFT + hand-written kernels) against
the reference's outputs and the oracle.

Tolerance: every output field within 1e-10 of the reference's largest
magnitude of that field (FP64 throughout; the transforms differ from
NumPy/SciPy's in rounding only), and the equilibrium residual below 1e-12
(the reference's own audit demands 1e-10).
"""
import types

import numpy as np
import pytest

from gpk import GPKError, SpectralElasticity, spectral_elasticity
from gpk.spectral import variant_eigenstrains
from oracle import spectral_oracle

from test_spectral_oracle import golden_cases, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _check(got, ref):
    d, e, h, r = got
    assert rel_err(d, ref["driving"]) < TOL
    assert rel_err(e, ref["energy"]) < TOL
    assert rel_err(h, ref["hydro"]) < TOL
    assert r < 1e-12


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0])
def test_gpu_matches_reference_outputs(case):
    name, vf, p, ref = case
    _check(spectral_elasticity(vf, p), ref)


def _plates(shape, seed, n_plates=6):
    rng = np.random.default_rng(seed)
    vf = np.zeros((3,) + shape)
    grids = np.indices(shape)
    for k in range(n_plates):
        v = k % 3
        c = [rng.integers(0, n) for n in shape]
        half = [int(rng.integers(2, max(3, n // 4))) for n in shape]
        half[v % len(shape)] = 1
        box = np.ones(shape, dtype=bool)
        for a, n in enumerate(shape):
            box &= np.abs((grids[a] - c[a] + n // 2) % n - n // 2) <= half[a]
        vf[v][box] = 1.0
    return vf


ALCU = types.SimpleNamespace(dx=1.5e-9, c11=107.07e9, c12=63.08e9, c44=28.52e9, eigen_small=0.00746,
                             eigen_large=-0.051)


@pytest.mark.parametrize("shape", [(512, 512), (64, 48, 40), (33, 31, 29)])
def test_gpu_matches_oracle_larger(shape):
    vf = _plates(shape, 7)
    d, e, h, r = spectral_oracle.spectral_elasticity(vf, ALCU)
    _check(spectral_elasticity(vf, ALCU), {"driving": d, "energy": e, "hydro": h})


def test_gpu_dilatational_sphere_128():
    """The 128^3 dilatational-misfit case (cubic 108/62/28 GPa, 0.5% misfit,
    nucleus radius 4) against the oracle, and the sphere's compressive core."""
    n = 128
    g = np.indices((n, n, n), dtype=np.int32) - n // 2
    inside = (g ** 2).sum(0) <= 16
    vf = np.zeros((3, n, n, n))
    vf[0][inside] = 1.0
    p = types.SimpleNamespace(dx=1.0, c11=108e9, c12=62e9, c44=28e9, eigen_small=0.005, eigen_large=0.005)
    got = spectral_elasticity(vf, p)
    d, e, h, r = spectral_oracle.spectral_elasticity(vf, p)
    _check(got, {"driving": d, "energy": e, "hydro": h})
    assert np.all(got[2][inside] < 0)


def test_device_path_equals_host_path_and_is_deterministic():
    torch = pytest.importorskip("torch")
    shape = (40, 36, 32)
    vf = _plates(shape, 3)
    s = SpectralElasticity(shape, ALCU.dx, ALCU.c11, ALCU.c12, ALCU.c44,
                           variant_eigenstrains(ALCU.eigen_small, ALCU.eigen_large))
    host = s.solve(vf)
    t = torch.from_numpy(vf).cuda()
    dev1 = s.solve(t)
    dev2 = s.solve(t)
    torch.cuda.synchronize()
    for a, b, c in zip(host[:3], dev1[:3], dev2[:3]):
        assert np.array_equal(a, b.cpu().numpy())
        assert np.array_equal(a, c.cpu().numpy())
    assert host[3] == dev1[3] == dev2[3]
    s.close()


def test_invalid_arguments():
    with pytest.raises(ValueError):
        SpectralElasticity((4,), 1.0, 1.0, 0.5, 0.3, np.eye(3))
    with pytest.raises(GPKError):
        SpectralElasticity((4, 0), 1.0, 1.0, 0.5, 0.3, np.eye(3))
    with pytest.raises(GPKError):
        SpectralElasticity((4, 4), -1.0, 1.0, 0.5, 0.3, np.eye(3))
    s = SpectralElasticity((8, 8), 1.0, 1.0, 0.5, 0.3, np.eye(3))
    with pytest.raises(ValueError):
        s.solve(np.zeros((3, 8, 9)))


@pytest.mark.gpu
def test_gpu_on_the_reference_trajectory():
    """The driver's own spectral solves of a 64^2 Al-Cu run (variant
    fractions of the evolving precipitates, tests/golden/alcu_trajectory.npz),
    through the device solve, every field within 1e-10."""
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import alcu_replay as R
    from gpk import spectral_elasticity as gpu_spectral

    for vf, p, ref, res in R.spectral_cases():
        d, e, h, r = gpu_spectral(vf, p)
        assert R.rel_err(d, ref["driving"]) < TOL and R.rel_err(e, ref["energy"]) < TOL
        assert R.rel_err(h, ref["hydro"]) < TOL and abs(r - res) < 1e-12
