"""The tiled separable Gaussian passes (src/gpk_gaussian.cpp:9-72).

gpk_gaussian_filter_3d and the separable geometry path run one periodic 1-D
pass per axis (x, then y, then z); every output is acc = 0; acc += w[k] *
in[wrap(q + k - R)] for k = 0 .. 2R, a float multiply and a float add per
tap.  The restatement below does exactly that in numpy float32, so the device
result must match it bit for bit: on grids whose axes are shorter than the
radius (several wraps), on axes that are and are not multiples of the
128-cell tile, and for radii whose tiles need more than the default 48 KB of shared
memory or do not fit at all (the one-thread-per-output form).
"""
import numpy as np
import pytest

from gpk_b200 import GPKGrid, lib, thermo
from gpk_b200._lib import check

from _cases import compare_all, polycrystal, rel_close

pytestmark = pytest.mark.gpu


def _restated(field, taps, r):
    x = field.astype(np.float32)
    axes = (2, 1, 0) if field.shape[0] > 1 else (2, 1)
    for ax in axes:
        acc = np.zeros_like(x)
        for k in range(2 * r + 1):
            acc = acc + taps[k] * np.roll(x, -(k - r), axis=ax)
        x = acc
    return x


def _gauss_taps(sigma):
    r = int(np.ceil(3.5 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float32)
    w = np.exp(-x * x / np.float32(2 * sigma * sigma)).astype(np.float32)
    return (w / w.sum(dtype=np.float32)).astype(np.float32), r


def _filter(field, taps, r):
    out = np.empty_like(field)
    Nz, Ny, Nx = field.shape
    check(lib().gpk_gaussian_filter_3d(field.ctypes.data, out.ctypes.data, Nz, Ny, Nx, taps.ctypes.data, r))
    return out


@pytest.mark.parametrize("shape,sigma", [((1, 96, 80), 2.0), ((20, 24, 28), 1.5), ((40, 48, 128), 5.0),
                                         ((8, 6, 10), 6.0), ((3, 70, 130), 4.0)])
def test_filter_matches_float32_restatement(shape, sigma):
    rng = np.random.default_rng(11)
    field = rng.random(shape, dtype=np.float32)
    taps, r = _gauss_taps(sigma)
    assert np.array_equal(_filter(field, taps, r), _restated(field, taps, r))


@pytest.mark.parametrize("r", [300, 900])
def test_filter_wide_radii(r):
    """r = 300 needs the opt-in shared-memory size; r = 900 does not fit and
    takes the one-thread-per-output form."""
    rng = np.random.default_rng(r)
    field = rng.random((2, 5, 700), dtype=np.float32)
    w = rng.random(2 * r + 1).astype(np.float32)
    taps = (w / w.sum(dtype=np.float32)).astype(np.float32)
    assert np.array_equal(_filter(field, taps, r), _restated(field, taps, r))


def _pair(oracle_mod, shape, sigma, precision):
    th = thermo.isotropic(1.0, 1.0)
    return (GPKGrid(*shape, 1.0, th, 0.0, sigma, precision=precision),
            oracle_mod.OracleGrid(*shape, 1.0, th, 0.0, sigma, precision=precision))


@pytest.mark.parametrize("shape", [(40, 48, 128), (36, 30, 70)])
def test_separable_geometry_polycrystal_f32(oracle_mod, shape):
    """sigma 5 in 3-D: per-label smoothed indicators through the tiled passes
    (int4 label loads when x is a whole number of tiles), bit for bit."""
    phi, g = polycrystal(*shape, 6, 3)
    gpu, ora = _pair(oracle_mod, shape, 5.0, "f32")
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g)
        G.set("alpha", 1.0)
    for s in range(3):
        assert gpu.step() == ora.step(), s
        bad = compare_all(gpu, ora)
        assert not bad, (s, bad)


def test_separable_geometry_polycrystal_f64(oracle_mod):
    shape = (40, 48, 128)
    phi, g = polycrystal(*shape, 6, 4)
    gpu, ora = _pair(oracle_mod, shape, 5.0, "f64")
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g.astype(np.float64))
        G.set("alpha", 1.0)
    for s in range(3):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= 1e-10 * abs(do), s
        assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
        for f in ("kappa_f", "nx_f", "vn_f"):
            assert rel_close(gpu.get(f), ora.get(f), 1e-10), (s, f)


# velocity-projection radius ceil(3 clamp(0.375 sigma, 0.85, 3)): 4, 5, 8 — the
# tiled projection kernels beyond radius 3 (sigma 7 also takes the separable
# geometry).  Every extent is at least the Gaussian radius ceil(3.5 sigma):
# beyond it the reference's one-step wrap (src/gpk_gaussian.cpp:27, 42, 59)
# indexes outside the field, so it has no defined result to match.
@pytest.mark.parametrize("sigma,shape", [(3.0, (20, 22, 24)), (4.2, (20, 22, 24)), (7.0, (26, 28, 30))])
def test_projection_radii_f32(oracle_mod, sigma, shape):
    phi, g = polycrystal(*shape, 8, 5)
    gpu, ora = _pair(oracle_mod, shape, sigma, "f32")
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g)
        G.set("alpha", 1.0)
    for s in range(3):
        assert gpu.step() == ora.step(), s
        bad = compare_all(gpu, ora)
        assert not bad, (s, bad)
