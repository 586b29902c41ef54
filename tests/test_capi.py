"""Host-side checks of the C ABI library (no GPU needed).

The library must load, export every entry point declared in include/*.h, lay
out gpk_thermo_desc exactly as the header does, refuse to run without a
B200, and produce valid initial conditions.
"""
import ctypes as C

import numpy as np
import pytest

from gpk_b200 import GPKError, lib, thermo, voronoi
from gpk_b200._lib import exported_symbols
from gpk_b200.thermo import CThermoDesc


def test_library_exports_every_declared_symbol():
    L = lib()
    names = exported_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_thermo_desc_layout_matches_header():
    d = CThermoDesc()
    lib().gpk_thermo_desc_init(C.byref(d), 3)
    assert d.model == 3
    assert d.sigma0 == pytest.approx(0.5) and d.M0 == pytest.approx(1e-8)
    assert d.Rgas == pytest.approx(8.314) and d.kB == pytest.approx(1.380649e-23)
    assert d.k_partition == 1.0 and d.elastic_smooth_iters == 8 and d.noise_scale == 1.0
    assert C.sizeof(CThermoDesc) == 9 * 4 + 20 * 4 + 40 * 4


def test_thermo_factories_mirror_reference_constructors():
    iso = thermo.isotropic(2.0, 0.7)
    assert iso.grain_network and iso.eps4 == 0.0 and iso.model == "isotropic"
    dis = thermo.dislocation(1e-10, 0.5, 4e10, 2.5e-10, 0.5, 0.1, 1e12)
    f = np.float32
    assert np.float32(dis.disloc_coeff) == f(f(f(f(0.5) * f(0.5)) * f(4e10)) * f(2.5e-10)) * f(2.5e-10)
    pre = thermo.precipitation(1e-9, 0.3, 3, [1, 2, 3], [4, 5, 6], [7, 8, 9], [0, 0, 1])
    assert pre.phase_selection and pre.p[0] == 3 and pre.p[2 + 2] == 3 and pre.p[26 + 2] == 1
    with pytest.raises(ValueError):
        thermo.precipitation(1e-9, 0.3, 2, [1], [1], [1], [1])


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly():
    from gpk_b200 import GPKGrid
    with pytest.raises(GPKError) as e:
        GPKGrid(1, 8, 8, 1.0, thermo.isotropic(1.0))
    assert e.value.code == 7


def _components(phi):
    """Face-connected periodic components per label (BFS)."""
    Nz, Ny, Nx = phi.shape
    seen = np.zeros(phi.shape, bool)
    comps = {}
    for start in zip(*np.nonzero(np.ones_like(phi))):
        if seen[start]:
            continue
        lab = phi[start]
        comps[lab] = comps.get(lab, 0) + 1
        stack = [start]
        seen[start] = True
        while stack:
            z, y, x = stack.pop()
            nb = [(z, y, (x + 1) % Nx), (z, y, (x - 1) % Nx), (z, (y + 1) % Ny, x), (z, (y - 1) % Ny, x)]
            if Nz > 1:
                nb += [((z + 1) % Nz, y, x), ((z - 1) % Nz, y, x)]
            for n in nb:
                if not seen[n] and phi[n] == lab:
                    seen[n] = True
                    stack.append(n)
    return comps


@pytest.mark.parametrize("shape,n", [((1, 48, 40), 12), ((10, 12, 14), 9)])
def test_voronoi_initial_state(shape, n):
    phi, g = voronoi(*shape, n, 11)
    phi2, g2 = voronoi(*shape, n, 11)
    assert np.array_equal(phi, phi2) and np.array_equal(g, g2)
    assert sorted(np.unique(phi)) == list(range(1, n + 1))
    # every grain is one face-connected component (demos/gpk.cpp:100-185)
    assert all(v == 1 for v in _components(phi).values())
    assert np.all((g >= 0) & (g < np.pi / 2))
    # orientation is constant per grain
    for lab in range(1, n + 1):
        assert np.unique(g[phi == lab]).size == 1
