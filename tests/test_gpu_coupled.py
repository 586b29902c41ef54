"""Spectral elasticity coupled into the step (external elastic energy).

The coupled path (gpk_spectral_couple_grid + gpk_grid_set_external_elastic)
must equal, bit for bit, the same composition done by hand through host
copies: solid indicator -> spectral solve -> E_el upload -> step.  With a
zero elastic energy the external mode must leave the step unchanged.
"""
import numpy as np
import pytest

from gpk import GPKGrid, SpectralElasticity, thermo
from gpk.spectral import variant_eigenstrains

from _cases import PUBLIC_FIELDS

pytestmark = pytest.mark.gpu
N = 24
CUBIC = (108e9, 62e9, 28e9)


def _solid_seed(n, r=4, prec="f64", k_part=0.14):
    th = thermo.solidification(M0=5e-8, sigma0=0.2, eps4=0.04, m_liq=-500.0, k_part=k_part, T_melt=933.0, L=1e8)
    th.solute_rejection = True
    g = GPKGrid(n, n, n, 0.5e-6, th, 3e-9, 1.5, precision=prec)
    z, y, x = np.indices((n, n, n)) - n // 2
    g.set("phi", ((x * x + y * y + z * z) <= r * r).astype(np.int32))
    g.set("c", 0.02)
    g.set("T", 933.0 - 5.0)
    return g


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_coupled_step_equals_manual_composition(prec):
    a, b = _solid_seed(N, prec=prec), _solid_seed(N, prec=prec)
    for g in (a, b):
        g.set_external_elastic(True)
    eig = variant_eigenstrains(0.005, 0.005)
    sa = SpectralElasticity((N, N, N), 0.5e-6, *CUBIC, eig)
    sb = SpectralElasticity((N, N, N), 0.5e-6, *CUBIC, eig)
    for _ in range(6):
        r = sa.couple(a, want_residual=True)
        assert r < 1e-12
        a.step()
        f = np.zeros((3, N, N, N))
        f[0] = (b.get("phi")[...] != 0).astype(np.float64)
        _, energy, _, _ = sb.solve(f)
        b.set("E_el", energy)
        b.step()
    for name in PUBLIC_FIELDS:
        x, y = a.get(name), b.get(name)
        assert np.array_equal(x, y), name
    assert a.get("E_el").max() > 0


def test_zero_external_energy_changes_nothing():
    a, b = _solid_seed(N), _solid_seed(N)
    a.set_external_elastic(True)
    a.set("E_el", 0.0)
    for _ in range(6):
        a.step()
        b.step()
    for name in ("phi", "alpha", "c", "vn_f"):
        assert np.array_equal(a.get(name), b.get(name)), name
