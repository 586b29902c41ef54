"""Solid/liquid diffusivity ratio of the partitioned solute transport.

The reference diffuses the liquid composition only, through the smaller
liquid fraction of a face (src/gpk_transport.cpp:102-135).  With a ratio
r = D_solid / D_liquid the solid composition k cL also diffuses, with r D,
through the face's shared solid fraction (face weight
min(l_i, l_j) + r k min(s_i, s_j)); r = 0 is the reference.  The device
step equals the oracle's restatement of the same rule bit for bit in FP32
and within 1e-10 in FP64; parity with the reference itself holds at r = 0
only, since the reference has no such ratio.
"""
import numpy as np
import pytest

from gpk_b200 import GPKGrid, thermo

from _cases import compare_all, rel_close

pytestmark = pytest.mark.gpu


def _case(oracle_mod, shape, ratio, precision):
    th = thermo.solidification(5e-8, 0.2, 0.0, -500.0, 0.14, 933.0, 1e8)
    th.solute_rejection, th.k_partition = True, 0.14
    gpu = GPKGrid(*shape, 0.5e-6, th, 3e-9, 1.5, precision=precision)
    ora = oracle_mod.OracleGrid(*shape, 0.5e-6, th, 3e-9, 1.5, precision=precision)
    Nz, Ny, Nx = shape
    zz, yy, xx = np.mgrid[0:Nz, 0:Ny, 0:Nx]
    nucleus = (zz - Nz // 2) ** 2 + (yy - Ny // 2) ** 2 + (xx - Nx // 2) ** 2 <= 25
    rd = np.float32 if precision == "f32" else np.float64
    rng = np.random.default_rng(5)
    c = (0.02 + 0.002 * rng.standard_normal(shape)).astype(rd)
    c[nucleus] *= rd(0.14)
    for G in (gpu, ora):
        G.set("phi", nucleus.astype(np.int32))
        G.set("c", c)
        G.set("T", rd(933.0) - rd(30.0))
        G.set("alpha", 1.0)
        G.set_solid_diffusivity_ratio(ratio)
    return gpu, ora


@pytest.mark.parametrize("shape", [(1, 64, 64), (32, 32, 32)])
@pytest.mark.parametrize("ratio", [1e-4, 0.3])
def test_solid_diffusion_fp32_bitexact(oracle_mod, shape, ratio):
    gpu, ora = _case(oracle_mod, shape, ratio, "f32")
    for s in range(15):
        assert gpu.step() == ora.step(), s
        bad = compare_all(gpu, ora, ["phi", "alpha", "c"])
        assert not bad, f"step {s}: {bad}"


def test_solid_diffusion_fp64_within_1e10(oracle_mod):
    gpu, ora = _case(oracle_mod, (24, 24, 24), 1e-4, "f64")
    for s in range(10):
        gpu.step(); ora.step()
        assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
        assert rel_close(gpu.get("c"), ora.get("c"), 1e-10), s


def test_solid_diffusion_ratio_changes_the_solid_only(oracle_mod):
    """The ratio moves solute inside the solid; a liquid-only field is
    unchanged by it, and the ratio is validated."""
    from gpk_b200 import GPKError
    a, _ = _case(oracle_mod, (1, 48, 48), 0.0, "f32")
    b, _ = _case(oracle_mod, (1, 48, 48), 0.5, "f32")
    for _ in range(5):
        a.step(); b.step()
    solid = a.get("phi") != 0
    assert not np.array_equal(a.get("c")[solid], b.get("c")[solid])
    assert abs(float(a.get("c").sum(dtype=np.float64)) - float(b.get("c").sum(dtype=np.float64))) < 1e-5
    with pytest.raises(GPKError):
        a.set_solid_diffusivity_ratio(1.5)
