"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

In the reference's FP32 arithmetic every public field must be bit-identical
to the oracle after every step (the oracle is itself pinned bit-exact to the
reference and to its golden vectors).  Constitutive laws that call
transcendental functions (cos/sin/atan2/log/exp of per-cell values) cannot be
bit-exact across libm implementations; for those the fields agree to 1e-5
relative and the labels are compared.
"""
import os

import numpy as np
import pytest

from gpk_b200 import GPKGrid, thermo

from _cases import (PUBLIC_FIELDS, bits_equal, compare_all, neutral, polycrystal, rel_close,
                    topology_cases)

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _pair(oracle_mod, shape, dx, th, D, sigma, precision="f32"):
    g = GPKGrid(*shape, dx, th, D, sigma, precision=precision)
    o = oracle_mod.OracleGrid(*shape, dx, th, D, sigma, precision=precision)
    return g, o


def _load(grids, **fields):
    for G in grids:
        for k, v in fields.items():
            G.set(k, v)


def _lockstep(gpu, ora, steps, fields=PUBLIC_FIELDS, check_every=1, dt=-1.0):
    for s in range(steps):
        dg = gpu.step(dt)
        do = ora.step(dt)
        assert dg == do, f"step {s}: dt gpu={dg!r} oracle={do!r}"
        if (s + 1) % check_every == 0 or s == steps - 1:
            bad = compare_all(gpu, ora, fields)
            assert not bad, f"step {s}: {bad}"
            assert gpu.counters() == ora.counters(), f"step {s}: {gpu.counters()} vs {ora.counters()}"


def test_polycrystal_2d_bitexact(oracle_mod):
    phi, g = polycrystal(1, 128, 128, 48, 5)
    gpu, ora = _pair(oracle_mod, (1, 128, 128), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    _lockstep(gpu, ora, 60)


def test_polycrystal_3d_bitexact(oracle_mod):
    phi, g = polycrystal(28, 28, 28, 24, 9)
    gpu, ora = _pair(oracle_mod, (28, 28, 28), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    _lockstep(gpu, ora, 10)


# sigma 0.5 / 1.0 / 1.5 / 2.0 / 2.2 give geometry radii 4 / 6 / 8 / 9 / 10
@pytest.mark.parametrize("sigma", [0.5, 1.0, 1.5, 2.0, 2.2])
def test_geometry_kernels_agree_3d(oracle_mod, sigma):
    """Tiled (one and many bitmap batches; pair-bitmap and pair-compare
    projection) and per-cell kernels give the oracle's fields bit for bit."""
    phi, g = polycrystal(24, 30, 36, 20, 12)
    ora = oracle_mod.OracleGrid(24, 30, 36, 1.0, thermo.isotropic(1.0, 1.0), 0.0, sigma)
    _load((ora,), phi=phi, g=g, alpha=1.0)
    for _ in range(10):
        ora.step()
    for kind in ("tiled", "per_cell", "tiled_batched", "tiled_exact_scores"):
        gpu = GPKGrid(24, 30, 36, 1.0, thermo.isotropic(1.0, 1.0), 0.0, sigma)
        gpu.set_geometry_kernel(kind)
        _load((gpu,), phi=phi, g=g, alpha=1.0)
        for _ in range(10):
            gpu.step()
        assert not compare_all(gpu, ora), kind


@pytest.mark.parametrize("sigma", [0.5, 1.5, 2.2])
def test_geometry_kernels_agree_2d(oracle_mod, sigma):
    """2-D tiles (TX = 32 - 2R, 1024 / TX rows) on a grid that no tile
    width divides, against the oracle."""
    phi, g = polycrystal(1, 70, 90, 40, 5)
    ora = oracle_mod.OracleGrid(1, 70, 90, 1.0, thermo.isotropic(1.0, 1.0), 0.0, sigma)
    _load((ora,), phi=phi, g=g, alpha=1.0)
    for _ in range(10):
        ora.step()
    for kind in ("tiled", "tiled_batched", "tiled_exact_scores"):
        gpu = GPKGrid(1, 70, 90, 1.0, thermo.isotropic(1.0, 1.0), 0.0, sigma)
        gpu.set_geometry_kernel(kind)
        _load((gpu,), phi=phi, g=g, alpha=1.0)
        for _ in range(10):
            gpu.step()
        assert not compare_all(gpu, ora), kind


@pytest.mark.parametrize("shape,grains", [((40, 44, 36), 120), ((1, 160, 150), 90)])
def test_remap_screening_equals_exact_scores(oracle_mod, shape, grains):
    """The remap scores settle most cells from bitmap row sums and sum the
    rest tap by tap; every field equals the all-tap-by-tap kernel's and the
    oracle's after each step, through many remap exchanges."""
    phi, g = oracle_mod.voronoi(*shape, grains, 21)
    iso = thermo.isotropic(1.0, 1.0)
    a = GPKGrid(*shape, 1.0, iso, 0.0, 1.5)
    b = GPKGrid(*shape, 1.0, iso, 0.0, 1.5)
    b.set_geometry_kernel("tiled_exact_scores")
    ora = oracle_mod.OracleGrid(*shape, 1.0, iso, 0.0, 1.5)
    _load((a, b, ora), phi=phi, g=g, alpha=1.0)
    exchanges = 0
    for s in range(24):
        da, db, do = a.step(), b.step(), ora.step()
        assert da == db == do, s
        assert not compare_all(a, b), s
        assert not compare_all(a, ora, ["phi", "alpha", "phi_comp", "g"]), s
        exchanges += a.counters()[2]
    if shape[0] > 1:
        assert exchanges > 0   # the 3-D case runs both remap passes with exchanges


@pytest.mark.parametrize("shape", [(12, 20, 40), (1, 48, 64)])
def test_projection_many_pairs_per_tile(oracle_mod, shape):
    """Label noise: nearly every cell is an interface cell and a projection
    tile holds far more than the 64 label pairs its slot table takes (those
    tiles sum from global memory); two steps against the oracle and the
    pair-compare kernel, every public field bit for bit."""
    rng = np.random.default_rng(3)
    phi = rng.integers(0, 400, size=shape).astype(np.int32)
    iso = thermo.isotropic(1.0, 1.0)
    a = GPKGrid(*shape, 1.0, iso, 0.0, 1.5)
    b = GPKGrid(*shape, 1.0, iso, 0.0, 1.5)
    b.set_geometry_kernel("tiled_exact_scores")
    ora = oracle_mod.OracleGrid(*shape, 1.0, iso, 0.0, 1.5)
    _load((a, b, ora), phi=phi, g=0.0, alpha=1.0)
    for s in range(2):
        da, db, do = a.step(), b.step(), ora.step()
        assert da == db == do, s
        assert not compare_all(a, b), s
        assert not compare_all(a, ora), s


@pytest.mark.parametrize("divisor", [2, 4])
def test_geometry_tile_heights_2d(oracle_mod, divisor):
    """The 2-D tiles of 512 and 256 cells at sigma 1.5 (kernel radius 8),
    the shapes the sweep's autotuner chooses among, against the oracle."""
    phi, g = polycrystal(1, 70, 90, 40, 5)
    ora = oracle_mod.OracleGrid(1, 70, 90, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    gpu = GPKGrid(1, 70, 90, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    gpu.set_tile_rows(divisor)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    for _ in range(10):
        assert gpu.step() == ora.step()
    assert not compare_all(gpu, ora)


def test_config1_256_128_grains_200_steps(oracle_mod):
    """The CPU-runnable configuration: 256^2, 128 grains, sigma 1.5, 200 steps."""
    phi, g = polycrystal(1, 256, 256, 128, 42)
    gpu, ora = _pair(oracle_mod, (1, 256, 256), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    _lockstep(gpu, ora, 200, fields=["phi", "alpha", "g", "kappa_f", "vn_f", "phi_comp", "mask"], check_every=20)


@pytest.mark.parametrize("key", ["g13", "g14", "g15"])
def test_golden_curved_bicrystals(key):
    gd = np.load(os.path.join(GOLDEN, "curved_bicrystals_360.npz"))
    gpu = GPKGrid(1, 360, 360, 0.1e-6, thermo.isotropic(1e-8, 0.324), 0.0, 2.0)
    gpu.set("phi", gd[key + "_before"].astype(np.int32)[None])
    gpu.set("alpha", 1.0)
    gpu.step_n(800)
    assert np.array_equal(gpu.get("phi")[0], gd[key + "_after"].astype(np.int32))


def test_golden_rex_snapshots():
    rx = np.load(os.path.join(GOLDEN, "rex_192_snapshots.npz"))
    gpu = GPKGrid(1, 192, 192, 1e-6, thermo.recrystallisation(1e-12, 0.3, 1e6), 0.0, 2.0)
    gpu.set("phi", rx["phi"][0].astype(np.int32)[None])
    gpu.set("alpha", 1.0)
    for snap in range(1, len(rx["phi"])):
        while gpu.time < 44.0 / 24 * snap:
            gpu.step(-1.0)
        assert np.array_equal(gpu.get("phi")[0], rx["phi"][snap].astype(np.int32)), snap
        a = np.array([round(float("%.6f" % v) * 1e6) for v in gpu.get("alpha").ravel()])
        assert np.array_equal(a, rx["alpha_micro"][snap].ravel()), snap
        assert "%g" % gpu.time == str(rx["time_str"][snap])


@pytest.mark.parametrize("name,phi,cell,new,expected", topology_cases(), ids=[c[0] for c in topology_cases()])
def test_topology_known_answers(name, phi, cell, new, expected):
    gpu = GPKGrid(*phi.shape, 1.0, neutral())
    gpu.set("phi", phi)
    Nz, Ny, Nx = phi.shape
    assert gpu.topology_simple_move((cell[0] * Ny + cell[1]) * Nx + cell[2], new) == expected


def _solidification_case(oracle_mod, eps4, k, D, shape=(1, 64, 64), precision="f32"):
    th = thermo.solidification(5e-8, 0.2, eps4, -500.0, k, 933.0, 1e8)
    th.solute_rejection, th.k_partition = k < 1.0, k
    gpu, ora = _pair(oracle_mod, shape, 0.5e-6, th, D, 2.0, precision)
    Nz, Ny, Nx = shape
    zz, yy, xx = np.mgrid[0:Nz, 0:Ny, 0:Nx]
    seed = (zz - Nz // 2) ** 2 + (yy - Ny // 2) ** 2 + (xx - Nx // 2) ** 2 <= 16
    phi = np.zeros(shape, np.int32); phi[seed] = 1
    rd = np.float32 if precision == "f32" else np.float64
    c = np.full(shape, rd(0.02)); c[seed] = rd(0.02) * rd(k)
    T = rd(933.0) + rd(-500.0) * rd(0.02) - rd(5.0)
    _load((gpu, ora), phi=phi, c=c, T=T, alpha=1.0)
    return gpu, ora


def test_solidification_partitioned_bitexact(oracle_mod):
    gpu, ora = _solidification_case(oracle_mod, 0.0, 0.14, 3e-9)
    _lockstep(gpu, ora, 40)


def test_solidification_partitioned_3d_bitexact(oracle_mod):
    gpu, ora = _solidification_case(oracle_mod, 0.0, 0.14, 3e-9, shape=(24, 24, 24))
    _lockstep(gpu, ora, 12)


def test_anisotropic_solidification_close(oracle_mod):
    """eps4 != 0 evaluates cos/sin/atan2 per cell: fields within 1e-5."""
    gpu, ora = _solidification_case(oracle_mod, 0.04, 0.3, 3e-9)
    for _ in range(20):
        gpu.step(); ora.step()
    assert np.array_equal(gpu.get("phi"), ora.get("phi"))
    for f in ("c", "kappa_f", "alpha"):
        np.testing.assert_allclose(gpu.get(f), ora.get(f), rtol=1e-5, atol=1e-9)


def test_ostwald_diffusion_bitexact(oracle_mod):
    th = thermo.ostwald(1e-12, 0.3, 0.15, 5e8)
    Ny = Nx = 64
    gpu, ora = _pair(oracle_mod, (1, Ny, Nx), 1e-6, th, 1e-10, 2.0)
    yy, xx = np.mgrid[0:Ny, 0:Nx]
    phi = np.zeros((1, Ny, Nx), np.int32)
    for k, (cy, cx, r) in enumerate([(16, 16, 6), (44, 40, 9), (20, 48, 4)]):
        phi[0][(yy - cy) ** 2 + (xx - cx) ** 2 <= r * r] = k + 1
    rng = np.random.default_rng(1)
    c = (np.where(phi > 0, 0.9, 0.16) + rng.normal(0, 1e-3, phi.shape)).astype(np.float32)
    _load((gpu, ora), phi=phi, c=c, alpha=1.0)
    _lockstep(gpu, ora, 30)


def test_precipitation_phase_selection_bitexact(oracle_mod):
    th = thermo.precipitation(1e-12, 0.3, 3, [0.0, 1e7, 2e7], [0.0, -1e8, -2.5e8], [0.0, 0.0, 0.0],
                              [0.0, 0.0, 0.0], 900.0)
    Ny = Nx = 48
    gpu, ora = _pair(oracle_mod, (1, Ny, Nx), 1e-6, th, 1e-10, 2.0)
    yy, xx = np.mgrid[0:Ny, 0:Nx]
    phi = np.zeros((1, Ny, Nx), np.int32)
    phi[0][(yy - 24) ** 2 + (xx - 14) ** 2 <= 25] = 1
    phi[0][(yy - 24) ** 2 + (xx - 34) ** 2 <= 25] = 2
    c = np.full((1, Ny, Nx), 0.12, np.float32)
    _load((gpu, ora), phi=phi, c=c, alpha=1.0)
    _lockstep(gpu, ora, 25)


def test_dislocation_recovery_elastic_bitexact(oracle_mod):
    th = thermo.dislocation(1e-12, 0.3, 4e10, 2.5e-10, 0.5, 0.05, 1e12)
    th.elastic_enabled, th.elastic_modulus, th.eigenstrain_coeff, th.c_ref = True, 5e9, 0.02, 0.0
    th.elastic_smooth_iters = 4
    phi, g = polycrystal(1, 64, 64, 10, 2)
    gpu, ora = _pair(oracle_mod, (1, 64, 64), 1e-6, th, 0.0, 2.0)
    rng = np.random.default_rng(4)
    rho = (1e14 * (phi % 3 + 1)).astype(np.float32)
    c = rng.uniform(0, 0.05, phi.shape).astype(np.float32)
    _load((gpu, ora), phi=phi, g=g, rho=rho, c=c, alpha=1.0)
    _lockstep(gpu, ora, 20)


def test_grooving_bitexact(oracle_mod):
    th = thermo.grooving(1e-12, 0.4, 0.8)
    Ny = Nx = 48
    phi = np.zeros((1, Ny, Nx), np.int32)
    phi[0, 24:, :24] = 1
    phi[0, 24:, 24:] = 2
    gpu, ora = _pair(oracle_mod, (1, Ny, Nx), 1e-6, th, 0.0, 2.0)
    _load((gpu, ora), phi=phi, alpha=1.0)
    _lockstep(gpu, ora, 30)


def test_separable_geometry_path(oracle_mod):
    """sigma = 5 in 3-D selects the global separable geometry (geom radius 20 > 18)."""
    phi = np.zeros((40, 40, 40), np.int32)
    zz, yy, xx = np.mgrid[0:40, 0:40, 0:40]
    phi[(zz - 20) ** 2 + (yy - 20) ** 2 + (xx - 20) ** 2 <= 144] = 1
    gpu, ora = _pair(oracle_mod, (40, 40, 40), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 5.0)
    _load((gpu, ora), phi=phi, alpha=1.0)
    _lockstep(gpu, ora, 3)


def test_f64_mode_matches_f64_oracle(oracle_mod):
    phi, g = polycrystal(1, 96, 96, 24, 8)
    gpu, ora = _pair(oracle_mod, (1, 96, 96), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5, precision="f64")
    _load((gpu, ora), phi=phi, g=g.astype(np.float64), alpha=1.0)
    for s in range(40):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= 1e-10 * abs(do), s
        assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
        for f in ("kappa_f", "vn_f", "alpha"):
            assert rel_close(gpu.get(f), ora.get(f), 1e-10), (s, f)


def test_diagnostics_match(oracle_mod):
    phi, g = polycrystal(1, 80, 80, 20, 6)
    gpu, ora = _pair(oracle_mod, (1, 80, 80), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    for _ in range(15):
        gpu.step(); ora.step()
    assert gpu.n_grains() == ora.n_grains()
    assert gpu.interface_fraction() == ora.interface_fraction()
    assert gpu.max_dt() == ora.max_dt()
    for lab in (1, 5, 11):
        assert gpu.phase_volume(lab) == ora.phase_volume(lab)
    cells = np.nonzero(gpu.get("mask").ravel())[0][:40]
    pc = gpu.get("phi_comp").ravel()
    for c in cells:
        assert gpu.topology_simple_move(int(c), int(pc[c])) == ora.topology_simple_move(int(c), int(pc[c]))


def test_run_matches_oracle(oracle_mod):
    """GPKGrid::run(t_end): each step capped by the remaining time."""
    phi, g = polycrystal(1, 64, 64, 12, 4)
    gpu, ora = _pair(oracle_mod, (1, 64, 64), 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    _load((gpu, ora), phi=phi, g=g, alpha=1.0)
    t_end = 40.0
    n_g = gpu.run(t_end)
    n_o = ora.run(t_end)
    assert n_g == n_o
    assert gpu.time == ora.time
    assert not compare_all(gpu, ora, ["phi", "alpha"])


def test_label_range_rejected():
    from gpk_b200 import GPKError
    gpu = GPKGrid(1, 8, 8, 1.0, thermo.isotropic(1.0))
    good = (np.arange(64, dtype=np.int32) // 16).reshape(1, 8, 8) + 1
    gpu.set("phi", good)
    assert gpu.n_grains() == 4
    bad = np.zeros((1, 8, 8), np.int32); bad[0, 0, 0] = -3
    with pytest.raises(GPKError) as e:
        gpu.set("phi", bad)
    assert e.value.code == 5
    bad = good.copy(); bad[0, 5, 2] = 1 << 26; bad[0, 7, 7] = -1
    with pytest.raises(GPKError) as e:
        gpu.set("phi", bad)
    assert e.value.code == 5 and "at cell 42 " in str(e.value)
    # a rejected upload leaves the grid as it was
    assert np.array_equal(gpu.get("phi"), good) and gpu.n_grains() == 4
    with pytest.raises(GPKError):
        gpu.set("phi_comp", bad)
