"""Pins the CPU oracle: against the reference's golden vectors, its known-answer
topology tests, and (where its sources were built here) the reference itself.

These run without a GPU.
"""
import os

import numpy as np
import pytest

from gpk_b200 import thermo

from _cases import bits_equal, compare_all, neutral, polycrystal, topology_cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _ref_or_skip(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference library (oracle/_ref) not built here")


@pytest.mark.parametrize("name,phi,cell,new,expected", topology_cases(), ids=[c[0] for c in topology_cases()])
def test_topology_known_answers(oracle_mod, name, phi, cell, new, expected):
    # demos/validate_topology_transactions.cpp:28-80
    o = oracle_mod.OracleGrid(*phi.shape, 1.0, neutral(), 0.0, 2.0)
    o.set("phi", phi)
    Nz, Ny, Nx = phi.shape
    assert o.topology_simple_move((cell[0] * Ny + cell[1]) * Nx + cell[2], new) == expected


@pytest.mark.parametrize("key", ["g13", "g15"])
def test_golden_curved_bicrystal(oracle_mod, key):
    # demos/validate_extended_base_models.cpp:767-830: 360^2, 10 x 80 steps
    gd = np.load(os.path.join(GOLDEN, "curved_bicrystals_360.npz"))
    o = oracle_mod.OracleGrid(1, 360, 360, 0.1e-6, thermo.isotropic(1e-8, 0.324), 0.0, 2.0)
    o.set("phi", gd[key + "_before"].astype(np.int32)[None])
    o.set("alpha", 1.0)
    for _ in range(800):
        o.step()
    assert np.array_equal(o.get("phi")[0], gd[key + "_after"].astype(np.int32))


def _alpha_micro(alpha):
    return np.array([round(float("%.6f" % v) * 1e6) for v in np.asarray(alpha, dtype=np.float32).ravel()])


def test_golden_rex_snapshots(oracle_mod):
    # paper/inputs/validation_rex_current_2d.ini driven as run_recrystallisation does
    rx = np.load(os.path.join(GOLDEN, "rex_192_snapshots.npz"))
    o = oracle_mod.OracleGrid(1, 192, 192, 1e-6, thermo.recrystallisation(1e-12, 0.3, 1e6), 0.0, 2.0)
    o.set("phi", rx["phi"][0].astype(np.int32)[None])
    o.set("alpha", 1.0)
    for snap in range(1, 6):
        while o.time < 44.0 / 24 * snap:
            o.step(-1.0)
        assert np.array_equal(o.get("phi")[0], rx["phi"][snap].astype(np.int32)), snap
        assert np.array_equal(_alpha_micro(o.get("alpha")), rx["alpha_micro"][snap].ravel()), snap
        assert "%g" % o.time == str(rx["time_str"][snap])


def _run_pair(oracle_mod, shape, n_grains, steps, sigma, th=None, seed=7):
    _ref_or_skip(oracle_mod)
    phi, g = polycrystal(*shape, n_grains, seed)
    th = th or thermo.isotropic(1.0, 1.0)
    o = oracle_mod.OracleGrid(*shape, 1.0, th, 0.0, sigma)
    r = oracle_mod.RefGrid(*shape, 1.0, th, 0.0, sigma)
    for G in (o, r):
        G.set("phi", phi); G.set("g", g); G.set("alpha", 1.0)
    for s in range(steps):
        assert o.step() == r.step(), s
        bad = compare_all(o, r)
        assert not bad, f"step {s}: {bad}"
        assert o.counters() == r.counters(), s


def test_oracle_matches_reference_2d(oracle_mod):
    _run_pair(oracle_mod, (1, 96, 96), 30, 40, 1.5)


def test_oracle_matches_reference_3d(oracle_mod):
    _run_pair(oracle_mod, (20, 20, 20), 10, 6, 1.5)


def test_oracle_matches_reference_solidification(oracle_mod):
    _ref_or_skip(oracle_mod)
    th = thermo.solidification(5e-8, 0.2, 0.0, -500.0, 0.14, 933.0, 1e8)
    th.solute_rejection, th.k_partition = True, 0.14
    Ny = Nx = 48
    o = oracle_mod.OracleGrid(1, Ny, Nx, 0.5e-6, th, 3e-9, 2.0)
    r = oracle_mod.RefGrid(1, Ny, Nx, 0.5e-6, th, 3e-9, 2.0)
    phi = np.zeros((1, Ny, Nx), np.int32)
    yy, xx = np.mgrid[0:Ny, 0:Nx]
    seed = (yy - 24) ** 2 + (xx - 24) ** 2 <= 16
    phi[0][seed] = 1
    c = np.full((1, Ny, Nx), 0.02, np.float32); c[0][seed] = np.float32(0.02) * np.float32(0.14)
    T = np.float32(933.0 + -500.0 * 0.02) - np.float32(5.0)
    for G in (o, r):
        G.set("phi", phi); G.set("c", c); G.set("T", T); G.set("alpha", 1.0)
    for s in range(25):
        assert o.step() == r.step(), s
        assert not compare_all(o, r), s


def test_oracle_f64_tracks_f32(oracle_mod):
    """The FP64 build runs the same algorithm: on a short 2-D run its labels
    match the FP32 build and its curvature agrees to float rounding."""
    phi, g = polycrystal(1, 64, 64, 16, 3)
    th = thermo.isotropic(1.0, 1.0)
    a = oracle_mod.OracleGrid(1, 64, 64, 1.0, th, 0.0, 1.5, precision="f32")
    b = oracle_mod.OracleGrid(1, 64, 64, 1.0, th, 0.0, 1.5, precision="f64")
    for G in (a, b):
        G.set("phi", phi); G.set("g", g); G.set("alpha", 1.0)
    for _ in range(10):
        a.step(); b.step()
    assert np.array_equal(a.get("phi"), b.get("phi"))
    np.testing.assert_allclose(a.get("kappa_f"), b.get("kappa_f"), rtol=1e-4, atol=1e-5)
