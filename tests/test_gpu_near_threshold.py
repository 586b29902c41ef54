"""The near-threshold listing of the crossing decision.

The reference switches an interface cell when
    alpha_new <= 1e-6  &&  phi_comp != phi      (src/gpk_transitions.cpp:291-292)
with alpha_new = min(alpha + v dt / dx, 1) (:251-271).  Each step lists the
cells with phi_comp != phi whose margin alpha_new - 1e-6 lies within a
tolerance of zero (1e-12 by default): the decisions that arithmetic of
another precision or another operation order could flip.

* In the reference's FP32 arithmetic the device list equals the oracle's
  after every step, at the default tolerance and at a wide one that lists
  many cells, on the 256^2 / 128-grain configuration for 200 steps.
* In FP64 the device's labels equal the FP64 oracle's after every step of
  the same run except at listed cells, and the two lists are equal.
"""
import numpy as np
import pytest

from gpk_b200 import GPKGrid, thermo

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, precision, tol):
    phi, g = oracle_mod.voronoi(1, 256, 256, 128, 42)
    iso = thermo.isotropic(1.0, 1.0)
    gpu = GPKGrid(1, 256, 256, 1.0, iso, 0.0, 1.5, precision=precision)
    ora = oracle_mod.OracleGrid(1, 256, 256, 1.0, iso, 0.0, 1.5, precision=precision)
    rd = np.float32 if precision == "f32" else np.float64
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g.astype(rd))
        G.set("alpha", 1.0)
        G.set_near_threshold(tol)
    return gpu, ora


@pytest.mark.parametrize("tol", [1e-12, 5e-3])
def test_near_threshold_lists_equal_fp32(oracle_mod, tol):
    gpu, ora = _pair(oracle_mod, "f32", tol)
    listed = 0
    for s in range(200):
        assert gpu.step() == ora.step(), s
        a, b = gpu.near_threshold(), ora.near_threshold()
        assert np.array_equal(a, b), f"step {s}: {a[:8]} vs {b[:8]}"
        listed += a.size
        if s % 20 == 19:
            assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
    if tol > 1e-6:
        assert listed > 100, listed       # the wide tolerance does list cells


def test_near_threshold_f64_labels_equal_except_listed(oracle_mod):
    gpu, ora = _pair(oracle_mod, "f64", 1e-12)
    for s in range(200):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= 1e-10 * abs(do), s
        a, b = gpu.near_threshold(), ora.near_threshold()
        pg, po = gpu.get("phi").ravel(), ora.get("phi").ravel()
        diff = np.nonzero(pg != po)[0]
        assert np.isin(diff, np.union1d(a, b)).all(), f"step {s}: unlisted label differences at {diff[:8]}"
        if diff.size:   # continue from the device's state
            for f in ("phi", "alpha", "g"):
                ora.set(f, gpu.get(f))
        else:
            assert np.array_equal(a, b), f"step {s}"


def test_near_threshold_tolerance_is_validated():
    from gpk_b200 import GPKError
    g = GPKGrid(1, 16, 16, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    with pytest.raises(GPKError):
        g.set_near_threshold(-1.0)
    with pytest.raises(GPKError):
        g.set_near_threshold(float("nan"))
    g.set_near_threshold(0.0)
    g.step()
    assert g.near_threshold().dtype == np.int32
