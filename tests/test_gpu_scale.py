"""Parity at the benchmarked size and over long 3-D runs.

* The benchmarked workload itself — 256^3 periodic labels, 4096 Voronoi
  grains, sigma 1.5, IsotropicGrowthThermo(1, 1), the reference's FP32
  arithmetic — stepped on the GPU and by the reference's own GPKGrid (its
  src/*.cpp compiled into oracle/_ref, OpenMP on the host cores) from the same
  input: labels, alpha, orientations, dt and the three transaction counters
  equal after every step through the benchmark's 16 settling steps and 4
  more, the steps where crossings (src/gpk_transitions.cpp:273-313), the
  double balanced remap (:38-178, :320-324) and an extinction pass (:180-249)
  all run.  About 20 reference steps of ~7 s each on 16 host cores.
* A 48^3 lockstep of 40 steps against the oracle with every public field
  compared after every step: 60 Voronoi grains plus eight planted cubes of
  8 to 125 cells, so that grains are eroded by the extinction passes of
  steps 0, 16, 24 and 32 besides hundreds of crossings and remap exchanges
  per step.
* The solidification configuration at its size: 128^3 with solute
  partitioning (k = 0.14, c0 = 0.02, nucleus of radius 4), FP32 bit for bit
  and FP64 within 1e-10 of the FP64 oracle.
"""
import numpy as np
import pytest

from gpk_b200 import GPKGrid, thermo

from _cases import PUBLIC_FIELDS, bits_equal, compare_all, diff_report, rel_close

pytestmark = pytest.mark.gpu


def test_benchmarked_workload_256_matches_reference(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built")
    n, grains, seed, settle, extra = 256, 4096, 42, 16, 4
    iso = thermo.isotropic(1.0, 1.0)
    gpu = GPKGrid(n, n, n, 1.0, iso, 0.0, 1.5)
    gpu.voronoi(grains, seed)
    gpu.set("alpha", 1.0)
    ref = oracle_mod.RefGrid(n, n, n, 1.0, iso, 0.0, 1.5)
    ref.set("phi", gpu.get("phi"))
    ref.set("g", gpu.get("g"))
    ref.set("alpha", 1.0)
    seen = {"accepted": 0, "deferred": 0, "exchanges": 0}
    for s in range(settle + extra):
        dg, dr = gpu.step(), ref.step()
        assert dg == dr, f"step {s}: dt {dg!r} vs {dr!r}"
        cg, cr = gpu.counters(), ref.counters()
        assert cg == cr, f"step {s}: counters {cg} vs {cr}"
        for f in ("phi", "alpha", "g"):
            a, b = gpu.get(f), ref.get(f)
            assert bits_equal(a, b), f"step {s}: " + diff_report(f, a, b)
        seen["accepted"] += cg[0]
        seen["deferred"] += cg[1]
        seen["exchanges"] += cg[2]
    for f in ("kappa_f", "vn_f", "phi_comp", "mask"):
        a, b = gpu.get(f), ref.get(f)
        assert bits_equal(a, b), diff_report(f, a, b)
    # the compared steps did run the ordered label update
    assert seen["accepted"] > 1000 and seen["deferred"] > 0 and seen["exchanges"] > 0, seen


def _planted_polycrystal(oracle_mod, n=48):
    phi, g = oracle_mod.voronoi(n, n, n, 60, 5)
    rng = np.random.default_rng(3)
    lab = 61
    for side in (2, 2, 3, 3, 3, 4, 4, 5):
        z, y, x = rng.integers(0, n - 6, 3)
        phi[z:z + side, y:y + side, x:x + side] = lab
        g[z:z + side, y:y + side, x:x + side] = rng.random() * 1.5
        lab += 1
    return phi, g


def test_lockstep_3d_48_crossings_remap_extinction(oracle_mod):
    phi, g = _planted_polycrystal(oracle_mod)
    iso = thermo.isotropic(1.0, 1.0)
    gpu = GPKGrid(48, 48, 48, 1.0, iso, 0.0, 1.5)
    ora = oracle_mod.OracleGrid(48, 48, 48, 1.0, iso, 0.0, 1.5)
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g)
        G.set("alpha", 1.0)
    totals = np.zeros(3, dtype=np.int64)
    planted = {}
    for s in range(40):
        dg, do = gpu.step(), ora.step()
        assert dg == do, f"step {s}: dt {dg!r} vs {do!r}"
        assert gpu.counters() == ora.counters(), f"step {s}: {gpu.counters()} vs {ora.counters()}"
        bad = compare_all(gpu, ora, PUBLIC_FIELDS)
        assert not bad, f"step {s}: {bad}"
        totals += np.array(gpu.counters())
        ph = gpu.get("phi")
        planted[s] = [int((ph == lab).sum()) for lab in range(61, 69)]
    assert totals[0] > 5000 and totals[1] > 500 and totals[2] > 2000, totals
    # grains vanished in the extinction passes of steps 0, 16, 24 and 32
    assert planted[0][:2] == [0, 0]
    for s in (16, 24, 32):
        assert sum(v == 0 for v in planted[s]) > sum(v == 0 for v in planted[s - 1]), (s, planted)


def _solidification_128(oracle_mod, precision):
    th = thermo.solidification(5e-8, 0.2, 0.0, -500.0, 0.14, 933.0, 1e8)
    th.solute_rejection, th.k_partition = True, 0.14
    n = 128
    gpu = GPKGrid(n, n, n, 0.5e-6, th, 3e-9, 1.5, precision=precision)
    ora = oracle_mod.OracleGrid(n, n, n, 0.5e-6, th, 3e-9, 1.5, precision=precision)
    z, y, x = np.indices((n, n, n)) - n // 2
    nucleus = (x * x + y * y + z * z) <= 16
    rd = np.float32 if precision == "f32" else np.float64
    phi = nucleus.astype(np.int32)
    c = np.full((n, n, n), rd(0.02))
    c[nucleus] = rd(0.02) * rd(0.14)
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("c", c)
        G.set("T", rd(933.0) - rd(5.0))
        G.set("alpha", 1.0)
    return gpu, ora


def test_solidification_128_lockstep(oracle_mod):
    gpu, ora = _solidification_128(oracle_mod, "f32")
    for s in range(6):
        assert gpu.step() == ora.step(), s
        bad = compare_all(gpu, ora, ["phi", "alpha", "c", "kappa_f", "vn_f", "mask"])
        assert not bad, f"step {s}: {bad}"


def test_solidification_128_f64_within_1e10(oracle_mod):
    gpu, ora = _solidification_128(oracle_mod, "f64")
    for s in range(4):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= 1e-10 * abs(do), s
        assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
        for f in ("c", "alpha", "kappa_f", "vn_f"):
            assert rel_close(gpu.get(f), ora.get(f), 1e-10), (s, f)
