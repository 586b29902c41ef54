"""The step as a captured CUDA graph, alone and for a whole sweep.

A captured step runs the kernels of gpk_grid_step in the same order with no
decision on the host (device-read counts, the remap gated on the step's
accepted crossings, its proposals ordered by one block), so every field
must equal the ordinary step's bit for bit: for a single grid
(gpk_grid_step_graph) and for a batch of lamellar instances advanced as one
graph of per-instance child graphs (gpk_batch_step_graph).  The lamellar
instances (OstwaldThermo, D = 0.1, FP64) are also stepped against the FP64
oracle, fields within 1e-10 relative and labels equal.
"""
import numpy as np
import pytest

from gpk_b200 import GPKBatch, GPKError, GPKGrid, thermo
from gpk_b200.sweep import lamellar_grid, lamellar_instance

from _cases import PUBLIC_FIELDS, bits_equal, compare_all, rel_close

pytestmark = pytest.mark.gpu


def _same(a, b, fields=PUBLIC_FIELDS):
    bad = [f for f in fields if not bits_equal(a.get(f), b.get(f))]
    assert not bad, bad
    assert a.counters() == b.counters()
    assert a.time == b.time


def _same_remap_stats(a, b):
    """Remap statistics: the captured passes sum theirs on the device, the
    ordinary ones on the host; a captured pass without proposals still runs
    (and counts) one empty exchange wave."""
    sa, sb = a.wave_stats(), b.wave_stats()
    assert sa["remap_proposals"] == sb["remap_proposals"]
    assert sb["remap_waves"] >= sa["remap_waves"]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("seed", [5003, 5011])
def test_graph_step_equals_ordinary_steps_lamellar(seed, precision):
    a, _ = lamellar_grid(seed, precision=precision, side_range=(64, 160))
    b, _ = lamellar_grid(seed, precision=precision, side_range=(64, 160))
    assert a.graph_supported()
    a.step_n(21)
    b.step_graph(21)          # one ordinary, ten graph replays of two
    _same(a, b)
    a.step_n(7)
    b.step_graph(7)           # the captured graph again, and an odd step
    _same(a, b)
    _same_remap_stats(a, b)


def test_graph_step_equals_ordinary_steps_3d_solidification():
    """3-D: both remap passes run under their device-side gates."""
    th = thermo.solidification(5e-8, 0.2, 0.0, -500.0, 0.14, 933.0, 1e8)
    th.solute_rejection, th.k_partition = True, 0.14
    grids = []
    for _ in range(2):
        g = GPKGrid(40, 40, 40, 0.5e-6, th, 3e-9, 1.5)
        z, y, x = np.indices((40, 40, 40)) - 20
        g.set("phi", ((x * x + y * y + z * z) <= 25).astype(np.int32))
        g.set("c", 0.02)
        g.set("T", 933.0 - 40.0)
        g.set("alpha", 1.0)
        grids.append(g)
    a, b = grids
    a.step_n(25)
    b.step_graph(25)
    _same(a, b)
    _same_remap_stats(a, b)
    assert a.counters()[0] > 0 or a.get("phi").sum() > 515   # the nucleus grew through crossings


def test_graph_step_rejects_region_identity_models():
    g = GPKGrid(1, 32, 32, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    assert not g.graph_supported()
    with pytest.raises(GPKError) as e:
        g.step_graph(4)
    assert e.value.code == 2


def test_batch_tile_autotuner_keeps_results():
    """The tile-height autotuner only changes how the geometry is tiled: the
    instances it stepped equal the same instances stepped alone."""
    seeds = [5100 + i for i in range(6)]
    grids = [lamellar_grid(s, side_range=(64, 400))[0] for s in seeds]
    batch = GPKBatch(grids)
    choice, taken = batch.autotune_tiles(trial_steps=2)
    assert all(c in (1, 2, 4) for c in choice) and taken > 0
    alone = [lamellar_grid(s, side_range=(64, 400))[0] for s in seeds]
    for h in alone:
        h.step_n(taken)
    for g, h in zip(grids, alone):
        _same(g, h)
    batch.close()


def test_batch_graph_equals_instances_alone():
    seeds = [5000 + i for i in range(8)]
    alone = [lamellar_grid(s, side_range=(64, 192))[0] for s in seeds]
    for g in alone:
        g.step_n(13)
    grids = [lamellar_grid(s, side_range=(64, 192))[0] for s in seeds]
    batch = GPKBatch(grids, workers=4)
    batch.step_graph(13)
    for g, h in zip(grids, alone):
        _same(g, h)
    batch.step_graph(4)
    for h in alone:
        h.step_n(4)
    for g, h in zip(grids, alone):
        _same(g, h)
    batch.close()


@pytest.mark.parametrize("seed", [5001, 5002, 5007])
def test_lamellar_fp64_against_fp64_oracle(oracle_mod, seed):
    """OstwaldThermo lamellar instances, FP64, D = 0.1: labels equal to the
    FP64 oracle after every step, fields within 1e-10 relative."""
    inst = lamellar_instance(seed, side_range=(64, 128))
    L = inst["side"]
    th = thermo.ostwald(1.0, 1.0, c_sat=0.15, Omega=10.0)
    gpu = GPKGrid(1, L, L, 1.0, th, 0.1, 1.5, precision="f64")
    ora = oracle_mod.OracleGrid(1, L, L, 1.0, th, 0.1, 1.5, precision="f64")
    for G in (gpu, ora):
        G.set("phi", inst["phi"])
        G.set("c", inst["c"])
        G.set("alpha", 1.0)
    for s in range(40):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= 1e-10 * abs(do), s
        assert np.array_equal(gpu.get("phi"), ora.get("phi")), s
        for f in ("c", "alpha", "kappa_f", "vn_f"):
            assert rel_close(gpu.get(f), ora.get(f), 1e-10), (s, f)
