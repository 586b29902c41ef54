"""Batched sweep: every instance advanced in a batch equals the same instance
stepped alone, bit for bit, whatever the worker count."""
import numpy as np
import pytest

from gpk_b200 import GPKBatch, GPKError
from gpk_b200.sweep import lamellar_grid

from _cases import PUBLIC_FIELDS

pytestmark = pytest.mark.gpu
SEEDS = list(range(100, 112))
SMALL = (64, 160)


def _fields(g):
    return {f: g.get(f) for f in PUBLIC_FIELDS}


def _same(a, b):
    for f in a:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f
        else:
            assert np.array_equal(x, y), f


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_batch_equals_alone(precision):
    alone = [lamellar_grid(s, precision=precision, side_range=SMALL)[0] for s in SEEDS]
    for g in alone:
        for _ in range(12):
            g.step()
    batched = [lamellar_grid(s, precision=precision, side_range=SMALL)[0] for s in SEEDS]
    b = GPKBatch(batched, workers=5)
    b.step(7)
    b.workers = 3
    b.step(5)
    for ga, gb in zip(alone, batched):
        _same(_fields(ga), _fields(gb))
        assert ga.time == gb.time
    b.close()


def test_batch_run_and_autotune():
    grids = [lamellar_grid(s, side_range=SMALL)[0] for s in SEEDS[:6]]
    ref = [lamellar_grid(s, side_range=SMALL)[0] for s in SEEDS[:6]]
    b = GPKBatch(grids, workers=0)
    assert 1 <= b.workers <= 6
    w, taken = b.autotune(trial_steps=1)
    assert w in (1, 2, 4) and taken == 3
    for g in ref:
        for _ in range(taken):
            g.step()
    for g, r in zip(grids, ref):
        _same(_fields(g), _fields(r))
    t_end = max(g.time for g in grids) + 5.0
    steps = b.run(t_end)
    for g, r, n in zip(grids, ref, steps):
        assert n >= 1 and n == r.run(t_end)
        _same(_fields(g), _fields(r))
        assert g.time == r.time
    b.close()


def test_batch_rejects_bad_arguments():
    g, _ = lamellar_grid(1, side_range=SMALL)
    with pytest.raises(GPKError):
        GPKBatch([g, g])
    with pytest.raises(GPKError):
        GPKBatch([])
    b = GPKBatch([g], workers=1)
    with pytest.raises(GPKError):
        b.step(-1)
