"""The lamellar sweep generator (host logic, no GPU)."""
import numpy as np

from gpk_b200.sweep import C_PREC, C_SAT, lamellar_instance


def test_instances_follow_the_sweep_distribution():
    sides, hs, ratios = [], [], []
    for seed in range(200):
        inst = lamellar_instance(seed)
        L, h, d, phi, c = inst["side"], inst["h"], inst["d"], inst["phi"], inst["c"]
        assert 64 <= L <= 512 and 4 <= h <= 16 and 2.0 <= inst["ratio"] <= 12.0
        assert phi.shape == (1, L, L) and phi.dtype == np.int32
        rows = np.flatnonzero((phi[0] > 0).any(axis=1))
        assert len(rows) == h and rows[-1] - rows[0] == h - 1          # one stripe of thickness h
        stripe = phi[0, rows[0]]
        assert stripe.min() == 1 and np.all(np.diff(stripe) >= 0)      # grains of length d along x
        assert np.all(np.bincount(stripe)[1:-1] == d)
        dev = c - np.where(phi > 0, C_PREC, C_SAT)
        assert abs(dev.std() - 1e-3) < 2e-4
        sides.append(L); hs.append(h); ratios.append(inst["ratio"])
    assert min(sides) < 128 and max(sides) > 448 and set(range(4, 17)) <= set(hs)


def test_instances_are_seeded():
    a, b = lamellar_instance(7), lamellar_instance(7)
    assert a["side"] == b["side"] and np.array_equal(a["phi"], b["phi"]) and np.array_equal(a["c"], b["c"])
