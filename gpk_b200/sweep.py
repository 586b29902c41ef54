"""Seeded lamellar-precipitate instances for parameter sweeps.

One 2-D periodic square instance: side L ~ U{64..512}, one precipitate
stripe of thickness h ~ U{4..16} across x, cut into grains of length
d = round(r h) with r ~ U[2, 12] (the spacing-to-thickness ratio), as in the
reference's periodic lamellar stripe sweep (demos/gpk.cpp:1122-1150, where
grains of length d fill the stripe and each grain boundary pinches it).
Label 0 is the matrix (OstwaldThermo's parent phase), labels 1.. the stripe
grains.  Solute: c_sat in the matrix and c_prec in the stripe, each with
Gaussian noise of standard deviation 1e-3.
"""
from __future__ import annotations

import numpy as np

C_SAT = 0.15
C_PREC = 0.85


def lamellar_instance(seed: int, side_range=(64, 512)) -> dict:
    rng = np.random.default_rng(seed)
    side = int(rng.integers(side_range[0], side_range[1] + 1))
    h = int(rng.integers(4, 17))
    ratio = float(rng.uniform(2.0, 12.0))
    d = max(1, int(round(ratio * h)))
    phi = np.zeros((1, side, side), dtype=np.int32)
    y0 = side // 2 - h // 2
    phi[0, y0:y0 + h, :] = 1 + (np.arange(side, dtype=np.int32) // d)[None, :]
    c = np.where(phi > 0, C_PREC, C_SAT) + rng.normal(0.0, 1e-3, size=phi.shape)
    return {"side": side, "h": h, "ratio": ratio, "d": d, "phi": phi, "c": c}


def lamellar_side(seed: int, side_range=(64, 512)) -> int:
    """The side of instance `seed` (its first random draw), without building it."""
    return int(np.random.default_rng(seed).integers(side_range[0], side_range[1] + 1))


def shard(sizes, n: int) -> list:
    """Instances split over n ranks with balanced work: largest first, each
    to the least-loaded rank (ties to the lower rank); each part ascending."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * n
    parts = [[] for _ in range(n)]
    for i in order:
        r = min(range(n), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def lamellar_grid(seed: int, sigma: float = 1.5, precision: str = "f64", side_range=(64, 512)):
    """A GPKGrid holding instance `seed` (OstwaldThermo, M0 = sigma0 = 1,
    Omega = 10, D = 0.1, dx = 1)."""
    from . import thermo
    from .grid import GPKGrid
    inst = lamellar_instance(seed, side_range)
    L = inst["side"]
    g = GPKGrid(1, L, L, 1.0, thermo.ostwald(1.0, 1.0, c_sat=C_SAT, Omega=10.0), 0.1, sigma, precision=precision)
    g.set("phi", inst["phi"])
    g.set("c", inst["c"])
    g.set("alpha", 1.0)
    return g, inst
