"""Shared inputs and comparisons for the parity tests.

Every case builds one initial state on the host and feeds the same buffers
to the CUDA path and to the CPU oracle.
"""
from __future__ import annotations

import numpy as np

from gpk_b200 import thermo
from gpk_b200.thermo import FIELD_IDS

PUBLIC_FIELDS = list(FIELD_IDS)
STATE_FIELDS = ["phi", "alpha", "c", "T", "g", "rho"]


def polycrystal(Nz, Ny, Nx, n, seed=42):
    from gpk_b200.grid import voronoi
    return voronoi(Nz, Ny, Nx, n, seed)


def load_state(grid, phi, alpha=1.0, c=None, T=None, g=None, rho=None):
    grid.set("phi", phi)
    grid.set("alpha", alpha)
    if c is not None:
        grid.set("c", c)
    if T is not None:
        grid.set("T", T)
    if g is not None:
        grid.set("g", g)
    if rho is not None:
        grid.set("rho", rho)


def bits_equal(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-for-bit equality (distinguishes -0.0 from +0.0 and compares NaNs)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def diff_report(name, a, b) -> str:
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    if a.dtype.kind == "f":
        bad = np.nonzero(a.view(np.uint32 if a.dtype == np.float32 else np.uint64) !=
                         b.view(np.uint32 if b.dtype == np.float32 else np.uint64))[0]
    else:
        bad = np.nonzero(a != b)[0]
    if bad.size == 0:
        return f"{name}: equal"
    i = bad[0]
    return f"{name}: {bad.size} cells differ, first at {i}: gpu={a[i]!r} oracle={b[i]!r}"


def compare_all(gpu, ora, fields=PUBLIC_FIELDS):
    """Returns a list of mismatch descriptions (empty when bit-identical)."""
    out = []
    for f in fields:
        a, b = gpu.get(f), ora.get(f)
        if not bits_equal(a, b):
            out.append(diff_report(f, a, b))
    return out


def rel_close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b), 1e-300)
    d = np.abs(a - b)
    return bool(np.all((d <= rtol * scale) | (d == 0)))


# ---- the reference's topology known-answer cases ------------------------------
# demos/validate_topology_transactions.cpp:28-80: (name, dims, phi builder,
# cell (z, y, x), new label, expected)
def topology_cases():
    cases = []

    def g(dims):
        return np.zeros(dims, dtype=np.int32)

    p = g((1, 9, 9)); p[0, :, :5] = 1
    cases.append(("2D smooth boundary", p, (0, 4, 4), 0, True))
    p = g((1, 11, 11)); p[0, 3:8, 2:5] = 1; p[0, 3:8, 6:9] = 1; p[0, 5, 5] = 1
    cases.append(("2D component split", p, (0, 5, 5), 0, False))
    p = g((1, 9, 9)); p[0, 4, 3] = 1; p[0, 4, 5] = 1
    cases.append(("2D premature merger", p, (0, 4, 4), 1, False))
    p = g((1, 9, 9)); p[0, 4, 4] = 1
    cases.append(("2D terminal extinction", p, (0, 4, 4), 0, True))
    p = g((9, 9, 9)); p[3:6, 3:6, 1:4] = 2; p[3:6, 3:6, 5:8] = 2; p[4, 4, 4] = 2
    cases.append(("3D component split", p, (4, 4, 4), 0, False))
    p = g((7, 7, 7)); p[3, 3, 3] = 3
    cases.append(("3D terminal extinction", p, (3, 3, 3), 0, True))
    return cases


def neutral():
    """A plain ThermoModel with its member defaults."""
    return thermo.ThermoDesc("base")
