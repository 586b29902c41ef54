"""Generates tests/golden/spectral_elasticity.npz from the reference itself.

Imports `spectral_elasticity` and `Parameters` from the reference's
scripts/run_alcu_gpk_microstructure.py (lines 43-75 and 99-190) and runs it on
seeded variant-fraction fields of several shapes: even and odd extents in 2-D
and 3-D (the Nyquist planes of even extents are where the reference's
`ifftn(...).real` drops a non-Hermitian part), and a dilatational sphere with
the cubic constants 108/62/28 GPa and a 0.5% misfit.  Run it where the
reference tree is present:

    python tests/golden/make_spectral_golden.py [path/to/reference]
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "spectral_elasticity.npz")


def load_reference(root: str):
    path = os.path.join(root, "scripts", "run_alcu_gpk_microstructure.py")
    spec = importlib.util.spec_from_file_location("gpk_ref_alcu", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpk_ref_alcu"] = mod
    spec.loader.exec_module(mod)
    return mod


def fractions(shape, rng, kind):
    """Variant fractions in [0, 1] as multiples of 1/256, so they are exact
    in any format and can be stored as uint8."""
    if kind == "random":
        q = rng.integers(0, 256, size=(3,) + shape)
    elif kind == "plates":
        q = np.zeros((3,) + shape, dtype=np.int64)
        grids = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
        for v in range(3):
            for _ in range(2):
                c = [rng.integers(0, n) for n in shape]
                half = [rng.integers(1, max(2, n // 3)) for n in shape]
                half[v % len(shape)] = 1  # thin along one axis
                box = np.ones(shape, dtype=bool)
                for a, n in enumerate(shape):
                    d = np.abs((grids[a] - c[a] + n // 2) % n - n // 2)
                    box &= d <= half[a]
                q[v][box] = 255
    else:  # sphere of variant-0 fraction 1, used with equal eigenstrains
        q = np.zeros((3,) + shape, dtype=np.int64)
        grids = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
        r2 = sum((g - n // 2) ** 2 for g, n in zip(grids, shape))
        q[0][r2 <= 16] = 255
    return q.astype(np.uint8)


CASES = [
    # name, shape, kind, parameter overrides
    ("2d_even", (32, 24), "plates", {}),
    ("2d_odd", (21, 27), "random", {}),
    ("3d_even", (12, 8, 16), "random", {}),
    ("3d_odd", (9, 7, 11), "plates", {}),
    ("3d_sphere_dilatational", (16, 16, 16), "sphere",
     {"c11": 108e9, "c12": 62e9, "c44": 28e9, "eigen_small": 0.005, "eigen_large": 0.005, "dx": 1.0}),
]


def main(root: str) -> None:
    ref = load_reference(root)
    rng = np.random.default_rng(20240607)
    out = {}
    for name, shape, kind, over in CASES:
        p = ref.Parameters(**over)
        q = fractions(shape, rng, kind)
        vf = q.astype(np.float64) / 256.0
        driving, energy, hydro, residual = ref.spectral_elasticity(vf, p)
        out[f"{name}/q"] = q
        out[f"{name}/params"] = np.array([p.dx, p.c11, p.c12, p.c44, p.eigen_small, p.eigen_large])
        out[f"{name}/driving"] = driving
        out[f"{name}/energy"] = energy
        out[f"{name}/hydro"] = hydro
        out[f"{name}/residual"] = np.array(residual)
        print(f"{name}: shape {shape} residual {residual:.3e} energy mean {energy.mean():.6e}")
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPK_REFERENCE")
    if not _ref:
        sys.exit("usage: python %s <path to the reference checkout> (or set GPK_REFERENCE)" % sys.argv[0])
    main(_ref)
