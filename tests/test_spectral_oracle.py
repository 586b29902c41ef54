"""The spectral-elasticity oracle against the reference's own outputs.

tests/golden/spectral_elasticity.npz holds what the reference's
`spectral_elasticity` (scripts/run_alcu_gpk_microstructure.py:99-190)
returned for five seeded inputs (make_spectral_golden.py).  The numpy
restatement in oracle/spectral_oracle.py must reproduce them to FFT
rounding, so that the CUDA solve can be checked against the oracle at sizes
the fixtures do not cover.
"""
import os
import types

import numpy as np
import pytest

from oracle.spectral_oracle import spectral_elasticity

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "spectral_elasticity.npz")


def golden_cases():
    z = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    out = []
    for n in names:
        pr = z[n + "/params"]
        p = types.SimpleNamespace(dx=pr[0], c11=pr[1], c12=pr[2], c44=pr[3], eigen_small=pr[4], eigen_large=pr[5])
        out.append((n, z[n + "/q"].astype(np.float64) / 256.0, p,
                    {k: z[f"{n}/{k}"] for k in ("driving", "energy", "hydro", "residual")}))
    return out


def rel_err(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0])
def test_oracle_matches_reference_outputs(case):
    name, vf, p, ref = case
    d, e, h, r = spectral_elasticity(vf, p)
    assert rel_err(d, ref["driving"]) < 1e-13
    assert rel_err(e, ref["energy"]) < 1e-13
    assert rel_err(h, ref["hydro"]) < 1e-13
    # both residuals are at rounding level; the reference's own audit is 1e-10
    assert r < 1e-14 and float(ref["residual"]) < 1e-14


def test_oracle_dilatational_sphere_is_hydrostatic_inside():
    """Property of the solution: an equal-eigenstrain sphere in a cubic matrix
    carries an almost uniform compressive hydrostatic stress inside."""
    n = 24
    g = np.indices((n, n, n)) - n // 2
    inside = (g ** 2).sum(0) <= 25
    vf = np.zeros((3, n, n, n))
    vf[0][inside] = 1.0
    p = types.SimpleNamespace(dx=1.0, c11=108e9, c12=62e9, c44=28e9, eigen_small=0.005, eigen_large=0.005)
    d, e, h, r = spectral_elasticity(vf, p)
    assert r < 1e-12
    assert np.all(h[inside] < 0)
    assert np.all(e >= -1e-9 * e.max())


def test_oracle_on_the_reference_trajectory():
    """The driver's own spectral solves of a 64^2 Al-Cu run (recorded in
    tests/golden/alcu_trajectory.npz), through the oracle, within 1e-10."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import alcu_replay as R

    cases = R.spectral_cases()
    assert len(cases) >= 5
    for vf, p, ref, res in cases:
        d, e, h, r = spectral_elasticity(vf, p)
        assert R.rel_err(d, ref["driving"]) < 1e-10 and R.rel_err(e, ref["energy"]) < 1e-10
        assert R.rel_err(h, ref["hydro"]) < 1e-10 and abs(r - res) < 1e-12
