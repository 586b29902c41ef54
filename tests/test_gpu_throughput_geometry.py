"""FP64 separable tiles (the throughput geometry) against the FP64 oracle.

The oracle evaluates the reference's direct Gaussian-Hessian stencil in FP64.
The separable tiles smooth each label's indicator with the Gaussian and take
fourth-order differences at that label's interface cells (the reference's
separable formulas, src/gpk_geometry.cpp:185-347): the same linear operators
composed in another order, so the two agree to rounding, not bit for bit.

Tolerance: every field within 1e-10 of the oracle's, relative to the field's
largest magnitude; labels equal except at cells the near-threshold listing
names (the crossing decisions within 1e-12 of the switching threshold).
"""
import numpy as np
import pytest

from gpk_b200 import GPKError, GPKGrid, thermo

pytestmark = pytest.mark.gpu
FIELDS = ("nx_f", "ny_f", "nz_f", "kappa_f", "vn_f", "alpha")
TOL = 1e-10


def _close(a, b, tol=TOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) <= tol * scale


def _lockstep(oracle_mod, shape, grains, seed, steps, sigma=1.5):
    phi, g = oracle_mod.voronoi(*shape, grains, seed)
    iso = thermo.isotropic(1.0, 1.0)
    gpu = GPKGrid(*shape, 1.0, iso, 0.0, sigma, precision="f64")
    gpu.set_geometry_kernel("separable_tiles")
    ora = oracle_mod.OracleGrid(*shape, 1.0, iso, 0.0, sigma, precision="f64")
    for G in (gpu, ora):
        G.set("phi", phi)
        G.set("g", g.astype(np.float64))
        G.set("alpha", 1.0)
    accepted = 0
    for s in range(steps):
        dg, do = gpu.step(), ora.step()
        assert abs(dg - do) <= TOL * abs(do), s
        pa, pb = gpu.get("phi").ravel(), ora.get("phi").ravel()
        diff = np.flatnonzero(pa != pb)
        listed = set(gpu.near_threshold().tolist()) | set(ora.near_threshold().tolist())
        assert set(diff.tolist()) <= listed, (s, diff[:10])
        if diff.size:
            return accepted  # the runs parted at a listed tie: later steps are not comparable
        for f in FIELDS:
            assert _close(gpu.get(f), ora.get(f)), (s, f)
        assert np.array_equal(gpu.get("phi_comp"), ora.get("phi_comp")), s
        accepted += gpu.counters()[0]
    return accepted


def test_separable_tiles_3d_against_f64_oracle(oracle_mod):
    """28^3, 24 grains, 14 steps: crossings from step 8 on, with the remap."""
    assert _lockstep(oracle_mod, (28, 28, 28), 24, 9, 14) > 0


def test_separable_tiles_2d_against_f64_oracle(oracle_mod):
    """128^2, 48 grains, 60 steps."""
    assert _lockstep(oracle_mod, (1, 128, 128), 48, 5, 60) > 0


@pytest.mark.parametrize("sigma", [0.5, 1.0, 1.5, 2.2])
@pytest.mark.parametrize("shape", [(24, 30, 36), (1, 70, 90)])
def test_separable_tiles_geometry_every_radius(oracle_mod, sigma, shape):
    """Kernel radii 4, 6, 8 and 10 on grids no tile divides: one geometry
    evaluation of the separable tiles against the direct FP64 tiles."""
    phi, g = oracle_mod.voronoi(*shape, 20, 12)
    iso = thermo.isotropic(1.0, 1.0)
    out = []
    for kind in ("tiled", "separable_tiles"):
        G = GPKGrid(*shape, 1.0, iso, 0.0, sigma, precision="f64")
        G.set_geometry_kernel(kind)
        G.set("phi", phi)
        G.set("g", g.astype(np.float64))
        G.geometry()
        out.append({f: G.get(f) for f in ("nx_f", "ny_f", "nz_f", "kappa_f", "phi_comp")})
    for f in ("nx_f", "ny_f", "nz_f", "kappa_f"):
        assert _close(out[1][f], out[0][f]), f
    assert np.array_equal(out[1]["phi_comp"], out[0]["phi_comp"])


def test_separable_tiles_rejected_in_fp32():
    g = GPKGrid(8, 8, 8, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5)
    with pytest.raises(GPKError):
        g.set_geometry_kernel("separable_tiles")
    g64 = GPKGrid(8, 8, 8, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 6.0, precision="f64")  # kernel radius 23
    with pytest.raises(GPKError):
        g64.set_geometry_kernel("separable_tiles")


@pytest.mark.parametrize("shape", [(24, 30, 36), (1, 70, 90)])
def test_separable_tiles_many_labels_per_tile(oracle_mod, shape):
    """Hundreds of small grains: most tiles hold more labels than one bitmap
    batch (four), so the per-batch bitmaps, label boxes and passes repeat."""
    phi, g = oracle_mod.voronoi(*shape, 400, 7)
    iso = thermo.isotropic(1.0, 1.0)
    out = []
    for kind in ("tiled", "separable_tiles"):
        G = GPKGrid(*shape, 1.0, iso, 0.0, 1.5, precision="f64")
        G.set_geometry_kernel(kind)
        G.set("phi", phi)
        G.set("g", g.astype(np.float64))
        G.geometry()
        out.append({f: G.get(f) for f in ("nx_f", "ny_f", "nz_f", "kappa_f", "phi_comp")})
    for f in ("nx_f", "ny_f", "nz_f", "kappa_f"):
        assert _close(out[1][f], out[0][f]), f
    _competitors_equal_except_ties(phi, out[0], out[1])


def _competitors_equal_except_ties(phi, a, b):
    """The competitor (src/gpk_geometry.cpp:154-182) is the unlike face
    neighbour with the most like cells among the 26 around the cell, ties
    going to the larger outward-normal alignment.  Normals that agree to
    rounding can still order two equally supported candidates differently
    when their alignments agree to rounding; every other cell must match."""
    diff = np.argwhere(a["phi_comp"] != b["phi_comp"])
    Nz, Ny, Nx = phi.shape
    for z, y, x in diff:
        own = phi[z, y, x]

        def support(q):
            n = 0
            for dz in ((-1, 0, 1) if Nz > 1 else (0,)):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        if dz or dy or dx:
                            n += phi[(z + dz) % Nz, (y + dy) % Ny, (x + dx) % Nx] == q
            return n

        qa, qb = a["phi_comp"][z, y, x], b["phi_comp"][z, y, x]
        assert qa != own and qb != own, (z, y, x)
        assert support(qa) == support(qb), (z, y, x)
        faces = {(0, 0, -1): -a["nx_f"], (0, 0, 1): a["nx_f"], (0, -1, 0): -a["ny_f"], (0, 1, 0): a["ny_f"]}
        if Nz > 1:
            faces.update({(-1, 0, 0): -a["nz_f"], (1, 0, 0): a["nz_f"]})
        score = {}
        for (dz, dy, dx), field in faces.items():
            q = phi[(z + dz) % Nz, (y + dy) % Ny, (x + dx) % Nx]
            if q in (qa, qb):
                score[q] = max(score.get(q, -2.0), float(field[z, y, x]))
        assert abs(score[qa] - score[qb]) <= 1e-12, (z, y, x, score)
    print(f"competitors differing at near-ties: {len(diff)} of {a['phi_comp'].size} cells")
