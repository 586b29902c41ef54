"""The Al-Cu transport/remap oracle against the reference's own outputs.

tests/golden/alcu_transport.npz holds what the reference's functions
(scripts/run_alcu_gpk_microstructure.py:260-276, 562-594, 675-755) returned
on seeded 2-D and 3-D states (make_alcu_golden.py).  The numpy restatement
in oracle/alcu_oracle.py must reproduce every array bit for bit.  Its three
library primitives are checked against the installed numpy and scipy: the
pairwise sum against `np.sum`, the wrapped Gaussian against
`scipy.ndimage.gaussian_filter`, the components against `scipy.ndimage.label`.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np
import pytest

from oracle import alcu_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "alcu_transport.npz")


def params(z, name):
    return O.AlCuParams(dx=float(z[f"{name}_dx"]))


@pytest.fixture(scope="module")
def z():
    return np.load(GOLDEN)


def same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and a.dtype.kind == b.dtype.kind and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("n", [1, 7, 8, 128, 129, 1000, 4097, 33 * 35 * 37, 64 ** 3])
def test_pairwise_sum_is_numpy_sum(n):
    a = np.random.default_rng(n).standard_normal(n) * 10.0 ** np.random.default_rng(n + 1).integers(-8, 8, n)
    assert O.pairwise_sum(a) == float(np.sum(a))


@pytest.mark.parametrize("sigma", [0.1, 0.7, 0.75, 0.85, 1.2, 2.0, 8.0 / 3.0])
@pytest.mark.parametrize("shape", [(23, 17), (11, 13, 9), (5, 40)])
def test_gaussian_is_scipy(sigma, shape):
    ndi = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(int(sigma * 100) + sum(shape))
    for a in (rng.random(shape), (rng.random(shape) < 0.3).astype(float)):
        assert same(O.gaussian_filter_wrap(a, sigma), ndi.gaussian_filter(a, sigma, mode="wrap"))


@pytest.mark.parametrize("shape", [(40, 37), (17, 19, 23)])
def test_components_and_dilation_are_scipy(shape):
    ndi = pytest.importorskip("scipy.ndimage")
    m = np.random.default_rng(len(shape)).random(shape) < 0.45
    cc, n = ndi.label(m)
    c2, n2 = O.face_components(m)
    assert n == n2 and np.array_equal(cc, c2)
    box = ndi.binary_dilation(m, structure=np.ones((3,) * m.ndim, bool), iterations=1, border_value=0)
    assert np.array_equal(O.dilate_box(m), box)


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_competitor_fraction_composition(z, name):
    p = params(z, name)
    mask, comp = O.neighbor_competitor(z[f"{name}_labels"])
    assert np.array_equal(mask, z[f"{name}_mask"]) and np.array_equal(comp, z[f"{name}_competitor"])
    fp = O.precip_fraction(z[f"{name}_labels"], z[f"{name}_alpha"], comp)
    assert same(fp, z[f"{name}_fprec"])
    cm = O.matrix_composition(z[f"{name}_ctot"], fp, p)
    assert same(cm, z[f"{name}_cm"])
    assert same(O.interface_matrix_composition(cm, fp, p), z[f"{name}_trace"])


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_diffusion(z, name):
    p = params(z, name)
    c, cm, sub = O.diffuse_conservative_subcycled(z[f"{name}_ctot"].copy(), z[f"{name}_fprec"], p,
                                                  float(z[f"{name}_dt"]))
    assert sub == int(z[f"{name}_substeps"])
    assert same(c, z[f"{name}_diffused"]) and same(cm, z[f"{name}_cm_last"])


@pytest.mark.parametrize("kind", ["grow", "shrink", "none"])
@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_partition_transfer(z, name, kind):
    p = params(z, name)
    c = z[f"{name}_ctot"].copy()
    O.conservative_partition_transfer(c, z[f"{name}_fprec"], z[f"{name}_pt_{kind}_new"], z[f"{name}_trace"], p)
    assert same(c, z[f"{name}_pt_{kind}_out"])


def test_oracle_partition_transfer_errors():
    p = O.AlCuParams()
    shape = (12, 10)
    old = np.zeros(shape)
    new = np.zeros(shape)
    new[5, 5] = 0.5  # half a cell of theta-prime from a field without Cu above equilibrium
    c = np.full(shape, -0.5)
    with pytest.raises(RuntimeError, match="insufficient matrix Cu"):
        O.conservative_partition_transfer(c, old, new, np.full(shape, p.c_matrix_eq), p)
    # everything becomes precipitate: no matrix left to draw from
    c = np.full(shape, 0.2)
    with pytest.raises(RuntimeError, match="empty matrix neighbourhood"):
        O.conservative_partition_transfer(c, np.full(shape, 0.5), np.ones(shape), np.full(shape, 0.01), p)


@pytest.mark.parametrize("sigma", [0.70, 1.2])
@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_gaussian_remap(z, name, sigma):
    lab = z[f"{name}_labels"].copy()
    al = z[f"{name}_alpha"].copy()
    n = O.conservative_gaussian_remap(lab, al, sigma)
    tag = f"{name}_cgr_{int(round(sigma * 100))}"
    assert n == int(z[f"{tag}_changed"])
    assert np.array_equal(lab, z[f"{tag}_labels"]) and same(al, z[f"{tag}_alpha"])


@pytest.mark.parametrize("sigma", [0.70, 1.2])
@pytest.mark.parametrize("name", ["2d", "3d", "rough_2d", "rough_3d"])
def test_oracle_balanced_remap(z, name, sigma):
    lab = z[f"{name}_labels"].copy()
    al = z[f"{name}_alpha"].copy()
    n = O.balanced_gaussian_remap(lab, al, sigma)
    tag = f"{name}_bgr_{int(round(sigma * 100))}"
    assert n == int(z[f"{tag}_changed"])
    assert np.array_equal(lab, z[f"{tag}_labels"]) and same(al, z[f"{tag}_alpha"])


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_topology_transactions(z, name):
    lab = z[f"{name}_labels"].copy()
    al = z[f"{name}_tx_alpha_in"].copy()
    d = O.commit_topology_transactions(lab, al, z[f"{name}_competitor"], z[f"{name}_tx_crossing"])
    assert d == int(z[f"{name}_tx_deferred"])
    assert np.array_equal(lab, z[f"{name}_tx_labels"]) and same(al, z[f"{name}_tx_alpha"])


def test_oracle_certificate_known_answers(z):
    names = sorted({k[5:-7] for k in z.files if k.startswith("topo_") and k.endswith("_labels")})
    assert len(names) >= 9
    for n in names:
        lab = z[f"topo_{n}_labels"]
        index = tuple(int(v) for v in z[f"topo_{n}_index"])
        counts = {int(v): int(np.count_nonzero(lab == v)) for v in np.unique(lab)}
        got = O.simple_relabel_local(lab.copy(), index, int(lab[index]), int(z[f"topo_{n}_new"]), counts)
        assert got == bool(z[f"topo_{n}_local"]), n


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_variant_fractions(z, name):
    got = O.variant_fraction_fields(z[f"{name}_labels"], z[f"{name}_vf_alpha"], z[f"{name}_competitor"])
    assert same(got, z[f"{name}_vf"])


def test_oracle_replays_the_reference_trajectory():
    """Every recorded call of the reference's driver, through the oracle."""
    import alcu_replay as R

    def p_of(params):
        return O.AlCuParams(dx=params["dx"], diffusivity=params["diffusivity"], c_matrix_eq=params["c_matrix_eq"],
                            c_theta=params["c_theta"], remap_sigma_cells=params["remap_sigma_cells"],
                            composition_extension_sigma_cells=params["composition_extension_sigma_cells"])

    impl = {
        "neighbor_competitor": lambda a, pr, z: (O.neighbor_competitor(a[0]), {}),
        "precip_fraction": lambda a, pr, z: ((O.precip_fraction(a[0], a[1], a[2]),), {}),
        "variant_fraction_fields": lambda a, pr, z: ((O.variant_fraction_fields(a[0], a[1], a[2]),), {}),
        "interface_matrix_composition": lambda a, pr, z: ((O.interface_matrix_composition(a[0], a[1], p_of(pr)),), {}),
        "diffuse_conservative_subcycled": lambda a, pr, z: (O.diffuse_conservative_subcycled(a[0], a[1], p_of(pr),
                                                                                              a[3]), {}),
        "conservative_partition_transfer": lambda a, pr, z: (
            (O.conservative_partition_transfer(a[0], a[1], a[2], a[3], p_of(pr)),), {0: a[0]}),
        "commit_topology_transactions": lambda a, pr, z: (
            (O.commit_topology_transactions(a[0], a[1], a[2], a[3]),), {0: a[0], 1: a[1]}),
        "conservative_gaussian_remap": lambda a, pr, z: (
            (O.conservative_gaussian_remap(a[0], a[1], a[2]),), {0: a[0], 1: a[1]}),
    }
    assert R.replay(impl) == 97
