"""Generates tests/golden/alcu_transport.npz from the reference itself.

Imports the per-step transport and remap functions of the reference's Al-Cu
material module, scripts/run_alcu_gpk_microstructure.py:

  neighbor_competitor (260-276), variant_fraction_fields (278-283),
  precip_fraction (675-676),
  diffuse_conservative_subcycled (679-699),
  conservative_partition_transfer (702-737),
  interface_matrix_composition (740-755),
  conservative_gaussian_remap (562-594), balanced_gaussian_remap (597-672),
  commit_topology_transactions (526-559), topology_simple_relabel (464-523),

and runs them on seeded states shaped like the module's own: int8 labels
0..3 (alpha-Al and three theta-prime variants) with plates and spheres, one
crossing a periodic face (scipy's `label` splits it there), two touching
plates of different variants, single-cell specks and jagged interfaces as
left by committed crossings.  Run it where the reference tree is present:

    python tests/golden/make_alcu_golden.py [path/to/reference]
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "alcu_transport.npz")


def load_reference(root: str):
    path = os.path.join(root, "scripts", "run_alcu_gpk_microstructure.py")
    spec = importlib.util.spec_from_file_location("gpk_ref_alcu", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpk_ref_alcu"] = mod
    spec.loader.exec_module(mod)
    return mod


def ellipsoid(labels, centre, axes, value):
    shape = labels.shape
    coords = np.indices(shape)
    d2 = 0.0
    for a in range(len(shape)):
        delta = np.abs(coords[a] - centre[a])
        delta = np.minimum(delta, shape[a] - delta)  # minimum image
        d2 = d2 + (delta / axes[a]) ** 2
    labels[d2 <= 1.0] = value


def make_labels(shape, rng):
    labels = np.zeros(shape, dtype=np.int8)
    nd = len(shape)
    big = max(shape) / 5.0
    if nd == 2:
        ellipsoid(labels, (shape[0] // 4, shape[1] // 4), (big, big / 4), 1)
        ellipsoid(labels, (0, shape[1] // 2), (big / 3, big), 2)            # crosses axis-0 face
        ellipsoid(labels, (3 * shape[0] // 4, 2 * shape[1] // 3), (big / 1.5, big / 1.5), 1)
        # two touching plates of different variants
        labels[shape[0] // 2:shape[0] // 2 + 3, 4:16] = 2
        labels[shape[0] // 2 + 3:shape[0] // 2 + 5, 6:14] = 1
    else:
        ellipsoid(labels, (shape[0] // 4, shape[1] // 4, shape[2] // 4), (big / 4, big, big), 1)
        ellipsoid(labels, (shape[0] // 2, 0, shape[2] // 2), (big, big / 4, big), 2)  # crosses axis-1 face
        ellipsoid(labels, (3 * shape[0] // 4, 2 * shape[1] // 3, 3 * shape[2] // 4), (big, big, big / 4), 3)
        labels[2:5, shape[1] // 2:shape[1] // 2 + 6, 2:8] = 2
        labels[5:7, shape[1] // 2 + 1:shape[1] // 2 + 5, 3:7] = 3
    # jagged interfaces: random flips across matrix/precipitate faces
    for _ in range(2):
        nb_lab = np.zeros_like(labels)
        for axis in range(nd):
            for s in (-1, 1):
                r = np.roll(labels, s, axis=axis)
                nb_lab = np.where((nb_lab == 0) & (r > 0), r, nb_lab)
        grow = (labels == 0) & (nb_lab > 0) & (rng.random(shape) < 0.25)
        labels[grow] = nb_lab[grow]
        has_matrix = np.zeros(shape, dtype=bool)
        for axis in range(nd):
            for s in (-1, 1):
                has_matrix |= np.roll(labels, s, axis=axis) == 0
        shrink = (labels > 0) & has_matrix & (rng.random(shape) < 0.15)
        labels[shrink] = 0
    # isolated specks (components of one cell are left alone by the remap)
    for _ in range(4):
        idx = tuple(int(rng.integers(0, n)) for n in shape)
        labels[idx] = int(rng.integers(1, 4 if nd == 3 else 3))
    return labels


def make_state(shape, rng, ref, p):
    labels = make_labels(shape, rng)
    alpha = np.ones(shape)
    mask, comp = ref.neighbor_competitor(labels)
    alpha[mask] = rng.uniform(0.05, 1.0, size=int(mask.sum()))
    precip = labels > 0
    f0 = float(np.mean(precip))
    cm0 = (p.c0 - f0 * p.c_theta) / (1.0 - f0)
    ctot = np.full(shape, cm0) * (1.0 + 0.05 * rng.standard_normal(shape))
    ctot[precip] = p.c_theta
    return labels, alpha, ctot


def main(root: str) -> None:
    ref = load_reference(root)
    rng = np.random.default_rng(20240611)
    out = {}
    cases = [("2d", (64, 60), 0.5e-9), ("3d", (24, 26, 22), 1.5e-9)]
    for name, shape, dx in cases:
        p = ref.Parameters()
        p.dx = dx
        labels, alpha, ctot = make_state(shape, rng, ref, p)
        mask, comp = ref.neighbor_competitor(labels)
        fp = ref.precip_fraction(labels, alpha, comp)
        al_neg = alpha.copy()
        al_neg[mask & (rng.random(shape) < 0.2)] *= -1.0  # crossing cells carry alpha < 0
        out[f"{name}_vf_alpha"] = al_neg
        out[f"{name}_vf"] = ref.variant_fraction_fields(labels, al_neg, comp)
        matrix = np.maximum(1.0 - fp, 1e-8)
        cm = np.where(matrix > 1e-7, (ctot - fp * p.c_theta) / matrix, p.c_matrix_eq)
        cm = np.clip(cm, 0.0, p.c_theta)
        trace = ref.interface_matrix_composition(cm, fp, p)
        dt = 10.0
        c_new, cm_last, substeps = ref.diffuse_conservative_subcycled(ctot.copy(), fp, p, dt)
        out.update({f"{name}_labels": labels, f"{name}_alpha": alpha, f"{name}_ctot": ctot,
                    f"{name}_dx": np.float64(dx), f"{name}_dt": np.float64(dt),
                    f"{name}_mask": mask, f"{name}_competitor": comp, f"{name}_fprec": fp,
                    f"{name}_cm": cm, f"{name}_trace": trace, f"{name}_diffused": c_new,
                    f"{name}_cm_last": cm_last, f"{name}_substeps": np.int64(substeps)})
        # partition transfer: growth (correction < 0, capacity branch),
        # dissolution (correction > 0) and no change (early return)
        for kind in ("grow", "shrink", "none"):
            step = np.zeros(shape)
            if kind == "grow":
                step[mask] = rng.uniform(0.0, 0.3, size=int(mask.sum()))
            elif kind == "shrink":
                step[mask] = -rng.uniform(0.0, 0.3, size=int(mask.sum()))
            new_fp = np.clip(fp + step, -0.2, 1.2)
            c = ctot.copy()
            ref.conservative_partition_transfer(c, fp, new_fp, trace, p)
            out[f"{name}_pt_{kind}_new"] = new_fp
            out[f"{name}_pt_{kind}_out"] = c
        for sigma in (0.70, 1.2):
            lab = labels.copy()
            al = alpha.copy()
            n = ref.conservative_gaussian_remap(lab, al, sigma)
            tag = f"{name}_cgr_{int(round(sigma * 100))}"
            out[f"{tag}_labels"] = lab
            out[f"{tag}_alpha"] = al
            out[f"{tag}_changed"] = np.int64(n)
            lab = labels.copy()
            al = alpha.copy()
            n = ref.balanced_gaussian_remap(lab, al, sigma)
            tag = f"{name}_bgr_{int(round(sigma * 100))}"
            out[f"{tag}_labels"] = lab
            out[f"{tag}_alpha"] = al
            out[f"{tag}_changed"] = np.int64(n)
        # crossing commits on a random 40% of the interface cells
        crossing = mask & (rng.random(shape) < 0.4)
        lab = labels.copy()
        al = alpha.copy()
        al[crossing] = -rng.uniform(0.0, 0.2, int(crossing.sum()))
        al_in = al.copy()
        deferred = ref.commit_topology_transactions(lab, al, comp, crossing)
        out.update({f"{name}_tx_crossing": crossing, f"{name}_tx_alpha_in": al_in, f"{name}_tx_labels": lab,
                    f"{name}_tx_alpha": al, f"{name}_tx_deferred": np.int64(deferred)})
    # balanced remap on rough boundaries between variants (proposals both ways)
    for name, shape in (("rough_2d", (48, 50)), ("rough_3d", (20, 22, 18))):
        nd = len(shape)
        coords = np.indices(shape)
        wobble = rng.integers(-2, 3, size=shape[1:])
        lab = np.where(coords[0] < shape[0] // 2 + wobble[None], 1, 2).astype(np.int8)
        if nd == 3:
            lab[(coords[2] > shape[2] * 2 // 3 + rng.integers(-1, 2, size=shape))] = 3
        flip = rng.random(shape) < 0.06
        lab[flip] = rng.integers(1, 4 if nd == 3 else 3, size=int(flip.sum()))
        lab[:, :2] = 0  # a matrix strip: its pairs with the variants are not exchanged
        alpha = rng.uniform(0.1, 1.0, shape)
        out[f"{name}_labels"] = lab
        out[f"{name}_alpha"] = alpha
        for sigma in (0.70, 1.2):
            l2 = lab.copy()
            a2 = alpha.copy()
            n = ref.balanced_gaussian_remap(l2, a2, sigma)
            tag = f"{name}_bgr_{int(round(sigma * 100))}"
            out[f"{tag}_labels"] = l2
            out[f"{tag}_alpha"] = a2
            out[f"{tag}_changed"] = np.int64(n)
    # canonical certificate configurations, with the reference's verdicts in
    # its local form (used by both callers) and its global form
    topo = []
    a = np.zeros((9, 9), np.int8); a[:, :5] = 1
    topo.append(("smooth_2d", a, (4, 4), 0))
    a = np.zeros((11, 11), np.int8); a[3:8, 2:5] = 1; a[3:8, 6:9] = 1; a[5, 5] = 1
    topo.append(("split_2d", a, (5, 5), 0))
    a = np.zeros((9, 9), np.int8); a[4, 3] = 1; a[4, 5] = 1
    topo.append(("merge_2d", a, (4, 4), 1))
    a = np.zeros((9, 9), np.int8); a[4, 4] = 1
    topo.append(("extinct_2d", a, (4, 4), 0))
    a = np.zeros((9, 9), np.int8); a[2:7, 2] = 1; a[2:7, 6] = 1; a[2, 2:7] = 1; a[6, 2:7] = 1
    topo.append(("ring_2d", a, (2, 4), 0))
    a = np.zeros((9, 9, 9), np.int8); a[3:6, 3:6, 1:4] = 2; a[3:6, 3:6, 5:8] = 2; a[4, 4, 4] = 2
    topo.append(("split_3d", a, (4, 4, 4), 0))
    a = np.zeros((7, 7, 7), np.int8); a[3, 3, 3] = 3
    topo.append(("extinct_3d", a, (3, 3, 3), 0))
    a = np.zeros((8, 8, 8), np.int8); a[2:6, 2:6, 2:6] = 1
    topo.append(("corner_3d", a, (2, 2, 2), 0))
    a = np.zeros((2, 5), np.int8); a[:, 2:] = 2
    topo.append(("narrow_2d", a, (0, 2), 0))
    for tname, lab, index, new in topo:
        counts = {int(v): int(np.count_nonzero(lab == v)) for v in np.unique(lab)}
        local = ref.topology_simple_relabel(lab.copy(), index, int(lab[index]), new, counts, local_only=True)
        glob = ref.topology_simple_relabel(lab.copy(), index, int(lab[index]), new, counts, local_only=False)
        out[f"topo_{tname}_labels"] = lab
        out[f"topo_{tname}_index"] = np.asarray(index, dtype=np.int64)
        out[f"topo_{tname}_new"] = np.int64(new)
        out[f"topo_{tname}_local"] = np.bool_(local)
        out[f"topo_{tname}_global"] = np.bool_(glob)
    # the taps scipy sampled in this process (numpy's exp), for callers whose
    # numpy rounds exp differently
    for sigma in (0.70, 0.75, 1.2):
        r = int(4.0 * sigma + 0.5)
        x = np.arange(-r, r + 1)
        phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
        out[f"taps_{int(round(sigma * 100))}"] = phi / phi.sum()
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, {k: v.shape for k, v in out.items() if np.ndim(v)})


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPK_REFERENCE")
    if not _ref:
        sys.exit("usage: python %s <path to the reference checkout> (or set GPK_REFERENCE)" % sys.argv[0])
    main(_ref)
