"""CPU oracle of the Al-Cu material module's per-step transport and remap.

TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the CPU
baseline leg of the benchmark use this file; the product path
(gpk.alcu over the CUDA library) never does.

Restates, in numpy, the functions of the reference's
scripts/run_alcu_gpk_microstructure.py that move Cu and relabel cells once
per step:

  neighbor_competitor              lines 260-276
  precip_fraction                  lines 675-676
  variant_fraction_fields          lines 278-283
  matrix composition c_m           lines 680-682 (also 917-919)
  diffuse_conservative             lines 679-688
  diffuse_conservative_subcycled   lines 691-699
  conservative_partition_transfer  lines 702-737
  interface_matrix_composition     lines 740-755
  conservative_gaussian_remap      lines 562-594
  balanced_gaussian_remap          lines 597-672
  commit_topology_transactions     lines 526-559
  topology_simple_relabel          lines 464-523, with local_only=True (the
                                   form both callers above use), and its
                                   helpers _periodic_patch / _topological_number
                                   (lines 383-428)

with the reference's operand order, so that the results are bit-identical.
The reference calls two third-party pieces, both restated here from their
published algorithms and checked against the installed libraries by
tests/test_alcu_oracle.py:

  numpy 2.3 `np.sum` of a float64 array: pairwise summation over the
      flattened array (blocks of at most 128 values summed with 8 running
      partial sums, larger ranges split at half the length rounded down to a
      multiple of 8)                                          -> pairwise_sum
  scipy 1.18 `scipy.ndimage.gaussian_filter(a, sigma, mode="wrap")`: the
      normalised sampled Gaussian of radius int(4 sigma + 0.5) applied along
      axis 0, 1, 2 in turn; each output is x[i] w0 plus (x[i-j] + x[i+j]) w_j
      added from the outermost tap j = r inwards                 -> gaussian_filter_wrap
  scipy `label` (face connectivity, no wrap): components numbered by their
      first cell in C order                                   -> face_components
  scipy `binary_dilation` with the 3^d structure, border 0     -> dilate_box
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class AlCuParams:
    """The transport parameters of the reference's `Parameters` (lines 43-76)."""
    dx: float = 1.5e-9
    diffusivity: float = 1.66e-20
    c_matrix_eq: float = 3.7189506575706577e-4
    c_theta: float = 1.0 / 3.0
    remap_sigma_cells: float = 0.70
    composition_extension_sigma_cells: float = 0.75


# --------------------------------------------------------------------------
# library primitives
# --------------------------------------------------------------------------

def _pairwise_block(a: np.ndarray) -> float:
    n = a.size
    if n < 8:
        res = 0.0
        for v in a:
            res += float(v)
        return res
    r = a[:8].astype(np.float64).copy()
    i = 8
    while i < n - (n % 8):
        r += a[i:i + 8]
        i += 8
    res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]))
    while i < n:
        res += a[i]
        i += 1
    return float(res)


def pairwise_sum(a: np.ndarray) -> float:
    """numpy's float64 `np.sum(a)`: pairwise summation of a.ravel()."""
    flat = np.ascontiguousarray(a, dtype=np.float64).ravel()

    def rec(lo: int, n: int) -> float:
        if n <= 128:
            return _pairwise_block(flat[lo:lo + n])
        n2 = n // 2
        n2 -= n2 % 8
        return rec(lo, n2) + rec(lo + n2, n - n2)

    return rec(0, flat.size)


def gauss_weights(sigma: float, truncate: float = 4.0) -> np.ndarray:
    """The 2r+1 taps scipy samples for a Gaussian of width sigma (order 0)."""
    sd = float(sigma)
    radius = int(truncate * sd + 0.5)
    sigma2 = sigma * sigma
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / sigma2 * x ** 2)
    return phi / phi.sum()


def gaussian_filter_wrap(a: np.ndarray, sigma: float) -> np.ndarray:
    """scipy.ndimage.gaussian_filter(a, sigma, mode="wrap") in its operand order."""
    w = gauss_weights(sigma)
    r = (w.size - 1) // 2
    out = np.asarray(a, dtype=np.float64)
    for axis in range(out.ndim):
        acc = out * w[r]
        for j in range(r, 0, -1):
            acc = acc + (np.roll(out, j, axis=axis) + np.roll(out, -j, axis=axis)) * w[r + j]
        out = acc
    return out


def face_components(mask: np.ndarray) -> tuple[np.ndarray, int]:
    """Face-connected components of mask without wrap, numbered 1.. by their
    first cell in C order (0 off the mask)."""
    m = np.asarray(mask, dtype=bool)
    big = np.iinfo(np.int64).max
    lab = np.where(m, np.arange(m.size, dtype=np.int64).reshape(m.shape), big)
    while True:
        new = lab.copy()
        for axis in range(m.ndim):
            for step in (1, -1):
                sh = np.full_like(lab, big)
                src = [slice(None)] * m.ndim
                dst = [slice(None)] * m.ndim
                if step == 1:
                    src[axis] = slice(0, -1)
                    dst[axis] = slice(1, None)
                else:
                    src[axis] = slice(1, None)
                    dst[axis] = slice(0, -1)
                sh[tuple(dst)] = lab[tuple(src)]
                new = np.where(m, np.minimum(new, sh), big)
        if np.array_equal(new, lab):
            break
        lab = new
    roots = np.unique(lab[m])
    out = np.zeros(m.shape, dtype=np.int64)
    out[m] = np.searchsorted(roots, lab[m]) + 1
    return out, int(roots.size)


def dilate_box(mask: np.ndarray) -> np.ndarray:
    """One dilation by the full 3^d structure, border value 0 (no wrap)."""
    m = np.asarray(mask, dtype=bool)
    p = np.pad(m, 1, constant_values=False)
    out = np.zeros_like(m)
    for off in np.ndindex(*([3] * m.ndim)):
        sl = tuple(slice(o, o + n) for o, n in zip(off, m.shape))
        out |= p[sl]
    return out


# --------------------------------------------------------------------------
# the module's functions
# --------------------------------------------------------------------------

def neighbor_competitor(labels: np.ndarray):
    """Interface mask and competitor variant (lines 260-276)."""
    ndim = labels.ndim
    mask = np.zeros(labels.shape, dtype=bool)
    support = np.zeros((3,) + labels.shape, dtype=np.int16)
    matrix_neighbor = np.zeros(labels.shape, dtype=bool)
    for axis in range(ndim):
        for shift in (-1, 1):
            nb = np.roll(labels, shift, axis=axis)
            mask |= nb != labels
            matrix_neighbor |= nb == 0
            for v in (1, 2, 3):
                support[v - 1] += nb == v
    competitor = np.argmax(support, axis=0).astype(np.int8) + 1
    competitor[(labels > 0) & matrix_neighbor] = 0
    competitor[~mask] = labels[~mask]
    return mask, competitor


def precip_fraction(labels, alpha, competitor):
    """Local theta-prime fraction (lines 675-676)."""
    return np.where(labels > 0, alpha, np.where(competitor > 0, 1.0 - alpha, 0.0))


def variant_fraction_fields(labels, alpha, competitor):
    """One precipitate-fraction field per habit variant (lines 278-283)."""
    fraction = precip_fraction(labels, alpha, competitor)
    variant = np.where(labels > 0, labels, competitor)
    return np.asarray([fraction * (variant == v) for v in (1, 2, 3)])


def matrix_composition(ctot, fprec, p: AlCuParams):
    """c_m of the lever rule, clipped (lines 680-682)."""
    matrix = np.maximum(1.0 - fprec, 1e-8)
    cm = np.where(matrix > 1e-7, (ctot - fprec * p.c_theta) / matrix, p.c_matrix_eq)
    return np.clip(cm, 0.0, p.c_theta)


def diffuse_conservative(ctot, fprec, p: AlCuParams, dt: float):
    """One explicit conservative matrix-diffusion step (lines 679-688)."""
    matrix = np.maximum(1.0 - fprec, 1e-8)
    cm = np.where(matrix > 1e-7, (ctot - fprec * p.c_theta) / matrix, p.c_matrix_eq)
    cm = np.clip(cm, 0.0, p.c_theta)
    dc = np.zeros_like(ctot)
    for axis in range(ctot.ndim):
        mf = 0.5 * (matrix + np.roll(matrix, -1, axis=axis))
        flux_plus = -p.diffusivity * mf * (np.roll(cm, -1, axis=axis) - cm) / p.dx
        dc -= (flux_plus - np.roll(flux_plus, 1, axis=axis)) / p.dx
    return ctot + dt * dc, cm


def diffuse_conservative_subcycled(ctot, fprec, p: AlCuParams, dt: float):
    """Sub-cycled at 0.4 dx^2 / (2 ndim D) (lines 691-699)."""
    stable_dt = 0.4 * p.dx * p.dx / (2.0 * ctot.ndim * p.diffusivity)
    substeps = max(1, int(np.ceil(dt / stable_dt)))
    sub_dt = dt / substeps
    cm = None
    for _ in range(substeps):
        ctot, cm = diffuse_conservative(ctot, fprec, p, sub_dt)
    return ctot, cm, substeps


def conservative_partition_transfer(ctot, old_fraction, new_fraction, matrix_composition, p: AlCuParams) -> None:
    """Stefan partition transfer with exact Cu conservation (lines 702-737);
    ctot is updated in place.  Raises RuntimeError as the reference does."""
    delta_fraction = np.clip(new_fraction, 0.0, 1.0) - old_fraction
    transfer = delta_fraction * (p.c_theta - matrix_composition)
    total_transfer = pairwise_sum(transfer)
    ctot += transfer
    if abs(total_transfer) <= 1.0e-30:
        return
    matrix = np.clip(1.0 - new_fraction, 0.0, 1.0)
    weight = gaussian_filter_wrap(np.abs(transfer), p.composition_extension_sigma_cells) * matrix
    correction = -total_transfer
    if correction < 0.0:
        capacity = np.maximum(ctot - p.c_matrix_eq * matrix, 0.0)
        weight *= capacity
        if pairwise_sum(capacity) < -correction * (1.0 - 1.0e-12):
            raise RuntimeError("insufficient matrix Cu for partition transfer")
    weight_sum = pairwise_sum(weight)
    if weight_sum <= 0.0:
        raise RuntimeError("empty matrix neighbourhood for partition transfer")
    ctot += correction * weight / weight_sum
    residue = total_transfer + pairwise_sum(correction * weight / weight_sum)
    ctot.ravel()[int(np.argmax(weight))] -= residue


def interface_matrix_composition(cm, fprec, p: AlCuParams):
    """Gaussian trace of c_m over the matrix side (lines 740-755)."""
    matrix_fraction = np.clip(1.0 - fprec, 0.0, 1.0)
    sigma = p.composition_extension_sigma_cells
    numerator = gaussian_filter_wrap(cm * matrix_fraction, sigma)
    denominator = gaussian_filter_wrap(matrix_fraction, sigma)
    trace = numerator / np.maximum(denominator, 1.0e-12)
    return np.clip(trace, 0.0, p.c_theta)


def conservative_gaussian_remap(labels: np.ndarray, alpha: np.ndarray, sigma_cells: float) -> int:
    """Volume-conserving Gaussian relabelling of each component (lines 562-594);
    labels and alpha are updated in place; returns the changed-cell count."""
    original = labels.copy()
    remapped = labels.copy()
    for value in (int(v) for v in np.unique(original) if v != 0):
        cc, count = face_components(original == value)
        for component in range(1, count + 1):
            support = cc == component
            target = int(np.count_nonzero(support))
            if target <= 1:
                continue
            admissible = dilate_box(support)
            admissible &= (remapped == 0) | support
            score = gaussian_filter_wrap(support.astype(float), sigma_cells)
            candidates = np.flatnonzero(admissible)
            order = np.lexsort((candidates, -score.ravel()[candidates]))
            selected = candidates[order[:target]]
            remapped[support] = 0
            remapped.ravel()[selected] = value
    changed = remapped != labels
    labels[:] = remapped
    alpha[changed] = 1.0
    return int(np.count_nonzero(changed))


# --------------------------------------------------------------------------
# topology transactions and the balanced remap


def _periodic_patch(labels: np.ndarray, index: tuple) -> np.ndarray:
    axes = [np.asarray([(i - 1) % n, i, (i + 1) % n]) for i, n in zip(index, labels.shape)]
    return labels[np.ix_(*axes)]


def _topological_number(mask: np.ndarray) -> int:
    """Face-connected components of the 3^d patch (centre cleared) that touch
    a face neighbour of the centre."""
    nd = mask.ndim
    occupied = {tuple(int(v) for v in c) for c in np.argwhere(mask)}
    if not occupied:
        return 0
    offsets, incident = [], set()
    centre = (1,) * nd
    for axis in range(nd):
        for shift in (-1, 1):
            off = [0] * nd
            off[axis] = shift
            offsets.append(tuple(off))
            pos = list(centre)
            pos[axis] += shift
            incident.add(tuple(pos))
    count = 0
    unseen = set(occupied)
    while unseen:
        seed = unseen.pop()
        stack = [seed]
        touches = seed in incident
        while stack:
            pt = stack.pop()
            for off in offsets:
                nb = tuple(a + b for a, b in zip(pt, off))
                if nb in unseen:
                    unseen.remove(nb)
                    stack.append(nb)
                    touches |= nb in incident
        count += int(touches)
    return count


def simple_relabel_local(labels, index, old_label, new_label, label_counts) -> bool:
    """The local certificate of topology_simple_relabel(..., local_only=True)."""
    if old_label == new_label:
        return False
    patch = _periodic_patch(labels, index)
    centre = (1,) * labels.ndim
    old_object = patch == old_label
    old_object[centre] = False
    oc = _topological_number(old_object)
    extinction = label_counts.get(old_label, 0) <= 1
    if oc == 0 and not extinction:
        return False
    if oc > 1:
        return False
    new_object = patch == new_label
    new_object[centre] = False
    nc = _topological_number(new_object)
    if nc == 0 or nc > 1:
        return False
    return True


def commit_topology_transactions(labels, alpha, competitor, crossing) -> int:
    """Serial relabel of the crossing cells in C order (lines 526-559);
    labels and alpha in place; returns the deferred count."""
    if not np.any(crossing):
        return 0
    label_counts = {int(v): int(np.count_nonzero(labels == v)) for v in np.unique(labels)}
    deferred = 0
    for coordinate in np.argwhere(crossing):
        index = tuple(int(x) for x in coordinate)
        old_label = int(labels[index])
        new_label = int(competitor[index])
        if simple_relabel_local(labels, index, old_label, new_label, label_counts):
            labels[index] = new_label
            alpha[index] = 1.0
            label_counts[old_label] = label_counts.get(old_label, 0) - 1
            label_counts[new_label] = label_counts.get(new_label, 0) + 1
        else:
            deferred += 1
            alpha[index] = max(float(alpha[index]), 1.0e-6)
    return deferred


def balanced_gaussian_remap(labels: np.ndarray, alpha: np.ndarray, sigma_cells: float) -> int:
    """Volume-balanced exchange of the strongest opposite proposals per label
    pair of one phase class (lines 597-672); in place; changed-cell count."""
    values = np.unique(labels)
    scores = {int(v): gaussian_filter_wrap((labels == v).astype(float), sigma_cells) for v in values}
    interface = np.zeros(labels.shape, dtype=bool)
    candidates = {int(v): np.zeros(labels.shape, dtype=bool) for v in values}
    for axis in range(labels.ndim):
        for shift in (-1, 1):
            nb = np.roll(labels, shift, axis=axis)
            interface |= nb != labels
            for v in values:
                candidates[int(v)] |= nb == v
    proposals = {}
    flat_labels = labels.ravel()
    for flat in np.flatnonzero(interface):
        old = int(flat_labels[flat])
        old_score = float(scores[old].ravel()[flat])
        best, best_gain = old, 0.0
        for v in values:
            v = int(v)
            if v == old or not candidates[v].ravel()[flat]:
                continue
            gain = float(scores[v].ravel()[flat]) - old_score
            if gain > best_gain:
                best, best_gain = v, gain
        if best != old:
            proposals.setdefault((old, best), []).append((best_gain, int(flat)))
    changed = np.zeros(labels.size, dtype=bool)
    label_counts = {int(v): int(np.count_nonzero(labels == v)) for v in values}
    for ia, first in enumerate(values):
        for second in values[ia + 1:]:
            first, second = int(first), int(second)
            if (first == 0) != (second == 0):
                continue
            forward = sorted(proposals.get((first, second), ()), reverse=True)
            reverse = sorted(proposals.get((second, first), ()), reverse=True)
            for (_, ff), (_, fr) in zip(forward, reverse):
                index_f = np.unravel_index(ff, labels.shape)
                index_r = np.unravel_index(fr, labels.shape)
                if int(flat_labels[ff]) != first or int(flat_labels[fr]) != second:
                    continue
                if not simple_relabel_local(labels, index_f, first, second, label_counts):
                    continue
                flat_labels[ff] = second
                label_counts[first] -= 1
                label_counts[second] += 1
                if not simple_relabel_local(labels, index_r, second, first, label_counts):
                    flat_labels[ff] = first
                    label_counts[first] += 1
                    label_counts[second] -= 1
                    continue
                flat_labels[fr] = first
                label_counts[second] -= 1
                label_counts[first] += 1
                changed[ff] = True
                changed[fr] = True
    alpha.ravel()[changed] = 1.0
    return int(np.count_nonzero(changed))
