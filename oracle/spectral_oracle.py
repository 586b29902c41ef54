"""CPU oracle for the spectral micro-elasticity solve (test infrastructure only).

A numpy restatement of `spectral_elasticity` in the reference's
scripts/run_alcu_gpk_microstructure.py:99-190: periodic Fourier solution of
div(C : (eps - eps*)) = 0 for a homogeneous cubic solid (C11, C12, C44)
holding three tetragonal eigenstrain variants.  Only tests and the bench's CPU
baseline use it; the product path is the CUDA solve in gpk_b200/csrc.

Pinned against tests/golden/spectral_elasticity.npz, which the reference's
own function produced (tests/golden/make_spectral_golden.py).

Steps (reference line numbers in brackets):
  eps*_j = sum_v eig[v, j] * f_v                              [106-111]
  k_a = 2 pi fftfreq(n_a, dx) on each array axis, 0 beyond ndim  [113-118]
  A_il = C_ijkl k_j k_k (cubic), identity at k = 0             [123-132]
  b_i = k_i (C11 e*_i + C12 (e*_others)), zero at k = 0         [134-139]
  u = -i A^-1 b;  e_ij = (i/2)(k_i u_j + k_j u_i)               [140-148]
  e_normal(k=0) = e*_normal(k=0)  (free mean expansion)         [151-153]
  strain = Re ifft(e); stress = C : (strain - eps*)             [154-167]
  energy = stress : (strain - eps*) / 2; driving_v = -stress : eig_v;
  hydrostatic = trace(stress) / 3; residual = rms|k . stress^| / rms|b|  [168-188]
"""
from __future__ import annotations

import numpy as np


def variant_eigenstrains(eigen_small: float, eigen_large: float) -> np.ndarray:
    """Rows: x-, y-, z-normal plate variants; columns: xx, yy, zz (reference
    lines 93-96)."""
    s, q = eigen_small, eigen_large
    return np.array([[q, s, s], [s, q, s], [s, s, q]], dtype=np.float64)


def solve(fractions: np.ndarray, dx: float, c11: float, c12: float, c44: float,
          eig: np.ndarray):
    """fractions: (3, *shape) float64, shape 2-D or 3-D.  Returns
    (driving (3, *shape), energy, hydrostatic, residual)."""
    f = np.asarray(fractions, dtype=np.float64)
    shape = f.shape[1:]
    nd = len(shape)
    if nd not in (2, 3) or f.shape[0] != 3:
        raise ValueError("fractions must have shape (3, n0, n1[, n2])")
    estar = np.zeros((3,) + shape)
    for v in range(3):
        for j in range(3):
            estar[j] += eig[v, j] * f[v]

    grids = np.meshgrid(*[2.0 * np.pi * np.fft.fftfreq(n, d=dx) for n in shape], indexing="ij")
    kv = [grids[a] if a < nd else np.zeros(shape) for a in range(3)]
    origin = (kv[0] == 0) & (kv[1] == 0) & (kv[2] == 0)

    eh = [np.fft.fftn(estar[j]) for j in range(3)]
    cs = c12 + c44
    acoustic = np.empty(shape + (3, 3))
    for i in range(3):
        o1, o2 = [a for a in range(3) if a != i]
        acoustic[..., i, i] = c11 * kv[i] * kv[i] + c44 * (kv[o1] * kv[o1] + kv[o2] * kv[o2])
    for i, j in ((0, 1), (0, 2), (1, 2)):
        acoustic[..., i, j] = acoustic[..., j, i] = cs * kv[i] * kv[j]
    acoustic[origin] = np.eye(3)

    rhs = np.empty(shape + (3,), dtype=np.complex128)
    for i in range(3):
        o1, o2 = [a for a in range(3) if a != i]
        rhs[..., i] = kv[i] * (c11 * eh[i] + c12 * (eh[o1] + eh[o2]))
    rhs[origin] = 0.0
    u = -1j * np.linalg.solve(acoustic, rhs[..., None])[..., 0]

    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]  # xx yy zz xy xz yz
    strain_h = []
    for i, j in pairs:
        if i == j:
            strain_h.append(1j * kv[i] * u[..., i])
        else:
            strain_h.append(0.5j * (kv[i] * u[..., j] + kv[j] * u[..., i]))
    for i in range(3):
        strain_h[i][origin] = eh[i][origin]
    strain = [np.fft.ifftn(s).real for s in strain_h]

    de = [strain[m] - estar[m] if m < 3 else strain[m] for m in range(6)]
    sig = [None] * 6
    for i in range(3):
        o1, o2 = [a for a in range(3) if a != i]
        sig[i] = c11 * de[i] + c12 * (de[o1] + de[o2])
    for m in range(3, 6):
        sig[m] = 2.0 * c44 * de[m]
    energy = 0.5 * (sig[0] * de[0] + sig[1] * de[1] + sig[2] * de[2]
                    + 2.0 * (sig[3] * de[3] + sig[4] * de[4] + sig[5] * de[5]))
    driving = np.stack([-(sig[0] * eig[v, 0] + sig[1] * eig[v, 1] + sig[2] * eig[v, 2]) for v in range(3)])
    hydro = (sig[0] + sig[1] + sig[2]) / 3.0

    dh = [strain_h[i] - eh[i] for i in range(3)]
    sh = [None] * 6
    for i in range(3):
        o1, o2 = [a for a in range(3) if a != i]
        sh[i] = c11 * dh[i] + c12 * (dh[o1] + dh[o2])
    for m in range(3, 6):
        sh[m] = 2.0 * c44 * strain_h[m]
    # rows of the symmetric stress in Voigt order: (xx xy xz), (xy yy yz), (xz yz zz)
    rows = ((0, 3, 4), (3, 1, 5), (4, 5, 2))
    r2 = sum(np.abs(kv[0] * sh[a] + kv[1] * sh[b] + kv[2] * sh[c]) ** 2 for a, b, c in rows)
    num = np.sqrt(np.mean(r2))
    den = np.sqrt(np.mean(np.sum(np.abs(rhs) ** 2, axis=-1)))
    return driving, energy, hydro, float(num / max(den, 1e-30))


def spectral_elasticity(variant_fractions: np.ndarray, p):
    """Same call as the reference: `p` carries dx, c11, c12, c44,
    eigen_small and eigen_large."""
    return solve(variant_fractions, p.dx, p.c11, p.c12, p.c44,
                 variant_eigenstrains(p.eigen_small, p.eigen_large))
