"""CPU oracle of the adjoint module's FP64 forward model (test infrastructure).

A numpy restatement of the loss that include/gpk_adjoint.h defines, for
checking the CUDA forward pass and, by central differences, its adjoint.
The geometry inputs (mask, phi_comp, normals, curvature) come from the
grid's geometry stage, which the step tests pin to the reference.  Pieces
restated: the plane-strain form of the spectral solve in
scripts/run_alcu_gpk_microstructure.py:99-190 (x the last array axis), the
elastic term of the velocity law src/gpk_physics.cpp:118-125, sigma(n, g) of
src/gpk_thermo.cpp:9-30 extended to four cos(4 m theta) terms, and the pair
projection src/gpk_physics.cpp:152-193.  Parity of the model itself is
unpinned: the reference has no such loss.
"""
from __future__ import annotations

import numpy as np


def elastic(eta, E, c11, c12, c44, dx):
    """Energy density and elastic strain of the eigenstrain field eta * E."""
    Ny, Nx = eta.shape
    ky = 2.0 * np.pi * np.fft.fftfreq(Ny, d=dx)[:, None] * np.ones((1, Nx))
    kx = 2.0 * np.pi * np.fft.fftfreq(Nx, d=dx)[None, :] * np.ones((Ny, 1))
    es = [eta * E[0], eta * E[1], eta * E[2]]
    h = [np.fft.fft2(f) for f in es]
    txx, tyy, txy = c11 * h[0] + c12 * h[1], c12 * h[0] + c11 * h[1], 2.0 * c44 * h[2]
    bx, by = kx * txx + ky * txy, kx * txy + ky * tyy
    a00, a11, a01 = c11 * kx * kx + c44 * ky * ky, c44 * kx * kx + c11 * ky * ky, (c12 + c44) * kx * ky
    origin = (kx == 0) & (ky == 0)
    det = np.where(origin, 1.0, a00 * a11 - a01 * a01)
    x0 = (a11 * bx - a01 * by) / det
    x1 = (a00 * by - a01 * bx) / det
    s = [kx * x0, ky * x1, 0.5 * (kx * x1 + ky * x0)]
    s[0] = np.where(origin, h[0], s[0])
    s[1] = np.where(origin, h[1], s[1])
    s[2] = np.where(origin, 0.0, s[2])
    de = [np.fft.ifft2(s[k]).real - es[k] for k in range(3)]
    sxx, syy, sxy = c11 * de[0] + c12 * de[1], c12 * de[0] + c11 * de[1], 2.0 * c44 * de[2]
    return 0.5 * (sxx * de[0] + syy * de[1] + 2.0 * sxy * de[2]), de


def forward(phi, comp, mask, nx, ny, kappa, g, mob_index, theta, c11, c12, c44, sigma0, m_fixed, wE, dx,
            target, radius, weight):
    """Loss and projected velocity (zero off the interface).  weight(r2) ->
    projection weight; all arrays 2-D (Ny, Nx)."""
    Ny, Nx = phi.shape
    E, a, M = theta[:3], theta[3:7], theta[7:]
    eta = (mob_index[phi] < 0).astype(np.float64)
    en, _ = elastic(eta, E, c11, c12, c44, dx)
    act = np.flatnonzero(mask.ravel())
    P, Q = phi.ravel(), comp.ravel()
    vr = np.zeros(Ny * Nx)
    for i in act:
        y, x = divmod(int(i), Nx)
        q = -1
        if Q[i] != P[i]:
            for j in (y * Nx + (x - 1) % Nx, y * Nx + (x + 1) % Nx, ((y - 1) % Ny) * Nx + x, ((y + 1) % Ny) * Nx + x):
                if P[j] == Q[i]:
                    q = j
                    break
        dE = en.ravel()[q] - en.ravel()[i] if q >= 0 else 0.0
        cg, sg = np.cos(g.ravel()[i]), np.sin(g.ravel()[i])
        ncx = nx.ravel()[i] * cg + ny.ravel()[i] * sg
        ncy = -nx.ravel()[i] * sg + ny.ravel()[i] * cg
        th = np.arctan2(ncy, ncx)
        sa = sigma0 * (1.0 + sum(a[m] * np.cos(4.0 * (m + 1) * th) for m in range(4)))
        p = mob_index[P[i]]
        vr[i] = (M[p] if p >= 0 else m_fixed) * (dE - sa * kappa.ravel()[i])
    v = np.zeros(Ny * Nx)
    mk = mask.ravel()
    for i in act:
        if P[i] == Q[i]:
            v[i] = vr[i]
            continue
        low, high = min(P[i], Q[i]), max(P[i], Q[i])
        y0, x0 = divmod(int(i), Nx)
        num = den = 0.0
        for dy in range(-radius, radius + 1):
            for dxs in range(-radius, radius + 1):
                j = ((y0 + dy) % Ny) * Nx + (x0 + dxs) % Nx
                if not mk[j] or P[j] == Q[j] or min(P[j], Q[j]) != low or max(P[j], Q[j]) != high:
                    continue
                w = weight(dxs * dxs + dy * dy)
                num += w * (1.0 if P[j] == low else -1.0) * vr[j]
                den += w
        v[i] = (1.0 if P[i] == low else -1.0) * (num / den)
    r = v[act] - target.ravel()[act]
    return 0.5 * float(np.sum(r * r)) + wE * float(np.sum(en)) * dx * dx, v.reshape(Ny, Nx)
