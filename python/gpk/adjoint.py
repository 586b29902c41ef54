"""Gradients of an interface-velocity loss at a fixed label map.

`AdjointProblem` wraps the FP64 forward model and its hand-written discrete
adjoint in libgpk_b200.so (include/gpk_adjoint.h): eigenstrain (E_xx, E_yy,
E_xy) of the precipitate labels through a plane-strain spectral elastic
solve, interface velocities v = M_l (e(q) - e(i) - sigma_a(n, g) kappa) with
four anisotropy coefficients a_m and one mobility per grain, the reference's
pair projection, and the loss 1/2 |v - v*|^2 + w_E sum e dx^2.

The torch.autograd.Function over it is `gpk.autograd.GPKLoss`.  The
reference has no adjoint: the gradients are checked against FP64 central
differences of the forward.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gpk_b200._lib import check, lib


class AdjointProblem:
    """grid: a 2-D float64 GPKGrid holding the labels and orientations g.
    mob_index[l]: mobility-parameter index of label l, or -1 for a
    precipitate label (eigenstrain carrier, fixed mobility m_fixed)."""

    def __init__(self, grid, mob_index, n_mob: int, m_fixed: float = 1.0, sigma0: float = 1.0,
                 c11: float = 1.08, c12: float = 0.62, c44: float = 0.28, energy_weight: float = 1.0) -> None:
        self.grid = grid
        mi = np.ascontiguousarray(mob_index, dtype=np.int32)
        self.n_mob = int(n_mob)
        self._h = C.c_void_p()
        check(lib().gpk_adjoint_create(grid._h, len(mi), mi.ctypes.data_as(C.POINTER(C.c_int32)), self.n_mob,
                                       float(m_fixed), float(sigma0), float(c11), float(c12), float(c44),
                                       float(energy_weight), C.byref(self._h)))
        grid.attach(self)  # the grid closes this handle first if it goes away first
        self.shape = (grid.Ny, grid.Nx)

    @property
    def num_params(self) -> int:
        return 7 + self.n_mob

    def _theta(self, theta) -> np.ndarray:
        t = np.ascontiguousarray(theta, dtype=np.float64)
        if t.shape != (self.num_params,):
            raise ValueError(f"theta must have {self.num_params} entries")
        return t

    def set_target(self, v_target) -> None:
        v = np.ascontiguousarray(v_target, dtype=np.float64).reshape(self.shape)
        check(lib().gpk_adjoint_set_target(self._h, v.ctypes.data_as(C.POINTER(C.c_double))))

    def forward(self, theta, want_v: bool = False):
        t = self._theta(theta)
        loss = C.c_double()
        v = np.zeros(self.shape) if want_v else None
        check(lib().gpk_adjoint_forward(self._h, t.ctypes.data_as(C.POINTER(C.c_double)), C.byref(loss),
                                        v.ctypes.data_as(C.POINTER(C.c_double)) if want_v else None))
        return (loss.value, v) if want_v else loss.value

    def gradient(self, theta):
        t = self._theta(theta)
        loss = C.c_double()
        g = np.empty(self.num_params)
        check(lib().gpk_adjoint_gradient(self._h, t.ctypes.data_as(C.POINTER(C.c_double)), C.byref(loss),
                                         g.ctypes.data_as(C.POINTER(C.c_double))))
        return loss.value, g

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            self._h = C.c_void_p()
            lib().gpk_adjoint_destroy(h)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def calibration_case(n: int = 512, grains: int = 256, precipitates: int = 64, seed: int = 11,
                     r_range=(6, 20)):
    """2-D periodic polycrystal of `grains` Voronoi grains (labels 1..grains,
    random orientations) carrying `precipitates` circular particles of radius
    U[r_range] (labels grains+1..grains+precipitates, orientation 0).
    Returns (phi, g, mob_index) with mob_index[l] = l - 1 for grains and -1
    for precipitates."""
    from gpk_b200.grid import voronoi
    phi, g = voronoi(1, n, n, grains, seed)
    g = g.astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    yy, xx = np.indices((n, n))
    for k in range(precipitates):
        cy, cx = rng.uniform(0, n, size=2)
        r = rng.uniform(*r_range)
        dy = (yy - cy + n / 2) % n - n / 2
        dx = (xx - cx + n / 2) % n - n / 2
        inside = dy * dy + dx * dx <= r * r
        phi[0][inside] = grains + 1 + k
        g[0][inside] = 0.0
    mob_index = np.full(grains + precipitates + 1, -1, dtype=np.int32)
    mob_index[1:grains + 1] = np.arange(grains, dtype=np.int32)
    mob_index[0] = 0
    return phi, g, mob_index
