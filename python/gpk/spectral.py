"""FP64 spectral micro-elasticity on the GPU, called like the reference.

`spectral_elasticity(variant_fractions, p)` has the signature and return
values of the reference's Al-Cu material module
(scripts/run_alcu_gpk_microstructure.py:99-190): `p` carries `dx`, `c11`,
`c12`, `c44`, `eigen_small` and `eigen_large`; the result is
`(driving, energy, hydro, residual)`.  NumPy inputs give NumPy outputs (host
copies in and out); CUDA torch tensors stay on the device and run on torch's
current stream.  The solve itself is libgpk_b200.so (cuFFT transforms and
hand-written kernels); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gpk_b200._lib import check, lib


def variant_eigenstrains(eigen_small: float, eigen_large: float) -> np.ndarray:
    """Rows: x-, y-, z-normal plate variants; columns: xx, yy, zz."""
    s, q = float(eigen_small), float(eigen_large)
    return np.array([[q, s, s], [s, q, s], [s, s, q]], dtype=np.float64)


class SpectralElasticity:
    """One planned solve for a fixed field shape (2-D or 3-D)."""

    def __init__(self, shape, dx: float, c11: float, c12: float, c44: float, eig) -> None:
        shape = tuple(int(n) for n in shape)
        if len(shape) not in (2, 3):
            raise ValueError("shape must be 2-D or 3-D")
        self.shape = shape
        self._h = C.c_void_p()
        ext = (C.c_int * len(shape))(*shape)
        e = np.ascontiguousarray(eig, dtype=np.float64).reshape(9)
        check(lib().gpk_spectral_create(len(shape), ext, float(dx), float(c11), float(c12), float(c44),
                                        e.ctypes.data_as(C.POINTER(C.c_double)), C.byref(self._h)))

    def set_constants(self, dx: float, c11: float, c12: float, c44: float, eig) -> None:
        e = np.ascontiguousarray(eig, dtype=np.float64).reshape(9)
        check(lib().gpk_spectral_set_constants(self._h, float(dx), float(c11), float(c12), float(c44),
                                               e.ctypes.data_as(C.POINTER(C.c_double))))

    def close(self) -> None:
        if self._h:
            lib().gpk_spectral_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def couple(self, grid, matrix_label: int = 0, want_residual: bool = False):
        """Elastic energy density of the grid's current labels (variant 0 =
        every label but matrix_label) written into grid's E_el field, on the
        grid's stream; returns the residual when asked."""
        res = C.c_double(0.0)
        check(lib().gpk_spectral_couple_grid(self._h, grid._h, int(matrix_label),
                                             C.byref(res) if want_residual else None))
        return res.value if want_residual else None

    def device_bytes(self) -> int:
        cells, nb = C.c_int64(), C.c_int64()
        check(lib().gpk_spectral_info(self._h, C.byref(cells), C.byref(nb)))
        return nb.value

    def solve(self, fractions, want_residual: bool = True):
        """fractions: (3, *shape) float64, NumPy (host) or a CUDA torch tensor."""
        res = C.c_double(0.0)
        rp = C.byref(res) if want_residual else None
        if isinstance(fractions, np.ndarray):
            f = np.ascontiguousarray(fractions, dtype=np.float64)
            if f.shape != (3,) + self.shape:
                raise ValueError(f"fractions must have shape {(3,) + self.shape}")
            drv = np.empty_like(f)
            en = np.empty(self.shape)
            hy = np.empty(self.shape)
            check(lib().gpk_spectral_solve_host(self._h, f.ctypes.data, drv.ctypes.data, en.ctypes.data,
                                                hy.ctypes.data, rp))
            return drv, en, hy, (res.value if want_residual else None)
        import torch

        f = fractions.contiguous()
        if f.dtype != torch.float64 or not f.is_cuda or tuple(f.shape) != (3,) + self.shape:
            raise ValueError(f"fractions must be a CUDA float64 tensor of shape {(3,) + self.shape}")
        drv = torch.empty_like(f)
        en = torch.empty(self.shape, dtype=torch.float64, device=f.device)
        hy = torch.empty_like(en)
        check(lib().gpk_spectral_set_stream(self._h, C.c_void_p(torch.cuda.current_stream(f.device).cuda_stream)))
        check(lib().gpk_spectral_solve(self._h, f.data_ptr(), drv.data_ptr(), en.data_ptr(), hy.data_ptr(), rp))
        return drv, en, hy, (res.value if want_residual else None)


_cache: dict = {}


def spectral_elasticity(variant_fractions, p):
    """Drop-in for the reference's `spectral_elasticity(variant_fractions, p)`."""
    shape = tuple(variant_fractions.shape[1:])
    eig = variant_eigenstrains(p.eigen_small, p.eigen_large)
    key = shape
    s = _cache.get(key)
    if s is None:
        s = _cache[key] = SpectralElasticity(shape, p.dx, p.c11, p.c12, p.c44, eig)
    else:
        s.set_constants(p.dx, p.c11, p.c12, p.c44, eig)
    return s.solve(variant_fractions)
