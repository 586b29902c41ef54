"""Al-Cu per-step Cu transport and Gaussian label remap on the GPU.

The module-level functions have the names, arguments, return values and
in-place behaviour of the reference's Al-Cu material module
(scripts/run_alcu_gpk_microstructure.py):

  neighbor_competitor(labels)                                     260-276
  precip_fraction(labels, alpha, competitor)                      675-676
  variant_fraction_fields(labels, alpha, competitor)              278-283
  diffuse_conservative_subcycled(ctot, fprec, p, dt)              691-699
  conservative_partition_transfer(ctot, old, new, c_m, p)         702-737
  interface_matrix_composition(cm, fprec, p)                      740-755
  conservative_gaussian_remap(labels, alpha, sigma_cells)         562-594
  balanced_gaussian_remap(labels, alpha, sigma_cells)             597-672
  commit_topology_transactions(labels, alpha, competitor, crossing) 526-559

`p` is any object with the reference's `Parameters` fields (dx, diffusivity,
c_matrix_eq, c_theta, composition_extension_sigma_cells).  NumPy inputs give
NumPy outputs (host copies in and out; in-place arguments are written back);
CUDA torch tensors stay on the device and run on torch's current stream.
Results are bit-identical to the reference's: the work is libgpk_b200.so
(include/gpk_alcu.h); there is no CPU path.  The Gaussian taps are computed
here with numpy, exactly as scipy computes them, so that they carry numpy's
exp bits.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gpk_b200._lib import CAlCuParams, check, lib

__all__ = ["AlCuTransport", "gauss_taps", "neighbor_competitor", "precip_fraction", "variant_fraction_fields",
           "matrix_composition",
           "diffuse_conservative_subcycled", "conservative_partition_transfer", "interface_matrix_composition",
           "conservative_gaussian_remap", "balanced_gaussian_remap", "commit_topology_transactions", "field_sum"]


def gauss_taps(sigma: float, truncate: float = 4.0) -> np.ndarray:
    """scipy.ndimage's sampled, normalised Gaussian of width sigma (order 0):
    radius int(truncate sigma + 0.5), exp(-0.5 / sigma^2 x^2) / sum."""
    sd = float(sigma)
    radius = int(truncate * sd + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return np.ascontiguousarray(phi / phi.sum(), dtype=np.float64)


def _params(p) -> CAlCuParams:
    return CAlCuParams(float(p.dx), float(p.diffusivity), float(p.c_matrix_eq), float(p.c_theta))


def _taps_arg(sigma):
    """sigma: a width (taps computed as scipy does) or the taps themselves."""
    if np.ndim(sigma) == 0:
        t = gauss_taps(float(sigma))
    else:
        t = np.ascontiguousarray(sigma, dtype=np.float64)
        if t.ndim != 1 or t.size % 2 == 0:
            raise ValueError("taps must be a 1-D array of odd length")
    return t, t.ctypes.data_as(C.POINTER(C.c_double)), (t.size - 1) // 2


class AlCuTransport:
    """Device buffers and launches for one field shape (2-D or 3-D).

    Every method takes CUDA torch tensors (float64 fields, int8 labels) of
    the handle's shape and runs on torch's current stream.  A `sigma`
    argument is a Gaussian width or an explicit array of 2r+1 taps."""

    def __init__(self, shape, p) -> None:
        shape = tuple(int(n) for n in shape)
        if len(shape) not in (2, 3):
            raise ValueError("shape must be 2-D or 3-D")
        self.shape = shape
        self._h = C.c_void_p()
        ext = (C.c_int * len(shape))(*shape)
        prm = _params(p)
        check(lib().gpk_alcu_create(len(shape), ext, C.byref(prm), C.byref(self._h)))

    def set_params(self, p) -> None:
        prm = _params(p)
        check(lib().gpk_alcu_set_params(self._h, C.byref(prm)))

    def close(self) -> None:
        if self._h:
            lib().gpk_alcu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        v = [C.c_int64() for _ in range(5)]
        check(lib().gpk_alcu_info(self._h, *[C.byref(x) for x in v]))
        return dict(cells=v[0].value, device_bytes=v[1].value, components=v[2].value, waves=v[3].value,
                    pairs=v[4].value)

    # ---- helpers
    def _bind(self, *tensors) -> None:
        import torch

        dev = None
        for t in tensors:
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise ValueError("expected contiguous CUDA tensors")
            if tuple(t.shape) != self.shape:
                raise ValueError(f"expected shape {self.shape}, got {tuple(t.shape)}")
            dev = t.device
        check(lib().gpk_alcu_set_stream(self._h, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))

    @staticmethod
    def _f64(t):
        import torch

        if t.dtype != torch.float64:
            raise ValueError("expected a float64 tensor")
        return t.data_ptr()

    @staticmethod
    def _i8(t):
        import torch

        if t.dtype != torch.int8:
            raise ValueError("expected an int8 label tensor")
        return t.data_ptr()

    # ---- the module's functions on device tensors
    def competitor(self, labels):
        import torch

        self._bind(labels)
        mask = torch.empty(self.shape, dtype=torch.uint8, device=labels.device)
        comp = torch.empty(self.shape, dtype=torch.int8, device=labels.device)
        check(lib().gpk_alcu_competitor(self._h, self._i8(labels), mask.data_ptr(), comp.data_ptr()))
        return mask.bool(), comp

    def precip_fraction(self, labels, alpha, competitor):
        import torch

        self._bind(labels, alpha, competitor)
        fp = torch.empty(self.shape, dtype=torch.float64, device=alpha.device)
        check(lib().gpk_alcu_precip_fraction(self._h, self._i8(labels), self._f64(alpha), self._i8(competitor),
                                             fp.data_ptr()))
        return fp

    def variant_fractions(self, labels, alpha, competitor):
        """(3, *shape) float64: the spectral solve's input."""
        import torch

        self._bind(labels, alpha, competitor)
        out = torch.empty((3,) + self.shape, dtype=torch.float64, device=alpha.device)
        check(lib().gpk_alcu_variant_fractions(self._h, self._i8(labels), self._f64(alpha), self._i8(competitor),
                                               out.data_ptr()))
        return out

    def matrix_composition(self, ctot, fprec):
        import torch

        self._bind(ctot, fprec)
        cm = torch.empty_like(ctot)
        check(lib().gpk_alcu_matrix_composition(self._h, self._f64(ctot), self._f64(fprec), cm.data_ptr()))
        return cm

    def diffuse(self, ctot, fprec, dt: float):
        """ctot advanced in place; returns (cm of the last substep, substeps)."""
        import torch

        self._bind(ctot, fprec)
        cm = torch.empty_like(ctot)
        n = C.c_int(0)
        check(lib().gpk_alcu_diffuse(self._h, self._f64(ctot), self._f64(fprec), float(dt), cm.data_ptr(),
                                     C.byref(n)))
        return cm, n.value

    def partition_transfer(self, ctot, old_fraction, new_fraction, matrix_composition, sigma) -> None:
        self._bind(ctot, old_fraction, new_fraction, matrix_composition)
        t, tp, r = _taps_arg(sigma)
        check(lib().gpk_alcu_partition_transfer(self._h, self._f64(ctot), self._f64(old_fraction),
                                                self._f64(new_fraction), self._f64(matrix_composition), tp, r))

    def interface_composition(self, cm, fprec, sigma):
        import torch

        self._bind(cm, fprec)
        out = torch.empty_like(cm)
        t, tp, r = _taps_arg(sigma)
        check(lib().gpk_alcu_interface_composition(self._h, self._f64(cm), self._f64(fprec), out.data_ptr(), tp, r))
        return out

    def gaussian_remap(self, labels, alpha, sigma) -> int:
        self._bind(labels, alpha)
        t, tp, r = _taps_arg(sigma)
        n = C.c_int64(0)
        check(lib().gpk_alcu_gaussian_remap(self._h, self._i8(labels), self._f64(alpha), tp, r, C.byref(n)))
        return int(n.value)

    def balanced_remap(self, labels, alpha, sigma) -> int:
        self._bind(labels, alpha)
        t, tp, r = _taps_arg(sigma)
        n = C.c_int64(0)
        check(lib().gpk_alcu_balanced_remap(self._h, self._i8(labels), self._f64(alpha), tp, r, C.byref(n)))
        return int(n.value)

    def commit_transactions(self, labels, alpha, competitor, crossing) -> int:
        """crossing: a CUDA bool or uint8 tensor; returns the deferred count."""
        import torch

        self._bind(labels, alpha, competitor, crossing)
        if crossing.dtype not in (torch.bool, torch.uint8):
            raise ValueError("crossing must be a bool or uint8 tensor")
        n = C.c_int64(0)
        check(lib().gpk_alcu_commit_transactions(self._h, self._i8(labels), self._f64(alpha), self._i8(competitor),
                                                 crossing.data_ptr(), C.byref(n)))
        return int(n.value)

    def sum(self, x) -> float:
        self._bind(x)
        out = C.c_double(0.0)
        check(lib().gpk_alcu_sum(self._h, self._f64(x), C.byref(out)))
        return out.value

    def gaussian_filter(self, x, sigma):
        import torch

        self._bind(x)
        out = torch.empty_like(x)
        t, tp, r = _taps_arg(sigma)
        check(lib().gpk_alcu_gaussian_filter(self._h, self._f64(x), out.data_ptr(), tp, r))
        return out


# ---------------------------------------------------------------------------
# drop-ins with the reference's signatures

_cache: dict = {}


class _Defaults:
    """The reference's Parameters defaults (lines 43-76) for the fields read."""
    dx = 1.5e-9
    diffusivity = 1.66e-20
    c_matrix_eq = 3.7189506575706577e-4
    c_theta = 1.0 / 3.0
    composition_extension_sigma_cells = 0.75


def _handle(shape, p=None) -> AlCuTransport:
    shape = tuple(int(n) for n in shape)
    h = _cache.get(shape)
    if h is None:
        h = _cache[shape] = AlCuTransport(shape, p if p is not None else _Defaults())
    elif p is not None:
        h.set_params(p)
    return h


def _is_np(*xs) -> bool:
    return all(isinstance(x, np.ndarray) for x in xs)


def _dev(x, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x, dtype=dtype)).cuda()


def neighbor_competitor(labels):
    """(mask, competitor) of int8 labels."""
    if _is_np(labels):
        m, c = _handle(labels.shape).competitor(_dev(labels, np.int8))
        return m.cpu().numpy(), c.cpu().numpy()
    return _handle(labels.shape).competitor(labels)


def precip_fraction(labels, alpha, competitor):
    if _is_np(labels, alpha, competitor):
        h = _handle(labels.shape)
        return h.precip_fraction(_dev(labels, np.int8), _dev(alpha, np.float64),
                                 _dev(competitor, np.int8)).cpu().numpy()
    return _handle(labels.shape).precip_fraction(labels, alpha, competitor)


def variant_fraction_fields(labels, alpha, competitor):
    """One precipitate-fraction field per variant, stacked (3, *shape)."""
    if _is_np(labels, alpha, competitor):
        h = _handle(labels.shape)
        return h.variant_fractions(_dev(labels, np.int8), _dev(alpha, np.float64),
                                   _dev(competitor, np.int8)).cpu().numpy()
    return _handle(labels.shape).variant_fractions(labels, alpha, competitor)


def matrix_composition(ctot, fprec, p):
    """c_m = clip((ctot - f c_theta) / max(1 - f, 1e-8), 0, c_theta) (lines 917-919)."""
    h = _handle(ctot.shape, p)
    if _is_np(ctot, fprec):
        return h.matrix_composition(_dev(ctot, np.float64), _dev(fprec, np.float64)).cpu().numpy()
    return h.matrix_composition(ctot, fprec)


def diffuse_conservative_subcycled(ctot, fprec, p, dt: float):
    """Returns (ctot advanced by dt, c_m of the last substep, substeps); the
    input ctot is not modified, as in the reference."""
    h = _handle(ctot.shape, p)
    if _is_np(ctot, fprec):
        c = _dev(ctot, np.float64)
        cm, n = h.diffuse(c, _dev(fprec, np.float64), dt)
        return c.cpu().numpy(), cm.cpu().numpy(), n
    c = ctot.clone()
    cm, n = h.diffuse(c, fprec, dt)
    return c, cm, n


def conservative_partition_transfer(ctot, old_fraction, new_fraction, matrix_composition, p) -> None:
    """ctot updated in place; RuntimeError (GPKError) as the reference raises."""
    h = _handle(ctot.shape, p)
    sigma = p.composition_extension_sigma_cells
    if _is_np(ctot, old_fraction, new_fraction, matrix_composition):
        c = _dev(ctot, np.float64)
        try:
            h.partition_transfer(c, _dev(old_fraction, np.float64), _dev(new_fraction, np.float64),
                                 _dev(matrix_composition, np.float64), sigma)
        finally:
            ctot[...] = c.cpu().numpy()
        return None
    h.partition_transfer(ctot, old_fraction, new_fraction, matrix_composition, sigma)
    return None


def interface_matrix_composition(cm, fprec, p):
    h = _handle(cm.shape, p)
    sigma = p.composition_extension_sigma_cells
    if _is_np(cm, fprec):
        return h.interface_composition(_dev(cm, np.float64), _dev(fprec, np.float64), sigma).cpu().numpy()
    return h.interface_composition(cm, fprec, sigma)


def conservative_gaussian_remap(labels, alpha, sigma_cells) -> int:
    """labels and alpha updated in place; returns the changed-cell count."""
    h = _handle(labels.shape)
    if _is_np(labels, alpha):
        if labels.dtype != np.int8:
            raise ValueError("labels must be int8, as in the reference")
        lab = _dev(labels, np.int8)
        al = _dev(alpha, np.float64)
        n = h.gaussian_remap(lab, al, sigma_cells)
        labels[...] = lab.cpu().numpy()
        alpha[...] = al.cpu().numpy()
        return n
    return h.gaussian_remap(labels, alpha, sigma_cells)


def balanced_gaussian_remap(labels, alpha, sigma_cells) -> int:
    """labels and alpha updated in place; returns the changed-cell count."""
    h = _handle(labels.shape)
    if _is_np(labels, alpha):
        if labels.dtype != np.int8:
            raise ValueError("labels must be int8, as in the reference")
        lab = _dev(labels, np.int8)
        al = _dev(alpha, np.float64)
        n = h.balanced_remap(lab, al, sigma_cells)
        labels[...] = lab.cpu().numpy()
        alpha[...] = al.cpu().numpy()
        return n
    return h.balanced_remap(labels, alpha, sigma_cells)


def commit_topology_transactions(labels, alpha, competitor, crossing) -> int:
    """labels and alpha updated in place; returns the deferred-cell count."""
    h = _handle(labels.shape)
    if _is_np(labels, alpha, competitor, crossing):
        if labels.dtype != np.int8:
            raise ValueError("labels must be int8, as in the reference")
        lab = _dev(labels, np.int8)
        al = _dev(alpha, np.float64)
        n = h.commit_transactions(lab, al, _dev(competitor, np.int8), _dev(crossing, np.uint8))
        labels[...] = lab.cpu().numpy()
        alpha[...] = al.cpu().numpy()
        return n
    return h.commit_transactions(labels, alpha, competitor, crossing)


def field_sum(x) -> float:
    """np.sum(x) of a float64 field, same bits (numpy's pairwise order)."""
    if _is_np(x):
        return _handle(x.shape).sum(_dev(x, np.float64))
    return _handle(x.shape).sum(x)
