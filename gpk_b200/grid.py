"""``GPKGrid`` — Python mirror of the reference's gpk::GPKGrid over the C ABI.

Same constructor arguments, method names, return values and field names as
include/gpk_core.hpp:205-326 of albert-hzbn/GPK.  The state lives on the B200;
the public fields are exposed as numpy arrays copied out of (``grid.phi``)
and written back into (``grid.phi = ...``) device memory, which is how the
reference's drivers use the public std::vector members.
"""
from __future__ import annotations

import ctypes as C
import math
import weakref
from typing import Callable, Optional

import numpy as np

from ._lib import check, lib
from .thermo import FIELD_IDS, INT_FIELDS, U8_FIELDS, ThermoDesc

PRECISIONS = {"f32": 0, "f64": 1}


class GPKGrid:
    """A periodic Nz x Ny x Nx GPK domain stepped by the sm_100a kernels."""

    def __init__(self, Nz: int, Ny: int, Nx: int, dx: float, thermo: ThermoDesc,
                 D: float = 0.0, gaussian_sigma: float = 2.0, precision: str = "f32"):
        self.Nz, self.Ny, self.Nx = int(Nz), int(Ny), int(Nx)
        self.dx = float(dx)
        self.precision = precision
        self.real_dtype = np.float32 if precision == "f32" else np.float64
        self._thermo = thermo
        self._cthermo = thermo.to_c()
        L = lib()
        h = C.c_void_p()
        check(L.gpk_grid_create(self.Nz, self.Ny, self.Nx, self.dx, C.byref(self._cthermo), float(D),
                                float(gaussian_sigma), PRECISIONS[precision], C.byref(h)))
        self._h = h
        self._dependents = weakref.WeakSet()

    # ---- lifetime --------------------------------------------------------
    def attach(self, dependent) -> None:
        """Registers a handle built on this grid (an adjoint problem) whose
        close() must run before the grid is destroyed, whatever order the
        garbage collector finalises them in."""
        self._dependents.add(dependent)

    def close(self) -> None:
        for dep in list(getattr(self, "_dependents", ())):
            dep.close()
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().gpk_grid_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def N(self) -> int:
        return self.Nz * self.Ny * self.Nx

    def idx(self, z: int, y: int, x: int) -> int:
        return z * self.Ny * self.Nx + y * self.Nx + x

    # ---- fields ----------------------------------------------------------
    def _dtype(self, name):
        if name in INT_FIELDS:
            return np.int32
        if name in U8_FIELDS:
            return np.uint8
        return self.real_dtype

    def get(self, name: str) -> np.ndarray:
        out = np.empty((self.Nz, self.Ny, self.Nx), dtype=self._dtype(name))
        check(lib().gpk_grid_download(self._h, FIELD_IDS[name], out.ctypes.data, out.size))
        return out

    def set(self, name: str, value) -> None:
        arr = np.ascontiguousarray(np.broadcast_to(np.asarray(value, dtype=self._dtype(name)),
                                                   (self.Nz, self.Ny, self.Nx)))
        check(lib().gpk_grid_upload(self._h, FIELD_IDS[name], arr.ctypes.data, arr.size))

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        check(lib().gpk_grid_device_ptr(self._h, FIELD_IDS[name], C.byref(p)))
        return p.value

    def __getattr__(self, name):
        if name in FIELD_IDS:
            return self.get(name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in FIELD_IDS:
            self.set(name, value)
        else:
            object.__setattr__(self, name, value)

    def set_thermo(self, thermo: ThermoDesc) -> None:
        self._thermo = thermo
        self._cthermo = thermo.to_c()
        check(lib().gpk_grid_set_thermo(self._h, C.byref(self._cthermo)))

    # ---- time --------------------------------------------------------------
    @property
    def time(self) -> float:
        t = C.c_double()
        check(lib().gpk_grid_get_time(self._h, C.byref(t)))
        return t.value

    @time.setter
    def time(self, t: float) -> None:
        check(lib().gpk_grid_set_time(self._h, float(t)))

    @property
    def step_id(self) -> int:
        s = C.c_uint64()
        check(lib().gpk_grid_get_step_id(self._h, C.byref(s)))
        return s.value

    # ---- stepping (src/gpk_simulation.cpp:31-73) -------------------------------
    def step(self, dt: float = -1.0, dt_cap: float = 1.0e30) -> float:
        used = C.c_double()
        check(lib().gpk_grid_step(self._h, float(dt), float(dt_cap), C.byref(used)))
        return used.value

    def step_graph(self, n: int, dt: float = -1.0, dt_cap: float = 1.0e30) -> float:
        """n steps through a captured two-step CUDA graph (bit-identical to
        step_n); returns the grid time."""
        t = C.c_double()
        check(lib().gpk_grid_step_graph(self._h, int(n), float(dt), float(dt_cap), C.byref(t)))
        return t.value

    def set_tile_rows(self, divisor: int) -> None:
        """2-D geometry tile height at kernel radius 8: rows divided by 1, 2 or 4."""
        check(lib().gpk_grid_set_tile_rows(self._h, int(divisor)))

    def graph_supported(self) -> bool:
        s = C.c_int()
        check(lib().gpk_grid_graph_supported(self._h, C.byref(s)))
        return bool(s.value)

    def step_n(self, n: int, dt: float = -1.0, dt_cap: float = 1.0e30) -> float:
        t = C.c_double()
        check(lib().gpk_grid_step_n(self._h, int(n), float(dt), float(dt_cap), C.byref(t)))
        return t.value

    def run(self, t_end: float, dt: float = -1.0,
            cb: Optional[Callable[["GPKGrid", int], None]] = None, cb_interval: int = 100) -> int:
        if cb is None:
            n = C.c_int()
            check(lib().gpk_grid_run(self._h, float(t_end), float(dt), 0, C.byref(n)))
            return n.value
        steps = 0
        while self.time < t_end:
            remaining = float(np.float32(t_end - self.time))
            self.step(dt, remaining)
            steps += 1
            if steps % cb_interval == 0:
                cb(self, steps)
        return steps

    def sync(self) -> None:
        check(lib().gpk_grid_sync(self._h))

    # ---- diagnostics (src/gpk_simulation.cpp:11-144) ---------------------------
    def max_dt(self) -> float:
        v = C.c_double()
        check(lib().gpk_grid_max_dt(self._h, C.byref(v)))
        return v.value

    def phase_volume(self, label: int) -> float:
        v = C.c_double()
        check(lib().gpk_grid_phase_volume(self._h, int(label), C.byref(v)))
        return v.value

    def n_grains(self) -> int:
        v = C.c_int()
        check(lib().gpk_grid_n_grains(self._h, C.byref(v)))
        return v.value

    def mean_grain_radius(self) -> float:
        ng = self.n_grains()
        if ng == 0:
            return 0.0
        mv = self.N() / ng
        R = math.cbrt(3.0 * mv / (4.0 * math.pi)) if self.Nz > 1 else math.sqrt(mv / math.pi)
        return R * float(np.float32(self.dx))

    def solid_fraction(self) -> float:
        return float(np.float32(self.phase_volume(1) / float(self.N())))

    def interface_fraction(self) -> float:
        v = C.c_double()
        check(lib().gpk_grid_interface_fraction(self._h, C.byref(v)))
        return v.value

    def counters(self):
        c = (C.c_uint64 * 3)()
        check(lib().gpk_grid_counters(self._h, c))
        return tuple(int(v) for v in c)

    @property
    def topology_accepted_last(self) -> int:
        return self.counters()[0]

    @property
    def topology_deferred_last(self) -> int:
        return self.counters()[1]

    @property
    def gaussian_remap_exchanges_last(self) -> int:
        return self.counters()[2]

    def topology_simple_move(self, cell: int, new_label: int) -> bool:
        r = C.c_int()
        check(lib().gpk_grid_topology_simple_move(self._h, int(cell), int(new_label), C.byref(r)))
        return bool(r.value)

    def device_bytes(self) -> int:
        v = C.c_size_t()
        check(lib().gpk_grid_device_bytes(self._h, C.byref(v)))
        return v.value

    STAGES = ("mask", "geometry", "velocity", "projection", "alpha", "crossings", "remap",
              "extinction", "transport")

    def wave_stats(self) -> dict:
        out = (C.c_uint64 * 10)()
        check(lib().gpk_grid_wave_stats(self._h, out))
        return {"crossing_waves": int(out[0]), "remap_waves": int(out[1]), "candidates": int(out[2]),
                "remap_proposals": int(out[3]), "flood_fills": int(out[4]), "flood_cells": int(out[5]),
                "exact_counts": int(out[6]), "count_scanned": int(out[7]), "score_cells": int(out[8]),
                "score_cells_exact": int(out[9])}

    def set_geometry_kernel(self, kind: str) -> None:
        check(lib().gpk_grid_set_geometry_kernel(
            self._h, {"tiled": 0, "per_cell": 1, "tiled_batched": 2, "tiled_exact_scores": 3,
                      "separable_tiles": 4}[kind]))

    def set_external_elastic(self, on: bool = True) -> None:
        """E_el is supplied by the caller (e.g. SpectralElasticity.couple) and
        drives the interfaces; the model's elastic proxy is not run."""
        check(lib().gpk_grid_set_external_elastic(self._h, 1 if on else 0))

    def voronoi(self, n_grains: int, seed: int = 42) -> int:
        """Fills phi and g with the periodic Voronoi polycrystal of
        gpk_b200.voronoi(Nz, Ny, Nx, n_grains, seed), built on the device;
        returns the number of tie cells the connectivity step moved."""
        moved = C.c_int()
        check(lib().gpk_grid_voronoi(self._h, int(n_grains), int(seed), C.byref(moved)))
        return moved.value

    def voronoi_seeds(self, seeds, orientations) -> int:
        """The same construction on the device for an explicit seed list:
        ``seeds`` is (3, n) int (z, y, x rows), ``orientations`` (n,) float;
        seed k labels its Voronoi cell k + 1.  Returns the number of tie
        cells the connectivity step moved."""
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        sg = np.ascontiguousarray(orientations, dtype=np.float32)
        if s.ndim != 2 or s.shape[0] != 3 or sg.shape != (s.shape[1],):
            raise ValueError("seeds must be (3, n) and orientations (n,)")
        moved = C.c_int()
        check(lib().gpk_grid_voronoi_seeds(self._h, int(s.shape[1]), s[0].ctypes.data, s[1].ctypes.data,
                                           s[2].ctypes.data, sg.ctypes.data, C.byref(moved)))
        return moved.value

    def set_near_threshold(self, tol: float = 1e-12) -> None:
        """Tolerance of the near-threshold listing (see near_threshold)."""
        check(lib().gpk_grid_set_near_threshold(self._h, float(tol)))

    def near_threshold(self) -> np.ndarray:
        """Cells of the last step whose crossing decision lies within the
        tolerance of its threshold: interface cells with phi_comp != phi and
        |alpha_new - 1e-6| <= tol (src/gpk_transitions.cpp:291-292), in
        increasing cell order."""
        n = C.c_int()
        check(lib().gpk_grid_near_threshold(self._h, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.int32)
        if n.value:
            check(lib().gpk_grid_near_threshold(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out

    def set_solid_diffusivity_ratio(self, ratio: float) -> None:
        """Solid/liquid diffusivity ratio of the partitioned transport
        (0, the default, is the reference's transport)."""
        check(lib().gpk_grid_set_solid_diffusivity_ratio(self._h, float(ratio)))

    def geometry(self) -> None:
        """Mask and geometry of the current labels, without stepping."""
        check(lib().gpk_grid_geometry(self._h))

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().gpk_grid_stream(self._h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        check(lib().gpk_grid_profile(self._h, 1 if enable else 0))

    def stage_times(self) -> dict:
        ms = (C.c_double * len(self.STAGES))()
        calls = (C.c_uint64 * len(self.STAGES))()
        check(lib().gpk_grid_stage_times(self._h, ms, calls))
        return {s: (ms[k], int(calls[k])) for k, s in enumerate(self.STAGES)}

    def launch_count(self) -> int:
        v = C.c_uint64()
        check(lib().gpk_grid_launch_count(self._h, C.byref(v)))
        return v.value


def voronoi(Nz: int, Ny: int, Nx: int, n_grains: int, seed: int = 42):
    """Periodic Voronoi polycrystal (labels 1..n_grains) and per-grain orientations.

    Host-side, the same construction as the reference driver's voronoi_init
    (demos/gpk.cpp:51-189) with this library's own random stream.
    """
    phi = np.empty((Nz, Ny, Nx), dtype=np.int32)
    g = np.empty((Nz, Ny, Nx), dtype=np.float32)
    moved = C.c_int()
    rc = lib().gpk_voronoi_init(Nz, Ny, Nx, n_grains, seed, phi.ctypes.data, g.ctypes.data, C.byref(moved))
    if rc != 0:
        raise ValueError(f"gpk_voronoi_init failed with code {rc}")
    return phi, g
