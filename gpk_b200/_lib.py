"""ctypes binding of the C ABI in include/gpk_b200.h (libgpk_b200.so).

This is the Python-side stub a maintainer would bind against the library;
it raises instead of falling back to anything when the library or a B200 is
missing.
"""
from __future__ import annotations

import ctypes as C
import os

from .thermo import CThermoDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpk_b200.so")

GPK_OK = 0
ERRORS = {
    1: "invalid argument", 2: "unsupported thermodynamic model", 3: "CUDA error",
    4: "out of device memory", 5: "label out of range", 6: "device wait timed out",
    7: "no usable CUDA device", 8: "device consistency check failed",
    9: "no admissible result",
}


class CAlCuParams(C.Structure):
    """gpk_alcu_params of include/gpk_alcu.h."""
    _fields_ = [("dx", C.c_double), ("diffusivity", C.c_double), ("c_matrix_eq", C.c_double),
                ("c_theta", C.c_double)]


class GPKError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gpk_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Loads libgpk_b200.so (building it first when only sources are present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, u64, dbl, sz = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double, C.c_size_t
    sigs = {
        "gpk_version": ([], C.c_char_p),
        "gpk_last_error": ([], C.c_char_p),
        "gpk_device_init": ([i32], i32),
        "gpk_thermo_desc_init": ([vp, C.c_int32], None),
        "gpk_grid_create": ([i32, i32, i32, dbl, vp, dbl, dbl, i32, C.POINTER(vp)], i32),
        "gpk_grid_destroy": ([vp], i32),
        "gpk_grid_set_thermo": ([vp, vp], i32),
        "gpk_grid_upload": ([vp, i32, vp, sz], i32),
        "gpk_grid_download": ([vp, i32, vp, sz], i32),
        "gpk_grid_device_ptr": ([vp, i32, C.POINTER(vp)], i32),
        "gpk_grid_get_time": ([vp, C.POINTER(dbl)], i32),
        "gpk_grid_set_time": ([vp, dbl], i32),
        "gpk_grid_get_step_id": ([vp, C.POINTER(u64)], i32),
        "gpk_grid_set_step_id": ([vp, u64], i32),
        "gpk_grid_step": ([vp, dbl, dbl, C.POINTER(dbl)], i32),
        "gpk_grid_step_n": ([vp, i32, dbl, dbl, C.POINTER(dbl)], i32),
        "gpk_grid_run": ([vp, dbl, dbl, i32, C.POINTER(i32)], i32),
        "gpk_grid_sync": ([vp], i32),
        "gpk_grid_geometry": ([vp], i32),
        "gpk_grid_max_dt": ([vp, C.POINTER(dbl)], i32),
        "gpk_grid_phase_volume": ([vp, C.c_int32, C.POINTER(dbl)], i32),
        "gpk_grid_n_grains": ([vp, C.POINTER(i32)], i32),
        "gpk_grid_interface_fraction": ([vp, C.POINTER(dbl)], i32),
        "gpk_grid_counters": ([vp, C.POINTER(u64)], i32),
        "gpk_grid_topology_simple_move": ([vp, i32, C.c_int32, C.POINTER(i32)], i32),
        "gpk_grid_device_bytes": ([vp, C.POINTER(sz)], i32),
        "gpk_grid_launch_count": ([vp, C.POINTER(u64)], i32),
        "gpk_gaussian_filter_3d": ([vp, vp, i32, i32, i32, vp, i32], i32),
        "gpk_gaussian_filter_3d_noalloc": ([vp, vp, i32, i32, i32, vp, i32], i32),
        "gpk_grid_stream": ([vp, C.POINTER(vp)], i32),
        "gpk_grid_wave_stats": ([vp, C.POINTER(u64)], i32),
        "gpk_grid_set_geometry_kernel": ([vp, i32], i32),
        "gpk_grid_profile": ([vp, i32], i32),
        "gpk_grid_stage_times": ([vp, C.POINTER(dbl), C.POINTER(u64)], i32),
        "gpk_voronoi_init": ([i32, i32, i32, i32, u64, vp, vp, C.POINTER(i32)], i32),
        "gpk_grid_voronoi": ([vp, i32, u64, C.POINTER(i32)], i32),
        "gpk_grid_voronoi_seeds": ([vp, i32, vp, vp, vp, vp, C.POINTER(i32)], i32),
        "gpk_grid_set_near_threshold": ([vp, dbl], i32),
        "gpk_grid_near_threshold": ([vp, vp, i32, C.POINTER(i32)], i32),
        "gpk_grid_set_solid_diffusivity_ratio": ([vp, dbl], i32),
        "gpk_grid_inject_wait_timeout": ([vp, C.c_longlong], i32),
        "gpk_grid_step_graph": ([vp, i32, dbl, dbl, C.POINTER(dbl)], i32),
        "gpk_grid_graph_supported": ([vp, C.POINTER(i32)], i32),
        "gpk_batch_step_graph": ([vp, i32, dbl, dbl], i32),
        "gpk_batch_graph_stream": ([vp, C.POINTER(vp)], i32),
        "gpk_batch_autotune_tiles": ([vp, i32, C.POINTER(i32), C.POINTER(i32)], i32),
        "gpk_grid_set_tile_rows": ([vp, i32], i32),
        "gpk_spectral_create": ([i32, C.POINTER(i32), dbl, dbl, dbl, dbl, C.POINTER(dbl), C.POINTER(vp)], i32),
        "gpk_spectral_destroy": ([vp], i32),
        "gpk_spectral_set_constants": ([vp, dbl, dbl, dbl, dbl, C.POINTER(dbl)], i32),
        "gpk_spectral_set_stream": ([vp, vp], i32),
        "gpk_spectral_solve": ([vp, vp, vp, vp, vp, C.POINTER(dbl)], i32),
        "gpk_spectral_solve_host": ([vp, vp, vp, vp, vp, C.POINTER(dbl)], i32),
        "gpk_spectral_info": ([vp, C.POINTER(i64), C.POINTER(i64)], i32),
        "gpk_spectral_couple_grid": ([vp, vp, C.c_int32, C.POINTER(dbl)], i32),
        "gpk_grid_set_external_elastic": ([vp, i32], i32),
        "gpk_batch_create": ([i32, C.POINTER(vp), i32, C.POINTER(vp)], i32),
        "gpk_batch_destroy": ([vp], i32),
        "gpk_batch_set_workers": ([vp, i32], i32),
        "gpk_batch_workers": ([vp, C.POINTER(i32)], i32),
        "gpk_batch_step": ([vp, i32, dbl, dbl], i32),
        "gpk_batch_run": ([vp, dbl, dbl, i32, C.POINTER(i32)], i32),
        "gpk_batch_autotune": ([vp, i32, C.POINTER(i32), C.POINTER(i32)], i32),
        "gpk_adjoint_create": ([vp, i32, C.POINTER(C.c_int32), i32, dbl, dbl, dbl, dbl, dbl, dbl, C.POINTER(vp)], i32),
        "gpk_adjoint_destroy": ([vp], i32),
        "gpk_adjoint_num_params": ([vp, C.POINTER(i32)], i32),
        "gpk_adjoint_set_target": ([vp, C.POINTER(dbl)], i32),
        "gpk_adjoint_forward": ([vp, C.POINTER(dbl), C.POINTER(dbl), C.POINTER(dbl)], i32),
        "gpk_adjoint_gradient": ([vp, C.POINTER(dbl), C.POINTER(dbl), C.POINTER(dbl)], i32),
        "gpk_alcu_create": ([i32, C.POINTER(i32), C.POINTER(CAlCuParams), C.POINTER(vp)], i32),
        "gpk_alcu_destroy": ([vp], i32),
        "gpk_alcu_set_params": ([vp, C.POINTER(CAlCuParams)], i32),
        "gpk_alcu_set_stream": ([vp, vp], i32),
        "gpk_alcu_gauss_taps": ([dbl, C.POINTER(dbl), i32, C.POINTER(i32)], i32),
        "gpk_alcu_competitor": ([vp, vp, vp, vp], i32),
        "gpk_alcu_precip_fraction": ([vp, vp, vp, vp, vp], i32),
        "gpk_alcu_matrix_composition": ([vp, vp, vp, vp], i32),
        "gpk_alcu_variant_fractions": ([vp, vp, vp, vp, vp], i32),
        "gpk_alcu_diffuse": ([vp, vp, vp, dbl, vp, C.POINTER(i32)], i32),
        "gpk_alcu_partition_transfer": ([vp, vp, vp, vp, vp, C.POINTER(dbl), i32], i32),
        "gpk_alcu_interface_composition": ([vp, vp, vp, vp, C.POINTER(dbl), i32], i32),
        "gpk_alcu_gaussian_remap": ([vp, vp, vp, C.POINTER(dbl), i32, C.POINTER(i64)], i32),
        "gpk_alcu_sum": ([vp, vp, C.POINTER(dbl)], i32),
        "gpk_alcu_commit_transactions": ([vp, vp, vp, vp, vp, C.POINTER(i64)], i32),
        "gpk_alcu_balanced_remap": ([vp, vp, vp, C.POINTER(dbl), i32, C.POINTER(i64)], i32),
        "gpk_alcu_gaussian_filter": ([vp, vp, vp, C.POINTER(dbl), i32], i32),
        "gpk_alcu_info": ([vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)], i32),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(code: int) -> None:
    if code != GPK_OK:
        msg = lib().gpk_last_error().decode(errors="replace")
        raise GPKError(code, msg)


def exported_symbols() -> list:
    """Names of every entry point declared in the headers under include/."""
    import re
    names = []
    inc = os.path.join(HERE, "..", "include")
    for h in ("gpk_b200.h", "gpk_init.h", "gpk_spectral.h", "gpk_batch.h", "gpk_adjoint.h", "gpk_alcu.h"):
        text = open(os.path.join(inc, h)).read()
        names += re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(gpk_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


__all__ = ["lib", "check", "GPKError", "CThermoDesc", "CAlCuParams", "exported_symbols"]
