"""CPU checkers for the gpk_b200 CUDA path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  Two checkers are exposed with the same
interface:

* :class:`OracleGrid` — the C restatement in ``oracle/gpk_oracle.c`` of the
  reference's ``GPKGrid::step`` (float build = the reference's FP32
  arithmetic, double build = the FP64 variant).
* :class:`RefGrid` — the reference's own sources (src/*.cpp of
  albert-hzbn/GPK) compiled into ``oracle/_ref/libgpk_ref.so`` behind
  ``oracle/ref_harness.cpp``.

Both wrap the public fields of ``GPKGrid`` (include/gpk_core.hpp:211-228) as
numpy arrays copied in and out through plain pointers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gpk_b200.thermo import ThermoDesc, FIELD_IDS, INT_FIELDS, U8_FIELDS

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libgpk_ref.so")


def build(quiet: bool = True, demos: bool = False) -> None:
    """Compile the oracle (and the reference harness where its sources exist;
    with demos, also the reference's validation programs in their CPU and
    drop-in builds).  The reference checkout is named by GPK_REFERENCE."""
    targets = ["all"] + (["demos"] if demos else [])
    out = subprocess.run(["make", "-j8", "-f", os.path.join(_HERE, "Makefile")] + targets,
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_libs: dict = {}


def _load(path: str) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            if path == _ORACLE_SO:
                build()
            else:
                raise FileNotFoundError(path)
        _libs[path] = C.CDLL(path)
    return _libs[path]


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def _int_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def voronoi_seeds(Nz, Ny, Nx, n, seed):
    """Seed cells (z, y, x) and orientations in the draw order of the
    library's splitmix64 stream (oracle/voronoi_oracle.c)."""
    L = _load(_ORACLE_SO)
    s = np.empty((3, n), dtype=np.int32)
    g = np.empty(n, dtype=np.float32)
    rc = L.or_voronoi_seeds(C.c_int(Nz), C.c_int(Ny), C.c_int(Nx), C.c_int(n), C.c_uint64(seed),
                            _int_ptr(s[0]), _int_ptr(s[1]), _int_ptr(s[2]), _int_ptr(g))
    if rc:
        raise ValueError(f"or_voronoi_seeds failed ({rc})")
    return s, g


def voronoi_from_seeds(shape, seeds, orientations):
    """The reference driver's Voronoi construction (demos/gpk.cpp:51-189) for
    an explicit seed list: labels 1..n, orientations, reassigned tie cells."""
    L = _load(_ORACLE_SO)
    Nz, Ny, Nx = shape
    s = np.ascontiguousarray(seeds, dtype=np.int32)
    sg = np.ascontiguousarray(orientations, dtype=np.float32)
    n = s.shape[1]
    phi = np.empty(shape, dtype=np.int32)
    g = np.empty(shape, dtype=np.float32)
    re = C.c_int(0)
    rc = L.or_voronoi_from_seeds(C.c_int(Nz), C.c_int(Ny), C.c_int(Nx), C.c_int(n), _int_ptr(s[0]),
                                 _int_ptr(s[1]), _int_ptr(s[2]), _int_ptr(sg), _int_ptr(phi), _int_ptr(g),
                                 C.byref(re))
    if rc:
        raise ValueError(f"or_voronoi_from_seeds failed ({rc})")
    return phi, g, re.value


def voronoi(Nz, Ny, Nx, n, seed):
    """The polycrystal gpk_voronoi_init builds (seeds from the library's
    stream, the reference's construction), built without the library."""
    s, sg = voronoi_seeds(Nz, Ny, Nx, n, seed)
    phi, g, _ = voronoi_from_seeds((Nz, Ny, Nx), s, sg)
    return phi, g


def ref_voronoi_seeds(Nz, Ny, Nx, n, seed):
    """The seeds the reference's voronoi_init draws (std::mt19937 + libstdc++
    distributions, demos/gpk.cpp:56-71)."""
    L = _load(_REF_SO)
    s = np.empty((3, n), dtype=np.int32)
    g = np.empty(n, dtype=np.float32)
    rc = L.ref_voronoi_seeds(C.c_int(Nz), C.c_int(Ny), C.c_int(Nx), C.c_int(n), C.c_uint32(seed),
                             _int_ptr(s[0]), _int_ptr(s[1]), _int_ptr(s[2]), _int_ptr(g))
    if rc:
        raise ValueError("ref_voronoi_seeds failed")
    return s, g


def ref_voronoi(Nz, Ny, Nx, n, seed):
    """The reference driver's own voronoi_init (compiled from its source)."""
    L = _load(_REF_SO)
    phi = np.empty((Nz, Ny, Nx), dtype=np.int32)
    g = np.empty((Nz, Ny, Nx), dtype=np.float32)
    rc = L.ref_voronoi_init(C.c_int(Nz), C.c_int(Ny), C.c_int(Nx), C.c_int(n), C.c_uint32(seed),
                            _int_ptr(phi), _int_ptr(g))
    if rc:
        raise ValueError("ref_voronoi_init rejected its arguments")
    return phi, g


class _GridBase:
    """Shared numpy field access over a C grid handle."""

    real_dtype = np.float32

    def __init__(self, Nz: int, Ny: int, Nx: int):
        self.Nz, self.Ny, self.Nx = Nz, Ny, Nx
        self.N = Nz * Ny * Nx

    def _dtype(self, name: str):
        if name in INT_FIELDS:
            return np.int32
        if name in U8_FIELDS:
            return np.uint8
        return self.real_dtype

    def _ptr(self, name: str) -> int:
        raise NotImplementedError

    def get(self, name: str) -> np.ndarray:
        dt = self._dtype(name)
        ptr = self._ptr(name)
        buf = (C.c_byte * (self.N * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt).copy().reshape(self.Nz, self.Ny, self.Nx)

    def set(self, name: str, value) -> None:
        dt = self._dtype(name)
        arr = np.ascontiguousarray(np.broadcast_to(np.asarray(value, dtype=dt),
                                                   (self.Nz, self.Ny, self.Nx)))
        C.memmove(self._ptr(name), arr.ctypes.data, arr.nbytes)


class OracleGrid(_GridBase):
    """C restatement of GPKGrid (float or double build)."""

    def __init__(self, Nz, Ny, Nx, dx, thermo: ThermoDesc, D=0.0, sigma=2.0, precision="f32"):
        super().__init__(Nz, Ny, Nx)
        self.lib = _load(_ORACLE_SO)
        self.sfx = precision
        self.real_dtype = np.float32 if precision == "f32" else np.float64
        f = self._fn
        f("or_create").restype = C.c_void_p
        f("or_create").argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                   C.c_double, C.c_double]
        f("or_field").restype = C.c_void_p
        f("or_field").argtypes = [C.c_void_p, C.c_int]
        f("or_step").restype = C.c_double
        f("or_step").argtypes = [C.c_void_p, C.c_double, C.c_double]
        for n in ("or_get_time", "or_max_dt", "or_interface_fraction"):
            f(n).restype = C.c_double
            f(n).argtypes = [C.c_void_p]
        f("or_phase_volume").restype = C.c_double
        f("or_phase_volume").argtypes = [C.c_void_p, C.c_int32]
        f("or_set_time").argtypes = [C.c_void_p, C.c_double]
        f("or_counters").argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        f("or_n_grains").argtypes = [C.c_void_p]
        f("or_topology_simple_move").argtypes = [C.c_void_p, C.c_int, C.c_int32]
        f("or_run").argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        f("or_set_thermo").argtypes = [C.c_void_p, C.c_void_p]
        f("or_destroy").argtypes = [C.c_void_p]
        f("or_interface_mask").argtypes = [C.c_void_p]
        self._thermo = thermo.to_c()
        self.h = f("or_create")(Nz, Ny, Nx, float(dx), C.byref(self._thermo), float(D), float(sigma))
        if not self.h:
            raise RuntimeError("or_create failed")

    def _fn(self, name):
        return getattr(self.lib, f"{name}_{self.sfx}")

    def _ptr(self, name):
        return self._fn("or_field")(self.h, FIELD_IDS[name])

    def step(self, dt=-1.0, dt_cap=1e30) -> float:
        return self._fn("or_step")(self.h, dt, dt_cap)

    def run(self, t_end, dt=-1.0, max_steps=0) -> int:
        return self._fn("or_run")(self.h, t_end, dt, max_steps)

    @property
    def time(self) -> float:
        return self._fn("or_get_time")(self.h)

    @time.setter
    def time(self, t):
        self._fn("or_set_time")(self.h, t)

    def counters(self):
        out = (C.c_uint64 * 3)()
        self._fn("or_counters")(self.h, out)
        return tuple(int(v) for v in out)

    def set_thermo(self, thermo: ThermoDesc):
        self._thermo = thermo.to_c()
        self._fn("or_set_thermo")(self.h, C.byref(self._thermo))

    def max_dt(self):
        return self._fn("or_max_dt")(self.h)

    def phase_volume(self, label):
        return self._fn("or_phase_volume")(self.h, label)

    def n_grains(self):
        return self._fn("or_n_grains")(self.h)

    def interface_fraction(self):
        return self._fn("or_interface_fraction")(self.h)

    def topology_simple_move(self, cell, label):
        return bool(self._fn("or_topology_simple_move")(self.h, cell, label))

    def interface_mask(self):
        self._fn("or_interface_mask")(self.h)

    def set_near_threshold(self, tol=1e-12):
        f = self._fn("or_set_near_tol")
        f.argtypes = [C.c_void_p, C.c_double]
        f(self.h, float(tol))

    def near_threshold(self) -> np.ndarray:
        f = self._fn("or_near_threshold")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        f.restype = C.c_int
        n = f(self.h, None, 0)
        out = np.empty(n, dtype=np.int32)
        if n:
            f(self.h, out.ctypes.data, n)
        return out

    def set_solid_diffusivity_ratio(self, ratio):
        f = self._fn("or_set_solid_ratio")
        f.argtypes = [C.c_void_p, C.c_double]
        f(self.h, float(ratio))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self._fn("or_destroy")(h)
            self.h = None


class RefGrid(_GridBase):
    """The reference's own GPKGrid (compiled from its sources), float only."""

    def __init__(self, Nz, Ny, Nx, dx, thermo: ThermoDesc, D=0.0, sigma=2.0):
        super().__init__(Nz, Ny, Nx)
        self.lib = _load(_REF_SO)
        L = self.lib
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_double, C.c_double]
        L.ref_field.restype = C.c_void_p
        L.ref_field.argtypes = [C.c_void_p, C.c_int]
        L.ref_step.restype = C.c_double
        L.ref_step.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.ref_time_steps.restype = C.c_double
        L.ref_time_steps.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        for n in ("ref_get_time", "ref_max_dt", "ref_interface_fraction"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [C.c_void_p]
        L.ref_phase_volume.restype = C.c_double
        L.ref_phase_volume.argtypes = [C.c_void_p, C.c_int32]
        L.ref_set_time.argtypes = [C.c_void_p, C.c_double]
        L.ref_counters.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        L.ref_n_grains.argtypes = [C.c_void_p]
        L.ref_topology_simple_move.argtypes = [C.c_void_p, C.c_int, C.c_int32]
        L.ref_run.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.ref_destroy.argtypes = [C.c_void_p]
        self._thermo = thermo.to_c()
        self.h = L.ref_create(Nz, Ny, Nx, float(dx), C.byref(self._thermo), float(D), float(sigma))
        if not self.h:
            raise RuntimeError("ref_create failed (unknown model tag)")

    def _ptr(self, name):
        return self.lib.ref_field(self.h, FIELD_IDS[name])

    def step(self, dt=-1.0, dt_cap=1e30) -> float:
        return self.lib.ref_step(self.h, dt, dt_cap)

    def run(self, t_end, dt=-1.0) -> int:
        return self.lib.ref_run(self.h, t_end, dt)

    def time_steps(self, n, dt=-1.0, threads=0) -> float:
        return self.lib.ref_time_steps(self.h, n, dt, threads)

    @staticmethod
    def max_threads() -> int:
        lib = _load(_REF_SO)
        return lib.ref_max_threads()

    @property
    def time(self) -> float:
        return self.lib.ref_get_time(self.h)

    @time.setter
    def time(self, t):
        self.lib.ref_set_time(self.h, t)

    def counters(self):
        out = (C.c_uint64 * 3)()
        self.lib.ref_counters(self.h, out)
        return tuple(int(v) for v in out)

    def max_dt(self):
        return self.lib.ref_max_dt(self.h)

    def phase_volume(self, label):
        return self.lib.ref_phase_volume(self.h, label)

    def n_grains(self):
        return self.lib.ref_n_grains(self.h)

    def interface_fraction(self):
        return self.lib.ref_interface_fraction(self.h)

    def topology_simple_move(self, cell, label):
        return bool(self.lib.ref_topology_simple_move(self.h, cell, label))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.ref_destroy(h)
            self.h = None
