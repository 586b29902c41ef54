"""Many independent grids advanced together (parameter sweeps).

Mirrors a sweep that the reference writes as a loop of GPKGrid objects
(demos/gpk.cpp:1119-1200): `GPKBatch(grids)` advances every grid with the same
results as stepping each alone, with a pool of native worker threads driving
the instances' CUDA streams concurrently (libgpk_b200.so, gpk_batch.h).
"""
from __future__ import annotations

import ctypes as C

from ._lib import check, lib


class GPKBatch:
    """Holds references to the grids; they must outlive the batch and must
    not be used while a batch call runs."""

    def __init__(self, grids, workers: int = 0) -> None:
        self.grids = list(grids)
        arr = (C.c_void_p * len(self.grids))(*[g._h.value for g in self.grids])
        self._h = C.c_void_p()
        check(lib().gpk_batch_create(len(self.grids), arr, int(workers), C.byref(self._h)))

    @property
    def workers(self) -> int:
        w = C.c_int()
        check(lib().gpk_batch_workers(self._h, C.byref(w)))
        return w.value

    @workers.setter
    def workers(self, w: int) -> None:
        check(lib().gpk_batch_set_workers(self._h, int(w)))

    def step(self, steps: int = 1, dt: float = -1.0, dt_cap: float = 1e30) -> None:
        check(lib().gpk_batch_step(self._h, int(steps), float(dt), float(dt_cap)))

    def step_graph(self, steps: int = 2, dt: float = -1.0, dt_cap: float = 1e30) -> None:
        """The same steps with the whole sweep as one captured CUDA graph (two
        steps per launch); bit-identical to step()."""
        check(lib().gpk_batch_step_graph(self._h, int(steps), float(dt), float(dt_cap)))

    def graph_stream_ptr(self) -> int:
        """cudaStream_t of the sweep graph's launches (for timing events)."""
        p = C.c_void_p()
        check(lib().gpk_batch_graph_stream(self._h, C.byref(p)))
        return p.value or 0

    def run(self, t_end: float, dt: float = -1.0, max_steps: int = 1 << 30) -> list:
        out = (C.c_int * len(self.grids))()
        check(lib().gpk_batch_run(self._h, float(t_end), float(dt), int(max_steps), out))
        return list(out)

    def autotune(self, trial_steps: int = 2) -> tuple:
        """Returns (chosen worker count, steps every instance took while timing)."""
        w, n = C.c_int(), C.c_int()
        check(lib().gpk_batch_autotune(self._h, int(trial_steps), C.byref(w), C.byref(n)))
        return w.value, n.value

    def autotune_tiles(self, trial_steps: int = 2) -> tuple:
        """Picks the sweep graph's 2-D geometry tile height per instance-size
        group; returns (divisor per group (side <= 160, <= 320, larger),
        steps every instance took while timing)."""
        ch, n = (C.c_int * 3)(), C.c_int()
        check(lib().gpk_batch_autotune_tiles(self._h, int(trial_steps), ch, C.byref(n)))
        return list(ch), n.value

    def close(self) -> None:
        if self._h:
            lib().gpk_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
