"""Benchmark of the GPK per-step hot path on B200.

Workload (one "step" = one GPKGrid::step of the whole grid): 3-D isotropic
grain growth on a periodic 256^3 int32 label grid, 4096 Voronoi grains from
uniform random seeds, IsotropicGrowthThermo(M0=1, sigma0=1), dx=1, D=0,
Gaussian measurement length sigma = 1.5 cells, automatic (stable) dt, in the
reference's FP32 arithmetic (labels bit-identical to the reference).

Metric: cell-updates/s = cells x steps / device seconds (the reference's
"cell-steps/s", demos/benchmark.cpp:44).  The state (16.8 M cells x ~60 B)
is far larger than the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: a single grid does not shard without breaking the reference's
serial transaction order, so N GPUs run N independent replicas (weak
scaling); value = total cell-updates over all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "python"))

SIZE = 256
GRAINS = 4096
SIGMA = 1.5
SEED = 42
SETTLE = 16  # steps evolved while preparing the input state (untimed)
# single-thread CPU sample: same grain size (4096 cells per grain) on a 128^3 sub-volume
CPU_SIZE = 128
CPU_GRAINS = 512
# DRAM read + write bytes of one k_geometry_tiled launch on the 256^3 / 4096
# grain / sigma 1.5 workload, measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, one-pass metrics, the launch of the third warm-up step)
GEOMETRY_TRAFFIC_256 = 527.80e6
GEOMETRY_TRAFFIC_NOTE = ("DRAM bytes (read 300.98 MB + write 226.82 MB) of one launch of the kernel on this "
                         "256^3 workload, measured by ncu with the one-pass dram__bytes metrics")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _fp32_add_peak(sm_mhz: float) -> float:
    # 148 SMs x 128 FP32 lanes, one add per lane per clock
    return 148 * 128 * sm_mhz * 1e6


def _config(extra=None):
    c = {"workload": f"3-D isotropic grain growth {SIZE}^3, {GRAINS} Voronoi grains, sigma {SIGMA} cells, "
                     f"stable dt, reference FP32 arithmetic",
         "cells": SIZE ** 3, "grains": GRAINS, "sigma_cells": SIGMA, "model": "IsotropicGrowthThermo(1,1)",
         "l2": "state larger than L2 (16.8M cells x ~60 B); no flush needed",
         "initial_state": f"seeded Voronoi tessellation evolved {SETTLE} steps before warm-up (first crossings "
                          f"occur at step 8)",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                continue
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _allmax(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _ref_grid(n: int, phi, g):
    """The reference's own GPKGrid (oracle/_ref) loaded with a state."""
    import oracle
    from gpk_b200.thermo import isotropic
    if not oracle.ref_available():
        oracle.build()
    if not oracle.ref_available():
        return None
    r = oracle.RefGrid(n, n, n, 1.0, isotropic(1.0, 1.0), 0.0, SIGMA)
    r.set("phi", phi)
    r.set("g", g)
    return r


def single_thread_sample():
    """One step of the reference on one thread, on a 128^3 sub-volume with 512
    grains (the workload's 4096 cells per grain), after 16 settling steps on
    all threads; the same step on all threads beside it."""
    import oracle
    n, grains = CPU_SIZE, CPU_GRAINS
    phi, g = oracle.voronoi(n, n, n, grains, SEED)
    r = _ref_grid(n, phi, g)
    if r is None:
        return None
    r.set("alpha", 1.0)
    nproc = oracle.RefGrid.max_threads()
    r.time_steps(SETTLE, -1.0, nproc)
    t_all = r.time_steps(1, -1.0, nproc)
    t_one = r.time_steps(1, -1.0, 1)
    r.time_steps(0, -1.0, nproc)  # restore the thread count
    return {"value": n ** 3 / t_one, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
            "same_sample_all_cores": {"value": n ** 3 / t_all, "cores": nproc},
            "sample": f"one step of the reference's GPKGrid::step on a {n}^3 sub-volume with {grains} grains "
                      f"(4096 cells per grain, sigma {SIGMA}) after {SETTLE} settling steps; one thread, and all "
                      f"{nproc} threads on the next step"}


def cpu_sample_from_state(phi, alpha, g, steps: int = 2):
    """The reference's OpenMP step (oracle/_ref) on this host's cores, timed on
    a bounded sample of the benchmarked workload: the 256^3 state the GPU
    reached, one untimed step (the reference's step counter starts at zero,
    whose step runs the extinction pass), then `steps` timed steps."""
    import oracle
    n = phi.shape[0]
    r = _ref_grid(n, phi, g)
    if r is None:
        return None
    r.set("alpha", alpha)
    r.time_steps(1, -1.0, 0)
    sec = r.time_steps(steps, -1.0, 0)
    return {"value": n ** 3 * steps / sec, "unit": "cell-updates/s", "cores": oracle.RefGrid.max_threads(),
            "kind": "reference",
            "sample": f"{steps} step(s) of the reference's own GPKGrid::step (src/*.cpp, -O3, OpenMP) on the "
                      f"{n}^3 state the GPU run reached after its timed steps, after one untimed step"}


def run_reference_arm(args):
    """The reference's own OpenMP GPKGrid::step (its src/*.cpp compiled into
    oracle/_ref) on the same workload as the GPU arm: the 256^3 polycrystal
    built by the oracle's restatement of the driver's Voronoi construction
    (the GPU arm's input, cell for cell), SETTLE settling steps, W warm-up
    steps, then K timed steps on all host threads.  The CUDA library is
    never loaded on this path."""
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    import oracle
    t0 = time.perf_counter()
    phi, g = oracle.voronoi(SIZE, SIZE, SIZE, GRAINS, SEED)
    init_s = time.perf_counter() - t0
    r = _ref_grid(SIZE, phi, g)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library could not be built here"}))
        return 0
    del phi, g
    r.set("alpha", 1.0)
    nproc = oracle.RefGrid.max_threads()
    settle_s = r.time_steps(SETTLE + args.warmup, -1.0, nproc)
    per_step = [r.time_steps(1, -1.0, nproc) for _ in range(args.steps)]
    sec = sum(per_step)
    counters = list(r.counters())
    del r
    value = SIZE ** 3 * args.steps / sec
    one = None
    if not args.no_cpu:
        try:
            one = single_thread_sample()
        except Exception as exc:
            one = {"error": str(exc)}
    sample = (f"{args.steps} timed step(s) of the reference's own GPKGrid::step (src/*.cpp, -O3, OpenMP, "
              f"{nproc} threads) on the benchmarked {SIZE}^3 workload after {SETTLE} settling and "
              f"{args.warmup} warm-up steps (the GPU arm's step indices)")
    line = {"impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Voronoi polycrystal)",
            "config": _config(),
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": nproc, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "single_thread": one, "counters_last_step": counters,
            "input": {"builder": "oracle restatement of the driver's Voronoi construction (host, one thread)",
                      "seconds": init_s, "settle_and_warmup_seconds": settle_s}}
    print(json.dumps(line))
    return 0


def spectral_measurement(with_cpu: bool):
    """FP64 spectral micro-elasticity solve on the 128^3 solidification grid
    (cubic 108/62/28 GPa, 0.5% dilatational misfit, nucleus radius 4), inputs
    resident on the device, 10 timed solves after 3 warm-up solves."""
    import torch
    from gpk.spectral import SpectralElasticity, variant_eigenstrains
    n = 128
    g = torch.arange(n, device="cuda", dtype=torch.int32) - n // 2
    r2 = g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2
    vf = torch.zeros((3, n, n, n), dtype=torch.float64, device="cuda")
    vf[0][r2 <= 16] = 1.0
    s = SpectralElasticity((n, n, n), 1.0, 108e9, 62e9, 28e9, variant_eigenstrains(0.005, 0.005))
    for _ in range(3):
        out = s.solve(vf, want_residual=False)
    residual = s.solve(vf)[3]
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(10):
        out = s.solve(vf, want_residual=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 10
    cells = n ** 3
    # algorithmic bytes per cell: eigenstrain 24 + 24, forward half-spectrum
    # transforms 24 + 24, Green's kernel 24 + 48, inverse transforms 48 + 48,
    # epilogue 48 + 24 + 40
    per_cell = 48 + 48 + 72 + 96 + 112
    peak, peak_kind = _peaks()
    achieved = per_cell * cells / (ms / 1e3) / 1e9
    res = {"workload": "spectral elasticity 128^3 FP64 (3 D2Z + 6 Z2D cuFFT on half spectra, Green's-function "
                       "and epilogue kernels)", "ms_per_solve": ms, "cells_per_s": cells / (ms / 1e3),
           "residual": residual, "algorithmic_bytes_per_cell": per_cell,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": peak_kind},
           "own_kernels_per_solve": 4, "library_calls_per_solve": "cufftExecD2Z (batch 3), cufftExecZ2D (batch 6)"}
    if with_cpu:
        import types
        from oracle import spectral_oracle
        host = vf.cpu().numpy()
        p = types.SimpleNamespace(dx=1.0, c11=108e9, c12=62e9, c44=28e9, eigen_small=0.005, eigen_large=0.005)
        t0 = time.perf_counter()
        spectral_oracle.spectral_elasticity(host, p)
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": cells / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
                               "sample": "one 128^3 solve of the numpy restatement (numpy.fft, one thread)"}
    s.close()
    return res


def _alcu_state(shape, plates, rng):
    """int8 labels with theta-prime plates (thin along the variant's axis,
    aspect 8 as in the reference's embryos, periodic minimum image), alpha,
    and total Cu as the reference's initial_state sets them (matrix at the
    composition that keeps the mean at c0 = 0.0169, precipitates at
    c_theta).  Each plate is drawn in its own periodic window."""
    import numpy as np
    lab = np.zeros(shape, dtype=np.int8)
    for centre, v, scale in plates:
        axes = np.full(3, 6.0 * scale)
        axes[v - 1] /= 8.0
        half = [int(np.ceil(a)) for a in axes]
        offs = [np.arange(-h, h + 1) for h in half]
        idx = [(centre[a] + offs[a]) % shape[a] for a in range(3)]
        d2 = ((offs[0][:, None, None] / axes[0]) ** 2 + (offs[1][None, :, None] / axes[1]) ** 2
              + (offs[2][None, None, :] / axes[2]) ** 2)
        win = np.ix_(*idx)
        sub = lab[win]
        sub[d2 <= 1.0] = v
        lab[win] = sub
    f0 = float(np.mean(lab > 0))
    cm0 = (0.0169 - f0 / 3.0) / (1.0 - f0)
    ctot = np.full(shape, cm0)
    ctot[lab > 0] = 1.0 / 3.0
    alpha = np.ones(shape)
    return lab, alpha, ctot


def alcu_measurement(with_cpu: bool, steps: int = 10, warmup: int = 3):
    """The Al-Cu module's per-step transport and remap (competitor,
    precipitate fraction, matrix composition, interface composition, sub-cycled
    diffusion, partition transfer, crossing transactions, Gaussian remap), FP64, on the reference's
    three_dimensional case (96^3, three plates of its layout_3d_96) and on a
    256^3 field with 400 plates; inputs resident, each stage timed with CUDA
    events on the launching stream."""
    import numpy as np
    import torch
    from gpk.alcu import AlCuTransport
    from oracle import alcu_oracle as O

    out = {}
    cases = {
        "96^3 reference three_dimensional layout": ((96, 96, 96), [((24, 24, 24), 1, 1.05), ((72, 27, 68), 2, 0.95),
                                                                    ((29, 72, 69), 3, 1.00)]),
    }
    rng = np.random.default_rng(3)
    many = [(tuple(int(q) for q in rng.integers(0, 256, 3)), 1 + k % 3, float(rng.uniform(1.0, 2.5)))
            for k in range(400)]
    cases["256^3, 400 plates"] = ((256, 256, 256), many)
    p = O.AlCuParams()
    stages = ["competitor", "fraction", "composition", "interface", "diffuse", "transfer", "transactions", "remap"]
    # algorithmic bytes per cell of each stage (each field read or written
    # once; labels 1 B, fields 8 B): transactions (histogram 1, crossing
    # flags 1 + 4, ordered compaction 8), competitor 1 + 2, fraction 10 + 8,
    # composition 16 + 8, interface composition 16 + 16 in, 3 passes of 2
    # fields 32 each, 16 + 8 out, diffusion 2 substeps of 16 + 8 and the last
    # c_m 8, partition transfer (transfer 32 + 24, 4 sums 32, 3 passes 48,
    # weight 24 + 16, apply 16 + 8, argmax 16), remap (labels copy 2, union-
    # find 4 x 4, flags / scatter / vacate per wave 10, changed 1 + 8)
    per_cell = {"competitor": 3, "fraction": 18, "composition": 24, "interface": 152, "diffuse": 56,
                "transfer": 216, "transactions": 14, "remap": 37}
    peak, peak_kind = _peaks()
    for name, (shape, plates) in cases.items():
        lab, alpha, ctot = _alcu_state(shape, plates, rng)
        n = int(np.prod(shape))
        h = AlCuTransport(shape, p)
        dl = torch.from_numpy(lab).cuda()
        da = torch.from_numpy(alpha).cuda()
        dc = torch.from_numpy(ctot).cuda()
        # a fixed synthetic growth of the fraction at interface cells
        m0, _ = h.competitor(dl)
        grow = (0.05 * m0.double()).contiguous()
        # a fixed tenth of the initial interface cells cross in every step
        gen = torch.Generator(device="cuda").manual_seed(7)
        cross = (m0 & (torch.rand(shape, device="cuda", generator=gen) < 0.1)).to(torch.uint8).contiguous()
        stream = torch.cuda.current_stream()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(stages) + 1)]
        acc = {k: 0.0 for k in stages}
        info = {}

        def step(timed):
            if timed:
                ev[0].record(stream)
            mask, comp = h.competitor(dl)
            if timed:
                ev[1].record(stream)
            fp = h.precip_fraction(dl, da, comp)
            if timed:
                ev[2].record(stream)
            cm = h.matrix_composition(dc, fp)
            if timed:
                ev[3].record(stream)
            trace = h.interface_composition(cm, fp, 0.75)
            if timed:
                ev[4].record(stream)
            h.diffuse(dc, fp, 10.0)
            if timed:
                ev[5].record(stream)
            h.partition_transfer(dc, fp, fp + grow, trace, 0.75)
            if timed:
                ev[6].record(stream)
            info["deferred"] = h.commit_transactions(dl, da, comp, cross)
            if timed:
                ev[7].record(stream)
            info["changed"] = h.gaussian_remap(dl, da, 0.70)
            if timed:
                ev[8].record(stream)

        for _ in range(warmup):
            step(False)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            step(True)
            ev[-1].synchronize()
            for k, st in enumerate(stages):
                acc[st] += ev[k].elapsed_time(ev[k + 1])
        t1.record(stream)
        t1.synchronize()
        ms = t0.elapsed_time(t1) / steps
        st_ms = {k: v / steps for k, v in acc.items()}
        # the chain's largest single kernel: the tiled diffusion substep
        # (2 substeps per step at dt = 10 s, dx = 1.5 nm), 24 algorithmic B/cell
        sub_ms = st_ms["diffuse"] / 2.0
        diff_gbs = 24.0 * n / (sub_ms / 1e3) / 1e9
        roof = {"kernel": "k_diffuse_tiled (one explicit substep)", "bound": "hbm", "achieved": diff_gbs,
                "peak": peak, "unit": "GB/s", "frac": diff_gbs / peak, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": 24.0 * n,
                "traffic": 381.9e6 * n / 256 ** 3 if shape[0] == 256 else None,
                "traffic_note": "dram read + write of one 256^3 launch of the same kernel under ncu",
                "note": "issue-bound on its FP64 divisions in the reference's operand order, not on HBM"}
        res = {"ms_per_step": ms, "cells_per_s": n / (ms / 1e3), "stages_ms": st_ms, "roofline": roof,
               "components": h.info()["components"], "remap_waves": h.info()["waves"],
               "changed_last_step": info["changed"], "deferred_last_step": info["deferred"],
               "crossing_cells": int(cross.sum().item()),
               "stage_GBps": {k: per_cell[k] * n / (st_ms[k] / 1e3) / 1e9 for k in stages if st_ms[k] > 0},
               "algorithmic_bytes_per_cell": per_cell, "peak": peak, "peak_kind": peak_kind}
        if with_cpu and shape == (96, 96, 96):
            lab_h, al_h, c_h = lab.copy(), alpha.copy(), ctot.copy()
            g_h = grow.cpu().numpy()
            t_cpu = time.perf_counter()
            mask_h, comp_h = O.neighbor_competitor(lab_h)
            fp_h = O.precip_fraction(lab_h, al_h, comp_h)
            cm_h = O.matrix_composition(c_h, fp_h, p)
            tr_h = O.interface_matrix_composition(cm_h, fp_h, p)
            c_h, _, _ = O.diffuse_conservative_subcycled(c_h, fp_h, p, 10.0)
            O.conservative_partition_transfer(c_h, fp_h, fp_h + g_h, tr_h, p)
            O.commit_topology_transactions(lab_h, al_h, comp_h, cross.cpu().numpy().astype(bool))
            O.conservative_gaussian_remap(lab_h, al_h, 0.70)
            cpu_s = time.perf_counter() - t_cpu
            res["cpu_baseline"] = {"value": n / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
                                   "sample": "one step of the numpy restatement of the same eight functions "
                                             "(numpy/scipy order, one thread) on the 96^3 state"}
        out[name] = res
        h.close()
    return out


def batched_measurement(n_inst: int = 512, steps: int = 10, warmup: int = 4, ws: int = 1, rank: int = 0):
    """The lamellar-precipitate sweep: n_inst 2-D instances of sides
    U{64..512} (FP64, OstwaldThermo), all advanced by one captured CUDA graph
    per two steps (each instance's captured step a child graph), beside the
    plain loop over instances and the worker-pool engine (instances on their
    own streams, worker count autotuned).  Each figure times `steps` steps
    with CUDA events on the stream the work is issued on; the three run one
    after another on the same evolving instances.  With ws > 1 ranks the
    instances are sharded by cell count (no exchange); the time is the max
    over ranks and only the graph form runs."""
    import torch
    from gpk_b200 import GPKBatch
    from gpk_b200.sweep import lamellar_grid, lamellar_side, shard
    seeds = [5000 + i for i in range(n_inst)]
    sizes = [lamellar_side(s) ** 2 for s in seeds]
    mine = shard(sizes, ws)[rank] if ws > 1 else list(range(n_inst))
    grids = [lamellar_grid(seeds[i], precision="f64")[0] for i in mine]
    cells = sum(sizes) if ws == 1 else sum(sizes[i] for i in mine)
    total_cells = sum(sizes)
    streams = [torch.cuda.ExternalStream(g.stream_ptr()) for g in grids]
    batch = GPKBatch(grids)

    def timed_streams(nsteps):
        ts = torch.cuda.Stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(ts)
        for st in streams:
            st.wait_event(e0)
        batch.step(nsteps)
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            ts.wait_event(ev)
        e1.record(ts)
        e1.synchronize()
        return e0.elapsed_time(e1)

    gs = torch.cuda.ExternalStream(batch.graph_stream_ptr())

    def timed_graph(nsteps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = sum(g.launch_count() for g in grids)
        e0.record(gs)
        batch.step_graph(nsteps)
        e1.record(gs)
        e1.synchronize()
        return e0.elapsed_time(e1), sum(g.launch_count() for g in grids) - l0

    res = {"workload": f"{n_inst} lamellar-precipitate 2-D instances, sides U{{64..512}}, stripe thickness "
                       "U{4..16}, spacing/thickness U[2,12], OstwaldThermo, FP64, sigma 1.5",
           "instances": n_inst, "cells": total_cells, "steps": steps, "ranks": ws, "unit": "cell-updates/s"}
    if ws == 1:
        batch.workers = 1
        batch.step(2)
        ms_p = timed_streams(steps)
        workers, tune_steps = batch.autotune(trial_steps=1)
        ms_w = timed_streams(steps)
        res.update({"plain_value": cells * steps / (ms_p / 1e3), "plain_ms": ms_p,
                    "pool_value": cells * steps / (ms_w / 1e3), "pool_ms": ms_w, "pool_workers": workers})
    tiles, tile_steps = batch.autotune_tiles(trial_steps=2)
    batch.step_graph(warmup)  # one ordinary step where fresh, then capture and replays
    _barrier(ws)
    ms_g, launches = timed_graph(steps)
    ms_g = _allmax(ms_g, ws)
    res.update({"value": total_cells * steps / (ms_g / 1e3), "ms": ms_g, "warmup": warmup,
                "tile_rows_divisor_by_side": {"<=160": tiles[0], "161-320": tiles[1], ">320": tiles[2]},
                "autotune_steps": tile_steps,
                "gpu_launches_rank0": launches,
                "how": "each instance's step captured once (two steps per graph, counts read on the device, the "
                       "remap under a device-side gate), the instances' graphs the independent children of one "
                       "graph, launched once per two steps; plain = the instances stepped one after another; "
                       "pool = worker threads driving the instances' streams"})
    if ws == 1:
        res["speedup_vs_plain"] = ms_p / ms_g
        res["pool_speedup_vs_plain"] = ms_p / ms_w
    batch.close()
    for g in grids:
        g.close()
    return res


def adjoint_measurement(with_cpu: bool, evals: int = 20):
    """Gradients of the calibration loss on the 512^2 polycrystal (256 grains,
    64 precipitates of radius 6-20): 3 eigenstrain + 4 anisotropy + 256
    mobility derivatives per gradient, FP64."""
    import torch
    from gpk_b200 import GPKGrid, thermo
    from gpk.adjoint import AdjointProblem, calibration_case
    n, grains = 512, 256
    phi, g, mob_index = calibration_case(n, grains, 64, 11, (6, 20))
    grid = GPKGrid(1, n, n, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5, precision="f64")
    grid.set("phi", phi)
    grid.set("g", g)
    const = dict(m_fixed=1.0, sigma0=1e-3, c11=1.08, c12=0.62, c44=0.28, energy_weight=1e-6)
    prob = AdjointProblem(grid, mob_index, grains, **const)
    rng = np.random.default_rng(11)
    theta = np.concatenate([[0.01, -0.004, 0.003], [0.05, -0.02, 0.01, 0.005],
                            1.0 + 0.1 * rng.standard_normal(grains)])
    star = theta * 1.05
    prob.set_target(prob.forward(star, want_v=True)[1])
    for _ in range(3):
        prob.gradient(theta)
    stream = torch.cuda.ExternalStream(grid.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(evals):
        prob.gradient(theta)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / evals
    f0 = time.perf_counter()
    for _ in range(evals):
        prob.forward(theta)
    fwd_ms = (time.perf_counter() - f0) * 1e3 / evals
    res = {"workload": "adjoint calibration 512^2, 256 Voronoi grains + 64 precipitates, FP64; gradient = "
                       "forward + adjoint (2 spectral solves, projection and its transpose)",
           "params": len(theta), "ms_per_gradient": ms, "gradients_per_s": 1e3 / ms,
           "derivatives_per_s": len(theta) * 1e3 / ms, "forward_ms_wall": fwd_ms,
           "central_difference_gradients_per_s_gpu": 1e3 / (2 * len(theta) * fwd_ms)}
    if with_cpu:
        from oracle import adjoint_oracle
        f = {k: grid.get(k)[0] for k in ("phi", "phi_comp", "mask", "nx_f", "ny_f", "kappa_f", "g")}
        inv = 0.5 / (0.85 * 0.85)
        t0 = time.perf_counter()
        adjoint_oracle.forward(f["phi"], f["phi_comp"], f["mask"], f["nx_f"], f["ny_f"], f["kappa_f"], f["g"],
                               mob_index, theta, const["c11"], const["c12"], const["c44"], const["sigma0"],
                               const["m_fixed"], const["energy_weight"], 1.0, np.zeros((n, n)), 3,
                               lambda r2: float(np.exp(-r2 * inv)))
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": 1.0 / (2 * len(theta) * cpu_s), "unit": "gradients/s", "cores": 1,
                               "kind": "port", "sample": "one forward of the numpy restatement timed; a "
                               "central-difference gradient costs 2 x 263 of them"}
    prob.close()
    grid.close()
    return res


def coupled_measurement(steps: int = 300, warmup: int = 3, n: int = 128, elastic: bool = True,
                        undercooling: float = 40.0, solid_ratio: float = 1e-4):
    """3-D solidification with solute partitioning and a spectral elastic
    solve every step: n^3 (128 by default), FP64, nucleus of radius 4 at the
    centre in a melt undercooled by 40 K, c0 = 0.02, k = 0.14, solid/liquid
    diffusivity ratio 1e-4, cubic 108/62/28 GPa, 0.5% dilatational misfit of
    the solid (the reference's solidification deck otherwise).  The misfit
    energy density (about 2.5 MJ/m^3) exceeds the chemical driving force
    L dT / T_m below about 23 K, so at 5 K the nucleus dissolves; at 40 K it
    grows through the 300 steps.  The timed region is the whole 300-step run
    from the nucleus (a separate grid of the same case runs the warm-up
    steps).  Without elastic, the same step with no elastic solve: the
    solute transport alone on a field larger than L2."""
    import torch
    from gpk import GPKGrid, SpectralElasticity, thermo
    from gpk.spectral import variant_eigenstrains

    def make():
        th = thermo.solidification(M0=5e-8, sigma0=0.2, eps4=0.04, m_liq=-500.0, k_part=0.14, T_melt=933.0, L=1e8)
        th.solute_rejection, th.k_partition = True, 0.14  # as the reference's driver sets both from k_part
        g = GPKGrid(n, n, n, 0.5e-6, th, 3e-9, 1.5, precision="f64")
        z, y, x = np.indices((n, n, n)) - n // 2
        g.set("phi", ((x * x + y * y + z * z) <= 16).astype(np.int32))
        g.set("c", 0.02)
        g.set("T", 933.0 - undercooling)
        g.set_solid_diffusivity_ratio(solid_ratio)
        s = None
        if elastic:
            g.set_external_elastic(True)
            s = SpectralElasticity((n, n, n), 0.5e-6, 108e9, 62e9, 28e9, variant_eigenstrains(0.005, 0.005))
        return g, s

    g, s = make()
    for _ in range(warmup):
        if s:
            s.couple(g)
        g.step()
    g.sync()
    if s:
        s.close()
    g.close()
    g, s = make()
    solid0 = int((g.get("phi") != 0).sum())
    stream = torch.cuda.ExternalStream(g.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    l0 = g.launch_count()
    e0.record(stream)
    for _ in range(steps):
        if s:
            s.couple(g)
        g.step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = {"workload": f"3-D solidification {n}^3 FP64, nucleus of radius 4, {undercooling:g} K undercooling, "
                       f"solute partitioning (k 0.14), solid/liquid diffusivity ratio {solid_ratio:g}" +
                       (", a spectral elastic solve every step (cubic 108/62/28 GPa, 0.5% dilatational misfit)"
                        if elastic else ", no elastic solve"),
           "steps": steps, "warmup": warmup, "ms_per_step": ms, "value": n ** 3 / (ms / 1e3),
           "unit": "cell-updates/s", "gpu_launches_per_step": (g.launch_count() - l0) / steps,
           "solid_cells_start": solid0, "solid_cells": int((g.get("phi") != 0).sum()),
           "interface_fraction": g.interface_fraction(), "time_s": g.time}
    if s:
        s.close()
    g.close()
    return res


def separable_measurement(n: int = 256, grains: int = 32, sigma: float = 5.0, settle: int = 8, steps: int = 3,
                          warmup: int = 2):
    """3-D grain growth with the separable geometry: n^3, `grains` Voronoi
    grains, sigma 5 cells (Gaussian radius 18, geometry radius 20 > 18), FP32
    reference arithmetic.  Per step and interface label: the x pass of the
    indicator, the y and z passes, the evaluation on the label's interface
    cells.  Algorithmic bytes of the geometry stage: the labels read once
    per interface label (4 B per cell) and the normals and curvature of the
    interface cells written once (16 B each); the intermediate smoothed
    fields between the passes are not algorithmic bytes (the traffic they
    cause is in `intermediate_bytes_per_step`)."""
    import torch
    from gpk_b200 import GPKGrid, thermo
    g = GPKGrid(n, n, n, 1.0, thermo.isotropic(1.0, 1.0), 0.0, sigma)
    g.voronoi(grains, SEED)
    g.set("alpha", 1.0)
    g.step_n(settle)
    for _ in range(warmup):
        g.step()
    g.sync()
    g.profile(True)
    g.stage_times()
    stream = torch.cuda.ExternalStream(g.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    st = g.stage_times()
    g.profile(False)
    geo_ms = st["geometry"][0] / max(1, st["geometry"][1])
    cells = n ** 3
    n_active = g.interface_fraction() * cells
    geo_bytes = grains * cells * 4.0 + n_active * 16.0
    inter_bytes = grains * cells * 29.0  # x-pass output, y and z passes in/out, evaluation reads
    peak, peak_kind = _peaks()
    res = {"workload": f"3-D isotropic grain growth {n}^3, {grains} Voronoi grains, sigma {sigma} cells "
                       "(separable geometry: per-label x/y/z Gaussian passes + interface evaluation), FP32",
           "steps": steps, "warmup": warmup, "ms_per_step": ms, "value": cells / (ms / 1e3),
           "unit": "cell-updates/s", "geometry_ms_per_step": geo_ms,
           "stages_ms_per_step": {k: v[0] / max(1, v[1]) for k, v in st.items()},
           "roofline": {"kernels": "k_sep_x_indicator_f2, k_sep_pass (y, z), k_separable_eval per label",
                        "bound": "fp32 issue (the reference's unfused multiply + add per tap)",
                        "algorithmic_bytes_per_step": geo_bytes, "intermediate_bytes_per_step": inter_bytes,
                        "achieved": geo_bytes / (geo_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": geo_bytes / (geo_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind}}
    g.close()
    return res


def throughput_measurement(n: int = 256, grains: int = 4096, settle: int = 16, steps: int = 4, warmup: int = 2):
    """The FP64 step of the headline workload (n^3, `grains` Voronoi grains,
    sigma 1.5) with the direct FP64 geometry tiles and with the separable
    tiles (the throughput geometry: each tile label's indicator smoothed, then
    fourth-order differences), from the same settled state.  Algorithmic
    bytes of the geometry stage: the labels read once (4 B per cell) and, per
    interface cell, the normals and curvature written (4 x 8 B) and the
    competitor (4 B), i.e. 4 B per cell + 36 B per interface cell."""
    import torch
    from gpk_b200 import GPKGrid, thermo
    res = {"workload": f"3-D isotropic grain growth {n}^3, {grains} Voronoi grains, sigma 1.5 cells, FP64",
           "steps": steps, "warmup": warmup}
    peak, peak_kind = _peaks()
    cells = n ** 3
    for kind in ("tiled", "separable_tiles"):
        g = GPKGrid(n, n, n, 1.0, thermo.isotropic(1.0, 1.0), 0.0, 1.5, precision="f64")
        g.voronoi(grains, SEED)
        g.set("alpha", 1.0)
        g.step_n(settle)
        g.set_geometry_kernel(kind)
        for _ in range(warmup):
            g.step()
        g.sync()
        g.profile(True)
        g.stage_times()
        stream = torch.cuda.ExternalStream(g.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            g.step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        st = g.stage_times()
        g.profile(False)
        geo_ms = st["geometry"][0] / max(1, st["geometry"][1])
        geo_bytes = cells * 4.0 + g.interface_fraction() * cells * 36.0
        res[kind] = {"ms_per_step": ms, "value": cells / (ms / 1e3), "unit": "cell-updates/s",
                     "geometry_ms_per_step": geo_ms,
                     "stages_ms_per_step": {k: v[0] / max(1, v[1]) for k, v in st.items() if v[1]},
                     "geometry_roofline": {"algorithmic_bytes": geo_bytes,
                                           "achieved": geo_bytes / (geo_ms / 1e3) / 1e9, "peak": peak,
                                           "unit": "GB/s", "frac": geo_bytes / (geo_ms / 1e3) / 1e9 / peak,
                                           "peak_kind": peak_kind}}
        g.close()
    res["geometry_speedup"] = res["tiled"]["geometry_ms_per_step"] / res["separable_tiles"]["geometry_ms_per_step"]
    res["step_speedup"] = res["tiled"]["ms_per_step"] / res["separable_tiles"]["ms_per_step"]
    return res


def _summary(line):
    """A compact digest of the line's main figures, printed last so that a
    reader who keeps only the end of the output still has them."""
    def g(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def r3(v):
        return float("%.4g" % v) if isinstance(v, (int, float)) else v

    out = {"cell_updates_per_s": r3(line["value"]), "ms_per_step": r3(line["ms_per_step"]),
           "e2e_cell_updates_per_s": r3(g(line, "e2e", "value")),
           "geometry_ms": r3(g(line, "roofline", "ms_per_launch")),
           "geometry_fp32_add_frac": r3(g(line, "roofline", "compute", "frac")),
           "cpu_reference_cell_updates_per_s": r3(g(line, "cpu_baseline", "value")),
           "cpu_cores": g(line, "cpu_baseline", "cores"),
           "batched_cell_updates_per_s": r3(g(line, "batched", "value")),
           "batched_speedup_vs_plain": r3(g(line, "batched", "speedup_vs_plain")),
           "adjoint_gradients_per_s": r3(g(line, "adjoint", "gradients_per_s")),
           "spectral_ms_128": r3(g(line, "spectral", "ms_per_solve")),
           "coupled_ms_128": r3(g(line, "coupled", "ms_per_step")),
           "near_threshold_cells": g(line, "near_threshold", "cells_last_step"),
           "f64_step_ms_direct": r3(g(line, "throughput_f64", "tiled", "ms_per_step")),
           "f64_step_ms_separable_tiles": r3(g(line, "throughput_f64", "separable_tiles", "ms_per_step"))}
    st = line.get("stages_ms_per_step") or {}
    out["stages_ms"] = {k: r3(v) for k, v in st.items() if isinstance(v, (int, float)) and v > 0.01}
    return out


def run_gpu_arm(args):
    ws, rank, local = _dist()
    import torch
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from gpk_b200 import GPKGrid, lib, thermo, voronoi
    from gpk_b200._lib import check
    check(lib().gpk_device_init(local))
    torch.cuda.set_device(local)

    grid = GPKGrid(SIZE, SIZE, SIZE, 1.0, thermo.isotropic(1.0, 1.0), 0.0, SIGMA)
    stream = torch.cuda.ExternalStream(grid.stream_ptr())
    # the seeded Voronoi polycrystal, built on the device (cell for cell the
    # host construction, which is timed once beside it)
    i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    i0.record(stream)
    grid.voronoi(GRAINS, SEED + rank)
    i1.record(stream)
    i1.synchronize()
    init = {"workload": f"periodic Voronoi polycrystal {SIZE}^3, {GRAINS} grains, with connectivity normalisation",
            "device_ms": i0.elapsed_time(i1)}
    if rank == 0 and not args.no_cpu:
        t0 = time.perf_counter()
        voronoi(SIZE, SIZE, SIZE, GRAINS, SEED + rank)
        init["host_ms"] = (time.perf_counter() - t0) * 1e3
        init["host_threads"] = os.cpu_count()
    grid.set("alpha", 1.0)
    # Input preparation: from a fresh tessellation no cell crosses before
    # step 8 (|v| dt <= dx/8), so the state is first evolved SETTLE steps;
    # the timed steps then run the full pipeline, crossings and remap included.
    grid.step_n(SETTLE)
    for _ in range(args.warmup):
        grid.step()
    grid.sync()
    grid.profile(True)
    grid.stage_times()  # reset
    grid.wave_stats()  # reset
    l0 = grid.launch_count()
    _barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            grid.step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    _barrier(ws)
    ms = e0.elapsed_time(e1)
    launches = grid.launch_count() - l0
    stages = grid.stage_times()
    waves = {k: v / args.steps for k, v in grid.wave_stats().items()}
    grid.profile(False)
    iface = grid.interface_fraction()
    near = {"tolerance": 1e-12, "cells_last_step": int(grid.near_threshold().size),
            "what": "interface cells with phi_comp != phi whose switching margin alpha_new - 1e-6 lay within "
                    "the tolerance of zero in the last timed step"}
    ms_max = _allmax(ms, ws)
    cells = SIZE ** 3
    value = cells * args.steps * ws / (ms_max / 1e3)

    # ---- roofline of the dominant kernel (geometry) ----
    geo_ms = stages["geometry"][0] / max(1, stages["geometry"][1])
    n_active = iface * cells
    W = 2 * (int(np.ceil(3.5 * SIGMA)) + 2) + 1
    geo_bytes = cells * 4 + n_active * (4 * 4 + 4)
    peak, peak_kind = _peaks()
    achieved = geo_bytes / (geo_ms / 1e3) / 1e9
    # DRAM bytes (read + write) of one launch, from an ncu capture of the
    # same kernel on this workload; None for other sizes
    traffic = GEOMETRY_TRAFFIC_256 if (SIZE == 256 and GRAINS == 4096 and SIGMA == 1.5) else None
    clocks = clk.summary()
    tap_adds = n_active * W ** 3 * 9 / (geo_ms / 1e3)
    separable = (W - 1) // 2 > 18
    if separable:
        # per interface label the labels once (4 B per cell); the interface
        # cells' normals and curvature (16 B) once; intermediates excluded
        geo_bytes = GRAINS * cells * 4.0 + n_active * 16
        achieved = geo_bytes / (geo_ms / 1e3) / 1e9
    roofline = {"kernel": "k_geometry_tiled (label-bitmap Gaussian-Hessian tensor stencil + competitor)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": geo_bytes, "ms_per_launch": geo_ms,
                "note": "the reference-exact tensor stencil adds 9 products per matching tap over (2R+1)^3 "
                        "taps per interface cell in a fixed order; it is bound by FP32 add issue, not HBM "
                        "(compute: the reference's W^3 x 9 tap-adds per interface cell per second)",
                "traffic_note": GEOMETRY_TRAFFIC_NOTE,
                "compute": {"tap_adds_per_s": tap_adds,
                            "peak_fp32_adds_per_s": _fp32_add_peak(clocks["sm_mhz"] or 1965.0),
                            "frac": tap_adds / _fp32_add_peak(clocks["sm_mhz"] or 1965.0)}}
    if separable:
        roofline = {"kernel": "k_sep_pass x3 + k_separable_eval per interface label (separable geometry)",
                    "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": geo_bytes,
                    "ms_per_launch": geo_ms}
    step_bytes = 16.0 * cells
    step_roofline = {"algorithmic_bytes_per_step": step_bytes,
                     "achieved_GBps": step_bytes / (ms / args.steps / 1e3) / 1e9, "peak": peak,
                     "frac": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak}

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e_steps = max(1, min(args.steps, 5))
    h_phi = torch.empty((SIZE, SIZE, SIZE), dtype=torch.int32, pin_memory=True)
    h_alpha = torch.empty((SIZE, SIZE, SIZE), dtype=torch.float32, pin_memory=True)
    h_g = torch.empty((SIZE, SIZE, SIZE), dtype=torch.float32, pin_memory=True)
    h_phi.numpy()[...] = grid.get("phi")
    h_alpha.numpy()[...] = grid.get("alpha")
    h_g.numpy()[...] = grid.get("g")
    from gpk_b200.thermo import FIELD_IDS
    L = lib()
    _barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        for name, h in (("phi", h_phi), ("alpha", h_alpha), ("g", h_g)):
            check(L.gpk_grid_upload(grid._h, FIELD_IDS[name], h.data_ptr(), h.numel()))
        grid.step()
        for name, h in (("phi", h_phi), ("alpha", h_alpha), ("g", h_g)):
            check(L.gpk_grid_download(grid._h, FIELD_IDS[name], h.data_ptr(), h.numel()))
    f1.record(stream)
    f1.synchronize()
    e2e_ms = _allmax(f0.elapsed_time(f1), ws)
    e2e_value = cells * e2e_steps * ws / (e2e_ms / 1e3)
    io = cells * (4 + 4 + 4)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cpu = cpu_sample_from_state(grid.get("phi"), grid.get("alpha"), grid.get("g"))
        except Exception as exc:  # the GPU number stands on its own
            cpu = {"error": str(exc)}
    spectral = batched = adjoint = coupled = alcu = separable = transport = throughput = None
    # the sweep shards over all ranks (same collective order on every rank)
    if not args.headline_only:
        try:
            batched = batched_measurement(ws=ws, rank=rank)
        except Exception as exc:
            batched = {"error": str(exc)}
    if rank == 0 and not args.headline_only:
        try:
            spectral = spectral_measurement(not args.no_cpu and ws == 1)
        except Exception as exc:  # reported, never silent
            spectral = {"error": str(exc)}
        try:
            adjoint = adjoint_measurement(not args.no_cpu and ws == 1)
        except Exception as exc:
            adjoint = {"error": str(exc)}
        try:
            coupled = coupled_measurement()
        except Exception as exc:
            coupled = {"error": str(exc)}
        try:
            alcu = alcu_measurement(not args.no_cpu and ws == 1)
        except Exception as exc:
            alcu = {"error": str(exc)}
        try:
            separable = separable_measurement()
        except Exception as exc:
            separable = {"error": str(exc)}
        try:
            transport = coupled_measurement(5, 3, 256, elastic=False)
        except Exception as exc:
            transport = {"error": str(exc)}
        try:
            throughput = throughput_measurement()
        except Exception as exc:
            throughput = {"error": str(exc)}
    if rank == 0:
        line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Voronoi polycrystal)", "config": _config(),
                "roofline": roofline, "step_roofline": step_roofline,
                "stages_ms_per_step": {k: v[0] / max(1, v[1]) for k, v in stages.items()},
                "interface_fraction": iface, "counters_last_step": list(grid.counters()),
                "per_step_topology": waves, "near_threshold": near,
                "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches, "spectral": spectral, "batched": batched, "adjoint": adjoint, "coupled": coupled, "alcu": alcu, "separable": separable, "transport": transport, "throughput_f64": throughput, "init": init,
                "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": io,
                        "d2h_bytes_per_step": io, "steps": e2e_steps,
                        "path": "GPKGrid drop-in semantics: upload phi/alpha/g, step, download phi/alpha/g"}}
        line["summary"] = _summary(line)
        print(json.dumps(line))
    grid.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpk_b200")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--size", type=int, default=SIZE, help="cube side (profiling of smaller cases)")
    ap.add_argument("--grains", type=int, default=GRAINS)
    ap.add_argument("--batched-only", action="store_true",
                    help="time only the lamellar sweep, batched and plain")
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--adjoint-only", action="store_true", help="time only the 512^2 adjoint gradient")
    ap.add_argument("--coupled-only", action="store_true",
                    help="time only the 128^3 solidification step with a spectral solve per step")
    ap.add_argument("--separable-only", action="store_true",
                    help="time only the 256^3 sigma-5 grain-growth step (separable geometry)")
    ap.add_argument("--throughput-only", action="store_true",
                    help="time only the FP64 256^3 step with direct and with separable-tile geometry")
    ap.add_argument("--transport-only", action="store_true",
                    help="time only the solidification step without the elastic solve, on a --size cube")
    ap.add_argument("--sigma", type=float, default=SIGMA,
                    help="Gaussian width in cells (5 selects the per-label separable geometry)")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the grain-growth step and its e2e (profiling the headline kernels)")
    ap.add_argument("--alcu-only", action="store_true",
                    help="time only the Al-Cu transport and remap chain (96^3 and 256^3)")
    ap.add_argument("--spectral-only", action="store_true",
                    help="time only the 128^3 spectral elasticity solve (profiling its kernels)")
    args = ap.parse_args()
    globals()["SIZE"], globals()["GRAINS"], globals()["SIGMA"] = args.size, args.grains, args.sigma
    if args.spectral_only:
        print(json.dumps({"spectral": spectral_measurement(not args.no_cpu)}))
        return 0
    if args.alcu_only:
        print(json.dumps({"alcu": alcu_measurement(not args.no_cpu)}))
        return 0
    if args.coupled_only:
        print(json.dumps({"coupled": coupled_measurement()}))
        return 0
    if args.separable_only:
        print(json.dumps({"separable": separable_measurement()}))
        return 0
    if args.throughput_only:
        print(json.dumps({"throughput_f64": throughput_measurement(args.size, args.grains)}))
        return 0
    if args.transport_only:
        print(json.dumps({"transport": coupled_measurement(args.steps, args.warmup, args.size, elastic=False)}))
        return 0
    if args.adjoint_only:
        print(json.dumps({"adjoint": adjoint_measurement(not args.no_cpu)}))
        return 0
    if args.batched_only:
        print(json.dumps({"batched": batched_measurement(args.instances)}))
        return 0
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
