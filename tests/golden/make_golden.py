"""Converts the reference's committed golden data into compact test fixtures.

Run with the path of a reference checkout (argument or GPK_REFERENCE);
writes tests/golden/*.npz.  The sources are the reference's own outputs,
committed in its repository:

* paper/data/validate_extended_base_models/g{13,14,15}_grid_{before,after}.csv
  — label grids written by demos/validate_extended_base_models.cpp:91-100
  before and after 10 x 80 steps of the curved-bicrystal tests G13-G15
  (:767-830): 360^2, IsotropicGrowthThermo(M0=1e-8, sigma0=0.324),
  dx = 1e-7 m, D = 0, gaussian_sigma = 2 (the constructor default).
* paper/data/validation_rex_current_2d/snap_00NN.csv — full-state snapshots
  (utils/csv_writer.hpp:20-56 format) of paper/inputs/validation_rex_current_2d.ini
  (192^2, RecrystallisationThermo(M0=1e-12, sigma0=0.3, E_stored=1e6),
  dx = 1e-6 m, sigma_cells = 2, t_end = 44 s in 24 snapshots, Jdot = 0),
  produced by run_recrystallisation (demos/gpk.cpp:477-553): a loop of
  step(-1) until time >= snap*t_end/24, one CSV per snapshot.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_label_grid(path: str) -> np.ndarray:
    with open(path) as f:
        head = f.readline()
        assert head.startswith("# Ny=")
        parts = dict(p.split("=") for p in head[2:].split())
        ny, nx = int(parts["Ny"]), int(parts["Nx"])
        assert f.readline().strip() == "phi"
        vals = np.array([int(line) for line in f if line.strip()], dtype=np.int32)
    return vals.reshape(ny, nx)


def read_snapshot(path: str):
    with open(path) as f:
        lines = f.readlines()
    time_line = [l for l in lines[:6] if "time=" in l][0]
    time_str = time_line.split("time=")[1].strip()
    rows = [l.split() for l in lines if not l.startswith("#")]
    phi = np.array([int(r[3]) for r in rows], dtype=np.int32)
    alpha_str = np.array([r[4] for r in rows])
    alpha_u = np.array([round(float(a) * 1e6) for a in alpha_str], dtype=np.int64)
    return time_str, phi, alpha_u


def main(ref: str) -> None:
    base = os.path.join(ref, "paper", "data", "validate_extended_base_models")
    grids = {}
    for key in ("g13", "g14", "g15"):
        for when in ("before", "after"):
            g = read_label_grid(os.path.join(base, f"{key}_grid_{when}.csv"))
            assert g.min() >= 0 and g.max() <= 255
            grids[f"{key}_{when}"] = g.astype(np.uint8)
    np.savez_compressed(os.path.join(HERE, "curved_bicrystals_360.npz"), **grids)

    snapdir = os.path.join(ref, "paper", "data", "validation_rex_current_2d")
    files = sorted(f for f in os.listdir(snapdir) if f.startswith("snap_") and f.endswith(".csv"))
    times, phis, alphas = [], [], []
    for fn in files:
        t, phi, a = read_snapshot(os.path.join(snapdir, fn))
        times.append(t)
        phis.append(phi.reshape(192, 192))
        alphas.append(a.reshape(192, 192))
    phis = np.stack(phis)
    assert phis.min() >= 0 and phis.max() <= 255
    np.savez_compressed(os.path.join(HERE, "rex_192_snapshots.npz"),
                        phi=phis.astype(np.uint8),
                        alpha_micro=np.stack(alphas).astype(np.int32),
                        time_str=np.array(times))
    print("wrote", len(grids), "label grids and", len(files), "snapshots")


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPK_REFERENCE")
    if not _ref:
        sys.exit("usage: python %s <path to the reference checkout> (or set GPK_REFERENCE)" % sys.argv[0])
    main(_ref)
