"""Generates tests/golden/alcu_trajectory.npz from the reference's own driver.

Runs `run_case` of the reference's Al-Cu material module
(scripts/run_alcu_gpk_microstructure.py:847-1050) on a small 2-D case (64^2,
two sphere nuclei of variants 1 and 2, dx 0.5 nm, 200 s of simulated time)
with its per-step transport and remap functions wrapped, and records the
arguments and results of every call of

  neighbor_competitor, precip_fraction, variant_fraction_fields,
  interface_matrix_composition, diffuse_conservative_subcycled,
  conservative_partition_transfer, commit_topology_transactions,
  conservative_gaussian_remap

in the first two steps and in the steps around the first crossing events, so
that the device functions can be replayed on states the simulation itself
produces; and every call of spectral_elasticity (99-190) in the whole run,
with its variant fractions and results.  Arrays are stored once each
(deduplicated by content).  The driver's own output files go to a
temporary folder.  Run it where the reference tree is present:

    python tests/golden/make_alcu_trajectory.py [path/to/reference]
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "alcu_trajectory.npz")

NAMES = ["neighbor_competitor", "precip_fraction", "variant_fraction_fields", "interface_matrix_composition",
         "diffuse_conservative_subcycled", "conservative_partition_transfer", "commit_topology_transactions",
         "conservative_gaussian_remap"]
# arguments each function updates in place (recorded after the call too)
IN_PLACE = {"conservative_partition_transfer": [0], "commit_topology_transactions": [0, 1],
            "conservative_gaussian_remap": [0, 1]}


def load_reference(root: str):
    path = os.path.join(root, "scripts", "run_alcu_gpk_microstructure.py")
    spec = importlib.util.spec_from_file_location("gpk_ref_alcu", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpk_ref_alcu"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(root: str) -> None:
    ref = load_reference(root)
    ref.OUT = Path(tempfile.mkdtemp())
    calls = []      # (step, name, args (keys or scalars), outputs (keys), in-place outputs (keys))
    arrays = {}
    state = {"step": 0, "params": None}

    def key(a):
        a = np.ascontiguousarray(a)
        h = hashlib.sha1(a.tobytes() + str(a.dtype).encode() + str(a.shape).encode()).hexdigest()[:16]
        arrays.setdefault(h, a.copy())
        return h

    def encode(v):
        if isinstance(v, np.ndarray):
            return {"a": key(v)}
        if isinstance(v, (bool, np.bool_)):
            return {"b": bool(v)}
        if isinstance(v, (int, np.integer)):
            return {"i": int(v)}
        if isinstance(v, (float, np.floating)):
            return {"f": float(v)}
        return {"p": None}  # the Parameters object: recorded once below

    for name in NAMES:
        f = getattr(ref, name)

        def wrap(*args, _f=f, _n=name):
            if state["params"] is None:
                for a in args:
                    if hasattr(a, "c_theta"):
                        state["params"] = {k: float(getattr(a, k)) for k in
                                           ("dx", "diffusivity", "c_matrix_eq", "c_theta",
                                            "composition_extension_sigma_cells", "remap_sigma_cells")}
            before = [encode(a) for a in args]
            result = _f(*args)
            outs = result if isinstance(result, tuple) else (result,)
            after = {i: encode(args[i]) for i in IN_PLACE.get(_n, [])}
            calls.append({"step": state["step"], "name": _n, "args": before,
                          "out": [encode(o) for o in outs], "inplace": {str(k): v for k, v in after.items()}})
            if _n == "commit_topology_transactions":
                state["step"] += 1
            return result

        setattr(ref, name, wrap)
    spectral = []
    f_spec = ref.spectral_elasticity

    def spec_wrap(vf, p):
        r = f_spec(vf, p)
        spectral.append({"vf": key(vf), "driving": key(r[0]), "energy": key(r[1]), "hydro": key(r[2]),
                         "residual": float(r[3])})
        return r

    ref.spectral_elasticity = spec_wrap
    ref.run_case("trajectory", (64, 64), 2, 4.0, 200.0, [0.0], 7, dx=0.5e-9,
                 seed_layout=[((18, 20), 1, 1.0), ((44, 42), 2, 1.0)], initial_shape="sphere")
    # steps kept: the first two, and each crossing step with the next
    # (which holds that step's remap), for the first four crossing events
    keep = {0, 1}
    events = 0
    for c in calls:
        if c["name"] == "commit_topology_transactions" and arrays[c["args"][3]["a"]].any() and events < 4:
            keep |= {c["step"], c["step"] + 1}
            events += 1
    kept = [c for c in calls if c["step"] in keep]
    used = set()
    for c in spectral:
        used |= {c["vf"], c["driving"], c["energy"], c["hydro"]}
    for c in kept:
        for e in c["args"] + c["out"] + list(c["inplace"].values()):
            if "a" in e:
                used.add(e["a"])
    out = {f"arr_{k}": arrays[k] for k in used}
    # the taps scipy sampled in this process, for the two widths the module uses
    for sigma in (state["params"]["composition_extension_sigma_cells"], state["params"]["remap_sigma_cells"]):
        r = int(4.0 * sigma + 0.5)
        x = np.arange(-r, r + 1)
        phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
        out[f"taps_{int(round(sigma * 100))}"] = phi / phi.sum()
    out["calls"] = np.frombuffer(json.dumps(kept).encode(), dtype=np.uint8)
    out["spectral"] = np.frombuffer(json.dumps(spectral).encode(), dtype=np.uint8)
    out["elastic"] = np.asarray([float(getattr(ref.Parameters(), k)) for k in
                                 ("c11", "c12", "c44", "eigen_small", "eigen_large")])
    out["params"] = np.frombuffer(json.dumps(state["params"]).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, len(kept), "calls,", len(spectral), "spectral solves,", len(used), "arrays,", events,
          "crossing events")


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPK_REFERENCE")
    if not _ref:
        sys.exit("usage: python %s <path to the reference checkout> (or set GPK_REFERENCE)" % sys.argv[0])
    main(_ref)
