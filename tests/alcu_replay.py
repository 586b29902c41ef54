"""Replays the calls recorded in tests/golden/alcu_trajectory.npz (the
reference's driver on a 64^2 Al-Cu case, make_alcu_trajectory.py) through a
set of implementations and compares every result bit for bit."""
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(__file__), "golden", "alcu_trajectory.npz")


def load():
    z = np.load(PATH)
    calls = json.loads(bytes(z["calls"]).decode())
    params = json.loads(bytes(z["params"]).decode())
    return z, calls, params


def same(a, b):
    a = np.ascontiguousarray(np.asarray(a))
    b = np.ascontiguousarray(np.asarray(b))
    if a.dtype == bool or b.dtype == bool:
        return a.shape == b.shape and np.array_equal(a.astype(bool), b.astype(bool))
    return a.shape == b.shape and a.dtype.itemsize == b.dtype.itemsize and np.array_equal(a.view(np.uint8),
                                                                                          b.view(np.uint8))


def replay(impl, check_taps=None):
    """impl: name -> callable taking the decoded arguments (arrays copied) and
    returning (outputs tuple, in-place argument indices -> arrays after)."""
    z, calls, params = load()

    def dec(e):
        if "a" in e:
            return z["arr_" + e["a"]].copy()
        if "f" in e:
            return e["f"]
        if "i" in e:
            return e["i"]
        if "b" in e:
            return e["b"]
        return None  # the Parameters object

    checked = 0
    for c in calls:
        args = [dec(e) for e in c["args"]]
        outs, inplace = impl[c["name"]](args, params, z)
        for o, e in zip(outs, c["out"]):
            if "a" in e:
                assert same(o, z["arr_" + e["a"]]), (c["name"], c["step"])
            elif "i" in e:
                assert int(o) == e["i"], (c["name"], c["step"])
        for k, e in c["inplace"].items():
            assert same(inplace[int(k)], z["arr_" + e["a"]]), (c["name"], c["step"], "argument", k)
        checked += 1
    return checked


def spectral_cases():
    """(variant fractions, p, reference results) of every spectral solve the
    driver made in the recorded run."""
    import types

    z, _, params = load()
    el = z["elastic"]
    p = types.SimpleNamespace(dx=params["dx"], c11=el[0], c12=el[1], c44=el[2], eigen_small=el[3],
                              eigen_large=el[4])
    out = []
    for c in json.loads(bytes(z["spectral"]).decode()):
        out.append((z["arr_" + c["vf"]], p, {k: z["arr_" + c[k]] for k in ("driving", "energy", "hydro")},
                    c["residual"]))
    return out


def rel_err(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))
