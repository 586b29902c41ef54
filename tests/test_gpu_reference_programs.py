"""The reference's own validation programs, unchanged, run on a B200 through
the drop-in.

Each program (demos/validate_*.cpp of albert-hzbn/GPK) was compiled against
this repository's include/gpk_core.hpp and linked with libgpk_b200.so in
place of the reference's src/*.cpp (oracle/_ref/dropin/, built by
`make -f oracle/Makefile demos`).  Its standard output must equal, line for
line, the output of the same program built from the reference's sources and
run on the CPU (tests/golden/validate/*.txt, recorded by
tests/golden/make_validate_golden.py).  The programs exercise every
ThermoModel subclass of include/gpk_thermo.hpp that the step evaluates:
validate_real_materials alone covers TensorAnisotropy, AnisoOstwald,
Reduction, MagneticAnnealing, Magnetoelastic and NdFeB grain-boundary models
(demos/validate_real_materials.cpp:73-933).

One line differs by design: validate_interface_local_geometry prints the
bytes per cell of the grid's host arrays (allocated_array_bytes), and the
drop-in keeps fewer host arrays; both stay under the program's 110-byte gate.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
GOLDEN = os.path.join(ROOT, "tests", "golden", "validate")

PROGRAMS = [("validate_topology_transactions", 120), ("validate_extended_base_models", 600),
            ("validate_real_materials", 600), ("validate_dimensional_multiphase", 300),
            ("validate_interface_local_geometry", 300), ("validate_theory_foundations", 600)]


def _storage_line(line: str) -> bool:
    return "bytes/cell" in line and "PASS" not in line and "FAIL" not in line


@pytest.mark.parametrize("name,limit", PROGRAMS, ids=[p[0] for p in PROGRAMS])
def test_reference_program_output_on_gpu(name, limit, tmp_path):
    exe = os.path.join(DROPIN, name)
    gold = os.path.join(GOLDEN, name + ".txt")
    if not os.path.exists(exe):
        pytest.skip("drop-in build of the reference's programs not present")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=limit)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = r.stdout.splitlines()
    want = open(gold).read().splitlines()
    if name == "validate_interface_local_geometry":
        got = [l for l in got if not _storage_line(l)]
        want = [l for l in want if not _storage_line(l)]
    assert len(got) == len(want), f"{len(got)} lines vs {len(want)}"
    for k, (a, b) in enumerate(zip(got, want)):
        assert a == b, f"line {k}: drop-in {a!r} vs reference {b!r}"
    assert sum("PASS" in l for l in got) == sum("PASS" in l for l in want)
