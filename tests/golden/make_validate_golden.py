"""Records the standard output of the reference's own validation programs.

The programs (demos/validate_*.cpp of albert-hzbn/GPK) are built unchanged
from the reference's sources by `make -f oracle/Makefile demos` into
oracle/_ref/cpu/ (GPK_REFERENCE names the checkout).  Each one is run here,
on the CPU, in an empty working directory (some write CSV files), and its
standard output is written to tests/golden/validate/<program>.txt.  The GPU
test runs the same programs built against the drop-in header and
libgpk_b200.so and compares their output with these files.

    python tests/golden/make_validate_golden.py [program ...]
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CPU = os.path.join(ROOT, "oracle", "_ref", "cpu")
OUT = os.path.join(HERE, "validate")
PROGRAMS = ["validate_topology_transactions", "validate_extended_base_models", "validate_real_materials",
            "validate_dimensional_multiphase", "validate_theory_foundations", "validate_interface_local_geometry"]


def main(names):
    os.makedirs(OUT, exist_ok=True)
    for name in names:
        exe = os.path.join(CPU, name)
        if not os.path.exists(exe):
            sys.exit(f"{exe} is missing: run make -f oracle/Makefile demos with GPK_REFERENCE set")
        with tempfile.TemporaryDirectory() as wd:
            r = subprocess.run([exe], cwd=wd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.exit(f"{name} exited with {r.returncode}:\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        with open(os.path.join(OUT, name + ".txt"), "w") as f:
            f.write(r.stdout)
        print(name, len(r.stdout.splitlines()), "lines")


if __name__ == "__main__":
    main(sys.argv[1:] or PROGRAMS)
