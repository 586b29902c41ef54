"""The reference's own demo programs build against the drop-in header.

A maintainer swaps include/gpk_core.hpp of the reference for this
repository's and links libgpk_b200.so in place of the reference's src/*.cpp.
This test does exactly that in a temporary directory (the reference's other
headers are linked in beside our gpk_core.hpp, so that their
`#include "gpk_core.hpp"` resolves to ours) and compiles and links four of
the reference's programs unchanged, the full `gpk` driver among them.
Skipped unless GPK_REFERENCE names a reference checkout.
"""
import os
import subprocess

import pytest

REF = os.environ.get("GPK_REFERENCE", "")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gpk_b200")
DEMOS = ["validate_topology_transactions", "grain_growth", "validate_interface_local_geometry", "gpk"]


@pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF, "demos")),
                    reason="reference tree not given (GPK_REFERENCE)")
@pytest.mark.parametrize("demo", DEMOS)
def test_reference_demo_builds_against_dropin(demo, tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libgpk_b200.so")):
        pytest.skip("library not built")
    inc = tmp_path / "include"
    inc.mkdir()
    os.symlink(os.path.join(ROOT, "include", "gpk_core.hpp"), inc / "gpk_core.hpp")
    os.symlink(os.path.join(ROOT, "include", "gpk_b200.h"), inc / "gpk_b200.h")
    for h in os.listdir(os.path.join(REF, "include")):
        if h != "gpk_core.hpp":
            os.symlink(os.path.join(REF, "include", h), inc / h)
    cmd = ["g++", "-std=c++17", "-O1", "-fopenmp", "-I", str(inc), "-I", os.path.join(REF, "utils"),
           os.path.join(REF, "demos", demo + ".cpp"), "-o", str(tmp_path / demo),
           "-L", LIBDIR, "-lgpk_b200", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


PROBE_SRC = r"""
#include <cstdio>
#include <stdexcept>
#include "gpk_core.hpp"
using namespace gpk;
// the reference's demos/validate_interface_local_geometry.cpp defines one like this
struct ConstantMobility final : ThermoModel {
    ConstantMobility() { sigma0 = 0.5f; grain_network = true; }
    float mobility(float, float, float, float, float, float) const override { return 1.0f; }
};
struct PlainCopy : ThermoModel {};   // every virtual inherited: the base law
struct Driven : ThermoModel {
    float bulk_driving_force(int, int, float c, float) const override { return c; }
};
int main() {
    gpk_thermo_desc a = describe_thermo(ConstantMobility());
    gpk_thermo_desc b = describe_thermo(PlainCopy());
    std::printf("%d %g %d %g\n", a.model, a.M0, a.grain_network, a.sigma0);
    std::printf("%d\n", b.model);
    try { describe_thermo(Driven()); std::printf("described\n"); }
    catch (const std::runtime_error&) { std::printf("rejected\n"); }
    return 0;
}
"""


def test_unknown_subclasses_are_described_by_behaviour(tmp_path):
    """Subclasses the shim does not know by name: described when every
    virtual matches a device law (constant mobility -> the
    AnisotropicGrowthThermo law), rejected otherwise.  Host only."""
    if not os.path.exists(os.path.join(LIBDIR, "libgpk_b200.so")):
        pytest.skip("library not built")
    src = tmp_path / "probe.cpp"
    src.write_text(PROBE_SRC)
    exe = tmp_path / "probe"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", LIBDIR, "-lgpk_b200", "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120).stdout.split("\n")
    assert out[0] == "2 1 1 0.5"          # GPK_MODEL_ANISOTROPIC, M0 = 1, grain_network, sigma0
    assert out[1] == "0"                  # GPK_MODEL_BASE
    assert out[2] == "rejected"
