"""GPKGrid::run with GPK_ASYNC_CALLBACKS=1: callbacks on snapshot copies,
on a writer thread, see exactly what they see in the reference's
synchronous order (same steps, labels and times), and a callback's
exception is rethrown by run().  A small C++ driver is built against the
drop-in header."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gpk_b200")

SRC = r"""
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <utility>
#include <vector>
#include "gpk_core.hpp"
#include "gpk_init.h"
using namespace gpk;
struct Iso : ThermoModel {
    Iso() { M0 = 1.f; sigma0 = 1.f; grain_network = true; }
    float mobility(float, float, float, float, float, float) const override { return M0; }
};
static unsigned long long fnv(const std::vector<int32_t>& v) {
    unsigned long long h = 1469598103934665603ull;
    for (int32_t x : v) { h ^= (unsigned)x; h *= 1099511628211ull; }
    return h;
}
int main() {
    auto th = std::make_shared<Iso>();
    for (int mode = 0; mode < 2; ++mode) {
        setenv("GPK_ASYNC_CALLBACKS", mode ? "1" : "0", 1);
        GPKGrid g(1, 96, 96, 1.f, th, 0.f, 1.5f);
        gpk_voronoi_init(1, 96, 96, 40, 7, g.phi.data(), g.g.data(), nullptr);
        std::vector<std::pair<int, unsigned long long>> rec;
        const int n = g.run(40.0, -1.f, [&](const GPKGrid& s, int step) {
            rec.push_back({step, fnv(s.phi) ^ (unsigned long long)(s.time * 1e6)});
        }, 5);
        std::printf("run %d steps %d callbacks %zu final %llx\n", mode, n, rec.size(), fnv(g.phi));
        for (auto& r : rec) std::printf("cb %d %d %llx\n", mode, r.first, r.second);
    }
    setenv("GPK_ASYNC_CALLBACKS", "1", 1);
    GPKGrid g(1, 64, 64, 1.f, th, 0.f, 1.5f);
    gpk_voronoi_init(1, 64, 64, 20, 3, g.phi.data(), g.g.data(), nullptr);
    try {
        g.run(20.0, -1.f, [](const GPKGrid&, int step) { if (step == 10) throw std::runtime_error("stop"); }, 5);
        std::printf("not rethrown\n");
    } catch (const std::runtime_error& e) {
        std::printf("rethrown %s\n", e.what());
    }
    return 0;
}
"""


def test_async_callbacks_match_synchronous(tmp_path):
    src = tmp_path / "cb.cpp"
    src.write_text(SRC)
    exe = tmp_path / "cb"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", LIBDIR, "-lgpk_b200", "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.splitlines()
    runs = [l.split() for l in lines if l.startswith("run ")]
    assert len(runs) == 2 and runs[0][2:] == runs[1][2:] and int(runs[0][5]) > 0
    cb0 = [l.split()[2:] for l in lines if l.startswith("cb 0 ")]
    cb1 = [l.split()[2:] for l in lines if l.startswith("cb 1 ")]
    assert cb0 and cb0 == cb1
    assert "rethrown stop" in lines
