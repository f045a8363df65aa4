"""The partition threshold loop of qpart_ptr_EF (graph_cuda_partition.hpp:27-54),
`while (avg < g && bump < limit) { avg += 1; ++bump; }`, runs on the device as
`bump_until` (f2m_b200/csrc/f2m_device.cuh), which takes the stretches where
every `+= 1` is exact in one addition.  This test compiles that function for
the host with the system C++ compiler (no FP contraction, as on the device:
the function has no multiply-add to contract) and compares it with the plain
loop on random and edge cases: binade crossings, values around zero, huge
targets and the bump limit."""
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "f2m_b200", "csrc", "f2m_device.cuh")

HARNESS = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#define __device__
#define __forceinline__ inline
%(func)s
static void plain(double& avg, int& bump, double g, int limit) {
    while (avg < g && bump < limit) { avg += 1; ++bump; }
}
int main() {
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> U(0, 1);
    const double sp[] = {0.0, -0.0, 0.3, -0.3, 1.0, -1.0, 0.999999999, -0.999999999, 2.0, 4.0 - 1e-15,
                         1024.5, -1024.5, 4503599627370495.5, 4503599627370496.0, -5.3, 1e-300, 7.7e5};
    const int nsp = sizeof(sp) / sizeof(sp[0]);
    long long bad = 0;
    for (int it = 0; it < 300000; ++it) {
        double avg, g;
        int bump = (int)(U(rng) * 100), limit = 1 << 20;
        switch (it %% 6) {
            case 0: avg = (U(rng) - 0.5) * 2e4; g = avg + U(rng) * 3e4; break;
            case 1: avg = std::ldexp(1.0, (int)(U(rng) * 30)) - U(rng) * 5; g = avg + U(rng) * 100; break;
            case 2: avg = (U(rng) - 0.5) * 4; g = avg + U(rng) * 8; break;
            case 3: avg = sp[it %% nsp]; g = sp[(it / nsp) %% nsp] + U(rng) * 10; break;
            case 4: avg = (U(rng) - 0.5) * 1e6; g = INFINITY; limit = bump + (int)(U(rng) * 2e5); break;
            default: avg = std::ldexp(U(rng) + 1, 40 + (int)(U(rng) * 12)); g = avg + U(rng) * 1e5;
                     limit = bump + 100000;
        }
        double a1 = avg, a2 = avg;
        int b1 = bump, b2 = bump;
        plain(a1, b1, g, limit);
        bump_until(a2, b2, g, limit);
        if (std::memcmp(&a1, &a2, 8) != 0 || b1 != b2) {
            if (bad < 5) std::printf("mismatch avg %%.17g g %%.17g: %%.17g/%%d vs %%.17g/%%d\n", avg, g, a1, b1, a2, b2);
            ++bad;
        }
    }
    std::printf("mismatches %%lld\n", bad);
    return bad != 0;
}
"""


def _function_source():
    text = open(HEADER).read()
    m = re.search(r"__device__ __forceinline__ void bump_until\(.*?\n}\n", text, re.S)
    assert m, "bump_until not found in f2m_device.cuh"
    return m.group(0)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_bump_until_matches_the_plain_loop(tmp_path):
    src = tmp_path / "bump.cpp"
    exe = tmp_path / "bump"
    src.write_text(HARNESS % {"func": _function_source()})
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-o", str(exe), str(src)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
