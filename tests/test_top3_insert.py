"""The node gradient of cuda_get_Nodes_grad_R (graph_cuda_grad.hpp:65-84) keeps
the three smallest reduced costs with a compare chain: `if (v < v0) ...;
if (v < v1) ...; if (v < v2) ...`.  On the device that chain runs as
`top3_insert` (f2m_b200/csrc/f2m_device.cuh): three FP64 compares and selects,
used while the first value is below the 1e6 sentinels (the triple then stays
sorted).  This test compiles `top3_insert` and `half_grad` for the host with
the system C++ compiler and compares them with the reference's chain, bit for
bit, on random lists with ties, signed zeros, infinities and NaN."""
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "f2m_b200", "csrc", "f2m_device.cuh")
KERNELS = os.path.join(os.path.dirname(HERE), "f2m_b200", "csrc", "f2m_kernels.cu")

HARNESS = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#define __device__
#define __forceinline__ inline
%(insert)s
%(half)s
// the reference's chain (graph_cuda_grad.hpp:71-81), returning grad/2
static double chain(int n, const double* a) {
    double v0 = a[0], v1 = 1e6, v2 = 1e6;
    for (int i = 1; i < n; ++i) {
        const double v = a[i];
        if (v < v0) { v2 = v1; v1 = v0; v0 = v; continue; }
        if (v < v1) { v2 = v1; v1 = v; continue; }
        if (v < v2) { v2 = v; continue; }
    }
    return (-(v1 + v2) / 2) * 0.5;
}
int main() {
    std::mt19937_64 rng(5);
    std::uniform_real_distribution<double> U(0, 1);
    const double sp[] = {0.0, -0.0, 1e6, -1e6, 1e6 + 1, INFINITY, -INFINITY, NAN, 0.5, 0.5, -3.25};
    const int nsp = sizeof(sp) / sizeof(sp[0]);
    long long bad = 0;
    double a[40];
    for (int it = 0; it < 400000; ++it) {
        const int n = 1 + (int)(U(rng) * 39);
        const int mode = it %% 4;
        for (int k = 0; k < n; ++k) {
            if (mode == 0) a[k] = (U(rng) - 0.5) * 20;                 // distinct values
            else if (mode == 1) a[k] = (double)(int)(U(rng) * 6) - 2;  // many ties
            else if (mode == 2) a[k] = sp[(int)(U(rng) * nsp)];        // specials
            else a[k] = (U(rng) < 0.2) ? sp[(int)(U(rng) * nsp)] : (U(rng) - 0.3) * 4e6;
        }
        const double r = chain(n, a);
        const double g = half_grad(n, [&](int k) { return a[k]; });
        if (std::memcmp(&r, &g, 8) != 0 && !(r != r && g != g)) {
            if (bad < 5) std::printf("mismatch n %%d: %%.17g vs %%.17g\n", n, r, g);
            ++bad;
        }
    }
    std::printf("mismatches %%lld\n", bad);
    return bad != 0;
}
"""


def _source(path, pattern):
    text = open(path).read()
    m = re.search(pattern, text, re.S)
    assert m, f"{pattern} not found in {path}"
    return m.group(0)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_top3_insert_matches_the_reference_chain(tmp_path):
    insert = _source(HEADER, r"__device__ __forceinline__ void top3_insert\(.*?\n}\n")
    half = _source(KERNELS, r"template <class Get>\n__device__ __forceinline__ double half_grad\(.*?\n}\n")
    half = half.replace("#pragma unroll 4\n", "")
    src = tmp_path / "top3.cpp"
    exe = tmp_path / "top3"
    src.write_text(HARNESS % {"insert": insert, "half": half})
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", str(exe), str(src)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
