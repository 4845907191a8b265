"""The window rows of the window magnet kernels (csrc/seg_magnet.cuh): where one wrap reaches every row
-- a pencil of N >= C + reach rows, reach the halo the window has beyond its segment -- the select-only
form win_row_once gives the same row as the looping win_row_multi, and every row is inside the pencil,
for circ and const ends, every segment start the tilings make and the chain's and CT's windows (host
build of the header with nvcc; no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include "magnet_sweep.cuh"
#include "seg_magnet.cuh"
int main() {
    unsigned long long bad = 0, checks = 0, multi_only = 0;
    const int Cs[] = {1, 2, 3, 4, 8};
    for (int C : Cs) {
        const int shapes[2][2] = {{C + 8, 4}, {C + 2, 1}};   // (W, H): the chain's window, CT's
        for (const auto& sh : shapes) {
            const int W = sh[0], H = sh[1];
            const int reach = H > W - C - H ? H : W - C - H;
            for (int N = 1; N <= 200; ++N) {
                const int S = (N + C - 1) / C;
                for (int s = 0; s < S; ++s)
                    for (int lo = 0; lo < 2; ++lo)
                        for (int hi = 0; hi < 2; ++hi)
                            for (int j = 0; j < W; ++j) {
                                const int r = s * C + j - H;
                                const int m = img::win_row_multi(r, N, lo, hi);
                                ++checks;
                                if (m < 0 || m >= N) ++bad;
                                if (N >= C + reach) {
                                    const int o = img::win_row_once(r, N, lo, hi);
                                    if (o != m && bad++ < 5) std::printf("bad C=%d N=%d r=%d\n", C, N, r);
                                } else {
                                    ++multi_only;
                                }
                            }
            }
        }
    }
    std::printf("checks %llu multi_only %llu bad %llu\n", checks, multi_only, bad);
    return bad != 0;
}
"""


def test_select_rows_match_looping_rows(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "winrows.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "winrows"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "imogen_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "bad 0" in r.stdout
