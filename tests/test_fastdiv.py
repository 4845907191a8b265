"""The multiply-shift division of the pencil tiles (FastDiv in csrc/pencil.cuh) against true integer
division: every divisor the tilings can use, dense small dividends, the ends of the range and random
pairs (host build of the header with nvcc; no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include "pencil.cuh"
int main() {
    unsigned long long bad = 0, checks = 0;
    auto check = [&](unsigned n, unsigned D, const img::FastDiv& f) {
        ++checks;
        if (f.div(n) != n / D && bad++ < 5) std::printf("bad n=%u D=%u\n", n, D);
    };
    for (unsigned D = 1; D <= 4096; ++D) {
        const img::FastDiv f = img::make_fastdiv(D);
        for (unsigned n = 0; n < 20000; ++n) check(n, D, f);
        const unsigned top = 2147483647u;
        for (unsigned k = 0; k < 64; ++k) check(top - k, D, f);
        check((top / D) * D, D, f);
        check((top / D) * D - 1, D, f);
    }
    unsigned long long x = 88172645463325252ull;
    for (int r = 0; r < 3000000; ++r) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        const unsigned D = 1 + (unsigned)(x % 2000000u);
        const unsigned n = (unsigned)(x >> 33) & 0x7fffffffu;
        check(n, D, img::make_fastdiv(D));
    }
    std::printf("checks %llu bad %llu\n", checks, bad);
    return bad != 0;
}
"""


def test_fastdiv_matches_integer_division(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "fastdiv.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "fastdiv"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "imogen_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "bad 0" in r.stdout
