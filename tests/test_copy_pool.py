"""Host copy threads of the blocking render (dr::CopyPool, csrc/dr_host.h):
compiled here into a small host program that copies random ranges of random
sizes -- below and above the 4 MB floor, zero-length ones, two ranges per
call, one pool reused across calls and then destroyed -- and compares every
byte.  No GPU is involved."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "droplet-render_b200", "csrc")

PROGRAM = r"""
#include "dr_host.h"
#include <cstdio>
#include <random>
int main() {
    std::mt19937 rng(7);
    for (int pools = 0; pools < 3; ++pools) {
        dr::CopyPool pool;
        for (int it = 0; it < 40; ++it) {
            size_t n = it % 7 == 0 ? 0 : (it % 3 == 0 ? (rng() % (1u << 20)) : (rng() % (12u << 20))) + 1;
            std::vector<unsigned char> a(n + 1), b(n + 1, 0), c(n / 3 + 1), d(n / 3 + 1, 0);
            for (auto &x : a) x = (unsigned char)rng();
            for (auto &x : c) x = (unsigned char)rng();
            const dr::CopyPool::Range r[2] = {{b.data(), a.data(), n}, {d.data(), c.data(), c.size()}};
            pool.copy(r, 2);
            for (size_t i = 0; i < n; ++i)
                if (a[i] != b[i]) { std::printf("range 0 differs at %zu (call %d)\n", i, it); return 1; }
            if (b[n] != 0) { std::printf("wrote past range 0 (call %d)\n", it); return 1; }
            if (c != d) { std::printf("range 1 differs (call %d)\n", it); return 1; }
        }
    }
    std::printf("ok\n");
    return 0;
}
"""


def cuda_include():
    for d in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "cuda_runtime.h")):
            return os.path.join(d, "include")
    return None


def test_copy_pool_copies_every_byte(tmp_path):
    inc = cuda_include()
    if shutil.which("g++") is None or inc is None:
        pytest.skip("needs g++ and the CUDA headers")
    src = tmp_path / "copy_pool.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "copy_pool"
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", f"-I{CSRC}", f"-I{inc}", str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
