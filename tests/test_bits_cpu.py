"""Host checks of the prune's bit assembly: the 8 x 4 bit transpose that moves
the appended in-range bits (position 4 jj + ii) to the list's mask layout
(8 ii + jj), compiled from the library's own header as host code."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("SOFIA_NVCC", "/usr/local/cuda/bin/nvcc")

SRC = r"""
#include "common.cuh"
#include <cstdio>
#include <cstdlib>
int main() {
    for (int s = 0; s < 32; ++s) {
        const uint32_t y = sofia::transpose_8x4(1u << s);
        if (y != (1u << (8 * (s & 3) + (s >> 2)))) { printf("bit %d -> %08x\n", s, y); return 1; }
    }
    srand(7);
    for (int k = 0; k < 200000; ++k) {
        const uint32_t x = ((uint32_t)rand() << 16) ^ (uint32_t)rand();
        uint32_t r = 0;
        for (int s = 0; s < 32; ++s)
            if ((x >> s) & 1u) r |= 1u << (8 * (s & 3) + (s >> 2));
        if (sofia::transpose_8x4(x) != r) { printf("word %08x\n", x); return 1; }
    }
    // the prune's append order: j atoms 7..0, within one i atoms 3..0, one
    // funnel-shift append each, then the transpose gives bit 8 ii + jj
    for (int k = 0; k < 20000; ++k) {
        const uint32_t want = ((uint32_t)rand() << 16) ^ (uint32_t)rand();
        uint32_t acc = 0;
        for (int jj = 7; jj >= 0; --jj)
            for (int ii = 3; ii >= 0; --ii) acc = (acc << 1) | ((want >> (8 * ii + jj)) & 1u);
        if (sofia::transpose_8x4(acc) != want) { printf("append %08x\n", want); return 1; }
    }
    printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(not (os.path.exists(NVCC) or shutil.which("nvcc")), reason="needs nvcc")
def test_transpose_8x4_matches_the_mask_layout(tmp_path):
    src = tmp_path / "bits.cu"
    src.write_text(SRC)
    exe = tmp_path / "bits"
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    inc = os.path.join(ROOT, "molecular_simulation_code_b200", "csrc")
    subprocess.run([nvcc, "-std=c++17", "-I", inc, "-I", os.path.join(ROOT, "include"),
                    "-o", str(exe), str(src)], check=True, capture_output=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
