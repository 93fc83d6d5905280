"""Host logic of the INT8 product's tile width (fb::i8_tile_width, tc_gemm.h).

The width of 64, 48 or 32 columns that minimises (CTA waves on 148 SMs) x
width, ties to the wider tile: the time step's choice for its two eigen
transforms.  Compiled on the host with g++; no GPU.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

PROGRAM = r"""
#include "tc_gemm.h"
#include <cstdio>
int main() {
    const int cases[][3] = {{768, 1024, 148}, {256, 384, 148}, {1536, 2048, 148}, {128, 64, 148},
                            {768, 1024, 132}, {1024, 1024, 148}, {200, 100, 148}};
    for (const auto &c : cases) std::printf("%d\n", fb::i8_tile_width(c[0], c[1], c[2]));
}
"""


def _waves_cost(rows, cols, w, sms):
    ctas = ((rows + 127) // 128) * ((cols + w - 1) // w)
    return ((ctas + sms - 1) // sms) * w


def _model(rows, cols, sms):
    best_w, best = 64, None
    for w in (64, 48, 32):
        cost = _waves_cost(rows, cols, w, sms)
        if best is None or cost < best:
            best, best_w = cost, w
    return best_w


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(os.path.join(CUDA, "include")),
                    reason="needs g++ and the CUDA headers")
def test_i8_tile_width(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.check_call(["g++", "-std=c++17", "-I", os.path.join(ROOT, "fribois2d_b200", "csrc"),
                           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
                           str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    cases = [(768, 1024, 148), (256, 384, 148), (1536, 2048, 148), (128, 64, 148),
             (768, 1024, 132), (1024, 1024, 148), (200, 100, 148)]
    assert got == [_model(*c) for c in cases]
    # the benchmark grids: the galloping rectangle fills one wave with 48 columns
    # (132 CTAs; 64 leaves a third of the SMs idle, 32 needs two waves), the
    # small cylinder spreads over the most SMs with 32, and on the 2048 x 1536
    # cylinder the three widths tie (whole waves) and the widest is taken
    assert got[:3] == [48, 32, 64]
