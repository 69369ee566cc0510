"""The column passes' work schedule (tmk::ColSchedule in csrc/tm_kernels.cuh),
compiled for the host and run on the CPU.

tests/test_colpass_rg_cpu.py checks a Python restatement of the schedule; this
test builds the C++ struct itself (nvcc, host code only) and checks, for
launch shapes of the library's geometries and batches, that every (column
group, orientation) item goes to exactly one block, that the blocks of one
round hold adjacent groups at the same orientation step, and that no block has
more than max_items() items (the bound k_pass_b_rg's item list relies on).
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cistem_downstream_bah_b200", "csrc")

PROGRAM = r"""
#include "tm_kernels.cuh"
#include <cstdio>
#include <vector>

static int check(int ngroups, int nb, int nblk) {
    std::vector<int> seen((size_t)ngroups * nb, 0);
    int longest = 0;
    for (int b = 0; b < nblk; b++) {
        const tmk::ColSchedule s(ngroups, nb, b, nblk);
        if (s.n > longest) longest = s.n;
        for (int i = 0; i < s.n; i++) {
            int g, o;
            s.locate(i, g, o);
            if (g < 0 || g >= ngroups || o < 0 || o >= nb) return 1;
            seen[(size_t)g * nb + o]++;
        }
    }
    for (int c : seen)
        if (c != 1) return 2;
    if (longest > tmk::ColSchedule::max_items(ngroups, nb, nblk)) return 3;
    // within the whole rounds, step i of every block: one orientation, adjacent groups
    const int rounds = ngroups / nblk;
    for (int i = 0; i < rounds * nb; i++) {
        int g0 = -1, o0 = -1;
        for (int b = 0; b < nblk; b++) {
            const tmk::ColSchedule s(ngroups, nb, b, nblk);
            int g, o;
            s.locate(i, g, o);
            if (b == 0) { g0 = g; o0 = o; }
            else if (o != o0 || g != g0 + b) return 4;
        }
    }
    return 0;
}

int main() {
    const int shapes[][3] = {{513, 128, 148}, {513, 32, 148}, {513, 128, 296}, {257, 64, 148}, {129, 256, 148},
                             {1025, 64, 148}, {5, 16, 148}, {17, 1, 148}, {1458, 128, 148}};
    for (const auto& sh : shapes) {
        const int rc = check(sh[0], sh[1], sh[2]);
        if (rc) {
            std::printf("FAIL %d %d %d: %d\n", sh[0], sh[1], sh[2], rc);
            return 1;
        }
    }
    std::printf("OK\n");
    return 0;
}
"""


def test_col_schedule_compiled_for_the_host(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    src = tmp_path / "sched.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "sched"
    # the header's device code is compiled for sm_100a as in the library; only host code runs
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "--extended-lambda", "-I", CSRC,
                    "-o", str(exe), str(src)], check=True, capture_output=True, timeout=600)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout
