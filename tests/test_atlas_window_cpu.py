"""The composition's phi-index arithmetic on the CPU (no GPU): the helpers of
csrc/icp_atlas_window.cuh, compiled with g++ -- driven both directly (phi_sub, phi_cell per cell
and shift, as atlas_compose_kernel uses them) and through a sliding window (the first cell's
index set after a run of zero weights, stepped down by one per shift) -- give the cell
(p0 + k - s) mod np, phi-reflected when q = 1, for every output cell, shift and weight
pattern -- including strips past the row end and rows narrower than a strip."""
from __future__ import annotations

import subprocess

from conftest import ROOT

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "icp_atlas_window.cuh"
using namespace icp;
int main()
{
    const unsigned kPT = 8;
    const unsigned sizes[] = {1, 2, 3, 5, 7, 8, 9, 12, 31, 64, 257, 1800, 2100};
    unsigned long long checked = 0;
    srand(12345);
    for (unsigned np : sizes)
        for (int pattern = 0; pattern < 4; ++pattern) {
            std::vector<int> nz(np);
            for (unsigned s = 0; s < np; ++s)
                nz[s] = pattern == 0 ? 1 : pattern == 1 ? (s % 3 != 1) : pattern == 2 ? (rand() % 7 == 0) : (s > np / 2);
            for (unsigned p0 = 0; p0 < np + 2 * kPT * 256 && p0 < 5000; p0 += (np > 64 ? 37 : 1) * kPT / 8 + 1)
                for (int q = 0; q < 2; ++q) {
                    const unsigned pm = p0 % np;
                    unsigned m = 0;
                    bool gap = true;
                    unsigned idx[kPT];
                    for (unsigned s = 0; s < np; ++s) {
                        if (!nz[s]) { gap = true; continue; }
                        if (gap) {
                            m = phi_sub(pm, s, np);
                            for (unsigned k = 0; k < kPT; ++k) idx[k] = phi_cell(phi_add(m, k, np), np, q);
                            gap = false;
                        } else {
                            m = phi_prev(m, np);
                            for (unsigned k = kPT - 1; k > 0; --k) idx[k] = idx[k - 1];
                            idx[0] = phi_cell(m, np, q);
                        }
                        for (unsigned k = 0; k < kPT; ++k) {
                            const long long r = (((long long)p0 + k - (long long)s) % (long long)np + np) % np;
                            const unsigned want = q ? np - 1 - (unsigned)r : (unsigned)r;
                            const unsigned direct = phi_cell(phi_sub((p0 + k) % np, s, np), np, q);
                            if (idx[k] != want || idx[k] >= np || direct != want) {
                                printf("MISMATCH np=%u p0=%u q=%d s=%u k=%u got=%u want=%u\n", np, p0, q, s, k, idx[k], want);
                                return 1;
                            }
                            ++checked;
                        }
                    }
                }
        }
    printf("OK %llu\n", checked);
    return 0;
}
"""


def test_phi_window_indices(tmp_path):
    src = tmp_path / "window.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "window"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "ice_crystal_phase_b200" / "csrc"), str(src), "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert r.stdout.startswith("OK ") and int(r.stdout.split()[1]) > 1_000_000
