"""The covariance kernel's accumulator index map (csrc/gls_pca_pairs.h).

k_pca_cov finds the upper-triangle entry (r, c) its thread owns from the
thread index instead of a table loaded into constant memory, so the kernel
works on every device without per-device set-up. This compiles the same
header with the host compiler and checks the closed form against the
enumeration the accumulators are laid out by (row-major over r <= c, 325
entries); the eigen-solves read the accumulators back through the same
header's pca_tri_index."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HDR = ROOT / "glasscamerapublic_b200" / "csrc" / "gls_pca_pairs.h"

PROG = r"""
#include <cstdio>
#include "gls_pca_pairs.h"
int main() {
    int k = 0;
    for (int i = 0; i < 25; i++)
        for (int j = i; j < 25; j++, k++) {
            int r = -1, c = -1;
            gls::pca_pair(k, r, c);
            std::printf("%d %d %d %d\n", k, r, c, gls::pca_tri_index(i, j));
        }
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_pca_pair_closed_form_matches_enumeration(tmp_path):
    src = tmp_path / "pairs.cpp"
    src.write_text(PROG)
    exe = tmp_path / "pairs"
    r = subprocess.run(["g++", "-std=c++20", "-O1", "-Wall", "-Werror", f"-I{HDR.parent}", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [tuple(map(int, ln.split())) for ln in out if ln.strip()]
    expect = [(i, j) for i in range(25) for j in range(i, 25)]
    assert len(rows) == len(expect) == 325
    for k, (t, r, c, idx) in enumerate(rows):
        assert t == k and (r, c) == expect[k] and idx == k
