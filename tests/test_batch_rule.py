"""CPU: the batch graph's branch-count rule (csrc/batch_rule.h), compiled
with the host compiler into a small driver and checked on fixed L2 sizes
and per-plan bytes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "daggerfft.jl_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include "batch_rule.h"
int main(int argc, char** argv) {
  for (int i = 1; i + 3 < argc; i += 4)
    std::printf("%d\n", dfft::batch_branch_rule(std::atoi(argv[i]), std::atof(argv[i + 1]),
                                                std::atoll(argv[i + 2]), std::atoi(argv[i + 3])));
  return 0;
}
"""

CASES = [
    # (plans, total in+out bytes, L2 bytes, max branches) -> branches
    ((64, 64 * 24.0e6, 126 * 2 ** 20, 8), 4),      # the 64 uneven grids: 0.8 x 126 MiB / 24 MB
    ((64, 64 * 2.0e6, 126 * 2 ** 20, 8), 8),       # small grids: clamped to the stream count
    ((64, 64 * 200.0e6, 126 * 2 ** 20, 8), 2),     # grids larger than L2: at least two branches
    ((3, 3 * 2.0e6, 126 * 2 ** 20, 8), 3),         # never more branches than plans
    ((1, 1.0e6, 126 * 2 ** 20, 8), 1),
    ((16, 16 * 24.0e6, 0, 8), 8),                  # L2 size unknown: the stream count
    ((64, 64 * 24.0e6, 50 * 2 ** 20, 8), 2),       # a smaller L2
]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("batch_rule")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = d / "drv"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return str(exe)


def test_branch_rule(driver):
    args = []
    for (n, tot, l2, mx), _ in CASES:
        args += [str(n), repr(tot), str(l2), str(mx)]
    out = subprocess.run([driver] + args, check=True, capture_output=True, text=True).stdout.split()
    assert [int(x) for x in out] == [want for _, want in CASES]
