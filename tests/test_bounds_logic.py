"""The index check of the bounds-checked debug build (csrc/fsl_check.cuh),
compiled for the host and run on the CPU: an index out of range is counted,
the first one recorded (file id, line, index, extent) and the access
redirected to element 0; indices in range pass unchanged; a stencil's two
extremes are checked.  The mistakes are planted here, on the CPU: no test
plants an out-of-range index on the GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "freeshearlayer_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include "fsl_check.cuh"
using fsl::chk::Record;
int main()
{
    Record r{};
    const long long a = fsl::chk::at_into(&r, 5, 10, 3, 100);   // in range
    const long long b = fsl::chk::at_into(&r, 10, 10, 3, 101);  // one past the end: the first
    const long long c = fsl::chk::at_into(&r, -1, 10, 3, 102);  // negative
    const bool s1 = fsl::chk::span_into(&r, 5, -5, 4, 10, 4, 103); // 0 .. 9: inside
    const bool s2 = fsl::chk::span_into(&r, 5, -6, 4, 10, 4, 104); // -1: outside
    const bool s3 = fsl::chk::span_into(&r, 5, -5, 5, 10, 4, 105); // 10: outside
    std::printf("%lld %lld %lld %d %d %d %llu %d %d %lld %lld\n", a, b, c, (int)s1, (int)s2, (int)s3, r.hits,
                r.unit, r.line, r.index, r.extent);
    return 0;
}
"""


def test_index_check_counts_records_and_redirects(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "chk.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "chk"
    subprocess.run([nvcc, "-std=c++17", "-I" + CSRC, "-o", str(exe), str(src)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    a, b, c, s1, s2, s3, hits, unit, line, index, extent = (int(x) for x in out)
    assert (a, b, c) == (5, 0, 0)
    assert (s1, s2, s3) == (1, 0, 0)
    assert hits == 4
    assert (unit, line, index, extent) == (3, 101, 10, 10)
