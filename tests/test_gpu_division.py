"""The branch-free division the projector and backprojector use instead of
the compiler's (mk_recip / mk_div, Markstein's method) must round exactly as
__frcp_rn / __fdiv_rn: a test program compiled from the library's own header runs
every divisor significand for exponents -20 .. 19 (3.4e8 reciprocals, 1.3e9
quotients) and 2.4e9 random quotients.  The magic-number floor and
int-to-float conversions are checked for every float below 2^22 in
magnitude."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_branch_free_division_matches_the_compiler_bit_for_bit(tmp_path):
    exe = tmp_path / "div_check"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-I" + os.path.join(ROOT, "mcsart_b200", "csrc"),
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "div_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    counts = [int(x) for x in out.stdout.split()]
    assert counts == [0, 0, 0, 0, 0], counts
