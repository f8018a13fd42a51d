"""The reference's backprojector reads each projection cell through a
linear-filtered texture at the texel's centre; the engine reads memory and
applies tex_texel (csrc/common.cuh): the texel itself, denormals as signed
zeros.  A test program compiled from the library's own header compares tex_texel
with the texture unit on 65536 texels of every sign and magnitude class."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_texel_read_matches_the_texture_unit(tmp_path):
    exe = tmp_path / "texel_check"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-I" + os.path.join(ROOT, "mcsart_b200", "csrc"),
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "texel_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert int(out.stdout.split()[0]) == 0, out.stdout
