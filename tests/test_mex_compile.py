"""The MATLAB gateways in mcsart_b200/mex compile against the C ABI (MATLAB is
not installed here, so the MEX API comes from a declaration-only shim)."""
import os
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.parametrize("src", ["entry_AUMISART.cpp", "mex_backprojection.cpp", "mex_diff.cpp"])
def test_gateway_compiles(src, tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
           "-I" + os.path.join(ROOT, "tests", "mex_shim"), "-I" + os.path.join(ROOT, "include"),
           "-I/usr/local/cuda/include", os.path.join(ROOT, "mcsart_b200", "mex", src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
