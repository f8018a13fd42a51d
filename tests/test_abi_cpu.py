"""The C ABI without a GPU: the library loads, exports every function that
include/mcsart.h declares, and fails cleanly (status codes, messages) where a
device would be needed or an argument is invalid.  No compute is called."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def lib():
    from mcsart_b200 import _lib
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    from mcsart_b200 import _lib
    names = _lib.declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/mcsart.h but not exported"


def test_only_the_c_abi_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "mcsart_b200", "lib",
                                                                    "libmcsart.so")],
                         capture_output=True, text=True, check=True).stdout
    text = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert text and all(t.startswith("mcsart_") for t in text), \
        [t for t in text if not t.startswith("mcsart_")][:10]


def test_version(lib):
    assert lib.mcsart_version() == 10000


def test_create_without_a_device_reports_no_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    rc = lib.mcsart_create(ctypes.byref(h), 0)
    assert rc == -3
    assert b"no CUDA device" in lib.mcsart_last_error()
    assert not h.value


def test_null_context_is_rejected(lib):
    rc = lib.mcsart_projection(None, None, None, 0.0, 500.0, 750.0, 0.8, 128, -63.5, 0.8, 96,
                               -47.5, 64, 64, 64)
    assert rc == -1
    assert b"context is NULL" in lib.mcsart_last_error()
    assert lib.mcsart_set_interp(None, 0) == -1
    assert lib.mcsart_synchronize(None) == -1
    assert lib.mcsart_destroy(None) == 0


def test_default_options(lib):
    from mcsart_b200 import Options
    o = Options()
    lib.mcsart_default_options(ctypes.byref(o))
    assert (o.storage, o.interp, o.use_graph, o.fp_sum, o.fp_groups) == (0, 0, 1, 0, 0)
    assert (o.subset, o.dvf_inverse, o.geom64, o.autotune) == (1, 0, 0, 0)


def test_python_context_raises_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import mcsart_b200 as m
    with pytest.raises(m.McsartError) as e:
        m.Context(0)
    assert e.value.code == m.ERR_NO_DEVICE


def test_header_cites_the_reference_for_each_launcher():
    text = open(os.path.join(ROOT, "include", "mcsart.h")).read()
    for fn, ref in [("mcsart_projection", "host_projection"),
                    ("mcsart_backprojection", "host_backprojection"),
                    ("mcsart_deform", "host_deform"), ("mcsart_deform2", "host_deform2"),
                    ("mcsart_forward_dvf", "kernel_forwardDVF"), ("mcsart_add", "host_add"),
                    ("mcsart_add2", "host_add2"), ("mcsart_initial", "host_initial"),
                    ("mcsart_initial2", "host_initial2"), ("mcsart_division", "host_division"),
                    ("mcsart_multiple", "host_multiple"),
                    ("mcsart_update_udvf", "host_update_udvf"), ("mcsart_diff", "host_diff"),
                    ("mcsart_aumisart", "host_AUMISART")]:
        m = re.search(r"/\*(?:(?!\*/).)*\b" + ref + r"\b(?:(?!\*/).)*\*/\s*int " + fn + r"\(",
                      text, flags=re.S)
        assert m, f"{fn} lacks a comment naming {ref}"
