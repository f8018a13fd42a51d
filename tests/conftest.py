"""Shared fixtures of the McSART engine tests.

Markers: ``gpu`` tests need a CUDA GPU and call the engine through its C ABI;
everything else runs on CPU (oracle, host logic, library loading, gloo ranks).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU; calls the engine's C ABI")


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def max_rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def geo(nx=24, ny=20, nz=16, na=40, nb=28, SO=60.0, SD=90.0, da=0.9, db=0.8, ai=0.0, bi=0.0):
    """Small cone-beam geometry in the reference's conventions (ai/bi shifted)."""
    f = np.float32
    return dict(nx=nx, ny=ny, nz=nz, na=na, nb=nb, SO=float(f(SO)), SD=float(f(SD)),
                da=float(f(da)), db=float(f(db)),
                ai=float(f(f(ai) - (f(na) / f(2) - f(0.5)))),
                bi=float(f(f(bi) - (f(nb) / f(2) - f(0.5)))), dx=1.0)


# angles that exercise both driving axes, the 45-degree switch and all quadrants
ANGLES = [0.0, 0.3, 0.7853, 0.7863, 1.5707964, 2.1, 3.14159, 3.9, 4.712389, 5.5, 6.2]


def load_geo(z, prefix: str) -> dict:
    """Geometry dict stored as scalars named <prefix><key> in an npz file."""
    g = {k[len(prefix):]: z[k].item() for k in z.files if k.startswith(prefix)}
    for k in ("nx", "ny", "nz", "na", "nb"):
        g[k] = int(g[k])
    return g


def volume(shape, seed=0, smooth=True) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.random(shape, dtype=np.float32)
    if smooth:
        from scipy.ndimage import gaussian_filter
        v = gaussian_filter(v, 1.0).astype(np.float32)
        # add a few sharp edges
        nz, ny, nx = shape
        v[nz // 4: nz // 2, ny // 3: 2 * ny // 3, nx // 4: 3 * nx // 4] += 0.5
    return np.ascontiguousarray(v, np.float32)


def fields(shape, seed=1, scale=1.5) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    from scipy.ndimage import gaussian_filter
    return [np.ascontiguousarray(gaussian_filter(rng.normal(size=shape), 2.0) * scale * 3,
                                 np.float32) for _ in range(6)]


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch


@pytest.fixture(scope="session")
def ctx(torch_cuda):
    from mcsart_b200 import Context
    # torch's current stream, so that tensors torch fills are ready for the engine
    c = Context(0, stream=torch_cuda.cuda.current_stream().cuda_stream)
    yield c
    c.close()


@pytest.fixture(scope="session")
def ref(torch_cuda):
    from oracle import ref_runner
    return ref_runner.Ref()


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t) -> np.ndarray:
    return t.detach().cpu().numpy()
