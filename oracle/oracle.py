"""Test infrastructure: ctypes bindings of the CPU oracle (oracle/liboracle.so).

``orc_*`` functions are the FP64 restatement of the reference kernels of
bill52547/McSART; ``cpu_*`` the FP32 OpenMP transcription that serves as the
timed CPU baseline.  Only tests, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use this module; the product library never does.

All functions take and return numpy arrays in the reference layouts:
``img[iz, iy, ix]`` (C order == ix fastest) and ``proj[ib, ia]`` per view.
Geometry arguments are the reference's voxel-unit scalars (``ai``/``bi``
already shifted, as src/entry_AUMISART.cu:76-94 leaves them).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

TEX_EXACT, TEX_Q8_NEAREST, TEX_Q8_TRUNC = 0, 1, 2

_lib = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no reference sources)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p


def _declare(L: ctypes.CDLL) -> None:
    for pre in ("orc_", "cpu_"):
        geo = [_D, _D, _D, _D, _I, _D, _D, _I, _D, _I, _I, _I]
        getattr(L, pre + "projection").argtypes = [_P, _P] + geo
        getattr(L, pre + "backprojection").argtypes = [_P, _P] + geo
        getattr(L, pre + "backprojection_adjoint").argtypes = [_P, _P] + geo
        getattr(L, pre + "backprojection_sc").argtypes = [_P, _P, _D] + geo
        getattr(L, pre + "forward_dvf").argtypes = [_P] * 9 + [_D, _D, _I, _I, _I]
        getattr(L, pre + "deform").argtypes = [_P, _P, _I, _I, _I, _D, _D] + [_P] * 6 + [_I]
        getattr(L, pre + "deform2").argtypes = [_P, _P, _I, _I, _I, _D, _D] + [_P] * 6
        getattr(L, pre + "add").argtypes = [_P, _P, _I, _I, _I, _D]
        getattr(L, pre + "add2").argtypes = [_P, _P, _I, _I, _I, _P, _D, _I]
        getattr(L, pre + "initial").argtypes = [_P, _I, _I, _I, _D]
        getattr(L, pre + "initial2").argtypes = [_P, _I, _I, _I, _P, _D, _D]
        getattr(L, pre + "division").argtypes = [_P, _P, _I, _I, _I]
        getattr(L, pre + "multiple").argtypes = [_P, _I, _I, _I, _P, _D, _I]
        getattr(L, pre + "update_udvf").argtypes = [_P] * 8 + [_D, _D, _I, _I, _I, _I]
        getattr(L, pre + "diff").argtypes = [_P, _P, _I, _I, _I, _I]
        f = getattr(L, pre + "aumisart")
        f.argtypes = ([_P] * 6 + [_I] * 8 + [_P] + [_D] * 8 + [_P] * 3 + [_P] * 6 +
                      [_P, _I, _I, _I, _I, _I])
        getattr(L, pre + "invert_dvf").argtypes = [_P] * 9 + [_D, _D, _I, _I, _I, _I]
        f.restype = _I
    L.orc_num_threads.restype = _I
    L.orc_set_num_threads.argtypes = [_I]


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def _dt(prec: str):
    return np.float64 if prec == "orc" else np.float32


def _arr(a, prec):
    return np.ascontiguousarray(a, dtype=_dt(prec))


def _p(a) -> int:
    return a.ctypes.data if a is not None else None


def _geo(g) -> list:
    return [float(g["SO"]), float(g["SD"]), float(g["da"]), int(g["na"]), float(g["ai"]),
            float(g["db"]), int(g["nb"]), float(g["bi"]), int(g["nx"]), int(g["ny"]),
            int(g["nz"])]


# ------------------------------------------------------------------ kernels
def projection(img, angle, geo, prec="orc"):
    """Distance-driven forward projection of one view (src/cu_projection.cu:15)."""
    img = _arr(img, prec)
    out = np.zeros((geo["nb"], geo["na"]), _dt(prec))
    getattr(lib(), prec + "_projection")(_p(out), _p(img), float(angle), *_geo(geo))
    return out


def backprojection(proj, angle, geo, prec="orc"):
    """Backprojection of one view (src/cu_backprojection.cu:49)."""
    proj = _arr(proj, prec)
    out = np.zeros((geo["nz"], geo["ny"], geo["nx"]), _dt(prec))
    getattr(lib(), prec + "_backprojection")(_p(out), _p(proj), float(angle), *_geo(geo))
    return out


def invert_dvf(fields, volume, flow, iters, prec="orc"):
    """Fixed-point inverse of the warp's displacement (the engine's
    mcsart_invert_dvf); returns (inv_x, inv_y, inv_z)."""
    f = [_arr(x, prec) for x in fields]
    nz, ny, nx = f[0].shape
    out = [np.zeros_like(f[0]) for _ in range(3)]
    getattr(lib(), prec + "_invert_dvf")(*[_p(x) for x in out], *[_p(x) for x in f],
                                        float(volume), float(flow), nx, ny, nz, int(iters))
    return out


def backprojection_adjoint(proj, angle, geo, prec="orc"):
    """Exact adjoint (transpose) of projection(): scatters each ray's terms."""
    proj = _arr(proj, prec)
    out = np.zeros((geo["nz"], geo["ny"], geo["nx"]), _dt(prec))
    getattr(lib(), prec + "_backprojection_adjoint")(_p(out), _p(proj), float(angle), *_geo(geo))
    return out


def backprojection_sc(proj, cphi, sphi, geo, prec="orc"):
    """Backprojection with a given cos/sin pair (to mirror __cosf/__sinf)."""
    proj = _arr(proj, prec)
    out = np.zeros((geo["nz"], geo["ny"], geo["nx"]), _dt(prec))
    getattr(lib(), prec + "_backprojection_sc")(_p(out), _p(proj), float(cphi), float(sphi),
                                                 *_geo(geo))
    return out


def forward_dvf(fields, volume, flow, prec="orc"):
    """m = alpha*volume + beta*flow per component (src/cu_deform.cu:66)."""
    f = [_arr(x, prec) for x in fields]
    shp = f[0].shape
    m = [np.zeros(shp, _dt(prec)) for _ in range(3)]
    getattr(lib(), prec + "_forward_dvf")(*[_p(x) for x in m], *[_p(x) for x in f], float(volume),
                                          float(flow), shp[2], shp[1], shp[0])
    return m


def deform(img, volume, flow, fields, tex_mode=TEX_Q8_NEAREST, prec="orc"):
    """Trilinear warp (src/cu_deform.cu:3); fields = (ax, ay, az, bx, by, bz)."""
    img = _arr(img, prec)
    f = [_arr(x, prec) for x in fields]
    out = np.zeros_like(img)
    nz, ny, nx = img.shape
    getattr(lib(), prec + "_deform")(_p(out), _p(img), nx, ny, nz, float(volume), float(flow),
                                     *[_p(x) for x in f], int(tex_mode))
    return out


def deform2(img, volume, flow, fields, prec="orc"):
    """First-order warp (src/cu_deform.cu:49)."""
    img = _arr(img, prec)
    f = [_arr(x, prec) for x in fields]
    out = np.zeros_like(img)
    nz, ny, nx = img.shape
    getattr(lib(), prec + "_deform2")(_p(out), _p(img), nx, ny, nz, float(volume), float(flow),
                                      *[_p(x) for x in f])
    return out


def add(img1, img, weight, prec="orc"):
    """img1 += img*weight (src/cu_add.cu:9); returns a new array."""
    a = _arr(img1, prec).copy()
    b = _arr(img, prec)
    shp = (1,) * (3 - a.ndim) + a.shape
    getattr(lib(), prec + "_add")(_p(a), _p(b), shp[2], shp[1], shp[0], float(weight))
    return a


def add2(img1, img, img0, weight, ind, prec="orc"):
    """img1 += img[transposed]*weight*d_ind(img0) (src/cu_add.cu:28)."""
    a = _arr(img1, prec).copy()
    b, c = _arr(img, prec), _arr(img0, prec)
    nz, ny, nx = a.shape
    getattr(lib(), prec + "_add2")(_p(a), _p(b), nx, ny, nz, _p(c), float(weight), int(ind))
    return a


def initial(shape, value, prec="orc"):
    a = np.empty(shape, _dt(prec))
    nz, ny, nx = shape
    getattr(lib(), prec + "_initial")(_p(a), nx, ny, nz, float(value))
    return a


def initial2(img0, volume, flow, prec="orc"):
    """(dx+dy+dz img0)*(volume+flow) (src/cu_initial.cu:27)."""
    c = _arr(img0, prec)
    a = np.empty_like(c)
    nz, ny, nx = c.shape
    getattr(lib(), prec + "_initial2")(_p(a), nx, ny, nz, _p(c), float(volume), float(flow))
    return a


def division(img1, img, prec="orc"):
    """img1 / img with NaN/Inf -> 0 (src/cu_division.cu:11)."""
    a = _arr(img1, prec).copy()
    b = _arr(img, prec)
    nz, ny, nx = a.shape
    getattr(lib(), prec + "_division")(_p(a), _p(b), nx, ny, nz)
    return a


def multiple(img1, img0, weight, ind, prec="orc"):
    """img1 *= weight*d_ind(img0) (src/cu_multiple.cu:11)."""
    a = _arr(img1, prec).copy()
    c = _arr(img0, prec)
    nz, ny, nx = a.shape
    getattr(lib(), prec + "_multiple")(_p(a), nx, ny, nz, _p(c), float(weight), int(ind))
    return a


def update_udvf(fields, img, img0, volume_diff, flow_diff, it=0, prec="orc"):
    """Gauss-Newton DVF step (src/cu_update_udvf.cu:11); returns new fields."""
    f = [_arr(x, prec).copy() for x in fields]
    a, b = _arr(img, prec), _arr(img0, prec)
    nz, ny, nx = a.shape
    getattr(lib(), prec + "_update_udvf")(*[_p(x) for x in f], _p(a), _p(b), float(volume_diff),
                                          float(flow_diff), nx, ny, nz, int(it))
    return f


def diff(img, ind, prec="orc", init=None):
    """Backward difference, 0 on both faces (src/mex_diff.cu:75)."""
    b = _arr(img, prec)
    a = np.zeros_like(b) if init is None else _arr(init, prec).copy()
    nz, ny, nx = b.shape
    getattr(lib(), prec + "_diff")(_p(a), _p(b), nx, ny, nz, int(ind))
    return a


def aumisart(img, proj, geo, it, fields=None, tex_mode=TEX_Q8_NEAREST, prec="orc",
             view_lo=0, view_hi=-1, return_fields=False, subset=1, dvf_inverse=0):
    """The SART/motion loop of host_AUMISART (src/AUMISART.cu:3 and :143).

    ``it`` holds ``n_iter``, ``op_iter``, ``n_views``, ``lambda``, ``volumes``,
    ``flows``, ``angles`` (and optionally ``outIter``); ``fields`` = None selects
    overload 1 (DVF zero-initialised), a 6-tuple overload 2.  ``subset`` > 1:
    the engine's ordered-subset mode (views of a subset start from the same
    image, which then gets lambda/k times their corrections).
    Returns dict(img, norm, alpha_x, resid[, fields]).
    """
    dt = _dt(prec)
    img = _arr(img, prec)
    proj = _arr(proj, prec)
    nz, ny, nx = img.shape
    na, nb = int(geo["na"]), int(geo["nb"])
    n_views, n_iter = int(it["n_views"]), int(it["n_iter"])
    op = np.ascontiguousarray(it["op_iter"], dtype=np.int32)
    vols = np.ascontiguousarray(it["volumes"], dtype=np.float32)
    flows = np.ascontiguousarray(it["flows"], dtype=np.float32)
    angs = np.ascontiguousarray(it["angles"], dtype=np.float32)
    out_img = np.zeros_like(img)
    out_proj = np.zeros((n_views, nb, na), dt)
    out_norm = np.zeros(n_iter * n_views, dt)
    out_ax = np.zeros_like(img)
    f = [None] * 6 if fields is None else [_arr(x, prec) for x in fields]
    fo = np.zeros((6,) + img.shape, dt) if return_fields else None
    rc = getattr(lib(), prec + "_aumisart")(
        _p(out_img), _p(out_proj), _p(out_norm), _p(out_ax), _p(img), _p(proj), nx, ny, nz, na,
        nb, int(it.get("outIter", 1)), n_views, n_iter, _p(op), float(geo["da"]),
        float(geo["db"]), float(geo["ai"]), float(geo["bi"]), float(geo["SO"]),
        float(geo["SD"]), float(geo.get("dx", 1.0)), float(it["lambda"]), _p(vols), _p(flows),
        _p(angs), *[_p(x) for x in f], _p(fo), int(tex_mode), int(view_lo), int(view_hi),
        int(subset), int(dvf_inverse))
    if rc != 0:
        raise RuntimeError(f"oracle aumisart failed: {rc}")
    out = {"img": out_img, "norm": out_norm, "alpha_x": out_ax, "resid": out_proj}
    if return_fields:
        out["fields"] = fo
    return out
