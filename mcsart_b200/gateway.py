"""The reference's three MATLAB gateways, restated over the C ABI.

``entry_AUMISART``, ``mex_backprojection`` and ``mex_diff`` take the same
inputs as src/entry_AUMISART.cu, src/mex_backprojection.cu and src/mex_diff.cu
(MATLAB structs become dicts), apply the same field aliases, defaults and
detector-offset shift, raise with the reference's messages when a required
field is missing, and return the same outputs.  Volumes are numpy arrays whose
C order matches MATLAB's nx x ny x nz column-major memory ([nz, ny, nx]);
projection stacks are [n_views, nb, na].
"""
from __future__ import annotations

import numpy as np

from .engine import Context


class BadInput(ValueError):
    """Raised where the reference calls mexErrMsgIdAndTxt("MATLAB:badInput", ...)."""


def _get(d, *names):
    for n in names:
        if n in d and d[n] is not None:
            return d[n]
    return None


def parse_geo_para(geo: dict, need_angle: bool = False) -> dict:
    """src/entry_AUMISART.cu:18-108 (and src/mex_backprojection.cu:14-108)."""
    out = {}
    for k in ("nx", "ny", "nz"):
        v = _get(geo, k)
        if v is None:
            raise BadInput(f"Can't found valid volume resolution {k}.")
        out[k] = int(v)
    na = _get(geo, "na", "nv")
    if na is None:
        raise BadInput("Can't found valid number of detector in plane, which is denoted as na or nu.")
    nb = _get(geo, "nb", "nu")
    if nb is None:
        raise BadInput("Can't found valid number of detector across plane, which is denoted as nb or nv.")
    out["na"], out["nb"] = int(na), int(nb)
    out["dx"] = float(np.float32(_get(geo, "dx") if _get(geo, "dx") is not None else 1.0))
    out["da"] = float(np.float32(_get(geo, "da") if _get(geo, "da") is not None else 1.0))
    out["db"] = float(np.float32(_get(geo, "db") if _get(geo, "db") is not None else 1.0))
    # detector offsets are shifted to the first cell's centre (:76-94), in float
    f32 = np.float32
    ai = _get(geo, "ai")
    out["ai"] = float(f32(f32(ai if ai is not None else 0.0) - (f32(out["na"]) / f32(2) - f32(0.5))))
    bi = _get(geo, "bi")
    out["bi"] = float(f32(f32(bi if bi is not None else 0.0) - (f32(out["nb"]) / f32(2) - f32(0.5))))
    so = _get(geo, "SO", "SI")
    if so is None:
        raise BadInput("Can't found valid distance between source and isocenter, which is denoted with para.SO or para.DI.")
    out["SO"] = float(f32(so))
    sd = _get(geo, "SD")
    if sd is None:
        di = _get(geo, "DI")
        if di is None:
            raise BadInput("Can't found valid distance between source and detector plane, which is denoted with para.SD or para.SI + para.DI.")
        sd = f32(di) + f32(out["SO"])
    out["SD"] = float(f32(sd))
    if need_angle:
        ang = _get(geo, "angle")
        if ang is None:
            raise BadInput("Can't found valid projection angle, which is denoted with para.angle.")
        out["angle"] = float(f32(ang))
    return out


def parse_iter_para(it: dict) -> dict:
    """src/entry_AUMISART.cu:111-160."""
    out = {"n_iter": int(it["n_iter"]) if it.get("n_iter") is not None else 1}
    req = [("op_iter", "Can't found valid iteration distribution as iter_para.op_iter."),
           ("n_views", "Can't found valid number bins, which is denoted as iter_para.n_views."),
           ("lambda", "Can't found valid coefficience iter_para.lambda."),
           ("outIter", "Can't found valid coefficience iter_para.outIter."),
           ("volumes", "Can't found valid volume in iter_para.volumes."),
           ("flows", "Can't found valid flow in iter_para.flows."),
           ("err_weights", "Can't found valid flow in iter_para.err_weights."),
           ("angles", "Can't found valid angles iter_para.angles.")]
    for k, msg in req:
        if it.get(k) is None:
            raise BadInput(msg)
    out["op_iter"] = np.ascontiguousarray(it["op_iter"], dtype=np.int32)
    out["n_views"] = int(it["n_views"])
    out["lambda"] = float(np.float32(it["lambda"]))
    out["outIter"] = int(it["outIter"])
    for k in ("volumes", "flows", "err_weights", "angles"):
        out[k] = np.ascontiguousarray(it[k], dtype=np.float32).ravel()
    if it.get("alpha_x") is not None:  # :193 selects the overload
        out["fields"] = [np.ascontiguousarray(it[k], dtype=np.float32)
                         for k in ("alpha_x", "alpha_y", "alpha_z", "beta_x", "beta_y", "beta_z")]
    else:
        out["fields"] = None
    if out["op_iter"].size < out["n_iter"]:
        raise BadInput("iter_para.op_iter has fewer than n_iter entries.")
    for k in ("volumes", "flows", "angles"):
        if out[k].size < out["n_views"]:
            raise BadInput(f"iter_para.{k} has fewer than n_views entries.")
    return out


def entry_AUMISART(img, proj, geo_para: dict, iter_para: dict, ctx: Context | None = None):
    """[img, norm, alpha_x, resid] = entry_AUMISART(img0, proj, geo_para, iter_para)."""
    g = parse_geo_para(geo_para)
    it = parse_iter_para(iter_para)
    nx, ny, nz, na, nb = g["nx"], g["ny"], g["nz"], g["na"], g["nb"]
    nv, n_iter = it["n_views"], it["n_iter"]
    img = np.ascontiguousarray(img, dtype=np.float32).reshape(nz, ny, nx)
    proj = np.ascontiguousarray(proj, dtype=np.float32).reshape(nv, nb, na)
    out_img = np.zeros((nz, ny, nx), np.float32)
    out_norm = np.zeros(n_iter * nv, np.float32)
    out_ax = np.zeros((nz, ny, nx), np.float32)
    out_proj = np.zeros((nv, nb, na), np.float32)
    own = ctx is None
    ctx = ctx or Context()
    try:
        f = it["fields"] or [None] * 6
        ctx.host_AUMISART(out_img, out_proj, out_norm, out_ax, img, proj, nx, ny, nz, na, nb,
                          it["outIter"], nv, n_iter, it["op_iter"], g["da"], g["db"], g["ai"],
                          g["bi"], g["SO"], g["SD"], g["dx"], it["lambda"], it["volumes"],
                          it["flows"], it["err_weights"], it["angles"], *f)
    finally:
        if own:
            ctx.close()
    return out_img, out_norm.reshape(-1, 1), out_ax, out_proj


def mex_backprojection(proj, geo_para: dict, ctx: Context | None = None):
    """img = mex_backprojection(proj, geo_para) with geo_para.angle (src/mex_backprojection.cu)."""
    import torch
    g = parse_geo_para(geo_para, need_angle=True)
    p = torch.as_tensor(np.ascontiguousarray(proj, dtype=np.float32).reshape(g["nb"], g["na"]))
    own = ctx is None
    ctx = ctx or Context()
    try:
        dev = torch.device("cuda", ctx.device)
        d_proj = p.to(dev)
        d_img = torch.empty((g["nz"], g["ny"], g["nx"]), dtype=torch.float32, device=dev)
        torch.cuda.current_stream(dev).synchronize()
        ctx.host_backprojection(d_img, d_proj, g["angle"], g["SO"], g["SD"], g["da"], g["na"],
                                g["ai"], g["db"], g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
        ctx.synchronize()
        return d_img.cpu().numpy()
    finally:
        if own:
            ctx.close()


def mex_diff(img, geo_para: dict, ctx: Context | None = None):
    """img1 = mex_diff(img, struct(nx, ny, nz, ind)) (src/mex_diff.cu)."""
    import torch
    dims = {}
    for k in ("nx", "ny", "nz"):
        if geo_para.get(k) is None:
            raise BadInput(f"Can't found valid volume resolution {k}.")
        dims[k] = int(geo_para[k])
    if geo_para.get("ind") is None:
        raise BadInput("Can't found ind.")
    ind = int(geo_para["ind"])
    a = torch.as_tensor(np.ascontiguousarray(img, dtype=np.float32).reshape(dims["nz"], dims["ny"],
                                                                           dims["nx"]))
    own = ctx is None
    ctx = ctx or Context()
    try:
        dev = torch.device("cuda", ctx.device)
        d_img = a.to(dev)
        # the reference's output buffer is uninitialised for ind outside 1..3
        d_out = torch.zeros_like(d_img)
        torch.cuda.current_stream(dev).synchronize()
        ctx.host_diff(d_out, d_img, dims["nx"], dims["ny"], dims["nz"], ind)
        ctx.synchronize()
        return d_out.cpu().numpy()
    finally:
        if own:
            ctx.close()
