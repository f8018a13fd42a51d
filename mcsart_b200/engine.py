"""Host-side mirror of the reference's launcher interface over libmcsart.so.

``Context`` exposes one method per reference launcher with the reference's
name and positional argument order (``host_projection``, ``host_backprojection``,
``host_deform`` ... as declared in include/cu_*.h of bill52547/McSART), taking
device buffers as torch CUDA tensors (float32, contiguous) or raw device
pointers, plus ``host_AUMISART`` (host arrays, src/AUMISART.cu:3/:143) and the
device-resident ``aumisart_device``.  All work is stream-ordered on the
context's stream; ``synchronize()`` waits for it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (BF16, F16, F32, INTERP_EXACT, INTERP_TEXTURE, McsartError, Options,
                   Problem, check)

__all__ = ["Context", "McsartError", "Options", "default_options", "projection_noalloc", "F32",
           "BF16", "F16", "INTERP_TEXTURE", "INTERP_EXACT"]


def _ptr(x, name="buffer", dtype_bytes=None):
    """Device pointer of a torch CUDA tensor (or an int pointer)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr") and hasattr(x, "is_cuda"):
        if not x.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if not x.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        if dtype_bytes is not None and x.element_size() != dtype_bytes:
            raise ValueError(f"{name} has element size {x.element_size()}, expected {dtype_bytes}")
        return x.data_ptr()
    raise TypeError(f"{name}: expected a torch CUDA tensor or an int device pointer")


def _hptr(a: np.ndarray) -> int:
    return a.ctypes.data


def projection_noalloc(d_proj, d_img, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz,
                       stream=None):
    """mcsart_projection_noalloc: the projection of mcsart_projection without a
    context and without allocating; scratch in a fixed device array of
    MCSART_NOALLOC_MAX_VOXELS voxels.  stream: an int cudaStream_t, a
    torch.cuda.Stream, or None for the legacy default stream.

    Torch tensors must sit on one device and hold nx*ny*nz (d_img) and na*nb
    (d_proj) elements; the call runs with that device current.  Raw int
    pointers are passed through unchecked, on the current device."""
    if stream is not None and not isinstance(stream, int):
        stream = stream.cuda_stream
    p_proj, p_img = _ptr(d_proj, "d_proj", 4), _ptr(d_img, "d_img", 4)
    tensors = [t for t in (d_proj, d_img) if hasattr(t, "is_cuda")]
    device = None
    if tensors:
        devs = {t.device for t in tensors}
        if len(devs) != 1:
            raise ValueError(f"d_proj and d_img must be on one device (got {sorted(map(str, devs))})")
        device = tensors[0].device
    if hasattr(d_img, "numel") and d_img.numel() != nx * ny * nz:
        raise ValueError(f"d_img holds {d_img.numel()} elements, nx*ny*nz = {nx * ny * nz}")
    if hasattr(d_proj, "numel") and d_proj.numel() != na * nb:
        raise ValueError(f"d_proj holds {d_proj.numel()} elements, na*nb = {na * nb}")
    L = _lib.load()

    def call():
        check(L.mcsart_projection_noalloc(stream, p_proj, p_img, angle, SO, SD, da, na, ai, db,
                                          nb, bi, nx, ny, nz),
              "mcsart_projection_noalloc")
    if device is None:
        call()
    else:
        import torch
        with torch.cuda.device(device):
            call()


def default_options(**kw) -> Options:
    o = Options()
    _lib.load().mcsart_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


class Context:
    """A libmcsart context on one CUDA device (its own stream by default)."""

    def __init__(self, device: int = 0, stream=None, synchronous: bool = False):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        check(self._L.mcsart_create(ctypes.byref(h), int(device)), "mcsart_create")
        self._h = h
        self.device = int(device)
        if stream is not None:
            self.set_stream(stream)
        if synchronous:
            self.set_synchronous(True)

    # ----------------------------------------------------------- plumbing
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.mcsart_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        check(getattr(self._L, name)(self._h, *args), name)

    def set_stream(self, stream) -> None:
        """Use a cudaStream_t (int) or a torch.cuda.Stream; 0 = legacy default stream."""
        s = getattr(stream, "cuda_stream", stream)
        self._call("mcsart_set_stream", int(s) if s else None)

    @property
    def stream(self) -> int:
        return int(self._L.mcsart_get_stream(self._h) or 0)

    def set_synchronous(self, on: bool) -> None:
        self._call("mcsart_set_synchronous", 1 if on else 0)

    def set_interp(self, interp: int) -> None:
        self._call("mcsart_set_interp", int(interp))

    def synchronize(self) -> None:
        self._call("mcsart_synchronize")

    @property
    def launches(self) -> int:
        """Kernels of this library launched through the context so far."""
        return int(self._L.mcsart_launch_count(self._h))

    def profile_begin(self) -> None:
        """Start per-kernel event timing (graphs are bypassed until profile_end)."""
        self._call("mcsart_profile_begin")

    def profile_end(self) -> dict:
        """Stop timing; returns {kernel name: (launches, total ms)}."""
        self._call("mcsart_profile_end")
        out = {}
        buf = ctypes.create_string_buffer(256)
        n = ctypes.c_longlong()
        ms = ctypes.c_double()
        for i in range(self._L.mcsart_profile_count(self._h)):
            check(self._L.mcsart_profile_entry(self._h, i, buf, 256, ctypes.byref(n),
                                               ctypes.byref(ms)), "mcsart_profile_entry")
            out[buf.value.decode()] = (int(n.value), float(ms.value))
        return out

    # ------------------------------------------------ reference launchers
    def host_projection(self, d_proj, d_img, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz):
        """include/cu_projection.h:7"""
        self._call("mcsart_projection", _ptr(d_proj, "d_proj", 4), _ptr(d_img, "d_img", 4),
                   angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz)

    def host_backprojection(self, d_img, d_proj, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny,
                            nz):
        """include/cu_backprojection.h:7"""
        self._call("mcsart_backprojection", _ptr(d_img, "d_img", 4), _ptr(d_proj, "d_proj", 4),
                   angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz)

    def invert_dvf(self, inv_x, inv_y, inv_z, alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z,
                   volume, flow, nx, ny, nz, n_iter):
        """True inverse of the warp's displacement (mcsart_invert_dvf); no counterpart in
        the reference, which negates the amplitudes (src/AUMISART.cu:222)."""
        self._call("mcsart_invert_dvf", *[_ptr(a, "field", 4) for a in (
            inv_x, inv_y, inv_z, alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z)],
            volume, flow, nx, ny, nz, n_iter)

    def host_backprojection_adjoint(self, d_img, d_proj, angle, SO, SD, da, na, ai, db, nb, bi,
                                    nx, ny, nz):
        """Exact adjoint of host_projection (mcsart_backprojection_adjoint); no
        counterpart in the reference."""
        self._call("mcsart_backprojection_adjoint", _ptr(d_img, "d_img", 4),
                   _ptr(d_proj, "d_proj", 4), angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz)

    @staticmethod
    def _storage_of(t):
        import torch
        return {torch.float32: F32, torch.bfloat16: BF16, torch.float16: F16}[t.dtype]

    def projection_ex(self, d_proj, d_img, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz, *,
                      fp_sum=0, geom64=0):
        """mcsart_projection_ex: d_img a float32, bfloat16 or float16 CUDA tensor."""
        self._call("mcsart_projection_ex", _ptr(d_proj, "d_proj", 4), _ptr(d_img, "d_img"),
                   self._storage_of(d_img), int(fp_sum), int(geom64), angle, SO, SD, da, na, ai,
                   db, nb, bi, nx, ny, nz)

    def backprojection_ex(self, d_img, d_proj, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz,
                          *, geom64=0):
        """mcsart_backprojection_ex (geom64 = 1: FP64 geometry)."""
        self._call("mcsart_backprojection_ex", _ptr(d_img, "d_img", 4), _ptr(d_proj, "d_proj", 4),
                   int(geom64), angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz)

    def deform_ex(self, d_img1, d_img, nx, ny, nz, volume, flow, fields, *, interp=INTERP_EXACT):
        """mcsart_deform_ex: fields a (6, nz, ny, nx) CUDA tensor whose dtype (float32,
        bfloat16, float16) is also the output's."""
        if d_img1.dtype != fields.dtype:
            raise ValueError("d_img1 and fields must have the same dtype")
        self._call("mcsart_deform_ex", _ptr(d_img1, "d_img1"), _ptr(d_img, "d_img", 4), nx, ny,
                   nz, volume, flow, _ptr(fields, "fields"), self._storage_of(fields), int(interp))

    def host_deform(self, d_img1, d_img, nx, ny, nz, volume, flow, alpha_x, alpha_y, alpha_z,
                    beta_x, beta_y, beta_z):
        """include/cu_deform.h:8"""
        self._call("mcsart_deform", _ptr(d_img1, "d_img1", 4), _ptr(d_img, "d_img", 4), nx, ny,
                   nz, volume, flow, *[_ptr(f, "field", 4) for f in
                                       (alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z)])

    def host_deform2(self, d_img1, d_img, nx, ny, nz, volume, flow, alpha_x, alpha_y, alpha_z,
                     beta_x, beta_y, beta_z):
        """include/cu_deform.h:9"""
        self._call("mcsart_deform2", _ptr(d_img1, "d_img1", 4), _ptr(d_img, "d_img", 4), nx, ny,
                   nz, volume, flow, *[_ptr(f, "field", 4) for f in
                                       (alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z)])

    def kernel_forwardDVF(self, mx, my, mz, alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z,
                          volume, flow, nx, ny, nz):
        """include/cu_deform.h:10"""
        self._call("mcsart_forward_dvf", *[_ptr(a, "buffer", 4) for a in
                                           (mx, my, mz, alpha_x, alpha_y, alpha_z, beta_x,
                                            beta_y, beta_z)], volume, flow, nx, ny, nz)

    def host_add(self, img1, img, nx, ny, nz, weight):
        """include/cu_add.h:4"""
        self._call("mcsart_add", _ptr(img1, "img1", 4), _ptr(img, "img", 4), nx, ny, nz, weight)

    def host_add2(self, img1, img, nx, ny, nz, img0, weight, ind):
        """include/cu_add.h:8"""
        self._call("mcsart_add2", _ptr(img1, "img1", 4), _ptr(img, "img", 4), nx, ny, nz,
                   _ptr(img0, "img0", 4), weight, ind)

    def host_initial(self, img, nx, ny, nz, value):
        """include/cu_initial.h:5"""
        self._call("mcsart_initial", _ptr(img, "img", 4), nx, ny, nz, value)

    def host_initial2(self, img, nx, ny, nz, img0, volume, flow):
        """include/cu_initial.h:8"""
        self._call("mcsart_initial2", _ptr(img, "img", 4), nx, ny, nz, _ptr(img0, "img0", 4),
                   volume, flow)

    def host_division(self, img1, img, nx, ny, nz):
        """include/cu_division.h:5"""
        self._call("mcsart_division", _ptr(img1, "img1", 4), _ptr(img, "img", 4), nx, ny, nz)

    def host_multiple(self, img1, nx, ny, nz, img0, weight, ind):
        """include/cu_multiple.h:4"""
        self._call("mcsart_multiple", _ptr(img1, "img1", 4), nx, ny, nz, _ptr(img0, "img0", 4),
                   weight, ind)

    def host_update_udvf(self, alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z, img, img0,
                         volume_diff, flow_diff, nx, ny, nz, iter=0):
        """include/cu_update_udvf.h:8"""
        self._call("mcsart_update_udvf", *[_ptr(a, "buffer", 4) for a in
                                           (alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z,
                                            img, img0)], volume_diff, flow_diff, nx, ny, nz, iter)

    def host_diff(self, img1, img, nx, ny, nz, ind):
        """src/mex_diff.cu:67"""
        self._call("mcsart_diff", _ptr(img1, "img1", 4), _ptr(img, "img", 4), nx, ny, nz, ind)

    def snrm2(self, n, d_x) -> float:
        """Euclidean norm of n floats (the cublasSnrm2 use of src/AUMISART.cu:48)."""
        out = ctypes.c_float()
        self._call("mcsart_snrm2", int(n), _ptr(d_x, "d_x", 4), ctypes.byref(out))
        return float(out.value)

    def projection_views(self, d_proj, d_img, angles, SO, SD, da, na, ai, db, nb, bi, nx, ny,
                         nz):
        """All views of one volume in one launch; angles is a host sequence."""
        a = np.ascontiguousarray(angles, dtype=np.float32)
        self._call("mcsart_projection_views", _ptr(d_proj, "d_proj", 4), _ptr(d_img, "d_img", 4),
                   _hptr(a), len(a), SO, SD, da, na, ai, db, nb, bi, nx, ny, nz)

    # --------------------------------------------------------------- drivers
    def host_AUMISART(self, h_outimg, h_outproj, h_outnorm, h_outalphax, h_img, h_proj, nx, ny,
                      nz, na, nb, outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx,
                      lambda_, volumes, flows, err_weights, angles, ax=None, ay=None, az=None,
                      bx=None, by=None, bz=None):
        """include/AUMISART.h:17 (fields omitted) and :19 (fields given).

        Host numpy arrays (float32, C-contiguous); outputs are written in place.
        """
        def h(a, dt=np.float32, name="array", out=False):
            if a is None:
                return None
            if not (isinstance(a, np.ndarray) and a.dtype == dt and a.flags.c_contiguous):
                raise ValueError(f"{name} must be a C-contiguous {np.dtype(dt).name} array")
            if out and not a.flags.writeable:
                raise ValueError(f"{name} must be writeable")
            return _hptr(a)
        self._call("mcsart_aumisart", h(h_outimg, name="h_outimg", out=True),
                   h(h_outproj, name="h_outproj", out=True), h(h_outnorm, name="h_outnorm", out=True),
                   h(h_outalphax, name="h_outalphax", out=True), h(h_img, name="h_img"),
                   h(h_proj, name="h_proj"), nx, ny, nz, na, nb, outIter, n_views, n_iter,
                   h(op_iter, np.int32, "op_iter"), da, db, ai, bi, SO, SD, dx, lambda_,
                   h(volumes, name="volumes"), h(flows, name="flows"),
                   h(err_weights, name="err_weights") if err_weights is not None else None,
                   h(angles, name="angles"), *[h(f, name="field") for f in (ax, ay, az, bx, by, bz)])

    def aumisart_host(self, img, proj, geo, *, n_iter, op_iter, lambda_, angles, volumes, flows,
                      fields=None):
        """host_AUMISART on host arrays through mcsart_aumisart_fields: returns a
        dict with the image, the residuals of the last image pass, the norm list
        and all six final DVF fields (alpha_x ... beta_z).  Passing the returned
        image and fields back continues the reconstruction exactly."""
        img = np.ascontiguousarray(img, np.float32)
        proj = np.ascontiguousarray(proj, np.float32)
        nz, ny, nx = img.shape
        nv = proj.shape[0]
        out = dict(img=np.zeros_like(img), resid=np.zeros_like(proj),
                   norm=np.zeros(int(n_iter) * nv, np.float32),
                   fields=[np.zeros_like(img) for _ in range(6)])
        f = [np.ascontiguousarray(x, np.float32) for x in fields] if fields is not None else None
        keep = [np.ascontiguousarray(x, np.float32) for x in (volumes, flows, angles)]
        op = np.ascontiguousarray(op_iter, np.int32)
        self._call("mcsart_aumisart_fields", _hptr(out["img"]), _hptr(out["resid"]),
                   _hptr(out["norm"]), *[_hptr(x) for x in out["fields"]], _hptr(img), _hptr(proj),
                   nx, ny, nz, int(geo["na"]), int(geo["nb"]), 1, nv, int(n_iter), _hptr(op),
                   geo["da"], geo["db"], geo["ai"], geo["bi"], geo["SO"], geo["SD"], 1.0,
                   float(lambda_), _hptr(keep[0]), _hptr(keep[1]), None, _hptr(keep[2]),
                   *([_hptr(x) for x in f] if f is not None else [None] * 6))
        return out

    @staticmethod
    def _problem(geo, n_views, lambda_, angles, volumes, flows, img, proj, fields, resid, norm,
                 options):
        """A Problem struct and the host arrays it points into (keep them alive)."""
        es = 4 if options is None or options.storage == F32 else 2
        p = Problem()
        p.nx, p.ny, p.nz = int(geo["nx"]), int(geo["ny"]), int(geo["nz"])
        p.na, p.nb, p.n_views = int(geo["na"]), int(geo["nb"]), int(n_views)
        p.SO, p.SD, p.da, p.db = geo["SO"], geo["SD"], geo["da"], geo["db"]
        p.ai, p.bi, p.lambda_ = geo["ai"], geo["bi"], float(lambda_)
        keep = [np.ascontiguousarray(x, dtype=np.float32) for x in (angles, volumes, flows)]
        p.h_angles, p.h_volumes, p.h_flows = [_hptr(x) for x in keep]
        p.d_img = _ptr(img, "img", 4)
        p.d_proj = _ptr(proj, "proj", es)
        p.d_fields = _ptr(fields, "fields", es)
        p.d_resid = _ptr(resid, "resid", 4)
        p.d_norm = _ptr(norm, "norm", 4)
        return p, keep

    def aumisart_device(self, *, geo, n_views, lambda_, angles, volumes, flows, img, proj,
                        fields=None, resid=None, norm=None, n_iter, op_iter, options=None):
        """Device-resident driver (mcsart_aumisart_device).

        img: float32 CUDA tensor (updated in place); proj, fields: CUDA tensors of
        the options' storage type; resid/norm: optional float32 outputs.
        """
        p, self._keep = self._problem(geo, n_views, lambda_, angles, volumes, flows, img, proj,
                                      fields, resid, norm, options)
        op = np.ascontiguousarray(op_iter, dtype=np.int32)
        self._call("mcsart_aumisart_device", ctypes.byref(p), int(n_iter), _hptr(op),
                   ctypes.byref(options) if options is not None else None)

    def batch_run(self, problems, *, n_iter, op_iter, options=None):
        """Independent reconstructions run concurrently (mcsart_batch_run).

        problems: list of dicts with the keyword arguments of aumisart_device
        (geo, n_views, lambda_, angles, volumes, flows, img, proj and optionally
        fields, resid, norm); every problem runs n_iter iterations of op_iter.
        """
        structs, keep = [], []
        for q in problems:
            p, k = self._problem(q["geo"], q["n_views"], q["lambda_"], q["angles"], q["volumes"],
                                 q["flows"], q["img"], q["proj"], q.get("fields"), q.get("resid"),
                                 q.get("norm"), options)
            structs.append(p)
            keep.append(k)
        arr = (Problem * len(structs))(*structs)
        self._keep = keep
        op = np.ascontiguousarray(op_iter, dtype=np.int32)
        self._call("mcsart_batch_run", arr, len(structs), int(n_iter), _hptr(op),
                   ctypes.byref(options) if options is not None else None)

    def autotune(self, *, geo, n_views, lambda_, angles, volumes, flows, img, proj, fields=None,
                 options=None) -> list:
        """mcsart_autotune for one problem (same keyword arguments as
        aumisart_device); returns the cached variant indices [fp1, fp3, bp, warp, fup]."""
        p, keep = self._problem(geo, n_views, lambda_, angles, volumes, flows, img, proj, fields,
                                None, None, options)
        self._call("mcsart_autotune", ctypes.byref(p),
                   ctypes.byref(options) if options is not None else None)
        storage = options.storage if options is not None else F32
        return self.tuning_get(geo, storage)

    def tuning_get(self, geo, storage=F32):
        """Cached launch-shape variants [fp1, fp3, bp, warp, fup] of a geometry, or None."""
        p = Problem()
        p.nx, p.ny, p.nz = int(geo["nx"]), int(geo["ny"]), int(geo["nz"])
        p.na, p.nb = int(geo["na"]), int(geo["nb"])
        p.SO, p.SD, p.da, p.db = geo["SO"], geo["SD"], geo["da"], geo["db"]
        p.ai, p.bi = geo["ai"], geo["bi"]
        out = (ctypes.c_int * 5)()
        rc = self._L.mcsart_tuning_get(self._h, ctypes.byref(p), int(storage), out)
        if rc < 0:
            check(rc, "mcsart_tuning_get")
        return list(out) if rc == 1 else None

    def tuning_save(self, path) -> None:
        self._call("mcsart_tuning_save", str(path).encode())

    def tuning_load(self, path) -> int:
        rc = self._L.mcsart_tuning_load(self._h, str(path).encode())
        if rc < 0:
            check(rc, "mcsart_tuning_load")
        return rc
