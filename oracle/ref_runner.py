"""Test infrastructure: run the rebuilt reference (oracle/_ref/libmcsart_ref.so).

The library is bill52547/McSART's own CUDA sources compiled unmodified for
sm_100a (oracle/Makefile, target ``ref``) plus oracle/ref_harness.cu.  Each
function here uploads numpy inputs, calls exactly one reference launcher and
downloads the result, so tests can compare the engine with the reference on
the same GPU and inputs.

``aumisart`` runs host_AUMISART in a child process: the reference ends every
call with cudaDeviceReset() (src/AUMISART.cu:140,312), which would destroy the
CUDA context of anything else in the calling process.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libmcsart_ref.so")

_F, _I, _P = ctypes.c_float, ctypes.c_int, ctypes.c_void_p
_GEO = [_F, _F, _F, _F, _I, _F, _F, _I, _F, _I, _I, _I]


def available() -> bool:
    return os.path.exists(REF_LIB)


class Ref:
    def __init__(self):
        if not available():
            raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle ref` where the "
                                    "reference sources are present")
        L = ctypes.CDLL(REF_LIB)
        L.ref_malloc.restype = _P
        L.ref_malloc.argtypes = [ctypes.c_size_t]
        for n in ("ref_free",):
            getattr(L, n).argtypes = [_P]
        L.ref_h2d.argtypes = [_P, _P, ctypes.c_size_t]
        L.ref_d2h.argtypes = [_P, _P, ctypes.c_size_t]
        L.ref_projection.argtypes = [_P, _P] + _GEO
        L.ref_backprojection.argtypes = [_P, _P] + _GEO
        L.ref_deform.argtypes = [_P, _P, _I, _I, _I, _F, _F] + [_P] * 6
        L.ref_deform2.argtypes = [_P, _P, _I, _I, _I, _F, _F] + [_P] * 6
        L.ref_forward_dvf.argtypes = [_P] * 9 + [_F, _F, _I, _I, _I]
        L.ref_add.argtypes = [_P, _P, _I, _I, _I, _F]
        L.ref_add2.argtypes = [_P, _P, _I, _I, _I, _P, _F, _I]
        L.ref_initial.argtypes = [_P, _I, _I, _I, _F]
        L.ref_initial2.argtypes = [_P, _I, _I, _I, _P, _F, _F]
        L.ref_division.argtypes = [_P, _P, _I, _I, _I]
        L.ref_multiple.argtypes = [_P, _I, _I, _I, _P, _F, _I]
        L.ref_update_udvf.argtypes = [_P] * 8 + [_F, _F, _I, _I, _I, _I]
        L.ref_diff.argtypes = [_P, _P, _I, _I, _I, _I]
        L.ref_aumisart1.argtypes = [_P] * 6 + [_I] * 8 + [_P] + [_F] * 8 + [_P] * 4
        L.ref_aumisart2.argtypes = [_P] * 6 + [_I] * 8 + [_P] + [_F] * 8 + [_P] * 4 + [_P] * 6
        self.L = L
        self._live = []

    # ------------------------------------------------------------ memory
    def _up(self, a) -> int:
        a = np.ascontiguousarray(a, dtype=np.float32)
        d = self.L.ref_malloc(max(a.nbytes, 4))
        if not d:
            raise MemoryError("ref_malloc failed")
        self.L.ref_h2d(d, a.ctypes.data, a.nbytes)
        self._live.append(d)
        return d

    def _new(self, nbytes) -> int:
        d = self.L.ref_malloc(max(nbytes, 4))
        if not d:
            raise MemoryError("ref_malloc failed")
        self._live.append(d)
        return d

    def _down(self, d, shape) -> np.ndarray:
        out = np.empty(shape, np.float32)
        self.L.ref_d2h(out.ctypes.data, d, out.nbytes)
        return out

    def _free(self):
        self.L.ref_sync()
        for d in self._live:
            self.L.ref_free(d)
        self._live = []

    @staticmethod
    def _g(geo):
        return [float(geo["SO"]), float(geo["SD"]), float(geo["da"]), int(geo["na"]),
                float(geo["ai"]), float(geo["db"]), int(geo["nb"]), float(geo["bi"]),
                int(geo["nx"]), int(geo["ny"]), int(geo["nz"])]

    # ---------------------------------------------------------- launchers
    def projection(self, img, angle, geo, init=None):
        """host_projection (src/cu_projection.cu:7)."""
        try:
            d_img = self._up(img)
            shape = (geo["nb"], geo["na"])
            d_proj = self._up(np.zeros(shape, np.float32) if init is None else init)
            self.L.ref_projection(d_proj, d_img, float(angle), *self._g(geo))
            return self._down(d_proj, shape)
        finally:
            self._free()

    def backprojection(self, proj, angle, geo):
        """host_backprojection (src/cu_backprojection.cu:8)."""
        try:
            d_proj = self._up(proj)
            shape = (geo["nz"], geo["ny"], geo["nx"])
            d_img = self._new(4 * int(np.prod(shape)))
            self.L.ref_backprojection(d_img, d_proj, float(angle), *self._g(geo))
            return self._down(d_img, shape)
        finally:
            self._free()

    def deform(self, img, volume, flow, fields, first_order=False):
        """host_deform / host_deform2 (src/cu_deform.cu:3, :49)."""
        try:
            nz, ny, nx = img.shape
            d_in = self._up(img)
            d_out = self._new(img.size * 4)
            d_f = [self._up(f) for f in fields]
            fn = self.L.ref_deform2 if first_order else self.L.ref_deform
            fn(d_out, d_in, nx, ny, nz, float(volume), float(flow), *d_f)
            return self._down(d_out, img.shape)
        finally:
            self._free()

    def forward_dvf(self, fields, volume, flow):
        """kernel_forwardDVF (src/cu_deform.cu:66)."""
        try:
            shape = fields[0].shape
            nz, ny, nx = shape
            d_f = [self._up(f) for f in fields]
            d_m = [self._new(fields[0].size * 4) for _ in range(3)]
            self.L.ref_forward_dvf(*d_m, *d_f, float(volume), float(flow), nx, ny, nz)
            return [self._down(d, shape) for d in d_m]
        finally:
            self._free()

    def _dims(self, a):
        s = (1,) * (3 - a.ndim) + a.shape
        return s[2], s[1], s[0]

    def add(self, img1, img, weight):
        try:
            d1, d = self._up(img1), self._up(img)
            self.L.ref_add(d1, d, *self._dims(np.asarray(img1)), float(weight))
            return self._down(d1, np.shape(img1))
        finally:
            self._free()

    def add2(self, img1, img, img0, weight, ind):
        try:
            d1, d, d0 = self._up(img1), self._up(img), self._up(img0)
            self.L.ref_add2(d1, d, *self._dims(np.asarray(img1)), d0, float(weight), int(ind))
            return self._down(d1, np.shape(img1))
        finally:
            self._free()

    def initial(self, shape, value):
        try:
            d = self._new(4 * int(np.prod(shape)))
            self.L.ref_initial(d, shape[2], shape[1], shape[0], float(value))
            return self._down(d, shape)
        finally:
            self._free()

    def initial2(self, img0, volume, flow):
        try:
            d0 = self._up(img0)
            d = self._new(img0.size * 4)
            nx, ny, nz = self._dims(img0)
            self.L.ref_initial2(d, nx, ny, nz, d0, float(volume), float(flow))
            return self._down(d, img0.shape)
        finally:
            self._free()

    def division(self, img1, img):
        try:
            d1, d = self._up(img1), self._up(img)
            self.L.ref_division(d1, d, *self._dims(np.asarray(img1)))
            return self._down(d1, np.shape(img1))
        finally:
            self._free()

    def multiple(self, img1, img0, weight, ind):
        try:
            d1, d0 = self._up(img1), self._up(img0)
            nx, ny, nz = self._dims(np.asarray(img1))
            self.L.ref_multiple(d1, nx, ny, nz, d0, float(weight), int(ind))
            return self._down(d1, np.shape(img1))
        finally:
            self._free()

    def update_udvf(self, fields, img, img0, vd, fd, it=0):
        try:
            d_f = [self._up(f) for f in fields]
            d, d0 = self._up(img), self._up(img0)
            nx, ny, nz = self._dims(img)
            self.L.ref_update_udvf(*d_f, d, d0, float(vd), float(fd), nx, ny, nz, int(it))
            return [self._down(x, img.shape) for x in d_f]
        finally:
            self._free()

    def diff(self, img, ind, init=None):
        try:
            d = self._up(img)
            d1 = self._up(np.zeros_like(img) if init is None else init)
            nx, ny, nz = self._dims(img)
            self.L.ref_diff(d1, d, nx, ny, nz, int(ind))
            return self._down(d1, img.shape)
        finally:
            self._free()

    def motion_projections(self, truth, fields, volumes, flows, angles, geo):
        """proj_v = host_projection(host_deform(truth, a_v - a_0, b_v - b_0), angle_v)
        for every view, with the volume and fields uploaded once (the
        measured projections of a motion workload, made by the reference's
        own kernels); fields None: the static truth's projections."""
        try:
            nz, ny, nx = truth.shape
            shape = (geo["nb"], geo["na"])
            d_truth = self._up(truth)
            d_tmp = self._new(truth.size * 4)
            d_f = [self._up(f) for f in fields] if fields is not None else None
            d_proj = self._new(int(np.prod(shape)) * 4)
            out = np.empty((len(angles),) + shape, np.float32)
            for v, a in enumerate(angles):
                src = d_truth
                if d_f is not None:
                    self.L.ref_deform(d_tmp, d_truth, nx, ny, nz,
                                      float(np.float32(volumes[v] - volumes[0])),
                                      float(np.float32(flows[v] - flows[0])), *d_f)
                    src = d_tmp
                self.L.ref_projection(d_proj, src, float(a), *self._g(geo))
                out[v] = self._down(d_proj, shape)
            return out
        finally:
            self._free()

    # ------------------------------------------------------ the SART loop
    def aumisart_inprocess(self, img, proj, geo, it, fields=None):
        """host_AUMISART in this process; ends in cudaDeviceReset()."""
        nz, ny, nx = img.shape
        na, nb = int(geo["na"]), int(geo["nb"])
        nv, n_iter = int(it["n_views"]), int(it["n_iter"])
        img = np.ascontiguousarray(img, np.float32)
        proj = np.ascontiguousarray(proj, np.float32)
        op = np.ascontiguousarray(it["op_iter"], np.int32)
        vols = np.ascontiguousarray(it["volumes"], np.float32)
        flows = np.ascontiguousarray(it["flows"], np.float32)
        angs = np.ascontiguousarray(it["angles"], np.float32)
        errw = np.zeros(nv, np.float32)
        out_img = np.zeros_like(img)
        out_proj = np.zeros((nv, nb, na), np.float32)
        out_norm = np.zeros(n_iter * nv, np.float32)
        out_ax = np.zeros_like(img)
        args = [out_img.ctypes.data, out_proj.ctypes.data, out_norm.ctypes.data,
                out_ax.ctypes.data, img.ctypes.data, proj.ctypes.data, nx, ny, nz, na, nb,
                int(it.get("outIter", 1)), nv, n_iter, op.ctypes.data, float(geo["da"]),
                float(geo["db"]), float(geo["ai"]), float(geo["bi"]), float(geo["SO"]),
                float(geo["SD"]), float(geo.get("dx", 1.0)), float(it["lambda"]),
                vols.ctypes.data, flows.ctypes.data, errw.ctypes.data, angs.ctypes.data]
        if fields is None:
            self.L.ref_aumisart1(*args)
        else:
            fl = [np.ascontiguousarray(f, np.float32) for f in fields]
            self.L.ref_aumisart2(*args, *[f.ctypes.data for f in fl])
        return {"img": out_img, "norm": out_norm, "alpha_x": out_ax, "resid": out_proj}


def aumisart(img, proj, geo, it, fields=None, timeout=1800):
    """host_AUMISART in a child process (see module docstring); returns a dict."""
    with tempfile.TemporaryDirectory() as td:
        inp, outp = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        payload = dict(img=img, proj=proj, **{f"geo_{k}": v for k, v in geo.items()},
                       **{f"it_{k}": np.asarray(v) for k, v in it.items()})
        if fields is not None:
            payload["fields"] = np.stack(fields)
        np.savez(inp, **payload)
        env = dict(os.environ)
        env["PYTHONPATH"] = os.path.dirname(HERE) + os.pathsep + env.get("PYTHONPATH", "")
        r = subprocess.run([sys.executable, "-m", "oracle.ref_runner", inp, outp], env=env,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference host_AUMISART failed:\n{r.stdout}\n{r.stderr}")
        with np.load(outp) as z:
            return {k: z[k] for k in z.files}


def _child(inp, outp):
    import time
    z = np.load(inp)
    geo = {k[4:]: z[k].item() for k in z.files if k.startswith("geo_")}
    it = {k[3:]: z[k] for k in z.files if k.startswith("it_")}
    for k in ("n_views", "n_iter", "outIter"):
        if k in it:
            it[k] = int(it[k])
    it["lambda"] = float(it["lambda"])
    fields = list(z["fields"]) if "fields" in z.files else None
    t0 = time.perf_counter()
    out = Ref().aumisart_inprocess(z["img"], z["proj"], geo, it, fields)
    out["seconds"] = np.float64(time.perf_counter() - t0)
    np.savez(outp, **out)


if __name__ == "__main__":
    _child(sys.argv[1], sys.argv[2])
