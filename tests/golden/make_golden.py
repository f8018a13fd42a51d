"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs bill52547/McSART's own CUDA kernels and host_AUMISART, rebuilt unmodified
from their sources (oracle/_ref/libmcsart_ref.so, see oracle/Makefile), on a GPU,
for small seeded inputs, and stores inputs and outputs:

  ref_kernels.npz   projector, backprojector, warps, forwardDVF and the
                    elementwise steps on three geometries / shapes
  ref_aumisart.npz  host_AUMISART overload 1 and overload 2 on a small problem

Usage (needs a CUDA GPU):  python tests/golden/make_golden.py [out_dir]
The CPU test tests/test_oracle_golden.py checks the FP64 oracle against them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import ANGLES, fields, geo, volume  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref_runner  # noqa: E402

GEOS = [geo(), geo(nx=20, ny=20, nz=12, na=36, nb=24, ai=1.5, bi=-2.0),
        geo(nx=33, ny=17, nz=9, na=45, nb=15, da=1.1, db=1.3, SO=70, SD=100)]
SHAPES = [(12, 20, 20), (16, 20, 24), (9, 17, 33)]
VF = [(1.3, -0.4), (-2.7, 0.9)]


def kernels(ref) -> dict:
    out = {}
    for gi, g in enumerate(GEOS):
        img = volume((g["nz"], g["ny"], g["nx"]), seed=gi)
        rng = np.random.default_rng(10 + gi)
        out[f"g{gi}_img"] = img
        for k, v in g.items():
            out[f"g{gi}_geo_{k}"] = np.float64(v)
        for ai, a in enumerate(ANGLES):
            proj = rng.random((g["nb"], g["na"]), dtype=np.float32)
            out[f"g{gi}_a{ai}_fp"] = ref.projection(img, a, g)
            out[f"g{gi}_a{ai}_bpin"] = proj
            out[f"g{gi}_a{ai}_bp"] = ref.backprojection(proj, a, g)
    for si, shape in enumerate(SHAPES):
        img = volume(shape, seed=3)
        F = fields(shape, seed=4)
        out[f"s{si}_img"] = img
        out[f"s{si}_fields"] = np.stack(F)
        for vi, (vol, flow) in enumerate(VF):
            out[f"s{si}_v{vi}_deform"] = ref.deform(img, np.float32(vol), np.float32(flow), F)
            out[f"s{si}_v{vi}_deform2"] = ref.deform(img, np.float32(vol), np.float32(flow), F,
                                                     first_order=True)
            out[f"s{si}_v{vi}_fdvf"] = np.stack(ref.forward_dvf(F, vol, flow))
    shape = SHAPES[2]
    a, b, c = volume(shape, 1), volume(shape, 2), volume(shape, 3)
    b[0, 0, :5] = 0.0
    F = fields(shape, seed=12)
    out.update(e_a=a, e_b=b, e_c=c, e_fields=np.stack(F))
    out["e_add"] = ref.add(a, b, -0.7)
    for ind in (1, 2, 3):
        out[f"e_add2_{ind}"] = ref.add2(a, b, c, 0.6, ind)
        out[f"e_multiple_{ind}"] = ref.multiple(a, c, 1.4, ind)
        out[f"e_diff_{ind}"] = ref.diff(b, ind)
    out["e_initial2"] = ref.initial2(c, -0.4, 1.9)
    out["e_division"] = ref.division(a, b)
    out["e_udvf"] = np.stack(ref.update_udvf(F, b, c, 0.9, -0.5))
    return out


def aumisart_cases() -> dict:
    out = {}
    shape = (12, 16, 16)
    g = geo(nx=16, ny=16, nz=12, na=32, nb=24, SO=60, SD=90, da=0.9, db=0.9)
    truth = np.zeros(shape, np.float32)
    truth[3:9, 4:12, 3:13] = 0.02
    truth[5:7, 6:9, 6:9] += 0.03
    nv = 12
    angles = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(0)
    t = np.arange(nv) / 15.0
    vols = ((8 * np.sin(2 * np.pi * t / 4) + rng.normal(0, 0.5, nv)) * 0.1).astype(np.float32)
    flows = (8 * 2 * np.pi / 4 * np.cos(2 * np.pi * t / 4) * 0.1).astype(np.float32)
    proj = np.stack([O.projection(truth, a, g).astype(np.float32) for a in angles])
    F = fields(shape, seed=5, scale=0.3)
    for k, v in g.items():
        out[f"geo_{k}"] = np.float64(v)
    out.update(truth=truth, angles=angles, volumes=vols, flows=flows, proj=proj,
               fields=np.stack(F))
    for name, ff, op in (("o1", None, (1, 0, 1, 1, 1)), ("o2", F, (1, 0, 1, 0, 1))):
        it = dict(n_iter=len(op), op_iter=np.array(op, np.int32), n_views=nv, outIter=1,
                  volumes=vols, flows=flows, angles=angles, **{"lambda": 1.0})
        r = ref_runner.aumisart(np.zeros(shape, np.float32), proj, g, it, ff)
        out[f"{name}_op_iter"] = np.array(op, np.int32)
        for k in ("img", "norm", "alpha_x", "resid"):
            out[f"{name}_{k}"] = r[k]
    return out


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    ref = ref_runner.Ref()
    np.savez_compressed(os.path.join(out_dir, "ref_kernels.npz"), **kernels(ref))
    np.savez_compressed(os.path.join(out_dir, "ref_aumisart.npz"), **aumisart_cases())
    print("wrote", out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
