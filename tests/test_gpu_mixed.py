"""Mixed precision against the FP64 oracle at the 256x256x160 workload's size
(detector 512x384): every kernel, and the reconstructed volume after 10
image passes.

Storage modes: the DVF fields, the warped volumes the projector reads and the
measured projections in BF16 or FP16 (the reconstructed volume, the
residuals and every accumulation stay FP32); FP64 geometry and normalisation
sums (geom64) with the Kahan-compensated projector.  The warp is the exact
FP32 trilinear model (INTERP_EXACT), which the oracle restates in FP64.

Inputs are given at BF16 precision (measured projections and DVF fields
rounded to BF16 once; such values are exact in FP16 and FP32 as well), so
that every mode reconstructs from the same numbers and one FP64 oracle run
is the reference for all of them: the errors below are those of the
engine's arithmetic and intermediate storage, not of quantising the inputs.

Measured errors are printed (pytest -s) and written to
gpurun_out/mixed_precision_errors.json when that folder exists.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, dev, host, max_rel, rel_l2

pytestmark = pytest.mark.gpu

# unit roundoff of the storage types (half an ulp, relative)
U_BF16, U_F16 = 2.0 ** -8, 2.0 ** -11

RESULTS = {}


def _record(name, **kw):
    RESULTS[name] = kw
    print(name, " ".join(f"{k}={v:.3e}" for k, v in kw.items()))
    out = os.path.join(ROOT, "gpurun_out")
    if os.path.isdir(out):
        with open(os.path.join(out, "mixed_precision_errors.json"), "w") as f:
            json.dump(RESULTS, f, indent=1, sort_keys=True)


def _bf16(torch, a):
    """a rounded to BF16 (round to nearest even), as float32."""
    return torch.as_tensor(np.ascontiguousarray(a)).to(torch.bfloat16).to(torch.float32).numpy()


def _args(g):
    return (g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"], g["nb"], g["bi"], g["nx"],
            g["ny"], g["nz"])


@pytest.fixture(scope="module")
def motion256_problem(ctx, torch_cuda):
    """The seeded 256x256x160 problem (phantom, DVF), inputs at BF16 precision."""
    from mcsart_b200 import synthetic as S
    torch = torch_cuda
    p = S.make_problem("motion256", 0)
    truth = _bf16(torch, p.truth)
    F = [_bf16(torch, f) for f in p.fields]
    return p, truth, F


def test_kernel_errors_vs_fp64_oracle_at_256x256x160(ctx, torch_cuda, oracle, motion256_problem):
    """One call of each kernel form against the FP64 oracle of the same
    inputs.  Bounds: FP32-storage forms within 1e-5 relative L2; forms whose
    input or output is stored in 16 bits within that type's unit roundoff
    (plus 1e-5); the texture-unit warp (the reference's 8-bit filter
    weights) within 1e-2."""
    import mcsart_b200 as m
    torch = torch_cuda
    p, truth, F = motion256_problem
    g = p.geo
    angle = 0.3  # x-driven rays
    o_fp = oracle.projection(truth, angle, g)
    d_vol = dev(torch, truth)
    d_p = torch.empty((g["nb"], g["na"]), device="cuda")
    cases = [("fp_f32_reference_order", torch.float32, 0, 0, 1e-5),
             ("fp_f32_split", torch.float32, 1, 0, 1e-5),
             ("fp_f32_kahan_geom64", torch.float32, 2, 1, 1e-5),
             ("fp_bf16_volume", torch.bfloat16, 0, 0, U_BF16 + 1e-5),
             ("fp_bf16_volume_kahan_geom64", torch.bfloat16, 2, 1, U_BF16 + 1e-5),
             ("fp_f16_volume", torch.float16, 0, 0, U_F16 + 1e-5)]
    for name, dt, fp_sum, g64, tol in cases:
        ctx.projection_ex(d_p, d_vol.to(dt), angle, *_args(g), fp_sum=fp_sum, geom64=g64)
        ctx.synchronize()
        e = rel_l2(host(d_p), o_fp)
        _record(name, rel_l2=e, max_rel=max_rel(host(d_p), o_fp))
        assert e <= tol, (name, e)

    # backprojector (the reference's operator, not the projector's adjoint)
    proj = o_fp.astype(np.float32)
    o_bp = oracle.backprojection(proj, angle, g)
    d_proj = dev(torch, proj)
    d_b = torch.empty_like(d_vol)
    for name, g64 in (("bp_f32", 0), ("bp_f32_geom64", 1)):
        ctx.backprojection_ex(d_b, d_proj, angle, *_args(g), geom64=g64)
        ctx.synchronize()
        e = rel_l2(host(d_b), o_bp)
        _record(name, rel_l2=e, max_rel=max_rel(host(d_b), o_bp))
        assert e <= 1e-5, (name, e)

    # warp at the largest breathing amplitude of the scan
    v = int(np.argmax(np.abs(p.volumes - p.volumes[0])))
    vol, flow = float(p.volumes[v] - p.volumes[0]), float(p.flows[v] - p.flows[0])
    o_w = oracle.deform(truth, vol, flow, F, tex_mode=oracle.TEX_EXACT)
    dF = dev(torch, np.stack(F))
    for name, dt, interp, tol in (("warp_f32_exact", torch.float32, m.INTERP_EXACT, 1e-5),
                                  ("warp_f32_texture", torch.float32, m.INTERP_TEXTURE, 1e-2),
                                  ("warp_bf16_exact", torch.bfloat16, m.INTERP_EXACT,
                                   U_BF16 + 1e-5),
                                  ("warp_f16_exact", torch.float16, m.INTERP_EXACT,
                                   U_F16 + 1e-5)):
        out = torch.empty(truth.shape, dtype=dt, device="cuda")
        ctx.deform_ex(out, d_vol, g["nx"], g["ny"], g["nz"], vol, flow, dF.to(dt), interp=interp)
        ctx.synchronize()
        got = host(out.float())
        e = rel_l2(got, o_w)
        _record(name, rel_l2=e, max_rel=max_rel(got, o_w))
        assert e <= tol, (name, e)


def test_volume_error_after_10_image_passes_at_256x256x160(ctx, torch_cuda, oracle,
                                                              motion256_problem):
    """Motion-compensated SART with the DVF held fixed (10 image passes; the
    DVF-update pass divides by a signed normaliser and so amplifies any
    rounding difference without bound, see test_golden_shows_the_dvf_update_
    is_ill_conditioned), 12 views spread over the 660-view scan (every 55th:
    angles and breathing phases of the whole scan), at the full volume and
    detector size.  Every storage mode with the exact warp stays within 1e-3
    relative L2 of the FP64 oracle."""
    import mcsart_b200 as m
    torch = torch_cuda
    p, truth, F = motion256_problem
    g = p.geo
    sel = np.arange(0, p.cfg.n_views, 55)
    nv = len(sel)
    angles, vols, flows = p.angles[sel], p.volumes[sel], p.flows[sel]
    # measured projections of the warped phantom (the engine's FP32 drop-in
    # warp and projector), then rounded to BF16
    d_truth = dev(torch, truth)
    d_F = [dev(torch, f) for f in F]
    tmp = torch.empty_like(d_truth)
    proj = torch.empty((nv, g["nb"], g["na"]), device="cuda")
    for j in range(nv):
        ctx.host_deform(tmp, d_truth, g["nx"], g["ny"], g["nz"], np.float32(vols[j] - vols[0]),
                        np.float32(flows[j] - flows[0]), *d_F)
        ctx.host_projection(proj[j], tmp, float(angles[j]), *_args(g))
    ctx.synchronize()
    proj = _bf16(torch, host(proj))
    n_iter = 10
    op = np.ones(n_iter, np.int32)
    it = dict(n_iter=n_iter, op_iter=op, n_views=nv, **{"lambda": p.cfg.lam}, outIter=1,
              volumes=vols, flows=flows, angles=angles)
    img0 = np.zeros_like(truth)
    o = oracle.aumisart(img0, proj, g, it, F, tex_mode=oracle.TEX_EXACT)["img"]
    modes = [("f32_drop_in_texture_warp", m.F32, dict(), 1e-2),
             ("f32_exact_warp", m.F32, dict(interp=m.INTERP_EXACT), 1e-3),
             ("f32_kahan_geom64", m.F32, dict(interp=m.INTERP_EXACT, fp_sum=2, geom64=1), 1e-3),
             ("bf16", m.BF16, dict(interp=m.INTERP_EXACT), 1e-3),
             ("bf16_kahan_geom64", m.BF16, dict(interp=m.INTERP_EXACT, fp_sum=2, geom64=1), 1e-3),
             ("f16", m.F16, dict(interp=m.INTERP_EXACT), 1e-3),
             ("f16_kahan_geom64", m.F16, dict(interp=m.INTERP_EXACT, fp_sum=2, geom64=1), 1e-3)]
    for name, storage, kw, tol in modes:
        dt = {m.F32: torch.float32, m.BF16: torch.bfloat16, m.F16: torch.float16}[storage]
        d_img = dev(torch, img0)
        opt = m.default_options(storage=storage, **kw)
        ctx.aumisart_device(geo=g, n_views=nv, lambda_=p.cfg.lam, angles=angles, volumes=vols,
                            flows=flows, img=d_img, proj=dev(torch, proj).to(dt),
                            fields=dev(torch, np.stack(F)).to(dt), n_iter=n_iter, op_iter=op,
                            options=opt)
        ctx.synchronize()
        got = host(d_img)
        e = rel_l2(got, o)
        _record("volume_after_10_passes_" + name, rel_l2=e, max_rel=max_rel(got, o))
        assert e <= tol, (name, e)
