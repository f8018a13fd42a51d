"""The true inverse of the warp's displacement (mcsart_invert_dvf) and its use
in SART's back-warps (options.dvf_inverse).  The reference approximates the
inverse warp by negating the breathing amplitudes (src/AUMISART.cu:222)."""
import numpy as np
import pytest

from conftest import dev, fields, host, rel_l2
from test_gpu_sart import make_case

pytestmark = pytest.mark.gpu


def _fields(shape, seed, scale):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(gaussian_filter(rng.normal(size=shape), 3.0) * scale,
                                 np.float32) for _ in range(6)]


def _invert(ctx, torch, F, volume, flow, iters):
    nz, ny, nx = F[0].shape
    out = [torch.empty((nz, ny, nx), device="cuda") for _ in range(3)]
    ctx.invert_dvf(*out, *[dev(torch, f) for f in F], volume, flow, nx, ny, nz, iters)
    ctx.synchronize()
    return [host(o) for o in out]


def test_inverse_matches_the_fp64_oracle(ctx, torch_cuda, oracle):
    F = _fields((14, 20, 20), 3, 8.0)
    for vol, flow in ((1.0, 0.0), (0.6, -0.4)):
        mine = _invert(ctx, torch_cuda, F, vol, flow, 8)
        o = oracle.invert_dvf(F, vol, flow, 8)
        for c in range(3):
            assert rel_l2(mine[c], o[c]) <= 1e-5, (vol, flow, c, rel_l2(mine[c], o[c]))


def test_true_inverse_composes_to_the_identity(ctx, torch_cuda):
    """The warp samples position q at q + D(q).  For the true inverse N the
    composition residual N(q) + D(q + N(q)) vanishes (up to the fixed point's
    convergence); for the reference's negated amplitudes it is of the order
    of D * grad D."""
    from scipy.ndimage import map_coordinates
    shape = (14, 24, 24)
    F = _fields(shape, 5, 10.0)
    vol = 1.0
    inv = _invert(ctx, torch_cuda, F, vol, 0.0, 12)
    mx, my, mz = [np.float64(f) * vol for f in F[:3]]  # beta * flow = 0
    Z, Y, X = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")

    def residual(NX, NY, NZ):
        c = [Z + NZ, Y + NY, X + NX]
        DX = map_coordinates(my, c, order=1, mode="nearest")
        DY = map_coordinates(mx, c, order=1, mode="nearest")
        DZ = map_coordinates(mz, c, order=1, mode="nearest")
        r = np.sqrt((NX + DX) ** 2 + (NY + DY) ** 2 + (NZ + DZ) ** 2)
        return r[3:-3, 4:-4, 4:-4].max()  # away from the clamped edges

    r_true = residual(np.float64(inv[1]), np.float64(inv[0]), np.float64(inv[2]))
    r_neg = residual(-my, -mx, -mz)
    print(f"composition residual: true inverse {r_true:.2e}, negated amplitudes {r_neg:.2e} voxels")
    assert r_true < 1e-3 and r_true < 0.01 * r_neg, (r_true, r_neg)


def test_sart_with_the_true_inverse_matches_the_oracle(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    torch = torch_cuda
    op = (1, 1)
    g, it, img0, proj, F = make_case(oracle, motion=True, op_iter=op, seed=14)
    d_img = dev(torch, img0)
    opt = m.default_options(dvf_inverse=6, interp=m.INTERP_EXACT)
    ctx.aumisart_device(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                        volumes=it["volumes"], flows=it["flows"], img=d_img, proj=dev(torch, proj),
                        fields=dev(torch, np.stack(F)), n_iter=len(op),
                        op_iter=np.array(op, np.int32), options=opt)
    ctx.synchronize()
    o = oracle.aumisart(img0, proj, g, it, F, tex_mode=oracle.TEX_EXACT, dvf_inverse=6)
    err = rel_l2(host(d_img), o["img"])
    print(f"SART with the true DVF inverse: rel L2 vs FP64 oracle {err:.2e}")
    assert err <= 2e-5, err


def test_dvf_inverse_options_are_validated(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    torch = torch_cuda
    g, it, img0, proj, F = make_case(oracle, motion=True, nx=20, ny=16, op_iter=(1,), seed=15)
    with pytest.raises(m.McsartError):  # non-square slices
        ctx.aumisart_device(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                            volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0),
                            proj=dev(torch, proj), fields=dev(torch, np.stack(F)), n_iter=1,
                            op_iter=np.array([1], np.int32),
                            options=m.default_options(dvf_inverse=4))
    with pytest.raises(m.McsartError):  # 16-bit storage
        m.default_options(dvf_inverse=4, storage=m.BF16)  # built fine; rejected on use
        ctx.aumisart_device(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                            volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0),
                            proj=dev(torch, proj).to(torch.bfloat16),
                            fields=dev(torch, np.stack(F)).to(torch.bfloat16), n_iter=1,
                            op_iter=np.array([1], np.int32),
                            options=m.default_options(dvf_inverse=4, storage=m.BF16))
