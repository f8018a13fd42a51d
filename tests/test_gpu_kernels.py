"""Per-kernel parity of the engine's C ABI against the rebuilt reference kernels
(same GPU, same inputs) and against the FP64 CPU oracle.

Against the reference the projector, backprojector and texture-unit warp are
compared bit for bit (the stated bar for the FP32 drop-in is 1e-5 relative L2
per call; the kernels meet it with zero difference), elementwise steps bit
for bit where the arithmetic is the same, else to 1e-6.  Against the FP64 oracle the projector
and warp are held to 1e-5 and the backprojector to 1e-4 (the reference and the
engine take __sinf/__cosf of the angle, the oracle exact sine and cosine).
"""
import numpy as np
import pytest

from conftest import ANGLES, dev, fields, geo, host, max_rel, rel_l2, volume

pytestmark = pytest.mark.gpu

GEOS = [geo(), geo(nx=20, ny=20, nz=12, na=36, nb=24, ai=1.5, bi=-2.0),
        geo(nx=33, ny=17, nz=9, na=45, nb=15, da=1.1, db=1.3, SO=70, SD=100)]


def _fp(ctx, torch, img, angle, g):
    d_img = dev(torch, img)
    d_proj = torch.zeros((g["nb"], g["na"]), dtype=torch.float32, device="cuda")
    ctx.host_projection(d_proj, d_img, angle, g["SO"], g["SD"], g["da"], g["na"], g["ai"],
                        g["db"], g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
    ctx.synchronize()
    return host(d_proj)


def _bp(ctx, torch, proj, angle, g):
    d_proj = dev(torch, proj)
    d_img = torch.full((g["nz"], g["ny"], g["nx"]), 7.0, dtype=torch.float32, device="cuda")
    ctx.host_backprojection(d_img, d_proj, angle, g["SO"], g["SD"], g["da"], g["na"], g["ai"],
                            g["db"], g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
    ctx.synchronize()
    return host(d_img)


@pytest.mark.parametrize("gi", range(len(GEOS)))
def test_projection_matches_reference_and_oracle(ctx, torch_cuda, ref, oracle, gi):
    g = GEOS[gi]
    img = volume((g["nz"], g["ny"], g["nx"]), seed=gi)
    for a in ANGLES:
        mine = _fp(ctx, torch_cuda, img, a, g)
        r = ref.projection(img, a, g)
        o = oracle.projection(img, a, g)
        assert rel_l2(mine, r) <= 1e-5, (a, rel_l2(mine, r))
        assert np.count_nonzero(mine != r) == 0, (a, np.count_nonzero(mine != r), mine.size)
        assert rel_l2(mine, o) <= 1e-5, (a, rel_l2(mine, o))


def test_projection_of_ones_counts_slabs(ctx, torch_cuda):
    """Known answer: rays through the volume's core see one unit per slab."""
    g = geo(nx=32, ny=32, nz=32, na=64, nb=48, SO=200, SD=300, da=0.8, db=0.8)
    p = _fp(ctx, torch_cuda, np.ones((32, 32, 32), np.float32), 0.0, g)
    np.testing.assert_allclose(p[23:25, 31:33], 32.0, rtol=1e-6)


@pytest.mark.parametrize("gi", range(len(GEOS)))
def test_backprojection_matches_reference_and_oracle(ctx, torch_cuda, ref, oracle, gi):
    g = GEOS[gi]
    rng = np.random.default_rng(10 + gi)
    for a in ANGLES:
        proj = rng.random((g["nb"], g["na"]), dtype=np.float32)
        mine = _bp(ctx, torch_cuda, proj, a, g)
        r = ref.backprojection(proj, a, g)
        o = oracle.backprojection(proj, a, g)
        # same arithmetic in the same order as the reference kernel: bit for bit
        np.testing.assert_array_equal(mine, r)
        assert rel_l2(mine, o) <= 1e-4, (a, rel_l2(mine, o))


def bp_geom_proven(g):
    """The condition under which the backprojector launches its form without
    division range tests (bp_geom_proven in csrc/backprojector.cuh)."""
    R = ((g["nx"] // 2) + (g["ny"] // 2) + 3.0) * (1.0 + 2.0 ** -10)
    dlo, dhi = g["SO"] - R, g["SO"] + R
    if not (dlo >= 2.0 ** -19 and dhi < 2.0 ** 19):
        return False
    rmin = g["SD"] / dhi * (1.0 - 2.0 ** -10)
    rmax = g["SD"] / dlo * (1.0 + 2.0 ** -10)
    ext = R + g["nz"] // 2 + 4.0
    return (2.0 ** -79 <= g["SD"] <= 2.0 ** 79 and 2.0 ** -19 <= g["da"] < 2.0 ** 19
            and 2.0 ** -19 <= g["db"] < 2.0 ** 19 and rmin * 2.0 ** -26 >= 2.0 ** -79
            and rmax * ext <= 2.0 ** 79)


# source 20 voxels from the centre of a 24x20 slice (half-diagonal 15.6): the
# geometry is fine, but outside the backprojector's proof
CLOSE = geo(nx=24, ny=20, nz=16, na=40, nb=28, SO=20, SD=30, da=0.9, db=0.8)


def test_backprojection_outside_the_geometry_proof_matches_reference(ctx, torch_cuda, ref):
    """Both backprojector forms are covered: the parity geometries above take
    the one without range tests, this close-source geometry the general one;
    each matches the reference bit for bit (and so does the projector)."""
    assert all(bp_geom_proven(g) for g in GEOS) and not bp_geom_proven(CLOSE)
    rng = np.random.default_rng(31)
    img = volume((CLOSE["nz"], CLOSE["ny"], CLOSE["nx"]), seed=32)
    for a in ANGLES:
        proj = rng.random((CLOSE["nb"], CLOSE["na"]), dtype=np.float32)
        np.testing.assert_array_equal(_bp(ctx, torch_cuda, proj, a, CLOSE),
                                      ref.backprojection(proj, a, CLOSE))
        np.testing.assert_array_equal(_fp(ctx, torch_cuda, img, a, CLOSE),
                                      ref.projection(img, a, CLOSE))


@pytest.mark.parametrize("shape", [(12, 20, 20), (16, 20, 24), (9, 17, 33)])
@pytest.mark.parametrize("vf", [(0.0, 0.0), (1.3, -0.4), (-2.7, 0.9)])
def test_deform_matches_reference(ctx, torch_cuda, ref, oracle, shape, vf):
    torch = torch_cuda
    img = volume(shape, seed=3)
    F = fields(shape, seed=4)
    vol, flow = np.float32(vf[0]), np.float32(vf[1])
    d_img, d_out = dev(torch, img), torch.zeros(shape, dtype=torch.float32, device="cuda")
    d_F = [dev(torch, f) for f in F]
    nz, ny, nx = shape
    ctx.host_deform(d_out, d_img, nx, ny, nz, vol, flow, *d_F)
    ctx.synchronize()
    mine = host(d_out)
    r = ref.deform(img, vol, flow, F)
    np.testing.assert_array_equal(mine, r)  # the texture unit, as in the reference
    if vf == (0.0, 0.0) and shape[1] == shape[2]:
        np.testing.assert_array_equal(mine, img)  # zero DVF on square slices: identity


def test_deform_in_place(ctx, torch_cuda, ref):
    torch = torch_cuda
    shape = (12, 20, 20)
    img, F = volume(shape, seed=5), fields(shape, seed=6)
    d = dev(torch, img)
    d_F = [dev(torch, f) for f in F]
    ctx.host_deform(d, d, 20, 20, 12, 0.8, 0.3, *d_F)
    ctx.synchronize()
    assert rel_l2(host(d), ref.deform(img, 0.8, 0.3, F)) <= 1e-5


def test_deform_exact_interp_matches_oracle(torch_cuda, oracle):
    import mcsart_b200 as m
    torch = torch_cuda
    shape = (12, 20, 20)
    img, F = volume(shape, seed=7), fields(shape, seed=8)
    with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
        c.set_interp(m.INTERP_EXACT)
        d_out = torch.zeros(shape, dtype=torch.float32, device="cuda")
        c.host_deform(d_out, dev(torch, img), 20, 20, 12, 1.1, -0.6, *[dev(torch, f) for f in F])
        c.synchronize()
        o = oracle.deform(img, 1.1, -0.6, F, tex_mode=oracle.TEX_EXACT)
        assert rel_l2(host(d_out), o) <= 1e-6


def test_deform2_matches_reference(ctx, torch_cuda, ref):
    torch = torch_cuda
    shape = (12, 20, 20)
    img, F = volume(shape, seed=9), fields(shape, seed=10)
    d_out = torch.zeros(shape, dtype=torch.float32, device="cuda")
    ctx.host_deform2(d_out, dev(torch, img), 20, 20, 12, 0.7, 0.2, *[dev(torch, f) for f in F])
    ctx.synchronize()
    r = ref.deform2 if hasattr(ref, "deform2") else None
    r = ref.deform(img, 0.7, 0.2, F, first_order=True)
    # the reference reads past the volume for the last slice's +nx neighbours
    assert rel_l2(host(d_out)[:-1], r[:-1]) <= 1e-6


def test_forward_dvf_bitwise(ctx, torch_cuda, ref):
    torch = torch_cuda
    shape = (9, 17, 33)
    F = fields(shape, seed=11)
    d_F = [dev(torch, f) for f in F]
    m = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    ctx.kernel_forwardDVF(*m, *d_F, 1.7, -0.3, 33, 17, 9)
    ctx.synchronize()
    for a, b in zip(m, ref.forward_dvf(F, 1.7, -0.3)):
        np.testing.assert_array_equal(host(a), b)


def test_elementwise_match_reference(ctx, torch_cuda, ref):
    torch = torch_cuda
    shape = (9, 17, 33)
    nz, ny, nx = shape
    a, b, c = volume(shape, 1), volume(shape, 2), volume(shape, 3)
    b[0, 0, :5] = 0.0  # division by zero -> 0
    F = fields(shape, seed=12)

    def run(fn, *arrs):
        ts = [dev(torch, x) for x in arrs]
        fn(*ts)
        ctx.synchronize()
        return [host(t) for t in ts]

    out = run(lambda x, y: ctx.host_add(x, y, nx, ny, nz, -0.7), a, b)[0]
    np.testing.assert_array_equal(out, ref.add(a, b, -0.7))
    for ind in (1, 2, 3):
        out = run(lambda x, y, z: ctx.host_add2(x, y, nx, ny, nz, z, 0.6, ind), a, b, c)[0]
        np.testing.assert_array_equal(out, ref.add2(a, b, c, 0.6, ind))
        out = run(lambda x, z: ctx.host_multiple(x, nx, ny, nz, z, 1.4, ind), a, c)[0]
        np.testing.assert_array_equal(out, ref.multiple(a, c, 1.4, ind))
        out = run(lambda x, y: ctx.host_diff(x, y, nx, ny, nz, ind), np.zeros_like(a), b)[0]
        np.testing.assert_array_equal(out, ref.diff(b, ind))
    out = run(lambda x: ctx.host_initial(x, nx, ny, nz, 2.5), a)[0]
    np.testing.assert_array_equal(out, ref.initial(shape, 2.5))
    out = run(lambda x, z: ctx.host_initial2(x, nx, ny, nz, z, -0.4, 1.9), a, c)[0]
    np.testing.assert_array_equal(out, ref.initial2(c, -0.4, 1.9))
    out = run(lambda x, y: ctx.host_division(x, y, nx, ny, nz), a, b)[0]
    np.testing.assert_array_equal(out, ref.division(a, b))
    assert np.all(out[0, 0, :5] == 0.0)
    outs = run(lambda *t: ctx.host_update_udvf(*t[:6], t[6], t[7], 0.9, -0.5, nx, ny, nz),
               *F, b, c)
    for x, y in zip(outs[:6], ref.update_udvf(F, b, c, 0.9, -0.5)):
        np.testing.assert_array_equal(x, y)


def test_projection_residual_on_projection_shape(ctx, torch_cuda, ref):
    """host_add on a projection (nx, ny, nz) = (na, nb, 1), AUMISART.cu:206."""
    torch = torch_cuda
    rng = np.random.default_rng(0)
    p, q = rng.random((28, 40), dtype=np.float32), rng.random((28, 40), dtype=np.float32)
    d_p, d_q = dev(torch, p), dev(torch, q)
    ctx.host_add(d_p, d_q, 40, 28, 1, -1.0)
    ctx.synchronize()
    np.testing.assert_array_equal(host(d_p), ref.add(p, q, -1.0))


def test_projection_views_matches_single_view(ctx, torch_cuda):
    torch = torch_cuda
    g = GEOS[0]
    img = volume((g["nz"], g["ny"], g["nx"]), seed=21)
    d_img = dev(torch, img)
    d_all = torch.zeros((len(ANGLES), g["nb"], g["na"]), dtype=torch.float32, device="cuda")
    ctx.projection_views(d_all, d_img, ANGLES, g["SO"], g["SD"], g["da"], g["na"], g["ai"],
                         g["db"], g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
    ctx.synchronize()
    allv = host(d_all)
    for v, a in enumerate(ANGLES):
        np.testing.assert_array_equal(allv[v], _fp(ctx, torch, img, a, g))


def test_snrm2(ctx, torch_cuda):
    x = np.random.default_rng(3).normal(size=100003).astype(np.float32)
    n = ctx.snrm2(x.size, dev(torch_cuda, x))
    assert abs(n - np.linalg.norm(x.astype(np.float64))) <= 1e-6 * n


def test_runs_are_bitwise_reproducible(ctx, torch_cuda):
    g = GEOS[1]
    img = volume((g["nz"], g["ny"], g["nx"]), seed=30)
    p1 = _fp(ctx, torch_cuda, img, 0.9, g)
    p2 = _fp(ctx, torch_cuda, img, 0.9, g)
    np.testing.assert_array_equal(p1, p2)
    b1 = _bp(ctx, torch_cuda, p1, 0.9, g)
    b2 = _bp(ctx, torch_cuda, p1, 0.9, g)
    np.testing.assert_array_equal(b1, b2)


def test_invalid_arguments_raise(ctx, torch_cuda):
    import mcsart_b200 as m
    with pytest.raises(m.McsartError) as e:
        ctx.host_projection(0, 0, 0.0, 60, 90, 1, 10, 0, 1, 10, 0, 8, 8, 8)
    assert e.value.code == m.ERR_INVALID_ARGUMENT
    t = torch_cuda.zeros(8, device="cuda")
    with pytest.raises(m.McsartError):
        ctx.host_add2(t, t, 2, 2, 2, t, 1.0, 4)
    with pytest.raises(m.McsartError):
        ctx.host_projection(t, t, 0.0, 60, 90, 1, 0, 0, 1, 10, 0, 8, 8, 8)
