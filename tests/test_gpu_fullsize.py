"""Parity at the benchmark workloads' full sizes.

The kernel-level parity tests use small volumes the CPU oracle finishes in
seconds.  Here the engine runs at the workloads' own sizes against the
reference's own kernels and loop, rebuilt from its sources, bit for bit:

* the static 64x64x64 workload (detector 128x96, 60 views): five image passes
  of host_AUMISART overload 1;
* the motion-compensated 256x256x160 workload (detector 512x384, 660 views):
  projector, backprojector and warp, and one outer iteration of the loop;
  the 128x128x96 workload (detector 256x192, 360 views): one outer
  iteration of the loop;
* the clinical 512x512x256 size (detector 1024x768): projector,
  backprojector and warp, whose 256 MiB volume no longer fits the 126 MB L2,
  plus a size-independent property: a ray that stays inside the volume
  through every slab sums normalised footprint weights, so its projection of
  a ones-volume is the number of slabs;
* the uneven batch (8 motion problems from 96x96x64 to 256x256x128, 120 to
  660 views, ordered subsets of 10 views) through mcsart_batch_run, bitwise
  equal to separate runs of each problem.
"""
import numpy as np
import pytest

from conftest import dev, host

pytestmark = pytest.mark.gpu


def _geo(cfg):
    from mcsart_b200 import synthetic as S
    return S.geometry(S.CONFIGS[cfg])


def _args(g):
    return (g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"], g["nb"], g["bi"], g["nx"],
            g["ny"], g["nz"])


def _smooth_volume(shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.random(shape, dtype=np.float32)
    # cheap smoothing: box average along each axis
    for ax in range(3):
        v = (v + np.roll(v, 1, axis=ax) + np.roll(v, -1, axis=ax)) / np.float32(3)
    return np.ascontiguousarray(v, np.float32)


@pytest.fixture(scope="module")
def motion256():
    g = _geo("motion256")
    return g, _smooth_volume((g["nz"], g["ny"], g["nx"]), 31)


@pytest.mark.parametrize("angle", [0.3, 0.7853982, 2.4, 4.0])
def test_projection_and_backprojection_match_the_reference_at_256x256x160(ctx, torch_cuda, ref, motion256,
                                                                      angle):
    torch = torch_cuda
    g, img = motion256
    args = (g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"], g["nb"], g["bi"], g["nx"],
            g["ny"], g["nz"])
    d_img = dev(torch, img)
    d_proj = torch.empty((g["nb"], g["na"]), device="cuda")
    ctx.host_projection(d_proj, d_img, angle, *args)
    ctx.synchronize()
    mine = host(d_proj)
    r = ref.projection(img, angle, g)
    assert np.count_nonzero(mine != r) == 0, np.count_nonzero(mine != r)
    d_bp = torch.empty_like(d_img)
    ctx.host_backprojection(d_bp, d_proj, angle, *args)
    ctx.synchronize()
    np.testing.assert_array_equal(host(d_bp), ref.backprojection(mine, angle, g))


def test_warp_matches_the_reference_at_256x256x160(ctx, torch_cuda, ref, motion256):
    torch = torch_cuda
    g, img = motion256
    shape = img.shape
    F = [(_smooth_volume(shape, 40 + c) - np.float32(0.5)) * np.float32(4) for c in range(6)]
    out = torch.empty_like(dev(torch, img))
    ctx.host_deform(out, dev(torch, img), g["nx"], g["ny"], g["nz"], 0.7, -0.3,
                    *[dev(torch, f) for f in F])
    ctx.synchronize()
    np.testing.assert_array_equal(host(out), ref.deform(img, 0.7, -0.3, F))


@pytest.mark.parametrize("cfg", ["motion128", "motion256"])
def test_motion_loop_matches_the_reference_at_full_size(ctx, torch_cuda, cfg):
    """The whole host_AUMISART loop at the motion workloads' full sizes
    (256x256x160 at 1 mm with a 512x384 detector and 660 views, the
    benchmark's seeded problem; 128x128x96 at 2 mm with 256x192 and 360
    views): one outer iteration, an image pass and a DVF-update pass,
    against the reference's own loop rebuilt from its sources.  Volume,
    alpha_x and every residual projection agree bit for bit."""
    import bench
    from oracle import ref_runner
    p, proj, fields = bench.build_problem(ctx, torch_cuda, cfg)
    g, nv = p.geo, p.cfg.n_views
    proj_h = np.ascontiguousarray(proj.cpu().numpy())
    F = [np.ascontiguousarray(f.cpu().numpy()) for f in fields]
    del proj, fields
    img0 = np.ascontiguousarray(p.img0, np.float32)
    op = np.array([1, 0], np.int32)
    it = dict(n_iter=2, op_iter=op, n_views=nv, **{"lambda": p.cfg.lam}, outIter=1,
              volumes=p.volumes, flows=p.flows, angles=p.angles)
    out = dict(img=np.zeros_like(img0), resid=np.zeros((nv, g["nb"], g["na"]), np.float32),
               norm=np.zeros(2 * nv, np.float32), alpha_x=np.zeros_like(img0))
    ctx.host_AUMISART(out["img"], out["resid"], out["norm"], out["alpha_x"], img0, proj_h,
                      g["nx"], g["ny"], g["nz"], g["na"], g["nb"], 1, nv, 2, op, g["da"], g["db"],
                      g["ai"], g["bi"], g["SO"], g["SD"], 1.0, p.cfg.lam, p.volumes, p.flows,
                      np.zeros(nv, np.float32), p.angles, *F)
    r = ref_runner.aumisart(img0, proj_h, g, it, F)
    np.testing.assert_array_equal(out["img"], r["img"])
    np.testing.assert_array_equal(out["alpha_x"], r["alpha_x"])
    np.testing.assert_array_equal(out["resid"], r["resid"])


def test_static_loop_matches_the_reference_at_64_cubed(ctx, torch_cuda, ref):
    """host_AUMISART overload 1 at the static workload's size (64x64x64 at 2 mm,
    detector 128x96, 60 views, 5 image passes), the measured projections made
    by the reference's own projector: volume and residuals bit for bit the
    reference's loop; norms (cublasSnrm2 there) to 1e-6."""
    from mcsart_b200 import synthetic as S
    from oracle import ref_runner
    from conftest import rel_l2
    p = S.make_problem("static64", 0)
    g, nv = p.geo, p.cfg.n_views
    proj = ref.motion_projections(p.truth, None, p.volumes, p.flows, p.angles, g)
    op = np.ones(5, np.int32)
    it = dict(n_iter=5, op_iter=op, n_views=nv, **{"lambda": p.cfg.lam}, outIter=1,
              volumes=p.volumes, flows=p.flows, angles=p.angles)
    img0 = np.zeros_like(p.truth)
    out = dict(img=np.zeros_like(img0), resid=np.zeros((nv, g["nb"], g["na"]), np.float32),
               norm=np.zeros(5 * nv, np.float32), alpha_x=np.zeros_like(img0))
    ctx.host_AUMISART(out["img"], out["resid"], out["norm"], out["alpha_x"], img0, proj,
                      g["nx"], g["ny"], g["nz"], g["na"], g["nb"], 1, nv, 5, op, g["da"], g["db"],
                      g["ai"], g["bi"], g["SO"], g["SD"], 1.0, p.cfg.lam, p.volumes, p.flows,
                      np.zeros(nv, np.float32), p.angles)
    r = ref_runner.aumisart(img0, proj, g, it, None)
    np.testing.assert_array_equal(out["img"], r["img"])
    np.testing.assert_array_equal(out["resid"], r["resid"])
    assert rel_l2(out["norm"], r["norm"]) <= 1e-6
    # and the reconstruction converges: the last pass's residuals are smaller
    assert out["norm"][-nv:].mean() < 0.5 * out["norm"][:nv].mean()


@pytest.fixture(scope="module")
def clinical512():
    g = _geo("clinical512")
    return g, _smooth_volume((g["nz"], g["ny"], g["nx"]), 51)


@pytest.mark.parametrize("angle", [0.3, 0.7853982, 2.4])
def test_projection_and_backprojection_match_the_reference_at_512x512x256(ctx, torch_cuda, ref, clinical512,
                                                                      angle):
    """512x512x256 volume, 1024x768 detector: both driving axes and the
    45-degree switch, bit for bit the reference's kernels."""
    torch = torch_cuda
    g, img = clinical512
    d_img = dev(torch, img)
    d_proj = torch.empty((g["nb"], g["na"]), device="cuda")
    ctx.host_projection(d_proj, d_img, angle, *_args(g))
    ctx.synchronize()
    mine = host(d_proj)
    np.testing.assert_array_equal(mine, ref.projection(img, angle, g))
    d_bp = torch.empty_like(d_img)
    ctx.host_backprojection(d_bp, d_proj, angle, *_args(g))
    ctx.synchronize()
    np.testing.assert_array_equal(host(d_bp), ref.backprojection(mine, angle, g))
    del d_img, d_bp


def test_warp_matches_the_reference_at_512x512x256(ctx, torch_cuda, ref, clinical512):
    torch = torch_cuda
    g, img = clinical512
    shape = img.shape
    F = [(_smooth_volume(shape, 60 + c) - np.float32(0.5)) * np.float32(6) for c in range(6)]
    d_img = dev(torch, img)
    out = torch.empty_like(d_img)
    ctx.host_deform(out, d_img, g["nx"], g["ny"], g["nz"], -0.9, 0.4, *[dev(torch, f) for f in F])
    ctx.synchronize()
    np.testing.assert_array_equal(host(out), ref.deform(img, -0.9, 0.4, F))


def test_uneven_batch_matches_separate_runs(ctx, torch_cuda):
    """The 8 seeded problems of the uneven batch (96x96x64 .. 256x256x128,
    detectors 192x128 .. 512x384, 120 .. 660 views), one outer iteration
    (image pass in ordered subsets of 10 views, then the DVF pass) through
    mcsart_batch_run: image, fields and norms bitwise those of one
    mcsart_aumisart_device call per problem."""
    import bench
    import mcsart_b200 as m
    from mcsart_b200 import synthetic as S
    torch = torch_cuda
    op = np.array([1, 0], np.int32)
    opt = m.default_options(subset=S.BATCH_SUBSET)
    probs = []
    for i, cfg in enumerate(S.batch_configs()):
        p, proj, fields = bench.build_problem(ctx, torch, cfg, seed=40 + i)
        probs.append(dict(geo=p.geo, n_views=cfg.n_views, lambda_=p.cfg.lam, angles=p.angles,
                          volumes=p.volumes, flows=p.flows, proj=proj,
                          fields0=torch.stack(fields).contiguous()))
        del fields

    def inputs(q):
        g = q["geo"]
        return dict(geo=g, n_views=q["n_views"], lambda_=q["lambda_"], angles=q["angles"],
                    volumes=q["volumes"], flows=q["flows"], proj=q["proj"],
                    img=torch.zeros((g["nz"], g["ny"], g["nx"]), device="cuda"),
                    fields=q["fields0"].clone(), norm=torch.zeros(2 * q["n_views"], device="cuda"))

    alone = []
    for q in probs:
        d = inputs(q)
        ctx.aumisart_device(n_iter=2, op_iter=op, options=opt, **d)
        ctx.synchronize()
        alone.append({k: host(d[k]) for k in ("img", "fields", "norm")})
        del d
    batch = [inputs(q) for q in probs]
    ctx.batch_run(batch, n_iter=2, op_iter=op, options=opt)
    ctx.synchronize()
    for i, d in enumerate(batch):
        for k, v in alone[i].items():
            np.testing.assert_array_equal(host(d[k]), v, err_msg=f"problem {i} {k}")
        assert np.isfinite(alone[i]["img"]).all()


def test_central_rays_count_slabs_at_512x512x256(ctx, torch_cuda):
    torch = torch_cuda
    g = _geo("clinical512")
    ones = torch.ones((g["nz"], g["ny"], g["nx"]), device="cuda")
    d_proj = torch.empty((g["nb"], g["na"]), device="cuda")
    ctx.host_projection(d_proj, ones, 0.0, g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"],
                        g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
    ctx.synchronize()
    p = host(d_proj)
    # at angle 0 the rays through the detector centre run along x inside the
    # volume over all nx slabs
    c = p[g["nb"] // 2 - 8: g["nb"] // 2 + 8, g["na"] // 2 - 8: g["na"] // 2 + 8]
    np.testing.assert_allclose(c, float(g["nx"]), rtol=1e-4)
    assert np.isfinite(p).all() and p.min() >= 0.0
