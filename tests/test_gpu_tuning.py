"""The launch-shape autotuner (mcsart_autotune) and its per-geometry cache.

Every candidate shape computes every ray and voxel with the same operations
in the same order, so whatever the tuner picks, the reconstruction is the
same bits: checked here for every variant of every kernel class, against the
untuned run (whose own parity with the reference the other tests check).
"""
import numpy as np
import pytest

from conftest import dev, host
from test_gpu_sart import make_case

pytestmark = pytest.mark.gpu

N_VARIANTS = (5, 4, 4, 3, 3)  # fp1, fp3, bp, warp, fup


def _run(ctx, torch, case, opt):
    g, it, img0, proj, F = case
    d = dict(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
             volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0), proj=dev(torch, proj),
             fields=dev(torch, np.stack(F)), norm=torch.zeros(it["n_iter"] * it["n_views"],
                                                              device="cuda"))
    ctx.aumisart_device(n_iter=it["n_iter"], op_iter=it["op_iter"], options=opt, **d)
    ctx.synchronize()
    return {k: host(d[k]) for k in ("img", "fields", "norm")}


def _problem(torch, case):
    g, it, img0, proj, F = case
    return dict(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0),
                proj=dev(torch, proj), fields=dev(torch, np.stack(F)))


def test_autotune_caches_shapes_and_keeps_the_bits(ctx, torch_cuda, oracle, tmp_path):
    import mcsart_b200 as m
    torch = torch_cuda
    case = make_case(oracle, motion=True, op_iter=(1, 0, 1), seed=21, nx=24, ny=24, nz=16,
                     na=40, nb=32)
    g = case[0]
    base = _run(ctx, torch, case, m.default_options())
    prob = _problem(torch, case)
    img_before = host(prob["img"])
    shapes = ctx.autotune(**prob)
    # the problem's own buffers are left as they were
    np.testing.assert_array_equal(host(prob["img"]), img_before)
    assert shapes is not None and len(shapes) == 5
    for s, n in zip(shapes, N_VARIANTS):
        assert -1 <= s < n
    tuned = _run(ctx, torch, case, m.default_options())
    for k in base:
        np.testing.assert_array_equal(tuned[k], base[k], err_msg=k)
    # the cache survives a save / load round trip into a fresh context
    path = tmp_path / "tuning.txt"
    ctx.tuning_save(path)
    with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c2:
        assert c2.tuning_get(g) is None
        assert c2.tuning_load(path) >= 1
        assert c2.tuning_get(g) == shapes


def test_every_launch_shape_gives_the_same_bits(ctx, torch_cuda, oracle, tmp_path):
    """Force each variant of each kernel class through the cache file and
    compare the whole loop (image and DVF passes) with the built-in shapes."""
    import mcsart_b200 as m
    torch = torch_cuda
    case = make_case(oracle, motion=True, op_iter=(1, 0, 1), seed=22, nx=32, ny=32, nz=20,
                     na=48, nb=40)
    g = case[0]
    with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
        base = _run(c, torch, case, m.default_options())
        c.autotune(**_problem(torch, case))
        path = tmp_path / "t.txt"
        c.tuning_save(path)
        lines = [ln for ln in open(path).read().splitlines() if not ln.startswith("#")]
        key = [ln.split()[0] for ln in lines if ln.split()[0].startswith("32x32x20/")][0]
    combos = set()
    for cls, n in enumerate(N_VARIANTS):  # each variant of each class at least once
        for v in range(n):
            shape = [-1, -1, -1, -1, -1]
            shape[cls] = v
            combos.add(tuple(shape))
    combos |= {tuple(v % n for n in N_VARIANTS) for v in range(5)}
    for shape in sorted(combos):
        p = tmp_path / "forced.txt"
        p.write_text(f"{key} {' '.join(map(str, shape))}\n")
        with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
            assert c.tuning_load(p) == 1
            assert c.tuning_get(g) == list(shape)
            got = _run(c, torch, case, m.default_options())
        for k in base:
            np.testing.assert_array_equal(got[k], base[k], err_msg=f"{shape} {k}")


def test_autotune_option_tunes_on_first_run(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    torch = torch_cuda
    case = make_case(oracle, motion=True, op_iter=(1, 0), seed=23, nx=20, ny=20, nz=12,
                     na=36, nb=28)
    with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
        assert c.tuning_get(case[0]) is None
        a = _run(c, torch, case, m.default_options(autotune=1))
        assert c.tuning_get(case[0]) is not None
    b = _run(ctx, torch, case, m.default_options())
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_malformed_tuning_file_is_rejected(ctx, tmp_path):
    import mcsart_b200 as m
    p = tmp_path / "bad.txt"
    p.write_text("somekey 9 0 0 0 0\n")
    with pytest.raises(m.McsartError):
        ctx.tuning_load(p)


@pytest.mark.parametrize("storage", [1, 2])
def test_fused_and_separate_dvf_field_updates_agree_with_16bit_storage(ctx, torch_cuda, oracle,
                                                                       tmp_path, storage):
    """The DVF pass's field update with the backprojection computed inside it
    (variant 0, the built-in choice) and after a separate backprojector launch
    (variants 1 and 2) give the same bits with BF16 and FP16 fields and
    projections too (the ratio is computed from the FP32 pairs either way)."""
    import mcsart_b200 as m
    torch = torch_cuda
    dt = torch.bfloat16 if storage == m.BF16 else torch.float16
    g, it, img0, proj, F = make_case(oracle, motion=True, op_iter=(1, 0, 1), seed=24, nx=32,
                                     ny=32, nz=20, na=48, nb=40)
    opt = m.default_options(storage=storage)

    def run(c):
        d_img = dev(torch, img0)
        d_F = dev(torch, np.stack(F)).to(dt)
        c.aumisart_device(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                          volumes=it["volumes"], flows=it["flows"], img=d_img,
                          proj=dev(torch, proj).to(dt), fields=d_F, n_iter=it["n_iter"],
                          op_iter=it["op_iter"], options=opt)
        c.synchronize()
        return host(d_img), host(d_F.float())

    with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
        c.autotune(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                   volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0),
                   proj=dev(torch, proj).to(dt), fields=dev(torch, np.stack(F)).to(dt),
                   options=opt)
        path = tmp_path / "t.txt"
        c.tuning_save(path)
        key = [ln.split()[0] for ln in open(path).read().splitlines()
               if not ln.startswith("#") and ln.split()[0].endswith(f"/s{storage}")][0]
    results = []
    for fup in (0, 1, 2):
        p = tmp_path / f"forced{fup}.txt"
        p.write_text(f"{key} -1 -1 -1 -1 {fup}\n")
        with m.Context(0, stream=torch.cuda.current_stream().cuda_stream) as c:
            assert c.tuning_load(p) == 1
            assert c.tuning_get(g, storage)[4] == fup
            results.append(run(c))
    for r in results[1:]:
        np.testing.assert_array_equal(r[0], results[0][0])
        np.testing.assert_array_equal(r[1], results[0][1])
