"""Ordered subsets (options.subset = k): the k views of a subset compute the
reference's corrections from the same image in one projector and one
backprojector launch, and the image receives lambda/k times their sum.  k = 1
is the reference's loop (bitwise, covered by the parity tests); k > 1 is a
different algorithm, checked against the FP64 oracle running the same one."""
import numpy as np
import pytest

from conftest import dev, host, rel_l2
from test_gpu_sart import make_case

pytestmark = pytest.mark.gpu


def _run(ctx, torch, case, opt, op):
    g, it, img0, proj, F = case
    d_img = dev(torch, img0)
    d_F = dev(torch, np.stack(F)) if F is not None else None
    norm = torch.zeros(len(op) * it["n_views"], device="cuda")
    ctx.aumisart_device(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
                        volumes=it["volumes"], flows=it["flows"], img=d_img, proj=dev(torch, proj),
                        fields=d_F, norm=norm, n_iter=len(op), op_iter=np.array(op, np.int32),
                        options=opt)
    ctx.synchronize()
    return host(d_img), host(norm)


@pytest.mark.parametrize("k", [4, 5])
def test_static_subsets_match_the_fp64_oracle(ctx, torch_cuda, oracle, k):
    import mcsart_b200 as m
    op = (1, 1, 1)
    case = make_case(oracle, motion=False, op_iter=op, seed=8)
    g, it, img0, proj, F = case
    img, norm = _run(ctx, torch_cuda, case, m.default_options(subset=k), op)
    o = oracle.aumisart(img0, proj, g, it, None, subset=k)
    err = rel_l2(img, o["img"])
    print(f"static subset {k}: rel L2 vs FP64 oracle {err:.2e}")
    assert err <= 1e-4, err
    assert rel_l2(norm, o["norm"]) <= 1e-4


@pytest.mark.parametrize("k", [4, 5])
def test_motion_subsets_match_the_fp64_oracle(ctx, torch_cuda, oracle, k):
    """Image passes with a fixed DVF, exact trilinear warps (the oracle's
    TEX_EXACT); 12 views in subsets of 4 or of 5, 5 and 2."""
    import mcsart_b200 as m
    op = (1, 1, 1)
    case = make_case(oracle, motion=True, op_iter=op, seed=9)
    g, it, img0, proj, F = case
    opt = m.default_options(subset=k, interp=m.INTERP_EXACT)
    img, norm = _run(ctx, torch_cuda, case, opt, op)
    o = oracle.aumisart(img0, proj, g, it, F, tex_mode=oracle.TEX_EXACT, subset=k)
    err = rel_l2(img, o["img"])
    print(f"motion subset {k}: rel L2 vs FP64 oracle {err:.2e}")
    assert err <= 2e-5, err


def test_subsets_reduce_the_residual(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    op = (1, 1, 1, 1, 1)
    case = make_case(oracle, motion=False, op_iter=op, seed=10)
    _, it, _, _, _ = case
    _, norm = _run(ctx, torch_cuda, case, m.default_options(subset=4), op)
    nv = it["n_views"]
    assert norm[-nv:].mean() < 0.5 * norm[:nv].mean()


def test_subset_with_texture_warps_runs_and_is_deterministic(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    op = (1, 0, 1)
    case = make_case(oracle, motion=True, op_iter=op, seed=11)
    a, _ = _run(ctx, torch_cuda, case, m.default_options(subset=4), op)
    b, _ = _run(ctx, torch_cuda, case, m.default_options(subset=4, use_graph=0), op)
    np.testing.assert_array_equal(a, b)
    assert np.isfinite(a).all()


def test_subset_options_are_validated(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    case = make_case(oracle, motion=False, op_iter=(1,), seed=12)
    for bad in (dict(subset=17), dict(subset=4, fp_sum=2)):
        with pytest.raises(m.McsartError):
            _run(ctx, torch_cuda, case, m.default_options(**bad), (1,))
