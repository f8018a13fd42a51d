"""mcsart_batch_run: independent reconstructions of different sizes run
concurrently, each on its own lane, with results bitwise those of separate
mcsart_aumisart_device calls."""
import numpy as np
import pytest

from conftest import dev, host
from test_gpu_sart import make_case

pytestmark = pytest.mark.gpu


def _inputs(torch, case, seed):
    g, it, img0, proj, F = case
    d = dict(geo=g, n_views=it["n_views"], lambda_=1.0, angles=it["angles"],
             volumes=it["volumes"], flows=it["flows"], img=dev(torch, img0), proj=dev(torch, proj),
             norm=torch.zeros(3 * it["n_views"], device="cuda"),
             resid=torch.zeros((it["n_views"], g["nb"], g["na"]), device="cuda"))
    if F is not None:
        d["fields"] = dev(torch, np.stack(F))
    return d


def _snapshot(d):
    out = {k: host(d[k]) for k in ("img", "norm", "resid")}
    if "fields" in d:
        out["fields"] = host(d["fields"])
    return out


def test_batch_matches_separate_runs(ctx, torch_cuda, oracle):
    import mcsart_b200 as m
    torch = torch_cuda
    op = np.array([1, 0, 1], np.int32)
    cases = [make_case(oracle, motion=True, op_iter=tuple(op), seed=1),
             make_case(oracle, motion=True, nx=20, ny=16, nz=12, op_iter=tuple(op), seed=2),
             make_case(oracle, motion=False, nx=24, ny=20, nz=16, na=40, nb=28,
                       op_iter=tuple(op), seed=3)]
    opt = m.default_options()
    alone = []
    for i, c in enumerate(cases):
        d = _inputs(torch, c, i)
        ctx.aumisart_device(n_iter=len(op), op_iter=op, options=opt, **d)
        ctx.synchronize()
        alone.append(_snapshot(d))
    for repeat in range(2):  # the second batch reuses the lanes and their graphs
        batch = [_inputs(torch, c, i) for i, c in enumerate(cases)]
        ctx.batch_run(batch, n_iter=len(op), op_iter=op, options=opt)
        ctx.synchronize()
        for i, d in enumerate(batch):
            got = _snapshot(d)
            for k, v in alone[i].items():
                np.testing.assert_array_equal(got[k], v, err_msg=f"problem {i} {k} batch {repeat}")


def test_batch_rejects_bad_counts(ctx, torch_cuda):
    from mcsart_b200 import _lib
    L = _lib.load()
    assert L.mcsart_batch_run(ctx._h, None, 1, 1, None, None) == _lib.ERR_INVALID_ARGUMENT
    assert b"problems is NULL" in L.mcsart_last_error()
