"""mcsart_projection_noalloc: the projector with its scratch in a fixed device
array (no allocation, no context), against mcsart_projection.

The file name sorts last so that the GPU test also runs after every other test
of a session, with the library's other modules already loaded.
"""
import numpy as np
import pytest

from conftest import geo, volume

GEO_ARGS = ("SO", "SD", "da", "na", "ai", "db", "nb", "bi", "nx", "ny", "nz")
MAX_VOXELS = 4194304  # MCSART_NOALLOC_MAX_VOXELS


def _args(g):
    return [g[k] for k in GEO_ARGS]


def test_oversize_volume_is_rejected_before_any_device_work():
    """The size check precedes every CUDA call, so it holds without a GPU."""
    from mcsart_b200 import _lib
    L = _lib.load()
    g = geo(nx=257, ny=256, nz=64, na=64, nb=48)
    assert g["nx"] * g["ny"] * g["nz"] > MAX_VOXELS
    rc = L.mcsart_projection_noalloc(None, 16, 16, 0.3, *_args(g))
    assert rc == _lib.ERR_INVALID_ARGUMENT
    msg = L.mcsart_last_error().decode()
    assert "static scratch" in msg and str(MAX_VOXELS) in msg


@pytest.mark.gpu
def test_noalloc_matches_mcsart_projection_on_calls_in_a_row(ctx, torch_cuda):
    import mcsart_b200 as m
    torch = torch_cuda
    g = geo(nx=40, ny=36, nz=24, na=64, nb=40, SO=80.0, SD=120.0, da=1.0, db=1.0)
    shape = (g["nz"], g["ny"], g["nx"])
    imgs = [torch.as_tensor(volume(shape, seed=s)).cuda() for s in (21, 22)]
    stream = torch.cuda.current_stream()

    def expected(img, angle):
        out = torch.empty((g["nb"], g["na"]), device="cuda")
        ctx.host_projection(out, img, angle, *_args(g))
        ctx.synchronize()
        return out.cpu().numpy()

    # 0.3 rad: x-driven rays, the scratch copy is used; 1.5 rad: y-driven only.
    # The two x-driven calls in a row project different volumes, so a stale
    # scratch copy would show.
    calls = [(imgs[0], 0.3), (imgs[1], 0.3), (imgs[1], 1.5), (imgs[0], 2.9)]
    outs = [torch.full((g["nb"], g["na"]), float("nan"), device="cuda") for _ in calls]
    for (img, a), o in zip(calls[:1], outs[:1]):  # first call: the per-device set-up
        m.projection_noalloc(o, img, a, *_args(g), stream=stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for (img, a), o in zip(calls[1:], outs[1:]):
        m.projection_noalloc(o, img, a, *_args(g), stream=stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "device memory changed during the calls"
    for (img, a), o in zip(calls, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), expected(img, a))

    # and the same two calls again, back to back, after the others
    again = [torch.empty_like(outs[0]) for _ in range(2)]
    for (img, a), o in zip(calls[:2], again):
        m.projection_noalloc(o, img, a, *_args(g), stream=stream)
    torch.cuda.synchronize()
    for k in range(2):
        np.testing.assert_array_equal(again[k].cpu().numpy(), outs[k].cpu().numpy())


@pytest.mark.gpu
def test_noalloc_on_the_legacy_default_stream(torch_cuda):
    import mcsart_b200 as m
    torch = torch_cuda
    g = geo(nx=24, ny=20, nz=16, na=40, nb=28)
    img = torch.as_tensor(volume((g["nz"], g["ny"], g["nx"]), seed=3)).cuda()
    torch.cuda.synchronize()
    out = torch.empty((g["nb"], g["na"]), device="cuda")
    m.projection_noalloc(out, img, 0.7, *_args(g), stream=None)
    ctx = m.Context(0)
    try:
        ref = torch.empty_like(out)
        ctx.host_projection(ref, img, 0.7, *_args(g))
        ctx.synchronize()
    finally:
        ctx.close()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())


def test_depth_beyond_the_grid_limit_is_rejected_before_any_device_work():
    """A volume within the voxel limit whose depth exceeds the 65535 slices a
    launch grid can index is refused with a message, without device work."""
    from mcsart_b200 import _lib
    L = _lib.load()
    g = geo(nx=1, ny=1, nz=100000, na=8, nb=8)
    assert g["nx"] * g["ny"] * g["nz"] <= MAX_VOXELS
    rc = L.mcsart_projection_noalloc(None, 16, 16, 0.3, *_args(g))
    assert rc == _lib.ERR_INVALID_ARGUMENT
    assert "nz must be at most 65535" in L.mcsart_last_error().decode()
