"""mcsart_backprojection_adjoint: the exact transpose of mcsart_projection.

Checked against the FP64 oracle's adjoint (which scatters each ray's terms of
the oracle projector) and by the dot-product identity with the engine's own
projector, at angles that exercise both driving axes and the 45-degree switch,
on square and non-square volumes with detector offsets."""
import numpy as np
import pytest

from conftest import ANGLES, dev, geo, host, rel_l2, volume

pytestmark = pytest.mark.gpu

GEOS = [geo(), geo(nx=20, ny=20, nz=12, na=36, nb=24, ai=1.5, bi=-2.0),
        geo(nx=33, ny=17, nz=9, na=45, nb=15, da=1.1, db=1.3, SO=70, SD=100)]


def _args(g):
    return (g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"], g["nb"], g["bi"], g["nx"],
            g["ny"], g["nz"])


def _adj(ctx, torch, proj, a, g):
    out = torch.full((g["nz"], g["ny"], g["nx"]), 7.0, device="cuda")
    ctx.host_backprojection_adjoint(out, dev(torch, proj), a, *_args(g))
    ctx.synchronize()
    return host(out)


def _fp(ctx, torch, img, a, g):
    out = torch.zeros((g["nb"], g["na"]), device="cuda")
    ctx.host_projection(out, dev(torch, img), a, *_args(g))
    ctx.synchronize()
    return host(out)


@pytest.mark.parametrize("gi", range(len(GEOS)))
def test_adjoint_matches_the_fp64_oracle(ctx, torch_cuda, oracle, gi):
    g = GEOS[gi]
    rng = np.random.default_rng(gi)
    p = rng.random((g["nb"], g["na"]), dtype=np.float32)
    for a in ANGLES:
        mine = _adj(ctx, torch_cuda, p, a, g)
        o = oracle.backprojection_adjoint(p, a, g)
        assert rel_l2(mine, o) <= 1e-5, (a, rel_l2(mine, o))


@pytest.mark.parametrize("gi", range(len(GEOS)))
def test_dot_product_identity_with_the_engine_projector(ctx, torch_cuda, gi):
    g = GEOS[gi]
    rng = np.random.default_rng(10 + gi)
    x = volume((g["nz"], g["ny"], g["nx"]), seed=gi)
    y = rng.random((g["nb"], g["na"]), dtype=np.float32)
    for a in ANGLES:
        lhs = float(np.sum(_fp(ctx, torch_cuda, x, a, g).astype(np.float64) * y))
        rhs = float(np.sum(x.astype(np.float64) * _adj(ctx, torch_cuda, y, a, g)))
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (a, lhs, rhs)


def test_adjoint_is_deterministic_and_overwrites(ctx, torch_cuda):
    g = GEOS[0]
    p = np.random.default_rng(3).random((g["nb"], g["na"]), dtype=np.float32)
    a = _adj(ctx, torch_cuda, p, 0.7853, g)
    b = _adj(ctx, torch_cuda, p, 0.7853, g)
    np.testing.assert_array_equal(a, b)
    assert np.isfinite(a).all() and a.min() >= 0.0
