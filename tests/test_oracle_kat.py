"""Known-answer tests of the CPU oracle derived from the kernel mathematics, and
the FP32 OpenMP transcription (the timed CPU baseline) against the FP64 oracle."""
import numpy as np
import pytest

from conftest import fields, geo, rel_l2, volume


def test_projection_of_ones_equals_number_of_slabs(oracle):
    """Each slab's normalised overlap weights sum to 1 inside the volume
    (src/cu_projection.cu:83,86), so a central ray through a ones-volume
    sums to the number of slabs along the driving axis."""
    g = geo(nx=32, ny=32, nz=32, na=64, nb=48, SO=200, SD=300, da=0.8, db=0.8)
    ones = np.ones((32, 32, 32))
    for angle in (0.0, np.pi / 2, np.pi, 0.3):
        p = oracle.projection(ones, angle, g)
        np.testing.assert_allclose(p[23:25, 31:33], 32.0, rtol=1e-12)


def test_projection_is_linear(oracle):
    g = geo()
    a = volume((16, 20, 24), 1).astype(np.float64)
    b = volume((16, 20, 24), 2).astype(np.float64)
    pa, pb = oracle.projection(a, 0.8, g), oracle.projection(b, 0.8, g)
    np.testing.assert_allclose(oracle.projection(2.5 * a - b, 0.8, g), 2.5 * pa - pb,
                               rtol=1e-10, atol=1e-10)


def test_backprojection_of_ones_is_the_footprint_area(oracle):
    """Unnormalised weights: BP of a ones-projection is the area of the voxel's
    detector bounding box (src/cu_backprojection.cu:150-168) for voxels whose
    box lies inside the detector."""
    g = geo(nx=16, ny=16, nz=16, na=96, nb=96, SO=200, SD=300, da=0.5, db=0.5)
    bp = oracle.backprojection(np.ones((96, 96)), 0.0, g)
    # central voxel, rotated frame at angle 0: x in [-0.5, 0.5] around xc
    xc = yc = zc = 0.5
    mag = lambda x: g["SD"] / (x + g["SO"])
    a = [mag(xc + dx) * (yc + dy) for dx in (-0.5, 0.5) for dy in (-0.5, 0.5)] + [mag(xc) * yc]
    b = [mag(xc - 0.5) * zc, mag(xc + 0.5) * zc, mag(xc) * (zc + 0.5), mag(xc) * (zc - 0.5)]
    area = (max(a) - min(a)) / g["da"] * (max(b) - min(b)) / g["db"]
    assert abs(bp[8, 8, 8] - area) <= 1e-9 * area


def test_warp_with_zero_field_is_identity_on_square_slices(oracle):
    img = volume((10, 12, 12), 4)
    z = [np.zeros_like(img)] * 6
    for mode in (oracle.TEX_EXACT, oracle.TEX_Q8_NEAREST):
        np.testing.assert_array_equal(oracle.deform(img, 1.7, -0.2, z, tex_mode=mode), img)


def test_warp_integer_shift_is_exact_with_edge_clamp(oracle):
    img = volume((8, 12, 12), 5)
    f = [np.zeros_like(img) for _ in range(6)]
    f[1][:] = 1.0  # alpha_y displaces along the memory x axis (in-slice transpose)
    out = oracle.deform(img, 2.0, 0.0, f, tex_mode=oracle.TEX_EXACT)
    np.testing.assert_array_equal(out[:, :, :-2], img[:, :, 2:])
    np.testing.assert_array_equal(out[:, :, -2:], np.repeat(img[:, :, -1:], 2, axis=2))


def test_division_zeroes_nan_and_inf(oracle):
    a = np.array([[[1.0, 0.0, -2.0, 5.0]]])
    b = np.array([[[0.0, 0.0, 4.0, np.inf]]])
    np.testing.assert_array_equal(oracle.division(a, b), [[[0.0, 0.0, -0.5, 0.0]]])


def test_backward_difference_is_zero_on_both_faces(oracle):
    img = volume((5, 6, 7), 6)
    for ind, ax in ((1, 2), (2, 1), (3, 0)):
        d = oracle.diff(img, ind)
        sl = [slice(None)] * 3
        sl[ax] = 0
        assert np.all(d[tuple(sl)] == 0)
        sl[ax] = -1
        assert np.all(d[tuple(sl)] == 0)
        sl[ax] = slice(1, -1)
        ref = np.diff(img.astype(np.float64), axis=ax)
        rs = [slice(None)] * 3
        rs[ax] = slice(0, -1)
        np.testing.assert_allclose(d[tuple(sl)], ref[tuple(rs)], rtol=1e-12)


def test_fp32_port_matches_fp64_oracle_per_kernel(oracle):
    g = geo()
    img = volume((16, 20, 24), 7)
    for a in (0.1, 1.0, 2.4, 4.0):
        p64 = oracle.projection(img, a, g)
        assert rel_l2(oracle.projection(img, a, g, prec="cpu"), p64) <= 1e-5
        b64 = oracle.backprojection(p64, a, g)
        assert rel_l2(oracle.backprojection(p64, a, g, prec="cpu"), b64) <= 1e-5
    F = fields((12, 20, 20), 8)
    sq = volume((12, 20, 20), 9)
    d64 = oracle.deform(sq, 0.9, -0.3, F, tex_mode=oracle.TEX_EXACT)
    d32 = oracle.deform(sq, 0.9, -0.3, F, tex_mode=oracle.TEX_EXACT, prec="cpu")
    assert rel_l2(d32, d64) <= 1e-5


def test_static_loop_fp32_port_tracks_fp64(oracle):
    g = geo(nx=16, ny=16, nz=12, na=32, nb=24, SO=60, SD=90, da=0.9, db=0.9)
    truth = volume((12, 16, 16), 10)
    angles = np.linspace(0, 2 * np.pi, 10, endpoint=False).astype(np.float32)
    proj = np.stack([oracle.projection(truth, a, g) for a in angles]).astype(np.float32)
    it = dict(n_iter=3, op_iter=np.ones(3, np.int32), n_views=10, outIter=1,
              volumes=np.zeros(10, np.float32), flows=np.zeros(10, np.float32), angles=angles,
              **{"lambda": 1.0})
    o64 = oracle.aumisart(np.zeros_like(truth), proj, g, it, None)
    o32 = oracle.aumisart(np.zeros_like(truth), proj, g, it, None, prec="cpu")
    assert rel_l2(o32["img"], o64["img"]) <= 1e-5
    assert o64["norm"][-10:].mean() < o64["norm"][:10].mean()


def test_oracle_adjoint_is_the_transpose_of_the_oracle_projection(oracle):
    """<A x, y> = <x, A^T y> for the FP64 oracle's projector and its adjoint."""
    import numpy as np
    from conftest import geo
    g = geo(nx=20, ny=18, nz=12, na=30, nb=20)
    rng = np.random.default_rng(5)
    x = rng.random((g["nz"], g["ny"], g["nx"]))
    y = rng.random((g["nb"], g["na"]))
    for a in (0.0, 0.5, 0.7853982, 2.2, 3.9, 5.6):
        ax = oracle.projection(x, a, g)
        aty = oracle.backprojection_adjoint(y, a, g)
        lhs, rhs = float(np.sum(ax * y)), float(np.sum(x * aty))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (a, lhs, rhs)
