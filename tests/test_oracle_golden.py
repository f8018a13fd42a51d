"""The CPU oracle against golden outputs of the reference itself.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which ran
bill52547/McSART's own CUDA kernels and host_AUMISART (rebuilt unmodified from
their sources, oracle/Makefile) on a B200.  These tests pin the FP64
restatement in oracle/ to the reference: every kernel to FP32-rounding level,
the static SART loop to 1e-6.  (The warp's pin depends on the texture-filter
model, see test_oracle_pins_texture_warp.)
"""
import os

import numpy as np
import pytest

from conftest import ANGLES, GOLDEN, load_geo, rel_l2

KER = os.path.join(GOLDEN, "ref_kernels.npz")
AUM = os.path.join(GOLDEN, "ref_aumisart.npz")


@pytest.fixture(scope="module")
def z():
    with np.load(KER) as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope="module")
def za():
    with np.load(AUM) as f:
        return {k: f[k] for k in f.files}


def _zgeo(z, prefix):
    class _Z(dict):
        files = property(lambda self: list(self.keys()))
    return load_geo(_Z(z), prefix)


@pytest.mark.parametrize("gi", [0, 1, 2])
def test_oracle_projection_matches_reference(oracle, z, gi):
    g = _zgeo(z, f"g{gi}_geo_")
    img = z[f"g{gi}_img"]
    for ai, a in enumerate(ANGLES):
        assert rel_l2(oracle.projection(img, a, g), z[f"g{gi}_a{ai}_fp"]) <= 1e-6


@pytest.mark.parametrize("gi", [0, 1, 2])
def test_oracle_backprojection_matches_reference(oracle, z, gi):
    """The reference takes __sinf/__cosf of the angle, the oracle exact values."""
    g = _zgeo(z, f"g{gi}_geo_")
    for ai, a in enumerate(ANGLES):
        r = z[f"g{gi}_a{ai}_bp"]
        assert rel_l2(oracle.backprojection(z[f"g{gi}_a{ai}_bpin"], a, g), r) <= 1e-5


@pytest.mark.parametrize("si", [0, 1, 2])
def test_oracle_first_order_warp_and_dvf_match_reference(oracle, z, si):
    img = z[f"s{si}_img"]
    F = list(z[f"s{si}_fields"])
    for vi, (vol, flow) in enumerate([(1.3, -0.4), (-2.7, 0.9)]):
        vol, flow = np.float32(vol), np.float32(flow)
        # the reference reads past the volume for the last slice's +nx neighbours
        d2 = oracle.deform2(img, vol, flow, F)
        assert rel_l2(d2[:-1], z[f"s{si}_v{vi}_deform2"][:-1]) <= 1e-6
        m = np.stack(oracle.forward_dvf(F, vol, flow))
        assert rel_l2(m, z[f"s{si}_v{vi}_fdvf"]) <= 1e-6


def test_oracle_elementwise_match_reference(oracle, z):
    a, b, c = z["e_a"], z["e_b"], z["e_c"]
    F = list(z["e_fields"])
    assert rel_l2(oracle.add(a, b, -0.7), z["e_add"]) <= 1e-6
    for ind in (1, 2, 3):
        assert rel_l2(oracle.add2(a, b, c, 0.6, ind), z[f"e_add2_{ind}"]) <= 1e-6
        assert rel_l2(oracle.multiple(a, c, 1.4, ind), z[f"e_multiple_{ind}"]) <= 1e-6
        assert rel_l2(oracle.diff(b, ind), z[f"e_diff_{ind}"]) <= 1e-6
    assert rel_l2(oracle.initial2(c, -0.4, 1.9), z["e_initial2"]) <= 1e-6
    d = oracle.division(a, b)
    assert rel_l2(d, z["e_division"]) <= 1e-6
    assert np.all(z["e_division"][0, 0, :5] == 0) and np.all(d[0, 0, :5] == 0)
    assert rel_l2(np.stack(oracle.update_udvf(F, b, c, 0.9, -0.5)), z["e_udvf"]) <= 1e-6


def _it(za, name):
    op = za[f"{name}_op_iter"]
    return dict(n_iter=len(op), op_iter=op, n_views=len(za["angles"]), outIter=1,
                volumes=za["volumes"], flows=za["flows"], angles=za["angles"],
                **{"lambda": 1.0})


def test_oracle_static_sart_loop_matches_reference(oracle, za):
    """host_AUMISART overload 1: static image passes (+ DVF passes whose fields
    never feed back into the image)."""
    g = _zgeo(za, "geo_")
    o = oracle.aumisart(np.zeros_like(za["truth"]), za["proj"], g, _it(za, "o1"), None)
    assert rel_l2(o["img"], za["o1_img"]) <= 1e-5
    assert rel_l2(o["norm"], za["o1_norm"]) <= 1e-5
    assert rel_l2(o["resid"], za["o1_resid"]) <= 1e-4


def test_golden_shows_the_dvf_update_is_ill_conditioned(za):
    """The reference's own DVF pass divides by BP(FP(initial2)), a signed image
    that crosses zero (AUMISART.cu:267-270): its DVF leaves the physical range.
    This is why parity after motion passes needs bitwise-identical arithmetic."""
    assert np.abs(za["o2_alpha_x"]).max() > 10 * np.abs(za["fields"][0]).max()
