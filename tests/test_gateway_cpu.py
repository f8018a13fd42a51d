"""Host logic: the gateways' struct parsing (aliases, defaults, offset shift,
error messages of src/entry_AUMISART.cu:18-160) and the synthetic workloads."""
import numpy as np
import pytest

from mcsart_b200 import gateway as G
from mcsart_b200 import synthetic as S


def base_geo():
    return dict(nx=64, ny=64, nz=32, na=128, nb=96, SO=500.0, SD=750.0, da=0.8, db=0.8)


def test_geo_defaults_and_shift():
    g = G.parse_geo_para(dict(nx=8, ny=9, nz=10, na=20, nb=12, SO=100.0, SD=150.0))
    assert (g["da"], g["db"], g["dx"]) == (1.0, 1.0, 1.0)
    assert g["ai"] == -(20 / 2 - 0.5) and g["bi"] == -(12 / 2 - 0.5)


def test_geo_offsets_are_shifted():
    g = G.parse_geo_para(dict(base_geo(), ai=2.0, bi=-1.0))
    assert g["ai"] == pytest.approx(2.0 - 63.5) and g["bi"] == pytest.approx(-1.0 - 47.5)


def test_geo_aliases():
    g = G.parse_geo_para(dict(nx=4, ny=4, nz=4, nv=10, nu=6, SI=300.0, DI=200.0))
    assert (g["na"], g["nb"]) == (10, 6)
    assert g["SO"] == 300.0 and g["SD"] == 500.0  # SD = DI + SO
    g2 = G.parse_geo_para(dict(nx=4, ny=4, nz=4, na=7, nv=10, nb=5, nu=6, SO=1.0, SD=2.0))
    assert (g2["na"], g2["nb"]) == (7, 5)  # na/nb take precedence


@pytest.mark.parametrize("missing,msg", [("nx", "volume resolution nx"),
                                         ("na", "number of detector in plane"),
                                         ("SO", "source and isocenter"),
                                         ("SD", "source and detector plane")])
def test_geo_missing_fields_raise(missing, msg):
    g = base_geo()
    del g[missing]
    with pytest.raises(G.BadInput, match=msg):
        G.parse_geo_para(g)


def test_backprojection_needs_angle():
    with pytest.raises(G.BadInput, match="projection angle"):
        G.parse_geo_para(base_geo(), need_angle=True)
    assert G.parse_geo_para(dict(base_geo(), angle=0.5), need_angle=True)["angle"] == \
        pytest.approx(0.5)


def iter_para(**kw):
    d = dict(n_iter=2, op_iter=np.array([1, 0], np.int32), n_views=4, outIter=1,
             volumes=np.zeros(4), flows=np.zeros(4), err_weights=np.zeros(4),
             angles=np.linspace(0, 6, 4), **{"lambda": 1.0})
    d.update(kw)
    return d


def test_iter_para_parsing_and_overload_selection():
    it = G.parse_iter_para(iter_para())
    assert it["fields"] is None and it["op_iter"].dtype == np.int32
    f = [np.zeros((2, 2, 2))] * 6
    it2 = G.parse_iter_para(iter_para(alpha_x=f[0], alpha_y=f[1], alpha_z=f[2], beta_x=f[3],
                                      beta_y=f[4], beta_z=f[5]))
    assert len(it2["fields"]) == 6
    assert G.parse_iter_para({k: v for k, v in iter_para().items() if k != "n_iter"})[
        "n_iter"] == 1


@pytest.mark.parametrize("missing", ["op_iter", "n_views", "lambda", "outIter", "volumes",
                                     "flows", "err_weights", "angles"])
def test_iter_para_missing_fields_raise(missing):
    d = iter_para()
    del d[missing]
    with pytest.raises(G.BadInput):
        G.parse_iter_para(d)


def test_synthetic_problem_is_seeded_and_shaped():
    cfg = S.small_config(nx=24, ny=24, nz=16, na=48, nb=32, n_views=10)
    p1 = S.make_problem(cfg, seed=3)
    p2 = S.make_problem(cfg, seed=3)
    assert p1.truth.shape == (16, 24, 24) and p1.truth.dtype == np.float32
    np.testing.assert_array_equal(p1.truth, p2.truth)
    for a, b in zip(p1.fields, p2.fields):
        np.testing.assert_array_equal(a, b)
    assert p1.truth.max() > 0 and p1.truth.min() >= 0
    assert p1.op_iter.tolist() == [1, 0, 1, 0]


def test_synthetic_geometry_matches_the_benchmark_configs():
    g = S.geometry(S.CONFIGS["static64"])
    assert (g["SO"], g["SD"], g["da"]) == (500.0, 750.0, pytest.approx(0.8))
    assert g["ai"] == -63.5 and g["bi"] == -47.5
    g2 = S.geometry(S.CONFIGS["motion128"])
    assert (g2["nx"], g2["nz"], g2["na"], g2["nb"]) == (128, 96, 256, 192)
    assert g2["da"] == pytest.approx(0.6)


def test_dvf_scaling_hits_the_configured_peak():
    cfg = S.small_config(nx=24, ny=24, nz=16, n_views=30)
    a, b = S.breathing(30, 0)
    F = S.dvf_fields(cfg, a, b, 0)
    da, db = (a - a[0]).astype(np.float64), (b - b[0]).astype(np.float64)
    peak_z = max(np.abs(da[v] * F[2] + db[v] * F[5]).max() for v in range(30))
    assert peak_z == pytest.approx(cfg.si_mm / cfg.vox_mm, rel=0.05)
