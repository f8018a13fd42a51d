"""Seeded synthetic McSART problems: phantom, cone-beam geometry, 5DCT motion.

The workloads (keys of CONFIGS; the batch is ``batch_configs``):

  static64:    static SART, 64^3 at 2 mm, detector 128x96 at 1.6 mm, 60 views, 5 iterations
  motion128:   motion-compensated, 128x128x96 at 2 mm, 256x192 at 1.2 mm, 360 views,
               10 outer iterations of SART + DVF update
  motion256:   motion-compensated, 256x256x160 at 1 mm, 512x384 at 0.776 mm, 660 views
  batch8:      8 independent motion-compensated problems of seeded uneven
               sizes (volumes 96x96x64 to 256x256x128 at 1-2 mm, detectors
               192x128 to 512x384, 120-660 views each), reconstructed together
               in ordered subsets of 10 views (``batch_configs``)
  clinical512: 512x512x256 at 0.5 mm, 1024x768 at 0.388 mm, 1320 views

Phantom: 10 ellipsoids with centres uniform in a 50 mm ball, semi-axes U[5, 40] mm,
random rotation, attenuation U[0, 0.04]/mm, added together; motion configs add a
dense lesion ellipsoid.  Geometry: SAD 1000 mm, SDD 1500 mm, converted to voxel
units; angles evenly spaced over 360 degrees.  Breathing: a(t) = 8 sin(2 pi t / 4 s)
+ N(0, 0.5), b = da/dt of the sine part, t_v = v / 15 s.  DVF fields v, f: three
components of N(0,1) noise smoothed with sigma = 8 voxels, scaled so that the
largest applied displacement (a_v - a_0) v + (b_v - b_0) f over the scan is the
configured SI (z) and AP/LR (x, y) peak.  Everything is float32 and seeded with
numpy.random.default_rng(seed).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SAD_MM, SDD_MM = 1000.0, 1500.0


@dataclass
class Config:
    name: str
    nx: int
    ny: int
    nz: int
    vox_mm: float
    na: int
    nb: int
    pitch_mm: float
    n_views: int
    n_outer: int
    motion: bool
    lesion: bool
    si_mm: float = 10.0
    aplr_mm: float = 3.0
    lam: float = 1.0


CONFIGS = {
    "static64": Config("static SART 64^3, 60 views", 64, 64, 64, 2.0, 128, 96, 1.6, 60, 5, False, False),
    "motion128": Config("motion-compensated McSART 128x128x96, 360 views", 128, 128, 96, 2.0, 256, 192,
                 1.2, 360, 10, True, True),
    "motion256": Config("motion-compensated McSART 256x256x160, 660 views", 256, 256, 160, 1.0, 512, 384,
                 0.776, 660, 10, True, True),
    "clinical512": Config("clinical McSART 512x512x256, 1320 views", 512, 512, 256, 0.5, 1024, 768, 0.388,
                 1320, 10, True, True, si_mm=15.0, aplr_mm=4.5),
}


# The uneven batch: sizes drawn from these sets with a seeded generator.
BATCH_SLICES = (96, 128, 160, 192, 224, 256)
BATCH_DEPTHS = (64, 96, 128)
BATCH_VOXEL_MM = (1.0, 1.5, 2.0)
BATCH_DETECTORS = ((192, 128), (256, 192), (384, 288), (512, 384))
BATCH_SUBSET = 10


def batch_configs(n: int = 8, seed: int = 0) -> list[Config]:
    """The uneven batch (batch8): n motion-compensated problems of seeded
    sizes.  The first two are the extremes (96x96x64 with a 192x128 detector
    and 120 views; 256x256x128 with 512x384 and 660 views), the others drawn
    from the size sets above; views are multiples of the subset size 10 in
    [120, 660].  The detector pitch makes the detector cover the volume's
    width magnified by SDD/SAD = 1.5 with a 10 % margin."""
    rng = np.random.default_rng(seed + 4)
    out = []
    for i in range(n):
        if i == 0:
            nxy, nz, vox, (na, nb), nv = 96, 64, 2.0, BATCH_DETECTORS[0], 120
        elif i == 1:
            nxy, nz, vox, (na, nb), nv = 256, 128, 1.0, BATCH_DETECTORS[-1], 660
        else:
            nxy = int(rng.choice(BATCH_SLICES))
            nz = int(rng.choice(BATCH_DEPTHS))
            vox = float(rng.choice(BATCH_VOXEL_MM))
            na, nb = BATCH_DETECTORS[int(rng.integers(len(BATCH_DETECTORS)))]
            nv = int(rng.integers(12, 67)) * BATCH_SUBSET
        pitch = round(1.5 * 1.1 * nxy * vox / na, 3)
        out.append(Config(f"batch problem {i}: {nxy}x{nxy}x{nz} at {vox} mm, {na}x{nb}, {nv} views",
                          nxy, nxy, nz, vox, na, nb, pitch, nv, 10, True, True))
    return out


def geometry(cfg: Config) -> dict:
    """Reference-convention geometry in voxel units (ai/bi shifted as the gateway does)."""
    f32 = np.float32
    na, nb = cfg.na, cfg.nb
    return dict(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, na=na, nb=nb,
                SO=float(f32(SAD_MM / cfg.vox_mm)), SD=float(f32(SDD_MM / cfg.vox_mm)),
                da=float(f32(cfg.pitch_mm / cfg.vox_mm)), db=float(f32(cfg.pitch_mm / cfg.vox_mm)),
                ai=float(-(f32(na) / f32(2) - f32(0.5))), bi=float(-(f32(nb) / f32(2) - f32(0.5))),
                dx=1.0)


def _rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _add_ellipsoid(vol, centre_mm, axes_mm, rot, value, vox_mm):
    nz, ny, nx = vol.shape
    xs = ((np.arange(nx) + 0.5 - nx / 2) * vox_mm).astype(np.float32)
    ys = ((np.arange(ny) + 0.5 - ny / 2) * vox_mm).astype(np.float32)
    zs = ((np.arange(nz) + 0.5 - nz / 2) * vox_mm).astype(np.float32)
    # bounding box of the ellipsoid to keep the work local
    r = float(np.max(axes_mm))
    sl = []
    for coords, c in ((zs, centre_mm[2]), (ys, centre_mm[1]), (xs, centre_mm[0])):
        lo = np.searchsorted(coords, c - r)
        hi = np.searchsorted(coords, c + r)
        sl.append(slice(lo, hi))
    if any(s.start >= s.stop for s in sl):
        return
    Z, Y, X = np.meshgrid(zs[sl[0]] - centre_mm[2], ys[sl[1]] - centre_mm[1],
                          xs[sl[2]] - centre_mm[0], indexing="ij")
    P = np.stack([X, Y, Z], axis=-1) @ rot.astype(np.float32)
    q = (P[..., 0] / axes_mm[0]) ** 2 + (P[..., 1] / axes_mm[1]) ** 2 + (P[..., 2] / axes_mm[2]) ** 2
    vol[sl[0], sl[1], sl[2]] += np.where(q <= 1.0, np.float32(value), np.float32(0))


def phantom(cfg: Config, seed: int = 0) -> np.ndarray:
    """[nz, ny, nx] float32 attenuation phantom (1/mm)."""
    rng = np.random.default_rng(seed)
    vol = np.zeros((cfg.nz, cfg.ny, cfg.nx), np.float32)
    for _ in range(10):
        while True:
            c = rng.uniform(-50, 50, 3)
            if np.linalg.norm(c) <= 50:
                break
        axes = rng.uniform(5, 40, 3)
        _add_ellipsoid(vol, c, axes, _rotation(rng), rng.uniform(0, 0.04), cfg.vox_mm)
    if cfg.lesion:
        c = rng.uniform(-20, 20, 3)
        _add_ellipsoid(vol, c, rng.uniform(6, 12, 3), _rotation(rng), 0.06, cfg.vox_mm)
    return vol


def breathing(n_views: int, seed: int = 0, fps: float = 15.0, period: float = 4.0):
    """Per-view amplitude a(t_v) and flow b(t_v) (float32)."""
    rng = np.random.default_rng(seed + 7)
    t = np.arange(n_views) / fps
    w = 2 * np.pi / period
    a = 8 * np.sin(w * t) + rng.normal(0, 0.5, n_views)
    b = 8 * w * np.cos(w * t)
    return a.astype(np.float32), b.astype(np.float32)


def _smooth(x, sigma):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(x, sigma, mode="nearest")


def dvf_fields(cfg: Config, volumes, flows, seed: int = 0) -> list[np.ndarray]:
    """[ax, ay, az, bx, by, bz] float32 volumes (voxel units)."""
    rng = np.random.default_rng(seed + 13)
    shape = (cfg.nz, cfg.ny, cfg.nx)
    comp = [_smooth(rng.normal(size=shape).astype(np.float32), 8.0) for _ in range(6)]
    da = (volumes - volumes[0]).astype(np.float64)
    db = (flows - flows[0]).astype(np.float64)
    out = [None] * 6
    # max over views of |da_v v(x) + db_v f(x)| is attained at a vertex of the
    # convex hull of the points (da_v, db_v): scan only those views
    pts = np.stack([da, db], axis=1)
    try:
        from scipy.spatial import ConvexHull
        hull = np.unique(ConvexHull(pts).vertices)
    except Exception:  # degenerate (collinear) point sets
        hull = np.arange(len(da))
    for c in range(3):
        v, f = comp[c].astype(np.float64), comp[3 + c].astype(np.float64)
        peak = max(np.max(np.abs(da[i] * v + db[i] * f)) for i in hull)
        target = (cfg.si_mm if c == 2 else cfg.aplr_mm) / cfg.vox_mm
        s = target / peak if peak > 0 else 0.0
        out[c] = (v * s).astype(np.float32)
        out[3 + c] = (f * s).astype(np.float32)
    return out


@dataclass
class Problem:
    cfg: Config
    geo: dict
    img0: np.ndarray
    truth: np.ndarray
    angles: np.ndarray
    volumes: np.ndarray
    flows: np.ndarray
    fields: list | None
    op_iter: np.ndarray
    n_iter: int
    proj: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


def make_problem(cfg: Config | str, seed: int = 0, with_proj: bool = False) -> Problem:
    """Seeded problem for a config; projections are added by ``make_projections``."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    geo = geometry(cfg)
    truth = phantom(cfg, seed)
    angles = np.linspace(0, 2 * np.pi, cfg.n_views, endpoint=False).astype(np.float32)
    if cfg.motion:
        volumes, flows = breathing(cfg.n_views, seed)
        fields = dvf_fields(cfg, volumes, flows, seed)
        op_iter = np.array([1, 0] * cfg.n_outer, np.int32)
    else:
        volumes = np.zeros(cfg.n_views, np.float32)
        flows = np.zeros(cfg.n_views, np.float32)
        fields = None
        op_iter = np.ones(cfg.n_outer, np.int32)
    p = Problem(cfg, geo, np.zeros_like(truth), truth, angles, volumes, flows, fields, op_iter,
                len(op_iter))
    return p


def make_projections(p: Problem, project, deform=None) -> np.ndarray:
    """proj_v = FP(warp(truth, a_v - a_0, b_v - b_0)) (static: FP(truth)).

    ``project(vol, angle) -> [nb, na]`` and ``deform(vol, volume, flow) -> vol``
    are supplied by the caller (GPU engine, rebuilt reference or oracle).
    """
    out = np.zeros((p.cfg.n_views, p.cfg.nb, p.cfg.na), np.float32)
    for v in range(p.cfg.n_views):
        vol = p.truth
        if p.fields is not None and deform is not None:
            vol = deform(p.truth, np.float32(p.volumes[v] - p.volumes[0]),
                         np.float32(p.flows[v] - p.flows[0]))
        out[v] = project(vol, float(p.angles[v]))
    p.proj = out
    return out


def small_config(nx=24, ny=24, nz=16, na=32, nb=24, n_views=12, motion=True, vox_mm=8.0,
                 pitch_mm=6.0, n_outer=2) -> Config:
    """A small problem the CPU oracle runs in seconds (for parity tests)."""
    return Config(f"small {nx}x{ny}x{nz}", nx, ny, nz, vox_mm, na, nb, pitch_mm, n_views,
                  n_outer, motion, motion)
