"""The projector runs one of two slab loops per warp: without per-slab
division range tests when every ray of the warp is proven safe (ray_axial in
mcsart_b200/csrc/projector.cuh: its axial footprint keeps away from the
volume's bottom face z = 0, among other bounds), with them otherwise.  Both
give the reference's bits; this checks, on the CPU, that the geometries and
angles of the bit-for-bit projector parity tests exercise both loops, so
that those tests cover each of them.  The restatement is in float64 and
drops the kernel's rounding margins, which only matter at the boundary."""
import numpy as np

from conftest import ANGLES
from test_gpu_kernels import GEOS  # the projector parity geometries

COLS, ROWS = 16, 8  # projector block: 16 detector columns x 8 rows, 2 rows per warp


def ray_exact(g, angle):
    """[nb, na] bool: the ray's axial coordinates never cross zero."""
    c, s = np.cos(angle), np.sin(angle)
    ia = np.arange(g["na"])[None, :]
    ib = np.arange(g["nb"])[:, None]
    x1, y1 = -g["SO"] * c, -g["SO"] * s
    y20 = (ia + g["ai"]) * g["da"]
    x20 = g["SD"] - g["SO"]
    x21 = x20 * c - y20 * s - x1
    y21 = y20 * c + x20 * s - y1
    xdrive = np.abs(x21) > np.abs(y21)
    drv = np.where(xdrive, x21, y21)
    nd = np.where(xdrive, g["nx"], g["ny"])
    src = np.where(xdrive, x1, y1)
    z2 = (ib + g["bi"]) * g["db"]
    dc_lo = 0.5 - nd / 2 - src - 1.0
    dc_hi = nd - 0.5 - nd / 2 - src + 1.0
    zh = g["nz"] // 2
    ok = (dc_lo > 0) | (dc_hi < 0)
    for z in (z2 - g["db"] / 2, z2 + g["db"] / 2):
        rz = z / drv
        ea, eb = rz * dc_lo + zh, rz * dc_hi + zh
        ok = ok & ((np.minimum(ea, eb) > 0) | (np.maximum(ea, eb) < 0))
    return ok


def warp_flags(g, angle):
    ok = ray_exact(g, angle)
    flags = set()
    for b0 in range(0, g["nb"], ROWS):
        for w in range(ROWS // 2):
            r0 = b0 + 2 * w
            for c0 in range(0, g["na"], COLS):
                lanes = ok[r0:min(r0 + 2, g["nb"]), c0:c0 + COLS]
                if lanes.size:
                    flags.add(bool(lanes.all()))
    return flags


def test_parity_geometries_exercise_both_slab_loops():
    for g in GEOS:
        seen = set()
        for a in ANGLES:
            seen |= warp_flags(g, a)
        assert seen == {True, False}, (g, seen)
