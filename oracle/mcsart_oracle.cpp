// Test infrastructure: CPU oracle for the McSART hot path (see mcsart_oracle.h).
//
// One templated restatement of the reference kernels, instantiated twice:
//   T = double -> orc_*  (FP64 oracle; the accuracy reference of the tests)
//   T = float  -> cpu_*  (FP32 OpenMP transcription; the timed CPU baseline)
// Each function cites the reference lines it restates.  Index conventions,
// integer divisions (nx/2 vs (float)nx/2), loop bounds and the order of the
// accumulations follow the reference exactly; only the scalar type changes.
//
// Two quantities are deliberately computed in float even in the FP64 oracle,
// because they are discrete decisions of the reference algorithm whose float
// outcome defines which formula applies:
//   * the projector's driving-axis choice |x21| > |y21| (cu_projection.cu:39);
//   * the warp's texture coordinates and the per-view amplitude differences,
//     which the reference forms in float before the texture unit quantises
//     them (cu_deform.cu:86-89, AUMISART.cu:193,222).
#include "mcsart_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

template <typename T> inline T tmin(T a, T b) { return (a < b) ? a : b; }  // universal.h:16
template <typename T> inline T tmax(T a, T b) { return (a > b) ? a : b; }  // universal.h:12
template <typename T> inline T min4(T a, T b, T c, T d) { return tmin(tmin(a, b), tmin(c, d)); }
template <typename T> inline T max4(T a, T b, T c, T d) { return tmax(tmax(a, b), tmax(c, d)); }
template <typename T> inline T min6(T a, T b, T c, T d, T e, T f) {
    return tmin(tmin(tmin(a, b), tmin(c, d)), tmin(e, f));
}
template <typename T> inline T max6(T a, T b, T c, T d, T e, T f) {
    return tmax(tmax(tmax(a, b), tmax(c, d)), tmax(e, f));
}

inline int64_t nvox(int nx, int ny, int nz) { return (int64_t)nx * ny * nz; }

// ---------------------------------------------------------------- projector
// src/cu_projection.cu:15-145: one detector cell (ia, ib) of one view.
// The terms of one ray (src/cu_projection.cu:22-144): visit(voxel index,
// in-plane weight, axial weight) in the reference's order.  project_ray sums
// img * w_u * w_z over them; the exact adjoint scatters p * w_u * w_z.
template <typename T, typename Visit>
void ray_walk(int ia, int ib, float anglef, T SO, T SD, T da, T ai, T db, T bi, int nx, int ny,
              int nz, Visit visit) {
    // Driving-axis decision in float, as the reference evaluates it (:23-39).
    const float cf = std::cos(anglef), sf = std::sin(anglef);
    const float SOf = (float)SO, SDf = (float)SD, daf = (float)da, aif = (float)ai;
    const float x1f = -SOf * cf, y1f = -SOf * sf;
    const float x20f = SDf - SOf, y20f = ((float)ia + aif) * daf;
    const float x21f = (x20f * cf - y20f * sf) - x1f;
    const float y21f = (x20f * sf + y20f * cf) - y1f;
    const bool xdrive = std::fabs(x21f) > std::fabs(y21f);

    const T cphi = (T)std::cos((double)anglef), sphi = (T)std::sin((double)anglef);
    const T x1 = -SO * cphi, y1 = -SO * sphi, z1 = 0;            // :25-27
    const T x20 = SD - SO, y20 = ((T)ia + ai) * da;              // :28-29
    const T x2 = x20 * cphi - y20 * sphi;                         // :30
    const T y2 = x20 * sphi + y20 * cphi;                         // :31
    const T z2 = ((T)ib + bi) * db;                               // :32
    const T x21 = x2 - x1, y21 = y2 - y1, z21 = z2 - z1;          // :34-36
    const T half_da = da / 2, half_db = db / 2;
    if (xdrive) {
        for (int ix = 0; ix < nx; ix++) {                          // :44
            const T xl = x21 - half_da * sphi, xr = x21 + half_da * sphi;  // :48-49
            const T yl = y21 - half_da * cphi, yr = y21 + half_da * cphi;  // :50-51
            const T xc = (T)ix + (T)0.5 - (T)nx / 2 - x1;          // :52 (float nx/2)
            const T cy = (T)(ny / 2);                              // :55 (integer ny/2)
            const T cyll = yl / xl * xc + y1 + cy, cylr = yl / xr * xc + y1 + cy;
            const T cyrl = yr / xl * xc + y1 + cy, cyrr = yr / xr * xc + y1 + cy;
            const T yi1 = min4(cyll, cylr, cyrl, cyrr), yi2 = max4(cyll, cylr, cyrl, cyrr);
            const int Yi1 = (int)std::floor(yi1), Yi2 = (int)std::floor(yi2);  // :63-64
            const T zl = z21 - half_db, zr = z21 + half_db;       // :67-68
            const T cz = (T)(nz / 2);                              // :72 (integer nz/2)
            const T czl = zl / x21 * xc + z1 + cz, czr = zr / x21 * xc + z1 + cz;
            const T zi1 = tmin(czl, czr), zi2 = tmax(czl, czr);
            const int Zi1 = (int)std::floor(zi1), Zi2 = (int)std::floor(zi2);  // :76-77
            for (int iy = std::max(0, Yi1); iy <= std::min(ny - 1, Yi2); iy++) {     // :81
                const T wy = (tmin((T)iy + 1, yi2) - tmax((T)iy, yi1)) / (yi2 - yi1);
                for (int iz = std::max(0, Zi1); iz <= std::min(nz - 1, Zi2); iz++) { // :84
                    const T wz = (tmin((T)iz + 1, zi2) - tmax((T)iz, zi1)) / (zi2 - zi1);
                    visit(ix + (int64_t)iy * nx + (int64_t)iz * nx * ny, wy, wz);  // :87
                }
            }
        }
    } else {
        for (int iy = 0; iy < ny; iy++) {                          // :97
            const T yl = y21 - half_da * cphi, yr = y21 + half_da * cphi;  // :101-102
            const T xl = x21 - half_da * sphi, xr = x21 + half_da * sphi;  // :103-104
            const T yc = (T)iy + (T)0.5 - (T)ny / 2 - y1;          // :105
            const T cx = (T)(nx / 2);                              // :108 (integer nx/2)
            const T cxll = xl / yl * yc + x1 + cx, cxlr = xl / yr * yc + x1 + cx;
            const T cxrl = xr / yl * yc + x1 + cx, cxrr = xr / yr * yc + x1 + cx;
            const T xi1 = min4(cxll, cxlr, cxrl, cxrr), xi2 = max4(cxll, cxlr, cxrl, cxrr);
            const int Xi1 = (int)std::floor(xi1), Xi2 = (int)std::floor(xi2);  // :116-117
            const T zl = z21 - half_db, zr = z21 + half_db;
            const T cz = (T)(nz / 2);                              // :125
            const T czl = zl / y21 * yc + z1 + cz, czr = zr / y21 * yc + z1 + cz;
            const T zi1 = tmin(czl, czr), zi2 = tmax(czl, czr);
            const int Zi1 = (int)std::floor(zi1), Zi2 = (int)std::floor(zi2);  // :129-130
            for (int ix = std::max(0, Xi1); ix <= std::min(nx - 1, Xi2); ix++) {     // :134
                const T wx = (tmin((T)ix + 1, xi2) - tmax((T)ix, xi1)) / (xi2 - xi1);
                for (int iz = std::max(0, Zi1); iz <= std::min(nz - 1, Zi2); iz++) { // :137
                    const T wz = (tmin((T)iz + 1, zi2) - tmax((T)iz, zi1)) / (zi2 - zi1);
                    visit(ix + (int64_t)iy * nx + (int64_t)iz * nx * ny, wx, wz);  // :140
                }
            }
        }
    }
}

template <typename T>
T project_ray(const T *img, int ia, int ib, float anglef, T SO, T SD, T da, T ai, T db, T bi,
              int nx, int ny, int nz) {
    T acc = 0;
    ray_walk<T>(ia, ib, anglef, SO, SD, da, ai, db, bi, nx, ny, nz,
                [&](int64_t i, T wu, T wz) { acc += img[i] * wu * wz; });
    return acc;
}

// Exact adjoint (transpose) of projection(): img = A^T proj, scattered ray by
// ray in the reference projector's terms.  Not a reference function (its
// backprojector is a different operator); the engine's
// mcsart_backprojection_adjoint is checked against it.
template <typename T>
void backprojection_adjoint(T *img, const T *proj, double angle, double SO, double SD, double da,
                            int na, double ai, double db, int nb, double bi, int nx, int ny,
                            int nz) {
    const float anglef = (float)angle;
    std::fill(img, img + nvox(nx, ny, nz), (T)0);
    for (int ib = 0; ib < nb; ib++)
        for (int ia = 0; ia < na; ia++) {
            const T p = proj[ia + (int64_t)ib * na];
            ray_walk<T>(ia, ib, anglef, (T)SO, (T)SD, (T)da, (T)ai, (T)db, (T)bi, nx, ny, nz,
                        [&](int64_t i, T wu, T wz) { img[i] += p * wu * wz; });
        }
}

template <typename T>
void projection(T *proj, const T *img, double angle, double SO, double SD, double da, int na,
                double ai, double db, int nb, double bi, int nx, int ny, int nz) {
    const float anglef = (float)angle;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int ib = 0; ib < nb; ib++)
        for (int ia = 0; ia < na; ia++)
            proj[ia + (int64_t)ib * na] = project_ray<T>(img, ia, ib, anglef, (T)SO, (T)SD,
                                                          (T)da, (T)ai, (T)db, (T)bi, nx, ny, nz);
}

// ------------------------------------------------------------ backprojector
// src/cu_backprojection.cu:49-170 for one voxel.  The reference reads the
// projection through a linear-filtered float texture exactly at texel centres
// (:167), which returns the texel itself, except that a texel below the
// float32 normal range reads as a zero of the same sign (the texture unit's
// behaviour, measured on B200); that read is restated here.
template <typename T>
T backproject_voxel(const T *proj, int ix, int iy, int iz, T cphi, T sphi, T SO, T SD, T da,
                    int na, T ai, T db, int nb, T bi, int nx, int ny, int nz) {
    const T xc = (T)ix - (T)(nx / 2) + (T)0.5;   // :66 (integer nx/2)
    const T yc = (T)iy - (T)(ny / 2) + (T)0.5;   // :67
    const T zc = (T)iz - (T)(nz / 2) + (T)0.5;   // :68
    const T h = (T)0.5;
    const T xrot = xc * cphi + yc * sphi, yrot = -xc * sphi + yc * cphi;
    // Six boundary points (:82-97): an axis-aligned unit square in the
    // rotated frame plus the top and bottom of the voxel.
    const T xll = xrot - h, yll = yrot - h, zll = zc;
    const T xrr = xrot + h, yrr = yrot + h, zrr = zc;
    const T xrl = xrot + h, yrl = yrot - h, zrl = zc;
    const T xlr = xrot - h, ylr = yrot + h, zlr = zc;
    const T xt = xrot, yt = yrot, zt = zc + h;
    const T xb = xrot, yb = yrot, zb = zc - h;
    T ratio;
    ratio = SD / (xll + SO); const T all = ratio * yll, bll = ratio * zll;   // :105-107
    ratio = SD / (xrr + SO); const T arr = ratio * yrr, brr = ratio * zrr;   // :108-110
    ratio = SD / (xlr + SO); const T alr = ratio * ylr, blr = ratio * zlr;   // :111-113
    ratio = SD / (xrl + SO); const T arl = ratio * yrl, brl = ratio * zrl;   // :114-116
    ratio = SD / (xt + SO); const T at = ratio * yt, bt = ratio * zt;        // :117-119
    ratio = SD / (xb + SO); const T ab = ratio * yb, bb = ratio * zb;        // :120-122
    T a_max = max6(all, arr, alr, arl, at, ab), a_min = min6(all, arr, alr, arl, at, ab);
    T b_max = max6(bll, brr, blr, brl, bt, bb), b_min = min6(bll, brr, blr, brl, bt, bb);
    a_max = a_max / da - ai + h;                  // :135-138
    a_min = a_min / da - ai + h;
    b_max = b_max / db - bi + h;
    b_min = b_min / db - bi + h;
    const int a_ind_min = (int)std::floor(a_min);
    const int b_ind_min = (int)std::floor(b_min);
    const T a_lim = ((T)na < a_max) ? (T)na : a_max;   // MIN(na, a_max), :150
    const T b_lim = ((T)nb < b_max) ? (T)nb : b_max;   // MIN(nb, b_max), :158
    T acc = 0;
    for (int ia = std::max(0, a_ind_min); (T)ia < a_lim; ia++) {
        const T wa = tmin((T)ia + 1, a_max) - tmax((T)ia, a_min);          // :156
        for (int ib = std::max(0, b_ind_min); (T)ib < b_lim; ib++) {
            const T wb = tmin((T)ib + 1, b_max) - tmax((T)ib, b_min);      // :164
            const T pv = proj[ia + (int64_t)ib * na];                       // :167
            const T tv = std::fabs(pv) < (T)0x1p-126 ? std::copysign((T)0, pv) : pv;
            acc += wa * wb * tv;
        }
    }
    return acc;
}

template <typename T>
void backprojection_sc(T *img, const T *proj, double cphi, double sphi, double SO, double SD,
                       double da, int na, double ai, double db, int nb, double bi, int nx,
                       int ny, int nz) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < nz; iz++)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++)
                img[ix + (int64_t)iy * nx + (int64_t)iz * nx * ny] = backproject_voxel<T>(
                    proj, ix, iy, iz, (T)cphi, (T)sphi, (T)SO, (T)SD, (T)da, na, (T)ai, (T)db,
                    nb, (T)bi, nx, ny, nz);
}

template <typename T>
void backprojection(T *img, const T *proj, double angle, double SO, double SD, double da, int na,
                    double ai, double db, int nb, double bi, int nx, int ny, int nz) {
    // The reference evaluates __sinf/__cosf of the float angle (:62-63); the
    // oracle uses the exact sine and cosine of that float.
    const double a = (double)(float)angle;
    backprojection_sc<T>(img, proj, std::cos(a), std::sin(a), SO, SD, da, na, ai, db, nb, bi, nx,
                         ny, nz);
}

// ------------------------------------------------------------------- warps
// src/cu_deform.cu:66-77
template <typename T>
void forward_dvf(T *mx, T *my, T *mz, const T *ax, const T *ay, const T *az, const T *bx,
                 const T *by, const T *bz, double volume, double flow, int nx, int ny, int nz) {
    const int64_t n = nvox(nx, ny, nz);
    const T v = (T)volume, f = (T)flow;
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < n; id++) {
        mx[id] = ax[id] * v + bx[id] * f;
        my[id] = ay[id] * v + by[id] * f;
        mz[id] = az[id] * v + bz[id] * f;
    }
}

inline double quantise_frac(double a, int tex_mode) {
    if (tex_mode == ORC_TEX_Q8_NEAREST) return std::floor(a * 256.0 + 0.5) / 256.0;
    if (tex_mode == ORC_TEX_Q8_TRUNC) return std::floor(a * 256.0) / 256.0;
    return a;
}

// Linear filtering of a 3D texture with clamp addressing at unnormalised
// coordinates (x, y, z), x the fastest axis of extent nx (the texture built at
// cu_deform.cu:13-38).  Texel centres sit at i + 0.5.
template <typename T>
T tex3d_linear(const T *img, int nx, int ny, int nz, double x, double y, double z, int tex_mode) {
    const double xb = x - 0.5, yb = y - 0.5, zb = z - 0.5;
    const double fi = std::floor(xb), fj = std::floor(yb), fk = std::floor(zb);
    const T a = (T)quantise_frac(xb - fi, tex_mode);
    const T b = (T)quantise_frac(yb - fj, tex_mode);
    const T c = (T)quantise_frac(zb - fk, tex_mode);
    auto clampi = [](double v, int n) -> int64_t {
        if (v < 0) return 0;
        if (v > n - 1) return n - 1;
        return (int64_t)v;
    };
    const int64_t i0 = clampi(fi, nx), i1 = clampi(fi + 1, nx);
    const int64_t j0 = clampi(fj, ny), j1 = clampi(fj + 1, ny);
    const int64_t k0 = clampi(fk, nz), k1 = clampi(fk + 1, nz);
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    auto t = [&](int64_t i, int64_t j, int64_t k) { return img[i + j * sy + k * sz]; };
    const T one = 1;
    return (one - a) * (one - b) * (one - c) * t(i0, j0, k0) + a * (one - b) * (one - c) * t(i1, j0, k0) +
           (one - a) * b * (one - c) * t(i0, j1, k0) + a * b * (one - c) * t(i1, j1, k0) +
           (one - a) * (one - b) * c * t(i0, j0, k1) + a * (one - b) * c * t(i1, j0, k1) +
           (one - a) * b * c * t(i0, j1, k1) + a * b * c * t(i1, j1, k1);
}

// src/cu_deform.cu:3-47 (forwardDVF + kernel_deformation, :79-90).  The output
// is written at the in-slice transposed index iy + ix*ny (:85).
template <typename T>
void deform(T *out, const T *img, int nx, int ny, int nz, double volume, double flow, const T *ax,
            const T *ay, const T *az, const T *bx, const T *by, const T *bz, int tex_mode) {
    const int64_t n = nvox(nx, ny, nz);
    std::vector<T> src(img, img + n);  // the reference samples a copy (cudaArray)
    const float vf = (float)volume, ff = (float)flow;
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int64_t id = iy + (int64_t)ix * ny + (int64_t)iz * nx * ny;
                double xs, ys, zs;
                if (tex_mode == ORC_TEX_EXACT) {
                    const double mx = (double)ax[id] * volume + (double)bx[id] * flow;
                    const double my = (double)ay[id] * volume + (double)by[id] * flow;
                    const double mz = (double)az[id] * volume + (double)bz[id] * flow;
                    xs = iy + 0.5 + my;
                    ys = ix + 0.5 + mx;
                    zs = iz + 0.5 + mz;
                } else {
                    // float coordinates exactly as formed at :74-76 and :86-89
                    const float mx = (float)ax[id] * vf + (float)bx[id] * ff;
                    const float my = (float)ay[id] * vf + (float)by[id] * ff;
                    const float mz = (float)az[id] * vf + (float)bz[id] * ff;
                    const float xi = (float)iy + 1.0f + my, yi = (float)ix + 1.0f + mx,
                                zi = (float)iz + 1.0f + mz;
                    xs = (double)(xi - 0.5f);
                    ys = (double)(yi - 0.5f);
                    zs = (double)(zi - 0.5f);
                }
                out[id] = tex3d_linear<T>(src.data(), nx, ny, nz, xs, ys, zs, tex_mode);
            }
}

// Inverse of the warp's displacement for square slices (the engine's
// mcsart_invert_dvf; not a reference function: the reference negates the
// amplitudes, src/AUMISART.cu:222).  The warp samples memory position
// q = (X, Y, Z) at q + D(q), D = (my, mx, mz)(q); N(q) = -D(q + N(q)) by
// fixed-point iteration from 0 with exact trilinear samples, returned in the
// forward layout (ox, oy, oz) = (N_Y, N_X, N_Z).
template <typename T>
void invert_dvf(T *ox, T *oy, T *oz, const T *ax, const T *ay, const T *az, const T *bx,
                const T *by, const T *bz, double volume, double flow, int nx, int ny, int nz,
                int iters) {
    const int64_t n = nvox(nx, ny, nz);
    std::vector<T> m(3 * n);
    forward_dvf<T>(m.data(), m.data() + n, m.data() + 2 * n, ax, ay, az, bx, by, bz, volume,
                   flow, nx, ny, nz);
    const T *mx = m.data(), *my = mx + n, *mz = my + n;
#pragma omp parallel for collapse(2) schedule(static)
    for (int Z = 0; Z < nz; Z++)
        for (int Y = 0; Y < ny; Y++)
            for (int X = 0; X < nx; X++) {
                double NX = 0, NY = 0, NZ = 0;
                for (int k = 0; k < iters; k++) {
                    const double px = X + 0.5 + NX, py = Y + 0.5 + NY, pz = Z + 0.5 + NZ;
                    const double dX = tex3d_linear<T>(my, nx, ny, nz, px, py, pz, ORC_TEX_EXACT);
                    const double dY = tex3d_linear<T>(mx, nx, ny, nz, px, py, pz, ORC_TEX_EXACT);
                    const double dZ = tex3d_linear<T>(mz, nx, ny, nz, px, py, pz, ORC_TEX_EXACT);
                    NX = -dX;
                    NY = -dY;
                    NZ = -dZ;
                }
                const int64_t id = X + (int64_t)Y * nx + (int64_t)Z * nx * ny;
                ox[id] = (T)NY;
                oy[id] = (T)NX;
                oz[id] = (T)NZ;
            }
}

// The warp of src/cu_deform.cu:79-90 with an explicit displacement (mx, my,
// mz) in place of alpha*volume + beta*flow, exact trilinear samples.
template <typename T>
void deform_disp(T *out, const T *img, int nx, int ny, int nz, const T *mx, const T *my,
                 const T *mz) {
    const int64_t n = nvox(nx, ny, nz);
    std::vector<T> src(img, img + n);
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int64_t id = iy + (int64_t)ix * ny + (int64_t)iz * nx * ny;
                out[id] = tex3d_linear<T>(src.data(), nx, ny, nz, iy + 0.5 + (double)my[id],
                                          ix + 0.5 + (double)mx[id], iz + 0.5 + (double)mz[id],
                                          ORC_TEX_EXACT);
            }
}

// src/cu_deform.cu:49-64,92-113 (first-order warp).  With the transposed index
// the +nx neighbour of the last x-row of the last slice lies past the end of
// the volume in the reference (an out-of-bounds read there); it reads 0 here.
template <typename T>
void deform2(T *out, const T *img, int nx, int ny, int nz, double volume, double flow,
             const T *ax, const T *ay, const T *az, const T *bx, const T *by, const T *bz) {
    const int64_t n = nvox(nx, ny, nz);
    std::vector<T> m(3 * n);
    forward_dvf<T>(m.data(), m.data() + n, m.data() + 2 * n, ax, ay, az, bx, by, bz, volume,
                   flow, nx, ny, nz);
    std::vector<T> src(img, img + n);
    auto at = [&](int64_t i) -> T { return i < n ? src[i] : (T)0; };
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int64_t id = iy + (int64_t)ix * ny + (int64_t)iz * nx * ny;
                const T dx = (ix == nx - 1) ? (T)0 : at(id + 1) - at(id);
                const T dy = (iy == ny - 1) ? (T)0 : at(id + nx) - at(id);
                const T dz = (iz == nz - 1) ? (T)0 : at(id + (int64_t)nx * ny) - at(id);
                out[id] = at(id) + dy * m[id] + dx * m[n + id] + dz * m[2 * n + id];
            }
}

// --------------------------------------------------------- elementwise ops
// Forward difference of img0 along ind at voxel id, 0 on the last plane
// (cu_add.cu:37-57, cu_multiple.cu:21-41, cu_initial.cu:36-47).
template <typename T>
inline T fwd_diff(const T *img0, int64_t id, int ix, int iy, int iz, int nx, int ny, int nz,
                  int ind) {
    switch (ind) {
        case 1: return (ix == nx - 1) ? (T)0 : img0[id + 1] - img0[id];
        case 2: return (iy == ny - 1) ? (T)0 : img0[id + nx] - img0[id];
        case 3: return (iz == nz - 1) ? (T)0 : img0[id + (int64_t)nx * ny] - img0[id];
        default: return (T)0;  // the reference leaves df unset for other ind
    }
}

#define FOR_VOXELS                                                                             \
    _Pragma("omp parallel for collapse(2) schedule(static)") for (int iz = 0; iz < nz; iz++)  \
        for (int iy = 0; iy < ny; iy++) for (int ix = 0; ix < nx; ix++)

// src/cu_add.cu:9-18
template <typename T> void add(T *img1, const T *img, int nx, int ny, int nz, double weight) {
    const T w = (T)weight;
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        img1[id] += img[id] * w;
    }
}

// src/cu_add.cu:28-59
template <typename T>
void add2(T *img1, const T *img, int nx, int ny, int nz, const T *img0, double weight, int ind) {
    const T w = (T)weight;
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        const T df = fwd_diff(img0, id, ix, iy, iz, nx, ny, nz, ind);
        img1[id] += img[iy + (int64_t)ix * ny + (int64_t)iz * nx * ny] * w * df;
    }
}

// src/cu_initial.cu:10-17
template <typename T> void initial(T *img, int nx, int ny, int nz, double value) {
    const T v = (T)value;
    FOR_VOXELS { img[ix + (int64_t)iy * nx + (int64_t)iz * nx * ny] = v; }
}

// src/cu_initial.cu:27-49
template <typename T>
void initial2(T *img, int nx, int ny, int nz, const T *img0, double volume, double flow) {
    const T s = (T)volume + (T)flow;
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        const T dfx = fwd_diff(img0, id, ix, iy, iz, nx, ny, nz, 1);
        const T dfy = fwd_diff(img0, id, ix, iy, iz, nx, ny, nz, 2);
        const T dfz = fwd_diff(img0, id, ix, iy, iz, nx, ny, nz, 3);
        img[id] = (dfx + dfy + dfz) * s;
    }
}

// src/cu_division.cu:11-25
template <typename T> void division(T *img1, const T *img, int nx, int ny, int nz) {
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        T q = img1[id] / img[id];
        if (std::isnan(q) || std::isinf(q)) q = 0;
        img1[id] = q;
    }
}

// src/cu_multiple.cu:11-43
template <typename T>
void multiple(T *img1, int nx, int ny, int nz, const T *img0, double weight, int ind) {
    const T w = (T)weight;
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        img1[id] *= w * fwd_diff(img0, id, ix, iy, iz, nx, ny, nz, ind);
    }
}

// src/cu_update_udvf.cu:11-62.  The reference pairs alpha_y/beta_y with the x
// gradient and alpha_x/beta_x with the y gradient when forming b (:45-50) but
// updates alpha_x with the x component (:55); both are kept.
template <typename T>
void update_udvf(T *alpha_x, T *alpha_y, T *alpha_z, T *beta_x, T *beta_y, T *beta_z,
                 const T *img, const T *img0, double volume_diff, double flow_diff, int nx,
                 int ny, int nz, int /*iter*/) {
    const T vd = (T)volume_diff, fd = (T)flow_diff;
    const T sixth = (T)1 / (T)6;
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        const T dfI = img0[id] - img[id];
        const T dfx = fwd_diff(img, id, ix, iy, iz, nx, ny, nz, 1);
        const T dfy = fwd_diff(img, id, ix, iy, iz, nx, ny, nz, 2);
        const T dfz = fwd_diff(img, id, ix, iy, iz, nx, ny, nz, 3);
        const T cax = dfx * vd, cay = dfy * vd, caz = dfz * vd;
        const T cbx = dfx * fd, cby = dfy * fd, cbz = dfz * fd;
        const T w = cax * cax + cay * cay + caz * caz + cbx * cbx + cby * cby + cbz * cbz;
        const T ax = alpha_y[id], ay = alpha_x[id], az = alpha_z[id];
        const T bx = beta_y[id], by = beta_x[id], bz = beta_z[id];
        T b = dfI - cax * ax - cay * ay - caz * az - cbx * bx - cby * by - cbz * bz;
        if (w == 0) continue;
        b /= w;
        alpha_x[id] += sixth * b * cax;
        alpha_y[id] += sixth * b * cay;
        alpha_z[id] += sixth * b * caz;
        beta_x[id] += sixth * b * cbx;
        beta_y[id] += sixth * b * cby;
        beta_z[id] += sixth * b * cbz;
    }
}

// src/mex_diff.cu:75-113: backward difference, 0 on both faces.
template <typename T> void diff(T *img1, const T *img, int nx, int ny, int nz, int ind) {
    FOR_VOXELS {
        const int64_t id = ix + (int64_t)iy * nx + (int64_t)iz * nx * ny;
        T v = 0;
        switch (ind) {
            case 1: v = (ix == nx - 1 || ix == 0) ? (T)0 : img[id] - img[id - 1]; break;
            case 2: v = (iy == ny - 1 || iy == 0) ? (T)0 : img[id] - img[id - nx]; break;
            case 3:
                v = (iz == nz - 1 || iz == 0) ? (T)0 : img[id] - img[id - (int64_t)nx * ny];
                break;
            default: continue;  // the reference writes nothing for other ind
        }
        img1[id] = v;
    }
}

template <typename T> double norm2(const T *x, int64_t n) {
    double s = 0;
    for (int64_t i = 0; i < n; i++) s += (double)x[i] * (double)x[i];
    return std::sqrt(s);
}

// ---------------------------------------------------------------- the loop
// src/AUMISART.cu:3-141 (overload 1, fields NULL) and :143-313 (overload 2).
// Views outside [view_lo, view_hi) are skipped in both passes; the full range
// reproduces the reference, a narrower one is a bounded sample for timing.
template <typename T>
int aumisart(T *outimg, T *outproj, T *outnorm, T *outalphax, const T *h_img, const T *h_proj,
             int nx, int ny, int nz, int na, int nb, int /*outIter*/, int n_views, int n_iter,
             const int *op_iter, double da, double db, double ai, double bi, double SO, double SD,
             double /*dx*/, double lambda, const float *volumes, const float *flows,
             const float *angles, const T *fax, const T *fay, const T *faz, const T *fbx,
             const T *fby, const T *fbz, T *fields_out, int tex_mode, int view_lo, int view_hi,
             int subset, int dvf_inverse) {
    const int64_t nv = nvox(nx, ny, nz), np = (int64_t)na * nb;
    const bool with_motion = fax != nullptr;  // overload 2
    if (view_hi < 0 || view_hi > n_views) view_hi = n_views;
    if (view_lo < 0) view_lo = 0;
    std::vector<T> img(h_img, h_img + nv), img0(nv), img1(nv), img_temp(nv), img_ones(nv);
    std::vector<T> proj(np), proj_temp(np), proj_ones(np);
    std::vector<T> F(6 * nv, (T)0);
    T *al_x = F.data(), *al_y = al_x + nv, *al_z = al_y + nv;
    T *be_x = al_z + nv, *be_y = be_x + nv, *be_z = be_y + nv;
    if (with_motion) {
        std::copy(fax, fax + nv, al_x); std::copy(fay, fay + nv, al_y);
        std::copy(faz, faz + nv, al_z); std::copy(fbx, fbx + nv, be_x);
        std::copy(fby, fby + nv, be_y); std::copy(fbz, fbz + nv, be_z);
    }
    const int motion_step = with_motion ? 1 : 10;  // AUMISART.cu:242 vs :72
    auto FP = [&](T *p, const T *v, int iv) {
        projection<T>(p, v, angles[iv], SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    };
    auto BP = [&](T *v, const T *p, int iv) {
        backprojection<T>(v, p, angles[iv], SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    };
    auto DEF = [&](T *o, const T *i, float vol, float flow) {
        deform<T>(o, i, nx, ny, nz, vol, flow, al_x, al_y, al_z, be_x, be_y, be_z, tex_mode);
    };
    for (int it = 0; it < n_iter; it++) {
        if (op_iter[it] == 1) {  // image update, AUMISART.cu:42-64 / :184-234
            // Ordered subsets of `subset` views (the engine's options.subset):
            // every view of a subset starts from the image as it was before the
            // subset, and the image then receives lambda/k times the views'
            // corrections (static: summed ratios, motion: each back-warped
            // ratio added in view order).  subset 1 is the reference's loop.
            const int sub = subset < 1 ? 1 : subset;
            for (int s0 = view_lo; s0 < view_hi; s0 += sub) {
                const int kk = std::min(sub, view_hi - s0);
                std::vector<T> snap;
                const T *cur = img.data();
                if (kk > 1) {
                    snap = img;
                    cur = snap.data();
                }
                const double lam = kk > 1 ? lambda / kk : lambda;
                std::vector<T> qsum;
            for (int iv = s0; iv < s0 + kk; iv++) {
                const T *fp_src = cur;
                if (with_motion) {
                    DEF(img1.data(), cur, volumes[iv] - volumes[0], flows[iv] - flows[0]);
                    fp_src = img1.data();
                }
                FP(proj_temp.data(), fp_src, iv);
                std::copy(h_proj + iv * np, h_proj + (iv + 1) * np, proj.begin());
                const double n0 = norm2(proj.data(), np);
                add<T>(proj.data(), proj_temp.data(), na, nb, 1, -1.0);
                const double n1 = norm2(proj.data(), np);
                outnorm[(int64_t)it * n_views + iv] = (T)(n1 / n0);
                std::copy(proj.begin(), proj.end(), outproj + iv * np);
                BP(img_temp.data(), proj.data(), iv);
                initial<T>(img_ones.data(), nx, ny, nz, 1.0);
                FP(proj_ones.data(), img_ones.data(), iv);
                BP(img_ones.data(), proj_ones.data(), iv);
                division<T>(img_temp.data(), img_ones.data(), nx, ny, nz);
                if (with_motion && dvf_inverse > 0) {  // the engine's options.dvf_inverse
                    std::vector<T> inv(3 * nv);
                    invert_dvf<T>(inv.data(), inv.data() + nv, inv.data() + 2 * nv, al_x, al_y,
                                  al_z, be_x, be_y, be_z, volumes[iv] - volumes[0],
                                  flows[iv] - flows[0], nx, ny, nz, dvf_inverse);
                    deform_disp<T>(img1.data(), img_temp.data(), nx, ny, nz, inv.data(),
                                   inv.data() + nv, inv.data() + 2 * nv);
                    add<T>(img.data(), img1.data(), nx, ny, nz, lam);
                } else if (with_motion) {
                    DEF(img1.data(), img_temp.data(), volumes[0] - volumes[iv],
                        flows[0] - flows[iv]);
                    add<T>(img.data(), img1.data(), nx, ny, nz, lam);
                } else if (kk == 1) {
                    add<T>(img.data(), img_temp.data(), nx, ny, nz, lambda);
                } else if (iv == s0) {
                    qsum = img_temp;
                } else {
                    add<T>(qsum.data(), img_temp.data(), nx, ny, nz, 1.0);
                }
            }
                if (!with_motion && kk > 1) add<T>(img.data(), qsum.data(), nx, ny, nz, lam);
            }
        } else {  // motion update, AUMISART.cu:66-118 / :236-288
            for (int iv = 1; iv < view_hi; iv += motion_step) {
                if (iv < view_lo) continue;
                FP(proj_temp.data(), img.data(), iv);
                std::copy(h_proj + iv * np, h_proj + (iv + 1) * np, proj.begin());
                const double n0 = norm2(proj.data(), np);
                const float vd = volumes[iv] - volumes[iv - 1];
                const float fd = flows[iv] - flows[iv - 1];
                add<T>(proj.data(), proj_temp.data(), na, nb, 1, -1.0);
                initial<T>(img0.data(), nx, ny, nz, 0.0);
                add2<T>(img0.data(), al_y, nx, ny, nz, img.data(), vd, 1);
                add2<T>(img0.data(), al_x, nx, ny, nz, img.data(), vd, 2);
                add2<T>(img0.data(), al_z, nx, ny, nz, img.data(), vd, 3);
                add2<T>(img0.data(), be_y, nx, ny, nz, img.data(), fd, 1);
                add2<T>(img0.data(), be_x, nx, ny, nz, img.data(), fd, 2);
                add2<T>(img0.data(), be_z, nx, ny, nz, img.data(), fd, 3);
                FP(proj_temp.data(), img0.data(), iv);
                add<T>(proj.data(), proj_temp.data(), na, nb, 1, 1.0);
                const double n1 = norm2(proj.data(), np);
                outnorm[(int64_t)it * n_views + iv] = (T)(n1 / n0);
                BP(img_temp.data(), proj.data(), iv);
                initial2<T>(img_ones.data(), nx, ny, nz, img.data(), -vd, -fd);
                FP(proj_ones.data(), img_ones.data(), iv);
                BP(img_ones.data(), proj_ones.data(), iv);
                division<T>(img_temp.data(), img_ones.data(), nx, ny, nz);
                const float nvd = volumes[iv - 1] - volumes[iv];
                const float nfd = flows[iv - 1] - flows[iv];
                add2<T>(al_y, img_temp.data(), nx, ny, nz, img.data(), nvd, 1);
                add2<T>(al_x, img_temp.data(), nx, ny, nz, img.data(), nvd, 2);
                add2<T>(al_z, img_temp.data(), nx, ny, nz, img.data(), nvd, 3);
                add2<T>(be_y, img_temp.data(), nx, ny, nz, img.data(), nfd, 1);
                add2<T>(be_x, img_temp.data(), nx, ny, nz, img.data(), nfd, 2);
                add2<T>(be_z, img_temp.data(), nx, ny, nz, img.data(), nfd, 3);
            }
        }
    }
    std::copy(img.begin(), img.end(), outimg);
    std::copy(al_x, al_x + nv, outalphax);
    if (fields_out) std::copy(F.begin(), F.end(), fields_out);
    return 0;
}

}  // namespace

// ------------------------------------------------------------------ exports
#define ORC_DEFINE(T, P)                                                                       \
    extern "C" void P##projection(T *proj, const T *img, double angle, double SO, double SD,    \
                                  double da, int na, double ai, double db, int nb, double bi,  \
                                  int nx, int ny, int nz) {                                    \
        projection<T>(proj, img, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);           \
    }                                                                                          \
    extern "C" void P##backprojection_adjoint(T *img, const T *proj, double angle, double SO,  \
                                              double SD, double da, int na, double ai,         \
                                              double db, int nb, double bi, int nx, int ny,    \
                                              int nz) {                                        \
        backprojection_adjoint<T>(img, proj, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny,     \
                                  nz);                                                         \
    }                                                                                          \
    extern "C" void P##backprojection(T *img, const T *proj, double angle, double SO,          \
                                      double SD, double da, int na, double ai, double db,      \
                                      int nb, double bi, int nx, int ny, int nz) {             \
        backprojection<T>(img, proj, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);       \
    }                                                                                          \
    extern "C" void P##backprojection_sc(T *img, const T *proj, double cphi, double sphi,      \
                                         double SO, double SD, double da, int na, double ai,   \
                                         double db, int nb, double bi, int nx, int ny,         \
                                         int nz) {                                             \
        backprojection_sc<T>(img, proj, cphi, sphi, SO, SD, da, na, ai, db, nb, bi, nx, ny,    \
                             nz);                                                              \
    }                                                                                          \
    extern "C" void P##forward_dvf(T *mx, T *my, T *mz, const T *ax, const T *ay,              \
                                   const T *az, const T *bx, const T *by, const T *bz,         \
                                   double volume, double flow, int nx, int ny, int nz) {       \
        forward_dvf<T>(mx, my, mz, ax, ay, az, bx, by, bz, volume, flow, nx, ny, nz);          \
    }                                                                                          \
    extern "C" void P##deform(T *out, const T *img, int nx, int ny, int nz, double volume,     \
                              double flow, const T *ax, const T *ay, const T *az,              \
                              const T *bx, const T *by, const T *bz, int tex_mode) {           \
        deform<T>(out, img, nx, ny, nz, volume, flow, ax, ay, az, bx, by, bz, tex_mode);       \
    }                                                                                          \
    extern "C" void P##deform2(T *out, const T *img, int nx, int ny, int nz, double volume,    \
                               double flow, const T *ax, const T *ay, const T *az,             \
                               const T *bx, const T *by, const T *bz) {                        \
        deform2<T>(out, img, nx, ny, nz, volume, flow, ax, ay, az, bx, by, bz);                \
    }                                                                                          \
    extern "C" void P##add(T *img1, const T *img, int nx, int ny, int nz, double w) {          \
        add<T>(img1, img, nx, ny, nz, w);                                                      \
    }                                                                                          \
    extern "C" void P##add2(T *img1, const T *img, int nx, int ny, int nz, const T *img0,      \
                            double w, int ind) {                                               \
        add2<T>(img1, img, nx, ny, nz, img0, w, ind);                                          \
    }                                                                                          \
    extern "C" void P##initial(T *img, int nx, int ny, int nz, double value) {                 \
        initial<T>(img, nx, ny, nz, value);                                                    \
    }                                                                                          \
    extern "C" void P##initial2(T *img, int nx, int ny, int nz, const T *img0, double volume,  \
                                double flow) {                                                 \
        initial2<T>(img, nx, ny, nz, img0, volume, flow);                                      \
    }                                                                                          \
    extern "C" void P##division(T *img1, const T *img, int nx, int ny, int nz) {               \
        division<T>(img1, img, nx, ny, nz);                                                    \
    }                                                                                          \
    extern "C" void P##multiple(T *img1, int nx, int ny, int nz, const T *img0, double w,      \
                                int ind) {                                                     \
        multiple<T>(img1, nx, ny, nz, img0, w, ind);                                           \
    }                                                                                          \
    extern "C" void P##update_udvf(T *ax, T *ay, T *az, T *bx, T *by, T *bz, const T *img,     \
                                   const T *img0, double vd, double fd, int nx, int ny,        \
                                   int nz, int iter) {                                         \
        update_udvf<T>(ax, ay, az, bx, by, bz, img, img0, vd, fd, nx, ny, nz, iter);           \
    }                                                                                          \
    extern "C" void P##diff(T *img1, const T *img, int nx, int ny, int nz, int ind) {          \
        diff<T>(img1, img, nx, ny, nz, ind);                                                   \
    }                                                                                          \
    extern "C" int P##aumisart(                                                                \
        T *outimg, T *outproj, T *outnorm, T *outalphax, const T *img, const T *proj, int nx,  \
        int ny, int nz, int na, int nb, int outIter, int n_views, int n_iter,                  \
        const int *op_iter, double da, double db, double ai, double bi, double SO, double SD,  \
        double dx, double lambda, const float *volumes, const float *flows,                    \
        const float *angles, const T *ax, const T *ay, const T *az, const T *bx, const T *by,  \
        const T *bz, T *fields_out, int tex_mode, int view_lo, int view_hi, int subset,        \
        int dvf_inverse) {                                                                     \
        return aumisart<T>(outimg, outproj, outnorm, outalphax, img, proj, nx, ny, nz, na, nb, \
                           outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx,      \
                           lambda, volumes, flows, angles, ax, ay, az, bx, by, bz, fields_out, \
                           tex_mode, view_lo, view_hi, subset, dvf_inverse);                   \
    }                                                                                          \
    extern "C" void P##invert_dvf(T *ox, T *oy, T *oz, const T *ax, const T *ay, const T *az,  \
                                  const T *bx, const T *by, const T *bz, double volume,        \
                                  double flow, int nx, int ny, int nz, int iters) {            \
        invert_dvf<T>(ox, oy, oz, ax, ay, az, bx, by, bz, volume, flow, nx, ny, nz, iters);    \
    }

ORC_DEFINE(double, orc_)
ORC_DEFINE(float, cpu_)

extern "C" int orc_num_threads(void) { return omp_get_max_threads(); }
extern "C" void orc_set_num_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}
