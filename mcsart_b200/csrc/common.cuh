// Internal definitions shared by the engine's translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "mcsart.h"

namespace mcsart {

// ------------------------------------------------------------------ errors
void set_error(const char *fmt, ...);
void clear_error();

#define MC_CHECK_CUDA(expr)                                                                     \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            ::mcsart::set_error("%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__,      \
                                __LINE__);                                                      \
            return MCSART_ERR_CUDA;                                                             \
        }                                                                                       \
    } while (0)

#define MC_REQUIRE(cond, ...)                                                                   \
    do {                                                                                        \
        if (!(cond)) {                                                                          \
            ::mcsart::set_error(__VA_ARGS__);                                                   \
            return MCSART_ERR_INVALID_ARGUMENT;                                                 \
        }                                                                                       \
    } while (0)

#define MC_TRY(expr)                                                                            \
    do {                                                                                        \
        int rc_ = (expr);                                                                       \
        if (rc_ != MCSART_OK) return rc_;                                                       \
    } while (0)

// Status after a kernel launch (configuration errors surface here).
int check_launch(const char *what);

struct DriverState;  // sart.cu

// Launch shapes of the driver's per-view kernels (mcsart_autotune).  Each
// field indexes the variant table of its kernel (tuning.cu); -1 selects the
// built-in choice.  Every variant computes every ray and voxel with the same
// operations in the same order, so the results do not depend on the choice.
struct Tuning {
    int fp1 = -1;   // one-volume projector (image passes): slab group depth, blocks per SM
    int fp3 = -1;   // three-volume projector (DVF-update passes)
    int bp = -1;    // backprojector: voxels per thread along z, voxel rows per block
    int warp = -1;  // image-pass warps: voxel rows per thread
    int fup = -1;   // DVF-pass field update + prep: field loads voxel by voxel or early
};

}  // namespace mcsart

struct mcsart_ctx {
    // per-kernel timing (mcsart_profile_begin/end): events around each launch
    struct ProfRec {
        const char *name;
        cudaEvent_t e0, e1;
    };
    struct ProfAgg {
        long long launches = 0;
        double ms = 0.0;
    };
    bool profiling = false;
    const char *label = nullptr;  // name of the next launch (else the kernel expression)
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    std::vector<std::pair<std::string, ProfAgg>> prof_table;
    int device = 0;
    int sms = 0;  // the device's SM count
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int synchronous = 0;
    int interp = MCSART_INTERP_TEXTURE;
    long long launches = 0;
    struct Buf {
        void *ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> ws;  // named device workspaces, grown on demand
    std::unique_ptr<mcsart::DriverState> driver;
    // mcsart_batch_run: one lane (child context with its own stream, buffers
    // and pass graphs) per concurrently running problem, and the events that
    // order the lanes against this context's stream
    std::vector<std::unique_ptr<mcsart_ctx>> lanes;
    std::vector<cudaEvent_t> lane_done;
    cudaEvent_t batch_start = nullptr;
    // tuned launch shapes per geometry and storage type (mcsart_autotune,
    // mcsart_tuning_load), keyed by tuning_key()
    std::map<std::string, mcsart::Tuning> tuning;
    // set while the tuner times a trial: the shapes every launch uses
    const mcsart::Tuning *tuning_override = nullptr;
    ~mcsart_ctx();
};

namespace mcsart {

// Device workspace `name` of at least `bytes` (contents undefined).
int workspace(mcsart_ctx *ctx, const char *name, size_t bytes, void **out);
// Called after enqueuing work: synchronises in synchronous mode.
int finish(mcsart_ctx *ctx, const char *what);
int validate_ctx(mcsart_ctx *ctx);

// ------------------------------------------------------------ geometry
struct Geom {
    float SO, SD, da, ai, db, bi;
    int na, nb, nx, ny, nz;
};

// Correctly rounded a / b without the slow-path branch of the compiler's
// division, for the operand ranges of the projector and backprojector.
// Method: P. W. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990: the hardware
// reciprocal seed (rcp.approx) refined by one Newton-Raphson step gives
// y = RN(1/b), and q = RN(a y) corrected by the exact residual r = a - b q
// gives RN(a/b) (Markstein's theorem; a, b and the quotient normal).  y was
// checked against __frcp_rn for every significand of b with exponents -20 to
// 19, and the quotient against __fdiv_rn on 2.2e10 operand pairs, with no
// difference.  mk_den_ok / mk_num_ok bound the operands to that range; the
// callers take __fdiv_rn (or '/') outside it.
__device__ __forceinline__ float mk_recip(float b) {
    float y0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(b));
    const float e = __fmaf_rn(-b, y0, 1.0f);
    return __fmaf_rn(y0, e, y0);
}
__device__ __forceinline__ float mk_div(float a, float b, float y) {
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-b, q0, a);
    return __fmaf_rn(r, y, q0);
}
__device__ __forceinline__ bool mk_den_ok(float b) {
    const float m = fabsf(b);
    return m >= 0x1p-20f && m < 0x1p20f;
}
// +0 is fine; -0 is not: the correction step returns +0 for -0 / b, b > 0,
// where the compiler's division returns -0.
__device__ __forceinline__ bool mk_num_ok(float a) {
    const float m = fabsf(a);
    return __float_as_uint(a) == 0u || (m >= 0x1p-80f && m <= 0x1p80f);
}

// floor to int and int to float on the FMA and integer pipes instead of the
// conversion unit (which the projector otherwise keeps busy), exact for
// |x| < 2^22: the floats in [2^23, 2^24) are the integers, so x + 1.5*2^23
// rounded toward -inf is 1.5*2^23 + floor(x), whose low significand bits are
// floor(x) + 2^22 (the magic-number conversion).  Callers keep their
// arguments inside the range.
constexpr float MK_MAGIC = 12582912.0f;  // 1.5 * 2^23
constexpr int MK_MAGIC_BITS = 0x4B400000;
constexpr float MK_MAGIC_RANGE = 4194304.0f;  // 2^22
// (the subtraction is unsigned: out of range it wraps instead of overflowing)
__device__ __forceinline__ int mk_floor_i(float x) {
    return (int)(__float_as_uint(__fadd_rd(x, MK_MAGIC)) - (unsigned)MK_MAGIC_BITS);
}
// floor(x) as an int and as a float
__device__ __forceinline__ int mk_floor(float x, float &fl) {
    const float t = __fadd_rd(x, MK_MAGIC);
    fl = __fsub_rn(t, MK_MAGIC);
    return (int)(__float_as_uint(t) - (unsigned)MK_MAGIC_BITS);
}
__device__ __forceinline__ float mk_i2f(int i) {
    return __fsub_rn(__int_as_float(MK_MAGIC_BITS + i), MK_MAGIC);
}

// The value the reference's backprojector reads for a projection cell: it
// samples a linear-filtered float texture at the texel's centre
// (src/cu_backprojection.cu:28-33,167), which returns the texel itself except
// that a denormal texel reads as a zero of the same sign (measured on B200
// for every sign and magnitude class).  The engine reads projections from
// memory and applies this where the reference's read happens.
__device__ __forceinline__ float tex_texel(float v) {
    return fabsf(v) < 0x1p-126f ? copysignf(0.0f, v) : v;
}

__host__ __device__ inline int64_t nvox(int nx, int ny, int nz) { return (int64_t)nx * ny * nz; }

int validate_geom(const Geom &g);
int validate_dims(int nx, int ny, int nz);

// -------------------------------------------------------- storage types
// Loads through the read-only data cache: every array read with ldv is
// either not written during the kernel or read and written at one index by
// one thread only.
template <typename T> __device__ __forceinline__ float ldv(const T *p, int64_t i);
template <> __device__ __forceinline__ float ldv<float>(const float *p, int64_t i) {
    return __ldg(p + i);
}
template <> __device__ __forceinline__ float ldv<__nv_bfloat16>(const __nv_bfloat16 *p, int64_t i) {
    return __bfloat162float(__ldg(p + i));
}
template <> __device__ __forceinline__ float ldv<__half>(const __half *p, int64_t i) {
    return __half2float(__ldg(p + i));
}
// Two consecutive storage-type values p[2i], p[2i+1] (8-byte aligned for
// FP32) as one load.
template <typename T> __device__ __forceinline__ float2 ldv2(const T *p, int64_t i);
template <> __device__ __forceinline__ float2 ldv2<float>(const float *p, int64_t i) {
    return __ldg(reinterpret_cast<const float2 *>(p) + i);
}
template <>
__device__ __forceinline__ float2 ldv2<__nv_bfloat16>(const __nv_bfloat16 *p, int64_t i) {
    return __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162 *>(p) + i));
}
template <> __device__ __forceinline__ float2 ldv2<__half>(const __half *p, int64_t i) {
    return __half22float2(__ldg(reinterpret_cast<const __half2 *>(p) + i));
}
// Stores (a, b) at p[2i], p[2i+1] as one two-element store.
__device__ __forceinline__ void stv2(float *p, int64_t i, float a, float b) {
    reinterpret_cast<float2 *>(p)[i] = make_float2(a, b);
}
__device__ __forceinline__ void stv2(__nv_bfloat16 *p, int64_t i, float a, float b) {
    reinterpret_cast<__nv_bfloat162 *>(p)[i] = __floats2bfloat162_rn(a, b);
}
__device__ __forceinline__ void stv2(__half *p, int64_t i, float a, float b) {
    reinterpret_cast<__half2 *>(p)[i] = __floats2half2_rn(a, b);
}

// A storage-type value as float (a value, not a load).
__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float tof(__half v) { return __half2float(v); }
template <typename T> __device__ __forceinline__ T cvt(float v);
template <> __device__ __forceinline__ float cvt<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 cvt<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}
template <> __device__ __forceinline__ __half cvt<__half>(float v) { return __float2half_rn(v); }

// ------------------------------------------------- trilinear sampling
// Source of a trilinear gather.  SrcTex samples a 3D texture with hardware
// linear filtering and clamp addressing, exactly the configuration the
// reference builds for its warp (src/cu_deform.cu:25-38); SrcLinear samples
// a linear x-fastest volume in software with full FP32 weights (the EXACT
// model).  Coordinates are unnormalised texture coordinates (texel centres at
// i + 0.5).
struct SrcTex {
    cudaTextureObject_t tex;
    __device__ __forceinline__ float fetch(float x, float y, float z, int, int, int) const {
        return tex3D<float>(tex, x, y, z);
    }
};

__device__ __forceinline__ void lin_axis(float x, int n, int &i0, int &i1, float &w) {
    const float xb = x - 0.5f;
    const float fl = floorf(xb);
    w = xb - fl;
    // clamp in float first so that far-out coordinates cannot overflow the conversion
    const int i = (int)fminf(fmaxf(fl, -1.0f), (float)n);
    i0 = min(max(i, 0), n - 1);
    i1 = min(max(i + 1, 0), n - 1);
}

template <typename T> struct SrcLinear {
    const T *p;
    __device__ __forceinline__ float fetch(float x, float y, float z, int nx, int ny,
                                           int nz) const {
        int x0, x1, y0, y1, z0, z1;
        float a, b, c;
        lin_axis(x, nx, x0, x1, a);
        lin_axis(y, ny, y0, y1, b);
        lin_axis(z, nz, z0, z1, c);
        const int64_t sy = nx, sz = (int64_t)nx * ny;
        const int64_t r00 = y0 * sy + z0 * sz, r10 = y1 * sy + z0 * sz;
        const int64_t r01 = y0 * sy + z1 * sz, r11 = y1 * sy + z1 * sz;
        const float t000 = ldv(p, x0 + r00), t100 = ldv(p, x1 + r00);
        const float t010 = ldv(p, x0 + r10), t110 = ldv(p, x1 + r10);
        const float t001 = ldv(p, x0 + r01), t101 = ldv(p, x1 + r01);
        const float t011 = ldv(p, x0 + r11), t111 = ldv(p, x1 + r11);
        // lerps along x, then y, then z
        const float c00 = fmaf(a, t100 - t000, t000), c10 = fmaf(a, t110 - t010, t010);
        const float c01 = fmaf(a, t101 - t001, t001), c11 = fmaf(a, t111 - t011, t011);
        const float c0 = fmaf(b, c10 - c00, c00), c1 = fmaf(b, c11 - c01, c01);
        return fmaf(c, c1 - c0, c0);
    }
};

// 3D array with texture (linear filtering, clamp) and surface views, used as
// the source of hardware-filtered warps.
struct TexVol {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    cudaSurfaceObject_t surf = 0;
    int nx = 0, ny = 0, nz = 0;
    int ensure(int nx, int ny, int nz);
    int upload(const float *src, cudaStream_t st);  // linear x-fastest volume -> array
    void release();
    ~TexVol() { release(); }
};

// Counted launch on the context stream.
int prof_before(mcsart_ctx *ctx, const char *name);
int prof_after(mcsart_ctx *ctx);

// Counted (and, while profiling, event-timed) launch on the context stream.
#define MC_LAUNCH(ctx, kernel, grid, block, smem, ...)                                          \
    do {                                                                                        \
        if ((ctx)->profiling) MC_TRY(::mcsart::prof_before((ctx), #kernel));                    \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);                        \
        (ctx)->launches++;                                                                      \
        MC_TRY(::mcsart::check_launch(#kernel));                                                \
        if ((ctx)->profiling) MC_TRY(::mcsart::prof_after(ctx));                                \
        (ctx)->label = nullptr;                                                                 \
    } while (0)

inline unsigned div_up(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace mcsart
