// Context, error reporting and workspaces of the C ABI.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "sart.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {

static thread_local char g_last_error[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

void clear_error() { g_last_error[0] = '\0'; }

int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("launch of %s failed: %s", what, cudaGetErrorString(e));
        return MCSART_ERR_CUDA;
    }
    return MCSART_OK;
}

int validate_ctx(mcsart_ctx *ctx) {
    MC_REQUIRE(ctx != nullptr, "context is NULL");
    MC_CHECK_CUDA(cudaSetDevice(ctx->device));
    return MCSART_OK;
}

int workspace(mcsart_ctx *ctx, const char *name, size_t bytes, void **out) {
    auto &b = ctx->ws[name];
    if (b.bytes < bytes) {
        if (b.ptr) {
            MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
            MC_CHECK_CUDA(cudaFree(b.ptr));
            b.ptr = nullptr;
            b.bytes = 0;
        }
        const cudaError_t e = cudaMalloc(&b.ptr, bytes);
        if (e != cudaSuccess) {
            b.ptr = nullptr;
            set_error("workspace '%s' of %zu bytes: %s", name, bytes, cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? MCSART_ERR_OUT_OF_MEMORY : MCSART_ERR_CUDA;
        }
        b.bytes = bytes;
    }
    *out = b.ptr;
    return MCSART_OK;
}

int finish(mcsart_ctx *ctx, const char *what) {
    if (ctx->synchronous) {
        const cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            set_error("%s: %s", what, cudaGetErrorString(e));
            return MCSART_ERR_CUDA;
        }
    }
    return MCSART_OK;
}

int validate_dims(int nx, int ny, int nz) {
    MC_REQUIRE(nx > 0 && ny > 0 && nz > 0, "volume dimensions must be positive (got %d x %d x %d)",
               nx, ny, nz);
    MC_REQUIRE(nvox(nx, ny, nz) < (int64_t)1 << 31, "volume of %lld voxels is too large",
               (long long)nvox(nx, ny, nz));
    return MCSART_OK;
}

int validate_geom(const Geom &g) {
    MC_TRY(validate_dims(g.nx, g.ny, g.nz));
    MC_REQUIRE(g.na > 0 && g.nb > 0, "detector dimensions must be positive (got %d x %d)", g.na,
               g.nb);
    MC_REQUIRE((int64_t)g.na * g.nb < (int64_t)1 << 31, "detector too large");
    // the projector converts slab indices with the magic-number conversion,
    // exact below 2^22
    const int lim = 1 << 20;
    MC_REQUIRE(g.nx <= lim && g.ny <= lim && g.nz <= lim && g.na <= lim && g.nb <= lim,
               "volume and detector dimensions must be at most 2^20");
    // kernels index slices (nz) and detector rows (nb) with a grid dimension,
    // whose limit is 65535
    MC_REQUIRE(g.nz <= 65535, "volume depth nz must be at most 65535 (got %d)", g.nz);
    MC_REQUIRE(g.nb <= 65535, "detector rows nb must be at most 65535 (got %d)", g.nb);
    MC_REQUIRE(g.SO > 0.0f && g.SD > 0.0f, "SO and SD must be positive");
    MC_REQUIRE(g.da > 0.0f && g.db > 0.0f, "detector pitches da, db must be positive");
    return MCSART_OK;
}

int TexVol::ensure(int x, int y, int z) {
    if (arr && nx == x && ny == y && nz == z) return MCSART_OK;
    release();
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    MC_CHECK_CUDA(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(x, y, z), cudaArraySurfaceLoadStore));
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    MC_CHECK_CUDA(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    MC_CHECK_CUDA(cudaCreateSurfaceObject(&surf, &rd));
    nx = x;
    ny = y;
    nz = z;
    return MCSART_OK;
}

int TexVol::upload(const float *src, cudaStream_t st) {
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr((void *)src, (size_t)nx * sizeof(float), nx, ny);
    cp.dstArray = arr;
    cp.extent = make_cudaExtent(nx, ny, nz);
    cp.kind = cudaMemcpyDeviceToDevice;
    MC_CHECK_CUDA(cudaMemcpy3DAsync(&cp, st));
    return MCSART_OK;
}

void TexVol::release() {
    if (tex) cudaDestroyTextureObject(tex);
    if (surf) cudaDestroySurfaceObject(surf);
    if (arr) cudaFreeArray(arr);
    tex = 0;
    surf = 0;
    arr = nullptr;
    nx = ny = nz = 0;
}

static cudaEvent_t pool_event(mcsart_ctx *ctx) {
    if (!ctx->prof_pool.empty()) {
        cudaEvent_t e = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

int prof_before(mcsart_ctx *ctx, const char *name) {
    mcsart_ctx::ProfRec r;
    r.name = ctx->label ? ctx->label : name;
    r.e0 = pool_event(ctx);
    r.e1 = pool_event(ctx);
    MC_CHECK_CUDA(cudaEventRecord(r.e0, ctx->stream));
    ctx->prof_pending.push_back(r);
    return MCSART_OK;
}

int prof_after(mcsart_ctx *ctx) {
    MC_CHECK_CUDA(cudaEventRecord(ctx->prof_pending.back().e1, ctx->stream));
    return MCSART_OK;
}

// Folds the recorded launches into the per-name table.
static int prof_collect(mcsart_ctx *ctx) {
    MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto &r : ctx->prof_pending) {
        float ms = 0.0f;
        MC_CHECK_CUDA(cudaEventElapsedTime(&ms, r.e0, r.e1));
        std::string name(r.name);
        auto it = ctx->prof_table.begin();
        for (; it != ctx->prof_table.end(); ++it)
            if (it->first == name) break;
        if (it == ctx->prof_table.end()) {
            ctx->prof_table.emplace_back(name, mcsart_ctx::ProfAgg());
            it = ctx->prof_table.end() - 1;
        }
        it->second.launches++;
        it->second.ms += ms;
        ctx->prof_pool.push_back(r.e0);
        ctx->prof_pool.push_back(r.e1);
    }
    ctx->prof_pending.clear();
    return MCSART_OK;
}

}  // namespace mcsart

mcsart_ctx::~mcsart_ctx() {
    lanes.clear();
    for (auto e : lane_done) cudaEventDestroy(e);
    if (batch_start) cudaEventDestroy(batch_start);
    for (auto &r : prof_pending) {
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
    }
    for (auto e : prof_pool) cudaEventDestroy(e);
    driver.reset();
    for (auto &kv : ws)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
    if (own_stream) cudaStreamDestroy(own_stream);
}

using namespace mcsart;

MC_EXPORT int mcsart_version(void) { return MCSART_VERSION; }

MC_EXPORT const char *mcsart_last_error(void) { return g_last_error; }

MC_EXPORT int mcsart_create(mcsart_ctx **out, int device) {
    clear_error();
    MC_REQUIRE(out != nullptr, "output pointer is NULL");
    *out = nullptr;
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error("no CUDA device available (%s)", cudaGetErrorString(e));
        return MCSART_ERR_NO_DEVICE;
    }
    MC_REQUIRE(device >= 0 && device < n, "device %d out of range [0, %d)", device, n);
    MC_CHECK_CUDA(cudaSetDevice(device));
    int sms = 0;
    MC_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    auto *ctx = new mcsart_ctx();
    ctx->device = device;
    ctx->sms = sms;
    const cudaError_t es = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (es != cudaSuccess) {
        delete ctx;
        set_error("cudaStreamCreate: %s", cudaGetErrorString(es));
        return MCSART_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return MCSART_OK;
}

MC_EXPORT int mcsart_destroy(mcsart_ctx *ctx) {
    clear_error();
    if (!ctx) return MCSART_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
    return MCSART_OK;
}

MC_EXPORT int mcsart_set_stream(mcsart_ctx *ctx, void *stream) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    ctx->stream = (cudaStream_t)stream;  // NULL: the legacy default stream
    if (ctx->driver) ctx->driver->invalidate_graphs();
    return MCSART_OK;
}

MC_EXPORT void *mcsart_get_stream(mcsart_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

MC_EXPORT int mcsart_set_synchronous(mcsart_ctx *ctx, int on) {
    clear_error();
    MC_REQUIRE(ctx != nullptr, "context is NULL");
    ctx->synchronous = on ? 1 : 0;
    return MCSART_OK;
}

MC_EXPORT int mcsart_set_interp(mcsart_ctx *ctx, int interp) {
    clear_error();
    MC_REQUIRE(ctx != nullptr, "context is NULL");
    MC_REQUIRE(interp == MCSART_INTERP_TEXTURE || interp == MCSART_INTERP_EXACT,
               "unknown interpolation model %d", interp);
    ctx->interp = interp;
    return MCSART_OK;
}

MC_EXPORT int mcsart_synchronize(mcsart_ctx *ctx) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    return MCSART_OK;
}

MC_EXPORT long long mcsart_launch_count(mcsart_ctx *ctx) { return ctx ? ctx->launches : -1; }

MC_EXPORT int mcsart_profile_begin(mcsart_ctx *ctx) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    ctx->prof_table.clear();
    ctx->profiling = true;
    return MCSART_OK;
}

MC_EXPORT int mcsart_profile_end(mcsart_ctx *ctx) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    ctx->profiling = false;
    return prof_collect(ctx);
}

MC_EXPORT int mcsart_profile_count(mcsart_ctx *ctx) {
    return ctx ? (int)ctx->prof_table.size() : -1;
}

MC_EXPORT int mcsart_profile_entry(mcsart_ctx *ctx, int i, char *name, int name_len,
                                   long long *launches, double *total_ms) {
    clear_error();
    MC_REQUIRE(ctx != nullptr, "context is NULL");
    MC_REQUIRE(i >= 0 && i < (int)ctx->prof_table.size(), "profile entry %d out of range", i);
    const auto &e = ctx->prof_table[i];
    if (name && name_len > 0) snprintf(name, (size_t)name_len, "%s", e.first.c_str());
    if (launches) *launches = e.second.launches;
    if (total_ms) *total_ms = e.second.ms;
    return MCSART_OK;
}
