// mcsart_projection_noalloc: the projector of mcsart_projection (the
// reference's host_projection, src/cu_projection.cu:7-12) with its one scratch
// buffer, the y-fastest copy of the volume that x-driven rays read, held in a
// fixed file-scope device array instead of a context workspace.  It allocates
// nothing and needs no context.  The kernels and their launch shapes are those
// of mcsart_projection, so the results are bitwise the same.
#include <cuda.h>  // CUcontext and CUresult, for the driver calls resolved below

#include <mutex>

#include "common.cuh"
#include "elementwise.cuh"
#include "projector.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {
bool view_has_xdrive(float angle, const Geom &g);  // abi_kernels.cu
}  // namespace mcsart

using namespace mcsart;

// The scratch: one y-fastest FP32 volume copy per device (16 MiB).
static __device__ __align__(256) float g_noalloc_volT[MCSART_NOALLOC_MAX_VOXELS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;

// The scratch's device address belongs to one CUDA context: each context
// that loads this library's module has its own instance of the array.  A
// cudaDeviceReset (which the reference's MEX functions call at the end of
// every call, and which may run in the same process) or a context created
// with the driver API gives the device a new context, and the address
// looked up in the old one is then invalid.  So the set-up is cached per
// device together with the unique id of the context it was done in
// (cuCtxGetId, never reused within a process), and redone when the calling
// thread's current context is another one.
struct Setup {
    unsigned long long ctx_id = 0;  // 0: not set up
    float *scratch = nullptr;       // device address of g_noalloc_volT in that context
};
Setup g_setup[kMaxDevices];

using PfnCtxGetCurrent = CUresult (*)(CUcontext *);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long *);
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;

// Driver entry points, resolved through the runtime (no link against the
// driver library); called with g_setup_mu held.
int resolve_driver_calls() {
    if (g_ctx_get_current && g_ctx_get_id) return MCSART_OK;
    void *f0 = nullptr, *f1 = nullptr;
    cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = q0;
    MC_CHECK_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000,
                                                    cudaEnableDefault, &q0));
    MC_CHECK_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault,
                                                    &q1));
    MC_REQUIRE(q0 == cudaDriverEntryPointSuccess && q1 == cudaDriverEntryPointSuccess && f0 && f1,
               "mcsart_projection_noalloc: the driver lacks cuCtxGetCurrent/cuCtxGetId");
    g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f0);
    g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f1);
    return MCSART_OK;
}

// Id of the calling thread's current context (called with g_setup_mu held).
int current_context_id(unsigned long long *id) {
    CUcontext c = nullptr;
    MC_REQUIRE(g_ctx_get_current(&c) == CUDA_SUCCESS && c != nullptr,
               "mcsart_projection_noalloc: no current CUDA context");
    MC_REQUIRE(g_ctx_get_id(c, id) == CUDA_SUCCESS && *id != 0,
               "mcsart_projection_noalloc: cuCtxGetId failed");
    return MCSART_OK;
}

// Set-up on the first call per device and context, with that device
// current: the scratch's address (cudaGetSymbolAddress, which also makes the
// runtime's context current), and both kernels loaded so that later calls
// load nothing.  Later calls in the same context only compare the id.
int scratch_of_current_device(float **out) {
    int dev = -1;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
        set_error("mcsart_projection_noalloc: no CUDA device (%s)", cudaGetErrorString(e));
        return MCSART_ERR_NO_DEVICE;
    }
    MC_CHECK_CUDA(e);
    MC_REQUIRE(dev >= 0 && dev < kMaxDevices,
               "mcsart_projection_noalloc: device ordinal %d above %d", dev, kMaxDevices - 1);
    std::lock_guard<std::mutex> lock(g_setup_mu);
    MC_TRY(resolve_driver_calls());
    Setup &s = g_setup[dev];
    if (s.ctx_id != 0) {
        unsigned long long id = 0;
        MC_TRY(current_context_id(&id));
        if (id == s.ctx_id) {
            *out = s.scratch;
            return MCSART_OK;
        }
    }
    void *p = nullptr;
    MC_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_volT));
    cudaFuncAttributes fa;
    MC_CHECK_CUDA(cudaFuncGetAttributes(&fa, transpose_kernel<float, float>));
    MC_CHECK_CUDA(cudaFuncGetAttributes(&fa, fp_ref_kernel<1, false, float>));
    unsigned long long id = 0;
    MC_TRY(current_context_id(&id));
    s.ctx_id = id;
    s.scratch = static_cast<float *>(p);
    *out = s.scratch;
    return MCSART_OK;
}

}  // namespace

MC_EXPORT int mcsart_projection_noalloc(void *stream, float *d_proj, const float *d_img,
                                        float angle, float SO, float SD, float da, int na,
                                        float ai, float db, int nb, float bi, int nx, int ny,
                                        int nz) {
    clear_error();
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    Geom g;
    g.SO = SO; g.SD = SD; g.da = da; g.ai = ai; g.db = db; g.bi = bi;
    g.na = na; g.nb = nb; g.nx = nx; g.ny = ny; g.nz = nz;
    MC_TRY(validate_geom(g));
    const int64_t n = nvox(nx, ny, nz);
    MC_REQUIRE(n <= MCSART_NOALLOC_MAX_VOXELS,
               "mcsart_projection_noalloc: the volume has %lld voxels, more than the %d its "
               "static scratch holds (use mcsart_projection)",
               (long long)n, MCSART_NOALLOC_MAX_VOXELS);
    float *scratch = nullptr;
    MC_TRY(scratch_of_current_device(&scratch));
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    const float *imgT = nullptr;
    if (view_has_xdrive(angle, g)) {
        const dim3 grid(div_up(nx, 32), div_up(ny, 32), nz), block(32, 8);
        transpose_kernel<float, float><<<grid, block, 0, s>>>(scratch, d_img, nx, ny);
        MC_CHECK_CUDA(cudaGetLastError());
        imgT = scratch;
    }
    FPArgs<float, 1> a{};
    a.vol.std[0] = d_img;
    a.vol.tr[0] = imgT;
    a.g = g;
    a.angle = angle;
    a.angles = nullptr;
    a.mode = FP_PLAIN;
    a.out = d_proj;
    const dim3 grid(div_up(na, FPC_COLS), div_up(nb, FPC_ROWS), 1);
    fp_ref_kernel<1, false, float><<<grid, dim3(FPC_THREADS), 0, s>>>(a);
    MC_CHECK_CUDA(cudaGetLastError());
    return MCSART_OK;
}
