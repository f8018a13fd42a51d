// mcsart_projection_noalloc: the projector of mcsart_projection (the
// reference's host_projection, src/cu_projection.cu:7-12) with its one scratch
// buffer, the y-fastest copy of the volume that x-driven rays read, held in a
// fixed file-scope device array instead of a context workspace.  It allocates
// nothing and needs no context.  The kernels and their launch shapes are those
// of mcsart_projection, so the results are bitwise the same.
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
float *g_scratch[kMaxDevices];  // device address of g_noalloc_volT, per device

// Set-up on first use per device, with that device current: the scratch's
// address, and both kernels loaded so that later calls load nothing.
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
    if (g_scratch[dev] == nullptr) {
        void *p = nullptr;
        MC_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_volT));
        cudaFuncAttributes fa;
        MC_CHECK_CUDA(cudaFuncGetAttributes(&fa, transpose_kernel<float, float>));
        MC_CHECK_CUDA(cudaFuncGetAttributes(&fa, fp_ref_kernel<1, false, float>));
        g_scratch[dev] = static_cast<float *>(p);
    }
    *out = g_scratch[dev];
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
