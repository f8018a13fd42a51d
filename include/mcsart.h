/* mcsart.h - C ABI of the B200-native McSART engine (libmcsart.so).
 *
 * Motion-compensated SART cone-beam CT reconstruction with the 5DCT breathing
 * model d(x,t) = a(t) v(x) + b(t) f(x), as in bill52547/McSART ("AUMISART").
 *
 * Every kernel-level entry point replaces one reference launcher and keeps its
 * argument meaning and order; the reference file:line is given beside each.
 * Differences from the reference at this boundary:
 *   - a context argument comes first (stream, workspaces, cached graphs);
 *   - every function returns an int status (MCSART_OK or a negative code) and
 *     mcsart_last_error() describes the failure (the reference returns void and
 *     checks nothing);
 *   - work is stream-ordered on the context's stream; call mcsart_synchronize
 *     (or set synchronous mode) where the reference relied on its
 *     cudaDeviceSynchronize after every launch.
 *
 * Layouts are the reference's: volumes img[ix + iy*nx + iz*nx*ny] (MATLAB
 * nx x ny x nz), projections proj[ia + ib*na (+ v*na*nb)].  Geometry is in voxel
 * units (SO = SAD/dx, SD = SDD/dx, da = pitch_a/dx, db = pitch_b/dx) with ai,
 * bi already shifted by -(n/2 - 0.5) (src/entry_AUMISART.cu:76-94).
 * Pointers named d_* are device pointers, h_* host pointers.
 */
#ifndef MCSART_H
#define MCSART_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCSART_VERSION 10000 /* 1.0.0 */

/* status codes */
#define MCSART_OK 0
#define MCSART_ERR_INVALID_ARGUMENT (-1)
#define MCSART_ERR_CUDA (-2)
#define MCSART_ERR_NO_DEVICE (-3)
#define MCSART_ERR_OUT_OF_MEMORY (-4)
#define MCSART_ERR_UNSUPPORTED (-5)

/* storage types of volumes, DVF fields and projections in the engine's own
 * driver (arithmetic is FP32 in every mode) */
typedef enum { MCSART_F32 = 0, MCSART_BF16 = 1, MCSART_F16 = 2 } mcsart_dtype;

/* trilinear interpolation model of the warp */
typedef enum {
    /* the reference's hardware linear texture filtering: fractional weights
     * carried with 8 bits (src/cu_deform.cu:29-38,89) */
    MCSART_INTERP_TEXTURE = 0,
    /* full FP32 trilinear weights */
    MCSART_INTERP_EXACT = 1
} mcsart_interp;

typedef struct mcsart_ctx mcsart_ctx;

/* ------------------------------------------------------------- context */
int mcsart_version(void);
/* Description of the last failure on the calling thread ("" if none). */
const char *mcsart_last_error(void);
/* Create a context on CUDA device `device` with its own non-blocking stream. */
int mcsart_create(mcsart_ctx **ctx, int device);
int mcsart_destroy(mcsart_ctx *ctx);
/* Enqueue on an external cudaStream_t from now on; NULL selects the legacy
 * default stream (the one torch uses unless told otherwise).  A new context
 * starts on its own non-blocking stream. */
int mcsart_set_stream(mcsart_ctx *ctx, void *cuda_stream);
void *mcsart_get_stream(mcsart_ctx *ctx);
/* Non-zero: every entry point synchronises before returning (reference
 * behaviour, src/cu_*.cu call cudaDeviceSynchronize after each launch). */
int mcsart_set_synchronous(mcsart_ctx *ctx, int on);
int mcsart_synchronize(mcsart_ctx *ctx);
/* Warp model for mcsart_deform and the drivers (default TEXTURE). */
int mcsart_set_interp(mcsart_ctx *ctx, int interp);
/* Number of this library's kernels launched through ctx so far. */
long long mcsart_launch_count(mcsart_ctx *ctx);
/* Per-kernel timing: between begin and end every launch is bracketed by CUDA
 * events on the context stream (CUDA graphs are bypassed meanwhile); end
 * synchronises and fills a table of (kernel name, launches, total ms). */
int mcsart_profile_begin(mcsart_ctx *ctx);
int mcsart_profile_end(mcsart_ctx *ctx);
int mcsart_profile_count(mcsart_ctx *ctx);
int mcsart_profile_entry(mcsart_ctx *ctx, int i, char *name, int name_len, long long *launches,
                         double *total_ms);

/* ------------------------------------------------- kernel-level (device) */
/* replaces host_projection, include/cu_projection.h:7 (src/cu_projection.cu:7) */
int mcsart_projection(mcsart_ctx *ctx, float *d_proj, const float *d_img, float angle, float SO,
                      float SD, float da, int na, float ai, float db, int nb, float bi, int nx,
                      int ny, int nz);
/* replaces host_backprojection, include/cu_backprojection.h:7 (src/cu_backprojection.cu:8) */
int mcsart_backprojection(mcsart_ctx *ctx, float *d_img, const float *d_proj, float angle,
                          float SO, float SD, float da, int na, float ai, float db, int nb,
                          float bi, int nx, int ny, int nz);
/* The exact adjoint (transpose) of mcsart_projection, same arguments as
 * mcsart_backprojection (d_img is overwritten).  No counterpart in the
 * reference: its backprojector (src/cu_backprojection.cu) is a different
 * operator, not the projector's transpose.  Deterministic gather with the
 * projector's own weights; <mcsart_projection(x), y> = <x, adjoint(y)> up to
 * FP32 rounding of the sums. */
int mcsart_backprojection_adjoint(mcsart_ctx *ctx, float *d_img, const float *d_proj,
                                  float angle, float SO, float SD, float da, int na, float ai,
                                  float db, int nb, float bi, int nx, int ny, int nz);
/* replaces host_deform, include/cu_deform.h:8 (src/cu_deform.cu:3); d_img1 may
 * equal d_img */
int mcsart_deform(mcsart_ctx *ctx, float *d_img1, const float *d_img, int nx, int ny, int nz,
                  float volume, float flow, const float *alpha_x, const float *alpha_y,
                  const float *alpha_z, const float *beta_x, const float *beta_y,
                  const float *beta_z);
/* replaces host_deform2, include/cu_deform.h:9 (src/cu_deform.cu:49) */
int mcsart_deform2(mcsart_ctx *ctx, float *d_img1, const float *d_img, int nx, int ny, int nz,
                   float volume, float flow, const float *alpha_x, const float *alpha_y,
                   const float *alpha_z, const float *beta_x, const float *beta_y,
                   const float *beta_z);
/* replaces kernel_forwardDVF, include/cu_deform.h:10 (src/cu_deform.cu:66) */
int mcsart_forward_dvf(mcsart_ctx *ctx, float *mx, float *my, float *mz, const float *alpha_x,
                       const float *alpha_y, const float *alpha_z, const float *beta_x,
                       const float *beta_y, const float *beta_z, float volume, float flow,
                       int nx, int ny, int nz);
/* The inverse of the warp's displacement m = alpha*volume + beta*flow (as
 * computed by mcsart_forward_dvf), for square slices: a fixed-point iteration
 * n(q) = -D(q + n(q)) from n = 0, n_iter steps, exact FP32 trilinear samples,
 * written in the layout of mcsart_forward_dvf (inv_x, inv_y, inv_z), so that
 * warping with it undoes the warp with m.  The reference approximates the
 * inverse by negating volume and flow (src/AUMISART.cu:222); a fixed-point
 * inverse appears only in its unused waste/kernel_invertDVF.cu. */
int mcsart_invert_dvf(mcsart_ctx *ctx, float *inv_x, float *inv_y, float *inv_z,
                      const float *alpha_x, const float *alpha_y, const float *alpha_z,
                      const float *beta_x, const float *beta_y, const float *beta_z, float volume,
                      float flow, int nx, int ny, int nz, int n_iter);
/* replaces host_add, include/cu_add.h:4 (src/cu_add.cu:2) */
int mcsart_add(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz,
               float weight);
/* replaces host_add2, include/cu_add.h:8 (src/cu_add.cu:20) */
int mcsart_add2(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz,
                const float *img0, float weight, int ind);
/* replaces host_initial, include/cu_initial.h:5 (src/cu_initial.cu:2) */
int mcsart_initial(mcsart_ctx *ctx, float *img, int nx, int ny, int nz, float value);
/* replaces host_initial2, include/cu_initial.h:8 (src/cu_initial.cu:20) */
int mcsart_initial2(mcsart_ctx *ctx, float *img, int nx, int ny, int nz, const float *img0,
                    float volume, float flow);
/* replaces host_division, include/cu_division.h:5 (src/cu_division.cu:2) */
int mcsart_division(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz);
/* replaces host_multiple, include/cu_multiple.h:4 (src/cu_multiple.cu:2) */
int mcsart_multiple(mcsart_ctx *ctx, float *img1, int nx, int ny, int nz, const float *img0,
                    float weight, int ind);
/* replaces host_update_udvf, include/cu_update_udvf.h:8 (src/cu_update_udvf.cu:3) */
int mcsart_update_udvf(mcsart_ctx *ctx, float *alpha_x, float *alpha_y, float *alpha_z,
                       float *beta_x, float *beta_y, float *beta_z, const float *img,
                       const float *img0, float volume_diff, float flow_diff, int nx, int ny,
                       int nz, int iter);
/* replaces host_diff, src/mex_diff.cu:67 (the mex_diff gateway's kernel) */
int mcsart_diff(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz, int ind);
/* replaces the cublasSnrm2 calls of src/AUMISART.cu:48,51 (FP64 accumulation);
 * writes the norm to *h_result after synchronising */
int mcsart_snrm2(mcsart_ctx *ctx, int n, const float *d_x, float *h_result);

/* ---------------------------------------------------- batched projector */
/* All n_views views of one volume in a single launch:
 * d_proj[v*na*nb + ia + ib*na] = FP(d_img, h_angles[v]).  Same operator as
 * mcsart_projection per view. */
int mcsart_projection_views(mcsart_ctx *ctx, float *d_proj, const float *d_img,
                            const float *h_angles, int n_views, float SO, float SD, float da,
                            int na, float ai, float db, int nb, float bi, int nx, int ny,
                            int nz);

/* -------------------------------------- mixed-precision kernel level */
/* The engine's non-drop-in kernel forms, one call each, for measuring them
 * against an FP64 reference.  No counterpart in the reference, whose
 * kernels are FP32 only (src/cu_projection.cu, src/cu_backprojection.cu,
 * src/cu_deform.cu).
 *
 * mcsart_projection_ex: the projection of a volume stored as `storage`
 * (mcsart_dtype; FP32 accumulation), with projector summation fp_sum (0 the
 * reference's order, as mcsart_projection; 1 per-slab partial sums; 2 the
 * same with Kahan compensation) and geom64 = 1 for FP64 geometry (fp_sum 1
 * or 2).  Output FP32. */
int mcsart_projection_ex(mcsart_ctx *ctx, float *d_proj, const void *d_img, int storage,
                         int fp_sum, int geom64, float angle, float SO, float SD, float da, int na,
                         float ai, float db, int nb, float bi, int nx, int ny, int nz);
/* mcsart_backprojection with geom64 = 1: voxel and detector boundary
 * coordinates and overlap weights in FP64, terms accumulated in FP32
 * (geom64 = 0 is mcsart_backprojection). */
int mcsart_backprojection_ex(mcsart_ctx *ctx, float *d_img, const float *d_proj, int geom64,
                             float angle, float SO, float SD, float da, int na, float ai,
                             float db, int nb, float bi, int nx, int ny, int nz);
/* mcsart_deform with the six DVF fields (contiguous, alpha_x .. beta_z) and
 * the output stored as `storage`, and the warp model `interp`
 * (mcsart_interp); d_img is FP32 and must not alias d_img1. */
int mcsart_deform_ex(mcsart_ctx *ctx, void *d_img1, const float *d_img, int nx, int ny, int nz,
                     float volume, float flow, const void *d_fields, int storage, int interp);

/* ------------------------------------------------------------ drivers */
/* replaces host_AUMISART, include/AUMISART.h:17 and :19 (src/AUMISART.cu:3,
 * :143).  Host pointers, the reference's argument list and order.  If alpha_x
 * is NULL the DVF starts at zero and the motion pass steps views by 10
 * (overload 1); otherwise all six fields are read and the motion pass steps
 * by 1 (overload 2).  Outputs: h_outimg (nx*ny*nz), h_outproj (na*nb*n_views
 * residuals of the last image pass), h_outnorm (n_iter*n_views ratios
 * ||b-Ax||/||b||; entries of skipped views are 0), h_outalphax (nx*ny*nz).
 * err_weights and outIter are accepted and unused, as in the reference. */
int mcsart_aumisart(mcsart_ctx *ctx, float *h_outimg, float *h_outproj, float *h_outnorm,
                    float *h_outalphax, const float *h_img, const float *h_proj, int nx, int ny,
                    int nz, int na, int nb, int outIter, int n_views, int n_iter,
                    const int *op_iter, float da, float db, float ai, float bi, float SO,
                    float SD, float dx, float lambda, const float *volumes, const float *flows,
                    const float *err_weights, const float *angles, const float *alpha_x,
                    const float *alpha_y, const float *alpha_z, const float *beta_x,
                    const float *beta_y, const float *beta_z);

/* Engine options for the device-resident driver. */
typedef struct {
    int storage;      /* mcsart_dtype of the DVF fields, warped volumes and projections */
    int interp;       /* mcsart_interp */
    int use_graph;    /* capture each pass as a CUDA graph and replay it */
    int fp_sum;       /* projector ray sums: 0 = the reference's order, one thread per
                         ray (bitwise drop-in); 1 = per-slab partial sums, slabs split
                         across warps; 2 = as 1 with Kahan-compensated slab sums */
    int fp_groups;    /* slab groups per ray in modes 1 and 2 (0 = auto) */
    int subset;       /* image passes: views per ordered subset, 1..16 (0 = 1).  1 is
                         the reference's view-by-view loop.  k > 1: the k views of a
                         subset each compute the reference's correction from the same
                         image, in one projector and one backprojector launch, and the
                         image receives lambda/k times their sum (a different
                         algorithm from the reference's, not a drop-in) */
    int dvf_inverse;  /* image passes with motion: 0 = warp corrections back with the
                         negated amplitudes (the reference); n > 0 = with the true
                         inverse of each view's displacement, n fixed-point steps
                         (mcsart_invert_dvf; FP32 storage, square slices; not a drop-in) */
    int geom64;       /* 1: projector and backprojector geometry (source, detector and
                         voxel boundary coordinates, overlap weights) in FP64 and the SART
                         normalisation sums (row sums FP(1), column sums BP(FP(1))) in
                         FP64; volume and residual terms still accumulate in FP32.  Needs
                         fp_sum 1 or 2 (not a drop-in) */
    int autotune;     /* 1: before the first run of a geometry (and storage type) that
                         the context has no tuned launch shapes for, run
                         mcsart_autotune; results are the same bits either way */
} mcsart_options;
void mcsart_default_options(mcsart_options *opt);

/* One reconstruction problem with device-resident state. */
typedef struct {
    int nx, ny, nz, na, nb, n_views;
    float SO, SD, da, db, ai, bi, lambda;
    const float *h_angles;   /* n_views, radians */
    const float *h_volumes;  /* n_views, a(t_v) */
    const float *h_flows;    /* n_views, b(t_v) */
    float *d_img;            /* in/out, FP32 volume */
    const void *d_proj;      /* measured projections, storage dtype, n_views*na*nb */
    void *d_fields;          /* 6*nx*ny*nz (ax,ay,az,bx,by,bz), storage dtype; NULL = overload 1 */
    float *d_resid;          /* optional out: residuals of the last image pass, FP32 */
    float *d_norm;           /* optional out: n_iter*n_views norm ratios, FP32 */
} mcsart_problem;

/* Run n_iter outer iterations (op_iter[i]==1: image pass, else motion pass)
 * of host_AUMISART's loop on device-resident buffers. */
int mcsart_aumisart_device(mcsart_ctx *ctx, const mcsart_problem *prob, int n_iter,
                           const int *h_op_iter, const mcsart_options *opt);

/* As mcsart_aumisart, returning all six final DVF fields (h_out_ax is
 * required, the other five may be NULL).  The reference returns alpha_x only
 * (src/AUMISART.cu:291).  The loop keeps no state between iterations other
 * than the image and the six fields, so passing the returned image and fields
 * back as inputs continues a reconstruction exactly where it stopped: n + m
 * iterations in two calls give the bits of one call of n + m iterations. */
int mcsart_aumisart_fields(mcsart_ctx *ctx, float *h_outimg, float *h_outproj, float *h_outnorm,
                           float *h_out_ax, float *h_out_ay, float *h_out_az, float *h_out_bx,
                           float *h_out_by, float *h_out_bz, const float *h_img,
                           const float *h_proj, int nx, int ny, int nz, int na, int nb,
                           int outIter, int n_views, int n_iter, const int *op_iter, float da,
                           float db, float ai, float bi, float SO, float SD, float dx,
                           float lambda, const float *volumes, const float *flows,
                           const float *err_weights, const float *angles, const float *alpha_x,
                           const float *alpha_y, const float *alpha_z, const float *beta_x,
                           const float *beta_y, const float *beta_z);

/* Independent reconstructions run concurrently on one GPU.  No counterpart
 * in the reference, which runs one problem per call (host_AUMISART,
 * src/AUMISART.cu:143): one view's kernels leave most of a B200 idle, and
 * problems of different sizes fill it together.  Each problem runs the same
 * loop as mcsart_aumisart_device (same n_iter, op_iter and options for all)
 * on a lane of its own (a stream, buffers and pass graphs kept by ctx, so
 * repeated batches reuse them); results are bitwise those of separate
 * mcsart_aumisart_device calls.  The lanes start after the work queued on
 * ctx's stream, and ctx's stream waits for all of them. */
#define MCSART_BATCH_MAX 64
int mcsart_batch_run(mcsart_ctx *ctx, const mcsart_problem *problems, int n_problems,
                     int n_iter, const int *h_op_iter, const mcsart_options *opt);

/* ------------------------------------------------------------ tuning */
/* Launch-shape autotuner, cached per geometry.  No counterpart in the
 * reference, whose kernels have fixed launch shapes (src/cu_projection.cu:9,
 * src/cu_backprojection.cu:46, src/cu_deform.cu:5).  Times the candidate
 * shapes of the driver's per-view kernels (projector slab-group depth and
 * blocks per SM, backprojector voxels per thread and rows per block, warp
 * rows per thread, the DVF-pass field update: with the backprojection ratio computed inside it, or after a
 * separate backprojector launch with either load order) on a sample of the problem's views (an image pass and a
 * DVF-update pass over up to 12 views, on copies of the image and fields;
 * the problem's buffers are not changed) and caches the fastest for the
 * problem's geometry and opt->storage.  Later driver runs of that geometry
 * use them.  Every candidate gives the same bits. */
int mcsart_autotune(mcsart_ctx *ctx, const mcsart_problem *prob, const mcsart_options *opt);
/* The cached shapes of prob's geometry and `storage` as five variant indices
 * (projector one-volume, projector three-volume, backprojector, warp, DVF-pass
 * field update; -1 = built-in): returns 1 and fills shapes[5], or 0 if none
 * are cached. */
int mcsart_tuning_get(mcsart_ctx *ctx, const mcsart_problem *prob, int storage, int *shapes);
/* Write / read the context's tuning cache as a text file (one geometry per
 * line); load returns the number of entries read. */
int mcsart_tuning_save(mcsart_ctx *ctx, const char *path);
int mcsart_tuning_load(mcsart_ctx *ctx, const char *path);

/* ------------------------------------------ allocation-free projector */
/* Largest volume, nx*ny*nz, that mcsart_projection_noalloc accepts: 2^22
 * voxels (e.g. 256x256x64), i.e. 16 MiB of FP32 scratch per device. */
#define MCSART_NOALLOC_MAX_VOXELS 4194304

/* mcsart_projection without any allocation.  This entry point has no
 * counterpart in the reference.
 *
 * Who needs it.  mcsart_projection keeps a scratch copy of the volume in its
 * context and allocates it (cudaMalloc) the first time a size is seen; the
 * context itself allocates a stream and events.  Some callers cannot allow
 * that: a MEX function or service whose device memory is owned by another
 * pool (MATLAB's gpuArray memory, PyTorch's caching allocator), where a
 * private cudaMalloc can fail for lack of free memory although the pool has
 * room; and a reconstruction loop running beside other GPU work, where a
 * cudaMalloc or cudaFree can stall work on other streams.  This entry point
 * takes a stream instead of a context, keeps its scratch in a fixed device
 * array that is part of the library, and calls no cudaMalloc, cudaFree or
 * allocating library.
 *
 * Same arguments and results as mcsart_projection (bitwise), except:
 * - stream: the CUDA stream (cudaStream_t) to run on; NULL = legacy default
 *   stream.  The call returns once the work is enqueued; kernel faults
 *   surface at the caller's next synchronisation;
 * - nx*ny*nz above MCSART_NOALLOC_MAX_VOXELS is rejected with
 *   MCSART_ERR_INVALID_ARGUMENT (use mcsart_projection for larger volumes);
 * - set-up: the first call on each device, with that device current, looks
 *   up the scratch's address (cudaGetSymbolAddress) and loads the kernels.
 *   Make that first call before any stream capture and outside time-critical
 *   code; later calls on that device do no set-up.  The address belongs to
 *   the device's current CUDA context: after a cudaDeviceReset, or from
 *   another context of the same device, the next call repeats the set-up
 *   (so make it, too, outside a stream capture);
 * - nothing has to start at zero: the scratch is written before it is read
 *   and every cell of d_proj is written;
 * - all calls on one device share the one scratch.  Calls in one stream are
 *   ordered and safe; calls whose execution can overlap (different streams
 *   or host threads with nothing ordering them) race on it and can return
 *   wrong projections.
 * The device reserves the 16 MiB array when it loads this part of the
 * library: at the first call under lazy module loading (the CUDA 12
 * default), at context creation under CUDA_MODULE_LOADING=EAGER. */
int mcsart_projection_noalloc(void *stream, float *d_proj, const float *d_img, float angle,
                              float SO, float SD, float da, int na, float ai, float db, int nb,
                              float bi, int nx, int ny, int nz);

#ifdef __cplusplus
}
#endif
#endif /* MCSART_H */
