/* Test infrastructure: the CPU oracle for the McSART hot path.
 *
 * orc_*  : FP64 restatement of every reference kernel and of the SART loop
 *          (the accuracy reference used by tests/, smoke() and bench.py's cpu_baseline leg).
 * cpu_*  : the same restatement instantiated in FP32 and parallelised with
 *          OpenMP; it is the timed CPU baseline (the reference has no CPU path).
 *
 * Arrays use the reference layouts: img[ix + iy*nx + iz*nx*ny],
 * proj[ia + ib*na (+ v*na*nb)].  Geometry is in voxel units, with ai/bi
 * already shifted by -(n/2 - 0.5) as src/entry_AUMISART.cu:76-94 does.
 * Nothing here is linked into the product library. */
#ifndef MCSART_ORACLE_H
#define MCSART_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Texture filtering model for the warp (src/cu_deform.cu:79-90 uses hardware
 * linear filtering, whose weights carry 8 fractional bits). */
enum { ORC_TEX_EXACT = 0, ORC_TEX_Q8_NEAREST = 1, ORC_TEX_Q8_TRUNC = 2 };

#define ORC_DECL(T, P)                                                                        \
    void P##projection(T *proj, const T *img, double angle, double SO, double SD, double da,   \
                       int na, double ai, double db, int nb, double bi, int nx, int ny,        \
                       int nz);                                                                \
    void P##backprojection_adjoint(T *img, const T *proj, double angle, double SO, double SD,  \
                                   double da, int na, double ai, double db, int nb, double bi, \
                                   int nx, int ny, int nz);                                    \
    void P##backprojection(T *img, const T *proj, double angle, double SO, double SD,          \
                           double da, int na, double ai, double db, int nb, double bi, int nx, \
                           int ny, int nz);                                                    \
    void P##backprojection_sc(T *img, const T *proj, double cphi, double sphi, double SO,      \
                              double SD, double da, int na, double ai, double db, int nb,      \
                              double bi, int nx, int ny, int nz);                              \
    void P##forward_dvf(T *mx, T *my, T *mz, const T *ax, const T *ay, const T *az,            \
                        const T *bx, const T *by, const T *bz, double volume, double flow,     \
                        int nx, int ny, int nz);                                               \
    void P##deform(T *out, const T *img, int nx, int ny, int nz, double volume, double flow,   \
                   const T *ax, const T *ay, const T *az, const T *bx, const T *by,            \
                   const T *bz, int tex_mode);                                                 \
    void P##deform2(T *out, const T *img, int nx, int ny, int nz, double volume, double flow,  \
                    const T *ax, const T *ay, const T *az, const T *bx, const T *by,           \
                    const T *bz);                                                              \
    void P##add(T *img1, const T *img, int nx, int ny, int nz, double weight);                 \
    void P##add2(T *img1, const T *img, int nx, int ny, int nz, const T *img0, double weight,  \
                 int ind);                                                                     \
    void P##initial(T *img, int nx, int ny, int nz, double value);                             \
    void P##initial2(T *img, int nx, int ny, int nz, const T *img0, double volume,             \
                     double flow);                                                             \
    void P##division(T *img1, const T *img, int nx, int ny, int nz);                           \
    void P##multiple(T *img1, int nx, int ny, int nz, const T *img0, double weight, int ind);   \
    void P##update_udvf(T *ax, T *ay, T *az, T *bx, T *by, T *bz, const T *img,               \
                        const T *img0, double volume_diff, double flow_diff, int nx, int ny,   \
                        int nz, int iter);                                                     \
    void P##diff(T *img1, const T *img, int nx, int ny, int nz, int ind);                      \
    int P##aumisart(T *outimg, T *outproj, T *outnorm, T *outalphax, const T *img,             \
                    const T *proj, int nx, int ny, int nz, int na, int nb, int outIter,        \
                    int n_views, int n_iter, const int *op_iter, double da, double db,         \
                    double ai, double bi, double SO, double SD, double dx, double lambda,      \
                    const float *volumes, const float *flows, const float *angles,             \
                    const T *ax, const T *ay, const T *az, const T *bx, const T *by,           \
                    const T *bz, T *fields_out, int tex_mode, int view_lo, int view_hi,       \
                    int subset, int dvf_inverse);                                             \
    void P##invert_dvf(T *ox, T *oy, T *oz, const T *ax, const T *ay, const T *az, const T *bx, \
                       const T *by, const T *bz, double volume, double flow, int nx, int ny,  \
                       int nz, int iters);

ORC_DECL(double, orc_)
ORC_DECL(float, cpu_)
#undef ORC_DECL

/* Number of OpenMP threads the library will use. */
int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
