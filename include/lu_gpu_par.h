/*
 * lu_gpu_par.h - single-block GPU sparse left-looking LU with partial
 * pivoting (pivots chosen on the device, pattern discovered on the fly) and
 * the matching triangular solve.
 *
 * Drop-in for LUspice src/lu_gpu_par.h:14-58: same macros, same kernel
 * names and parameter lists, same launch shape <<<1, 256, bytes>>>, same
 * outputs.  These kernels are the fp64 escalation path: they re-decide the
 * row permutation for values whose frozen pivots are no longer acceptable.
 *
 * Semantics (src/lu_gpu.cu:34-115, the single-thread kernel the parallel one
 * must equal column by column):
 *   P * A(:,q) = L * U, A given as q-ordered CSC with ORIGINAL row indices,
 *   diagrow[k] = q[k].  Per column: forward updates in ascending pivot
 *   order, entries that are exactly 0.0 are dropped, pivot = largest |x|
 *   over unpivoted rows with ties to the smallest row index, replaced by
 *   diagrow[k] when that row is unpivoted and |x[diagrow[k]]| >= max.
 *   L: CSC, unit diagonal first in each column, Li remapped to pivot
 *   positions after the last column; rows of a column ascending by original
 *   row index.  U: CSC, diagonal last, off-diagonal rows ordered by ascending
 *   original row index.  pinv[orig_row] = position.
 *   singular_out: -1 ok; >= 0 singular column; -2 capacity (Lcap/Ucap);
 *   -3 structure overflow (never raised by this implementation).
 * Work arrays: pinv[n]; xi[n + 2*LU_PAR_CAP] ints (xi[0..n) receives
 * rowat = inverse of pinv); xg unused (may be NULL).
 * Arithmetic is fp64 without fused multiply-add, so results are bitwise
 * reproducible against a host build with -ffp-contract=off.
 */
#ifndef DSH_LU_GPU_PAR_H
#define DSH_LU_GPU_PAR_H

#include <stddef.h>

/* src/lu_gpu_par.h:19 */
#define LU_PAR_CAP 1024

/* src/lu_gpu_par.h:28-29: dynamic shared bytes for lu_factor_par_kernel. */
#define LU_PAR_SHARED_BYTES(n) \
    ((size_t)(n) * 12 + (size_t)256)

#ifdef __CUDACC__
/* src/lu_gpu_par.h:41-50 */
__global__ void lu_factor_par_kernel(
    int n,
    const int  *Ap, const int *Ai, const double *Ax,
    const int  *diagrow,
    int        *Lp, int *Li, double *Lx, long Lcap,
    int        *Up, int *Ui, double *Ux, long Ucap,
    int        *pinv,
    int        *xi,
    double     *xg,
    int        *lnnz, int *unnz, int *singular_out);

/* src/lu_gpu_par.h:58-64 : pb = P b, L y = pb, U z = y, x = Q z.
 * work_i[n], work_d[2n]. */
__global__ void trisolve_par_kernel(
    int n,
    const int  *Lp, const int *Li, const double *Lx,
    const int  *Up, const int *Ui, const double *Ux,
    const int  *pinv, const int *q,
    const double *b, double *x,
    int        *work_i, double *work_d);
#endif /* __CUDACC__ */

#ifdef __cplusplus
extern "C" {
#endif
/* C-ABI launchers for callers that cannot use <<<>>> (C, ctypes, FFI).
 * They launch exactly <<<1, 256, LU_PAR_SHARED_BYTES(n), stream>>> and
 * return the cudaError_t of the launch (0 = success). */
int lusp_lu_factor_par_launch(
    int n, const int *Ap, const int *Ai, const double *Ax, const int *diagrow,
    int *Lp, int *Li, double *Lx, long Lcap,
    int *Up, int *Ui, double *Ux, long Ucap,
    int *pinv, int *xi, double *xg,
    int *lnnz, int *unnz, int *singular_out, void *stream);

int lusp_trisolve_par_launch(
    int n, const int *Lp, const int *Li, const double *Lx,
    const int *Up, const int *Ui, const double *Ux,
    const int *pinv, const int *q, const double *b, double *x,
    int *work_i, double *work_d, void *stream);

/* No counterpart in the reference.  The same solve as
 * lusp_trisolve_par_launch for callers that cannot allocate device memory at
 * solve time (a simulator time-step loop that sized all device memory up
 * front and must not call cudaMalloc mid-run, which synchronizes the device
 * and can fail with out-of-memory; host code that owns every device byte
 * through its own arena): the work arrays come from a fixed scratch area
 * inside the library instead of the caller.
 *   - n <= LUSP_NOALLOC_MAX_N, else LUSP_EARG (3) and lusp_last_error() says
 *     why; the scratch (1.25 MiB) is held by every GPU that loads the library
 *     until the process exits.
 *   - The first call on a device looks the scratch address up for that
 *     device (make it with that device current); make this first call
 *     before any stream capture.
 *   - Allocates nothing: no cudaMalloc, no cudaFree.
 *   - All calls share one scratch area per device: calls that overlap on the
 *     GPU (different streams, or a second call before the first finished on
 *     another stream) race and give wrong results; serialize them (one
 *     stream, or events).  Nothing needs clearing between calls.
 * Returns LUSP_OK (0), LUSP_EARG or LUSP_ECUDA (4). */
#define LUSP_NOALLOC_MAX_N 65536
int lusp_trisolve_par_noalloc(
    int n, const int *Lp, const int *Li, const double *Lx,
    const int *Up, const int *Ui, const double *Ux,
    const int *pinv, const int *q, const double *b, double *x, void *stream);
#ifdef __cplusplus
}
#endif

#endif /* DSH_LU_GPU_PAR_H */
