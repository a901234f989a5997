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
#ifdef __cplusplus
}
#endif

#endif /* DSH_LU_GPU_PAR_H */
