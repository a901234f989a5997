/*
 * lu_static.h - static-pattern sparse LU handle: host symbolic analysis once
 * per sparsity pattern, then numeric refactorizations and solves on one B200.
 *
 * Drop-in for LUspice src/lu_static.h:22-86 (same struct layout, same entry
 * points, same return codes).  Semantics of this implementation:
 *
 *   - COO indices are 1-based, as the reference actually consumes them
 *     (src/lu_static.c:78,84-85; fed 1-based by bench/test_lu.c:136) even
 *     though its header comment says 0-based.  Duplicate (row, col) entries
 *     are summed.
 *   - dsh_symbolic: converts the COO pattern to a column-sorted CSC, stores
 *     Q (COLAMD order, or natural when colamd_q is NULL).  Pivots and the
 *     L/U pattern need values, so they are fixed by the first dsh_numeric
 *     call (one fp64 left-looking LU with partial pivoting, tol = 1, the
 *     CSparse cs_lu algorithm used by the reference's splu.h:151-206); every
 *     later dsh_numeric with the same pattern is a GPU refactorization with
 *     the pivot order and L/U pattern frozen (fp32 factor storage, fp64
 *     work vector).
 *   - After dsh_numeric: F->lnnz / F->unnz are exact (unit diagonal counted
 *     in lnnz, U diagonal in unnz, as splu.h reports them), F->cap =
 *     lnnz + unnz - n (merged L+U slots), F->Ap / F->Ai describe the merged
 *     L+U columns in pivot-position space (rows ascending, diagonal
 *     included) and are HOST arrays; F->Ax is a DEVICE pointer to the fp32
 *     merged values (L below the diagonal holds multipliers, U on and above);
 *     F->P is a HOST array with P[orig_row] = pivot position (pinv);
 *     F->Q is a HOST array with the column order.
 *   - b and x of dsh_trisolve / dsh_gmres_ir are HOST arrays of n doubles.
 *   - Return codes: 0 OK, 1 SINGULAR, 2 ALLOC, 3 ARG/NOT_IMPL
 *     (src/lu_static.c:292-300); 4 IR_STAGNATED (dsh_gmres_ir only: the
 *     mixed-precision iteration stopped reducing the fp64 residual; the
 *     caller should escalate to the fp64 path, see selector.h).
 *   - Not thread-safe per handle.  dsh_symbolic_count() is process-global and
 *     atomic.
 */
#ifndef DSH_LU_STATIC_H
#define DSH_LU_STATIC_H

#ifdef __cplusplus
extern "C" {
#endif

/* Layout identical to src/lu_static.h:22-49. */
typedef struct {
    int     n;
    long    cnnz;
    long    lnnz;
    long    unnz;
    long    cap;

    int    *Ap;
    int    *Ai;
    float  *Ax;

    int    *P;
    int    *Q;

    double  min_diag_U;
    double  pivot_growth;

    int     dev_allocated;

    void   *factor_cache;
    double  pin;
} dsh_lu_static;

/* src/lu_static.h:56-59 */
int dsh_symbolic(int n, long cnnz,
                 const int *coo_row, const int *coo_col,
                 const int *colamd_q,
                 dsh_lu_static *F);

/* src/lu_static.h:64-66 */
int dsh_numeric(dsh_lu_static *F,
                const int *coo_row, const int *coo_col,
                const double *coo_val, int nnz);

/* src/lu_static.h:70 : x = Q U^-1 L^-1 P b with the stored factors. */
int dsh_trisolve(const dsh_lu_static *F, const double *b, double *x);

/* src/lu_static.h:73-75 (a stub returning 3 in the reference,
 * src/lu_static.c:283-290).  Here: right-preconditioned restarted GMRES
 * around the fp32 factors with fp64 residual, Arnoldi, Givens and update,
 * entirely on the device.  max_outer = restarts (<= 0 -> 3), max_inner =
 * Krylov dimension (<= 0 -> 50, capped at 64), rtol on ||b-Ax||/||b||
 * (<= 0 -> 1e-10).  residual_seq (may be NULL) receives up to
 * max_outer + 1 relative residuals; iters (may be NULL) the total inner
 * iterations. */
int dsh_gmres_ir(dsh_lu_static *F, const double *b, double *x,
                 int max_outer, int max_inner, double rtol,
                 double *residual_seq, int *iters);

/* src/lu_static.h:78-80 */
int dsh_lu_static_init(dsh_lu_static *F);
int dsh_lu_static_alloc(dsh_lu_static *F);
void dsh_lu_static_free(dsh_lu_static *F);

/* src/lu_static.h:83 */
const char *dsh_lu_status_str(int rc);

/* src/lu_static.h:86 */
long dsh_symbolic_count(void);

#ifdef __cplusplus
}
#endif

#endif /* DSH_LU_STATIC_H */
