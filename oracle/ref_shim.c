/* Test-only glue around the reference's header-only sparse LU (splu.h):
 * exposes lu_factor / lu_solve_perm through a handle so the checker can read
 * P, L, U and solve with them.  Compiled with the reference sources where
 * they lie; nothing here is shipped or called by the product.
 * lu_factor is called with a modest initial capacity (its growth logic,
 * splu.h:57-74, handles the rest) instead of cpu_ref_lu.c's n*n slots. */
#include <stdlib.h>
#include "splu.h"

typedef struct {
    int n;
    lu_factors F;
    int rc;
} ref_handle;

void *ref_lu_factor(int n, const int *Ap, const int *Ai, const double *Ax,
                    const int *q, double tol)
{
    ref_handle *h = (ref_handle *)calloc(1, sizeof(ref_handle));
    long cap = 4L * Ap[n] + 16L * n + 64;
    h->n = n;
    h->F.n = n;
    h->F.pinv = (int *)malloc((size_t)n * sizeof(int));
    h->F.L.n = h->F.U.n = n;
    h->F.L.Lp = (int *)malloc((size_t)(n + 1) * sizeof(int));
    h->F.L.Li = (int *)malloc((size_t)cap * sizeof(int));
    h->F.L.Lx = (double *)malloc((size_t)cap * sizeof(double));
    h->F.U.Up = (int *)malloc((size_t)(n + 1) * sizeof(int));
    h->F.U.Ui = (int *)malloc((size_t)cap * sizeof(int));
    h->F.U.Ux = (double *)malloc((size_t)cap * sizeof(double));
    h->F.L.Lcap = h->F.U.Ucap = cap;
    int *xi = (int *)malloc((size_t)(2 * n + 1) * sizeof(int));
    double *x = (double *)malloc((size_t)n * sizeof(double));
    h->rc = lu_factor(n, Ap, Ai, Ax, q, &h->F, tol, xi, x);
    free(xi);
    free(x);
    return h;
}

int ref_lu_status(void *hv) { return ((ref_handle *)hv)->rc; }
long ref_lu_lnnz(void *hv) { ref_handle *h = hv; return h->F.L.Lp[h->n]; }
long ref_lu_unnz(void *hv) { ref_handle *h = hv; return h->F.U.Up[h->n]; }

/* Copy out pinv, L (Lp, Li positions, Lx) and U (Up, Ui, Ux). */
void ref_lu_get(void *hv, int *pinv, int *Lp, int *Li, double *Lx,
                int *Up, int *Ui, double *Ux)
{
    ref_handle *h = (ref_handle *)hv;
    int n = h->n;
    long ln = h->F.L.Lp[n], un = h->F.U.Up[n];
    for (int i = 0; i < n; i++) pinv[i] = h->F.pinv[i];
    for (int i = 0; i <= n; i++) { Lp[i] = h->F.L.Lp[i]; Up[i] = h->F.U.Up[i]; }
    for (long p = 0; p < ln; p++) { Li[p] = h->F.L.Li[p]; Lx[p] = h->F.L.Lx[p]; }
    for (long p = 0; p < un; p++) { Ui[p] = h->F.U.Ui[p]; Ux[p] = h->F.U.Ux[p]; }
}

void ref_lu_solve(void *hv, const int *q, const double *b, double *x)
{
    ref_handle *h = (ref_handle *)hv;
    lu_solve_perm(h->n, &h->F, q, b, x);
}

void ref_lu_free(void *hv)
{
    ref_handle *h = (ref_handle *)hv;
    if (!h) return;
    free(h->F.pinv);
    free(h->F.L.Lp); free(h->F.L.Li); free(h->F.L.Lx);
    free(h->F.U.Up); free(h->F.U.Ui); free(h->F.U.Ux);
    free(h);
}
