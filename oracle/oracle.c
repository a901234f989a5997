/*
 * oracle.c - CPU restatement of the reference's refactor-and-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  The product never links, loads or calls this
 * file; tests, smoke() and bench.py's CPU-baseline leg use it as the checker.
 * Every function cites the reference code it restates (paths inside the
 * LUspice project).  Built with -ffp-contract=off: fp64 arithmetic is
 * plain multiply then add/subtract, as in a default x86-64 gcc build of the
 * reference, so results compare bitwise where the algorithm fixes the order.
 *
 * Pinned by the tests against the reference's own sources compiled in
 * oracle/_ref (splu.h lu_factor / lu_solve_perm, symbolic_dense.c,
 * level.c, selector.c) on generated matrices.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------
 * Left-looking LU with threshold partial pivoting, P A(:,q) = L U
 * (src/third_party/splu.h:76-206, CSparse cs_reach/cs_dfs/cs_spsolve/cs_lu).
 * Outputs in splu layout: L unit diagonal first (rows remapped to
 * positions), U diagonal last, rows in depth-first reach order.
 * Arrays Li/Lx/Ui/Ux must hold lcap/ucap entries; returns -1 ok, k >= 0 for
 * a singular column, -2 when a capacity is too small (counts still set).
 * ---------------------------------------------------------------------- */
int orc_lu_factor(int n, const int *Ap, const int *Ai, const double *Ax, const int *q,
                  double tol, int *pinv, int *Lp, int *Li, double *Lx, long lcap,
                  int *Up, int *Ui, double *Ux, long ucap, long *lnnz, long *unnz)
{
    int *stack = malloc(sizeof(int) * (size_t)(n + 1));
    int *resume = malloc(sizeof(int) * (size_t)(n + 1));
    int *order = malloc(sizeof(int) * (size_t)(n + 1));
    char *seen = calloc((size_t)n, 1);
    double *x = calloc((size_t)n, sizeof(double));
    long lz = 0, uz = 0;
    int status = -1;
    for (int i = 0; i < n; i++) pinv[i] = -1;
    for (int k = 0; k <= n; k++) Lp[k] = Up[k] = 0;
    for (int k = 0; k < n && status == -1; k++) {
        const int col = q ? q[k] : k;
        Lp[k] = (int)lz;
        Up[k] = (int)uz;
        if (lz + n + 1 > lcap || uz + n + 1 > ucap) { status = -2; break; }
        /* reach: iterative depth-first search from each entry of A(:,col);
         * finished nodes are pushed to the front of order[top..n). */
        int top = n;
        for (int p = Ap[col]; p < Ap[col + 1]; p++) {
            int root = Ai[p];
            if (seen[root]) continue;
            int sp = 0;
            stack[0] = root;
            while (sp >= 0) {
                const int v = stack[sp];
                const int J = pinv[v];
                if (!seen[v]) {
                    seen[v] = 1;
                    resume[sp] = J < 0 ? 0 : Lp[J];
                }
                const int end = J < 0 ? 0 : Lp[J + 1];
                int child = -1;
                for (int t = resume[sp]; t < end; t++) {
                    if (!seen[Li[t]]) { child = Li[t]; resume[sp] = t; break; }
                }
                if (child >= 0) {
                    stack[++sp] = child;
                } else {
                    sp--;
                    order[--top] = v;
                }
            }
        }
        for (int t = top; t < n; t++) seen[order[t]] = 0;
        /* numeric solve in reach order */
        for (int t = top; t < n; t++) x[order[t]] = 0.0;
        for (int p = Ap[col]; p < Ap[col + 1]; p++) x[Ai[p]] = Ax[p];
        for (int t = top; t < n; t++) {
            const int j = order[t], J = pinv[j];
            if (J < 0) continue;
            const double xj = x[j];
            for (int s = Lp[J] + 1; s < Lp[J + 1]; s++) x[Li[s]] -= Lx[s] * xj;
        }
        /* pivot: first strictly largest |x| in reach order, diagonal kept
         * when it is within tol of the largest */
        int ipiv = -1;
        double big = -1.0;
        for (int t = top; t < n; t++) {
            const int i = order[t];
            if (pinv[i] < 0) {
                if (fabs(x[i]) > big) { big = fabs(x[i]); ipiv = i; }
            } else {
                Ui[uz] = pinv[i];
                Ux[uz++] = x[i];
            }
        }
        if (ipiv == -1 || big <= 0.0) { status = k; break; }
        if (pinv[col] < 0 && fabs(x[col]) >= big * tol) ipiv = col;
        const double pv = x[ipiv];
        Ui[uz] = k;
        Ux[uz++] = pv;
        pinv[ipiv] = k;
        Li[lz] = ipiv;
        Lx[lz++] = 1.0;
        for (int t = top; t < n; t++) {
            const int i = order[t];
            if (pinv[i] < 0) {
                Li[lz] = i;
                Lx[lz++] = x[i] / pv;
            }
            x[i] = 0.0;
        }
    }
    if (status == -1) {
        Lp[n] = (int)lz;
        Up[n] = (int)uz;
        for (long p = 0; p < lz; p++) Li[p] = pinv[Li[p]];
    }
    if (lnnz) *lnnz = lz;
    if (unnz) *unnz = uz;
    free(stack); free(resume); free(order); free(seen); free(x);
    return status;
}

/* x = Q U^-1 L^-1 P b with splu-layout factors (splu.h:210-239). */
void orc_lu_solve(int n, const int *pinv, const int *Lp, const int *Li, const double *Lx,
                  const int *Up, const int *Ui, const double *Ux, const int *q,
                  const double *b, double *x)
{
    double *w = malloc(sizeof(double) * (size_t)n);
    double *y = malloc(sizeof(double) * (size_t)n);
    int *src = malloc(sizeof(int) * (size_t)n);
    for (int k = 0; k < n; k++) src[k] = -1;
    for (int i = 0; i < n; i++) if (pinv[i] >= 0) src[pinv[i]] = i;
    for (int k = 0; k < n; k++) w[k] = src[k] >= 0 ? b[src[k]] : 0.0;
    for (int k = 0; k < n; k++) {
        y[k] = w[k] / Lx[Lp[k]];
        for (int p = Lp[k] + 1; p < Lp[k + 1]; p++) w[Li[p]] -= Lx[p] * y[k];
    }
    for (int k = n - 1; k >= 0; k--) {
        y[k] /= Ux[Up[k + 1] - 1];
        for (int p = Up[k]; p < Up[k + 1] - 1; p++) y[Ui[p]] -= Ux[p] * y[k];
    }
    for (int k = 0; k < n; k++) x[q ? q[k] : k] = y[k];
    free(w); free(y); free(src);
}

/* ------------------------------------------------------------------------
 * Dense-scan single-thread GPU factorization semantics
 * (src/lu_gpu.cu:34-115, mirrored on the host by src/symbolic_dense.c:12-64):
 * forward updates for j = 0..k-1 skipping x[rowat[j]] == 0, exact zeros
 * dropped, pivot = largest |x| over unpivoted rows with the smallest row on
 * ties, diagrow[k] kept when |x[diagrow[k]]| >= max.  L rows remapped to
 * positions at the end.  Returns -1, a singular column, or -2 (capacity).
 * ---------------------------------------------------------------------- */
int orc_dense_factor(int n, const int *Ap, const int *Ai, const double *Ax, const int *diagrow,
                     int *pinv, int *Lp, int *Li, double *Lx, long lcap,
                     int *Up, int *Ui, double *Ux, long ucap, long *lnnz, long *unnz)
{
    int *rowat = malloc(sizeof(int) * (size_t)n);
    double *x = calloc((size_t)n, sizeof(double));
    long lz = 0, uz = 0;
    int status = -1;
    for (int i = 0; i < n; i++) { pinv[i] = -1; rowat[i] = -1; }
    for (int k = 0; k < n && status == -1; k++) {
        Lp[k] = (int)lz;
        Up[k] = (int)uz;
        for (int p = Ap[k]; p < Ap[k + 1]; p++) x[Ai[p]] = Ax[p];
        for (int j = 0; j < k; j++) {
            const double xr = x[rowat[j]];
            if (xr != 0.0)
                for (int p = Lp[j] + 1; p < Lp[j + 1]; p++) x[Li[p]] -= Lx[p] * xr;
        }
        int ipiv = -1;
        double big = -1.0;
        for (int i = 0; i < n; i++) {
            if (pinv[i] < 0) {
                if (fabs(x[i]) > big) { big = fabs(x[i]); ipiv = i; }
            } else if (x[i] != 0.0) {
                if (uz >= ucap) { status = -2; break; }
                Ui[uz] = pinv[i];
                Ux[uz++] = x[i];
            }
        }
        if (status != -1) break;
        if (ipiv == -1 || big <= 0.0) { status = k; break; }
        const int ck = diagrow[k];
        if (pinv[ck] < 0 && fabs(x[ck]) >= big) ipiv = ck;
        const double pv = x[ipiv];
        if (uz >= ucap || lz >= lcap) { status = -2; break; }
        Ui[uz] = k;
        Ux[uz++] = pv;
        pinv[ipiv] = k;
        rowat[k] = ipiv;
        Li[lz] = ipiv;
        Lx[lz++] = 1.0;
        for (int i = 0; i < n; i++) {
            if (pinv[i] < 0 && x[i] != 0.0) {
                if (lz >= lcap) { status = -2; break; }
                Li[lz] = i;
                Lx[lz++] = x[i] / pv;
            }
            x[i] = 0.0;
        }
    }
    if (status == -1) {
        Lp[n] = (int)lz;
        Up[n] = (int)uz;
        for (long p = 0; p < lz; p++) Li[p] = pinv[Li[p]];
    }
    if (lnnz) *lnnz = lz;
    if (unnz) *unnz = uz;
    free(rowat); free(x);
    return status;
}

/* Column levels from the U structure (src/level.c:20-38). */
int orc_levels(int n, const int *Up, const int *Ui, int *level)
{
    int deepest = 0;
    for (int k = 0; k < n; k++) {
        int l = 0;
        for (int p = Up[k]; p < Up[k + 1] - 1; p++) {
            const int j = Ui[p];
            if (j >= 0 && j < k && level[j] + 1 > l) l = level[j] + 1;
        }
        level[k] = l;
        if (l > deepest) deepest = l;
    }
    return deepest + 1;
}

/* ------------------------------------------------------------------------
 * Refactorization with frozen pivots and a static pattern: the fixed-pivot
 * wave factorization of src/lu_gpu_wave.cu:17-107 and
 * src/mp/multiblock_lu.cu:229-299 (x = A(:,k); for each dependency j in
 * ascending order: x -= L(:,j) x_j; U = x above the diagonal, L = x below
 * divided by the pivot), on the merged static layout:
 *   column k = slots [cp[k], cp[k+1]), rows ri ascending, diagonal at dg[k];
 *   input entries a_src[t] land in slot cp[k] + a_dst[t] for t in
 *   [a_ptr[k], a_ptr[k+1]) (duplicates summed in order).
 * store_fp32 != 0: factor values are rounded to float when stored and read
 * back as float (the work vector stays double).  Output vals[cap] (double,
 * holding the stored value).  Returns the first column with a zero or
 * non-finite pivot, or -1.
 * ---------------------------------------------------------------------- */
int orc_static_refactor(int n, const int *cp, const int *ri, const int *dg,
                        const int *a_ptr, const int *a_src, const int *a_dst,
                        const double *a_val, int store_fp32, double *vals)
{
    int maxlen = 1;
    for (int k = 0; k < n; k++) if (cp[k + 1] - cp[k] > maxlen) maxlen = cp[k + 1] - cp[k];
    double *x = malloc(sizeof(double) * (size_t)maxlen);
    int bad = -1;
    for (int k = 0; k < n; k++) {
        const int c0 = cp[k], len = cp[k + 1] - c0, d = dg[k] - c0;
        for (int t = 0; t < len; t++) x[t] = 0.0;
        for (int t = a_ptr[k]; t < a_ptr[k + 1]; t++) {
            if (t > a_ptr[k] && a_dst[t - 1] == a_dst[t]) continue;
            double s = a_val[a_src[t]];
            for (int u = t + 1; u < a_ptr[k + 1] && a_dst[u] == a_dst[t]; u++) s = s + a_val[a_src[u]];
            x[a_dst[t]] = s;
        }
        for (int u = 0; u < d; u++) {
            const int j = ri[c0 + u];
            const double xj = x[u];
            if (xj == 0.0) continue;
            int pos = u + 1;
            for (int p = dg[j] + 1; p < cp[j + 1]; p++) {
                const int i = ri[p];
                while (pos < len && ri[c0 + pos] < i) pos++;
                x[pos] = x[pos] - vals[p] * xj;
            }
        }
        const double pv = x[d];
        if ((!(fabs(pv) > 0.0) || !isfinite(pv)) && bad < 0) bad = k;
        for (int t = 0; t < len; t++) {
            double v = t > d ? x[t] / pv : x[t];
            if (store_fp32) v = (double)(float)v;
            vals[c0 + t] = v;
        }
    }
    free(x);
    return bad;
}

/* y = A x, CSR, row-sequential fp64 (src/spmv.cu:154-171). */
void orc_spmv_csr(int n, const int *rp, const int *ci, const double *v, const double *x, double *y)
{
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int p = rp[i]; p < rp[i + 1]; p++) s += v[p] * x[ci[p]];
        y[i] = s;
    }
}

/* ------------------------------------------------------------------------
 * Right-preconditioned restarted GMRES with iterative refinement, fp64
 * (bench/test_lu_gpu_f32.cu:540-715, bench/test_lu_gpu_ir64.cu:237-358):
 * r = b - A x; V0 = r/||r||; Arnoldi with two Gram-Schmidt passes; Givens
 * rotations; stop when |g_{j+1}|/||b|| <= rtol; x += M^-1 V y.  M^-1 is the
 * splu-layout factorization (pinv, L, U, q).  Differences from the
 * reference loop, all corrections: H is cleared at each restart, the
 * rotation of a breakdown column is applied before the back substitution.
 * A in CSR (original order).  Returns total inner iterations; res[] gets up
 * to max_outer+1 relative residuals (*nres set).
 * ---------------------------------------------------------------------- */
int orc_gmres_ir(int n, const int *rp, const int *ci, const double *av,
                 const int *pinv, const int *Lp, const int *Li, const double *Lx,
                 const int *Up, const int *Ui, const double *Ux, const int *q,
                 const double *b, double *x, int m, int max_outer, double rtol,
                 double *res, int *nres)
{
    double *V = malloc(sizeof(double) * (size_t)(m + 1) * n);
    double *H = malloc(sizeof(double) * (size_t)(m + 1) * m);
    double *cs = malloc(sizeof(double) * (size_t)m), *sn = malloc(sizeof(double) * (size_t)m);
    double *g = malloc(sizeof(double) * (size_t)(m + 1)), *yv = malloc(sizeof(double) * (size_t)(m + 1));
    double *w = malloc(sizeof(double) * (size_t)n), *z = malloc(sizeof(double) * (size_t)n);
    double *r = malloc(sizeof(double) * (size_t)n);
    double nb = 0.0;
    int total = 0, cnt = 0;
    for (int i = 0; i < n; i++) { x[i] = 0.0; nb += b[i] * b[i]; }
    nb = sqrt(nb);
    for (int outer = 0; ; outer++) {
        orc_spmv_csr(n, rp, ci, av, x, r);
        double beta = 0.0;
        for (int i = 0; i < n; i++) { r[i] = b[i] - r[i]; beta += r[i] * r[i]; }
        beta = sqrt(beta);
        const double rel = nb > 0 ? beta / nb : beta;
        if (cnt < max_outer + 1) res[cnt++] = rel;
        if (rel <= rtol || outer >= max_outer || !isfinite(rel)) break;
        for (int i = 0; i < n; i++) V[i] = r[i] / beta;
        for (int t = 0; t <= m; t++) g[t] = 0.0;
        for (int t = 0; t < (m + 1) * m; t++) H[t] = 0.0;
        g[0] = beta;
        int jj = 0;
        for (int j = 0; j < m; j++) {
            orc_lu_solve(n, pinv, Lp, Li, Lx, Up, Ui, Ux, q, V + (size_t)j * n, z);
            orc_spmv_csr(n, rp, ci, av, z, w);
            for (int pass = 0; pass < 2; pass++)
                for (int i = 0; i <= j; i++) {
                    double h = 0.0;
                    for (int e = 0; e < n; e++) h += V[(size_t)i * n + e] * w[e];
                    H[i * m + j] += h;
                    for (int e = 0; e < n; e++) w[e] -= h * V[(size_t)i * n + e];
                }
            double hn = 0.0;
            for (int e = 0; e < n; e++) hn += w[e] * w[e];
            hn = sqrt(hn);
            for (int i = 0; i < j; i++) {
                const double t1 = H[i * m + j], t2 = H[(i + 1) * m + j];
                H[i * m + j] = cs[i] * t1 + sn[i] * t2;
                H[(i + 1) * m + j] = -sn[i] * t1 + cs[i] * t2;
            }
            const double a = H[j * m + j], hb = hn < 1e-14 ? 0.0 : hn;
            const double rr = sqrt(a * a + hb * hb);
            cs[j] = rr > 0 ? a / rr : 1.0;
            sn[j] = rr > 0 ? hb / rr : 0.0;
            H[j * m + j] = rr;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            total++;
            jj = j + 1;
            if (hn < 1e-14 || fabs(g[j + 1]) / nb <= rtol) break;
            for (int e = 0; e < n; e++) V[(size_t)(j + 1) * n + e] = w[e] / hn;
        }
        for (int i = jj - 1; i >= 0; i--) {
            double s = g[i];
            for (int t = i + 1; t < jj; t++) s -= H[i * m + t] * yv[t];
            yv[i] = H[i * m + i] != 0.0 ? s / H[i * m + i] : 0.0;
        }
        for (int e = 0; e < n; e++) {
            double s = 0.0;
            for (int i = 0; i < jj; i++) s += yv[i] * V[(size_t)i * n + e];
            w[e] = s;
        }
        orc_lu_solve(n, pinv, Lp, Li, Lx, Up, Ui, Ux, q, w, z);
        for (int e = 0; e < n; e++) x[e] += z[e];
    }
    if (nres) *nres = cnt;
    free(V); free(H); free(cs); free(sn); free(g); free(yv); free(w); free(z); free(r);
    return total;
}
