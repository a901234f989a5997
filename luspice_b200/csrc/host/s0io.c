/* s0 matrix / RHS readers (format of src/spmv.h:9-14): a header line
 * "n <n>" then "A <i> <j> <val>" lines (1-based); RHS files list
 * "RHS <i> <val>".  The CSR keeps entries of a row in file order, as the
 * reference's reader does (src/spmv.cu:42-136). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spmv.h"

int read_s0_to_csr(const char *path, CSRMatrix *A)
{
    if (!path || !A) return 1;
    memset(A, 0, sizeof(*A));
    FILE *f = fopen(path, "r");
    if (!f) return 1;
    char line[512];
    int n = 0;
    if (!fgets(line, sizeof line, f) || sscanf(line, "n %d", &n) != 1 || n <= 0) {
        fclose(f);
        return 1;
    }
    long long cap = 1024, cnt = 0;
    int *ri = (int *)malloc((size_t)cap * sizeof(int));
    int *ci = (int *)malloc((size_t)cap * sizeof(int));
    double *vv = (double *)malloc((size_t)cap * sizeof(double));
    int ok = ri && ci && vv;
    while (ok && fgets(line, sizeof line, f)) {
        if (line[0] != 'A') continue;
        int i, j;
        double v;
        if (sscanf(line, "A %d %d %lf", &i, &j, &v) != 3) continue;
        if (i < 1 || i > n || j < 1 || j > n) { ok = 0; break; }
        if (cnt == cap) {
            cap *= 2;
            int *r2 = (int *)realloc(ri, (size_t)cap * sizeof(int));
            int *c2 = (int *)realloc(ci, (size_t)cap * sizeof(int));
            double *v2 = (double *)realloc(vv, (size_t)cap * sizeof(double));
            if (r2) ri = r2;
            if (c2) ci = c2;
            if (v2) vv = v2;
            if (!r2 || !c2 || !v2) { ok = 0; break; }
        }
        ri[cnt] = i - 1;
        ci[cnt] = j - 1;
        vv[cnt] = v;
        cnt++;
    }
    fclose(f);
    if (ok) {
        A->n = n;
        A->nnz = cnt;
        A->rowptr = (int *)calloc((size_t)n + 1, sizeof(int));
        A->colidx = (int *)malloc((size_t)(cnt ? cnt : 1) * sizeof(int));
        A->values = (double *)malloc((size_t)(cnt ? cnt : 1) * sizeof(double));
        ok = A->rowptr && A->colidx && A->values;
    }
    if (ok) {
        for (long long t = 0; t < cnt; t++) A->rowptr[ri[t] + 1]++;
        for (int i = 0; i < n; i++) A->rowptr[i + 1] += A->rowptr[i];
        int *cur = (int *)malloc((size_t)n * sizeof(int));
        ok = cur != NULL;
        if (ok) {
            memcpy(cur, A->rowptr, (size_t)n * sizeof(int));
            for (long long t = 0; t < cnt; t++) {
                int p = cur[ri[t]]++;
                A->colidx[p] = ci[t];
                A->values[p] = vv[t];
            }
            free(cur);
        }
    }
    free(ri);
    free(ci);
    free(vv);
    if (!ok) {
        csr_free(A);
        return 1;
    }
    return 0;
}

void csr_free(CSRMatrix *A)
{
    if (!A) return;
    free(A->rowptr);
    free(A->colidx);
    free(A->values);
    A->rowptr = NULL;
    A->colidx = NULL;
    A->values = NULL;
    A->n = 0;
    A->nnz = 0;
}

int read_rhs(const char *path, int n, double *x)
{
    if (!path || !x || n <= 0) return 1;
    FILE *f = fopen(path, "r");
    if (!f) return 1;
    char line[512];
    int got = 0;
    for (int i = 0; i < n; i++) x[i] = 0.0;
    while (fgets(line, sizeof line, f)) {
        int i;
        double v;
        if (sscanf(line, "RHS %d %lf", &i, &v) != 2) continue;
        if (i >= 1 && i <= n) { x[i - 1] = v; got++; }
    }
    fclose(f);
    return got > 0 ? 0 : 1;
}
