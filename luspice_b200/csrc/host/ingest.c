/* Netlist matrix ingest for replaying real circuits: s0 and Matrix Market
 * files as 1-based COO triplets, the floating-node pin list (".flt" files,
 * "F <row>" lines) applied to the COO diagonal, and COO -> CSC for
 * lusp_pattern_create.
 *
 * The pin follows the reference's replay programs (bench/test_lu.c:71-93,
 * bench/test_lu_gpu_par.cu apply_flt_pin): for each listed row i the first
 * stored (i, i) entry gains pin; a row without one gets a new (i, i) entry
 * of value pin appended at the end.  Nothing else changes. */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "luspice_b200.h"

static int coo_reserve(lusp_coo *A, long long want)
{
    if (want <= A->cap) return 0;
    long long cap = A->cap > 0 ? A->cap : 1024;
    while (cap < want) cap *= 2;
    int *r = (int *)realloc(A->row, (size_t)cap * sizeof(int));
    if (r) A->row = r;
    int *c = (int *)realloc(A->col, (size_t)cap * sizeof(int));
    if (c) A->col = c;
    double *v = (double *)realloc(A->val, (size_t)cap * sizeof(double));
    if (v) A->val = v;
    if (!r || !c || !v) return 1;
    A->cap = cap;
    return 0;
}

static int coo_push(lusp_coo *A, int i, int j, double v)
{
    if (A->nnz == A->cap && coo_reserve(A, A->nnz + 1)) return 1;
    A->row[A->nnz] = i;
    A->col[A->nnz] = j;
    A->val[A->nnz] = v;
    A->nnz++;
    return 0;
}

void lusp_coo_free(lusp_coo *A)
{
    if (!A) return;
    free(A->row);
    free(A->col);
    free(A->val);
    memset(A, 0, sizeof(*A));
}

int lusp_read_s0_coo(const char *path, lusp_coo *A)
{
    if (!path || !A) return LUSP_EARG;
    memset(A, 0, sizeof(*A));
    FILE *f = fopen(path, "r");
    if (!f) return LUSP_EARG;
    char line[512];
    int n = 0, rc = LUSP_OK;
    if (!fgets(line, sizeof line, f) || sscanf(line, "n %d", &n) != 1 || n <= 0) rc = LUSP_EARG;
    A->n = n;
    while (rc == LUSP_OK && fgets(line, sizeof line, f)) {
        if (line[0] != 'A') continue;
        int i, j;
        double v;
        if (sscanf(line, "A %d %d %lf", &i, &j, &v) != 3) continue;
        if (i < 1 || i > n || j < 1 || j > n) rc = LUSP_EARG;
        else if (coo_push(A, i, j, v)) rc = LUSP_EALLOC;
    }
    fclose(f);
    if (rc != LUSP_OK) lusp_coo_free(A);
    return rc;
}

/* Case-insensitive word test of the banner. */
static int has_word(const char *s, const char *w)
{
    size_t lw = strlen(w);
    for (; *s; s++) {
        size_t k = 0;
        while (k < lw && s[k] && tolower((unsigned char)s[k]) == w[k]) k++;
        if (k == lw) return 1;
    }
    return 0;
}

int lusp_read_mtx_coo(const char *path, lusp_coo *A)
{
    if (!path || !A) return LUSP_EARG;
    memset(A, 0, sizeof(*A));
    FILE *f = fopen(path, "r");
    if (!f) return LUSP_EARG;
    char line[1024];
    int rc = LUSP_OK;
    if (!fgets(line, sizeof line, f) || strncmp(line, "%%MatrixMarket", 14) != 0 || !has_word(line, "coordinate") ||
        has_word(line, "complex")) {
        fclose(f);
        return LUSP_EARG;
    }
    const int pattern = has_word(line, "pattern");
    const int sym = has_word(line, "symmetric") && !has_word(line, "skew");
    const int skew = has_word(line, "skew-symmetric");
    long long m = -1, ncol = -1, nz = -1;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%' || line[0] == '\n' || line[0] == '\r') continue;
        if (sscanf(line, "%lld %lld %lld", &m, &ncol, &nz) != 3) rc = LUSP_EARG;
        break;
    }
    if (rc == LUSP_OK && (m <= 0 || m != ncol || nz < 0 || m > 0x7fffffff)) rc = LUSP_EARG;
    if (rc == LUSP_OK) {
        A->n = (int)m;
        if (coo_reserve(A, (sym || skew) ? 2 * nz : nz)) rc = LUSP_EALLOC;
    }
    long long got = 0;
    while (rc == LUSP_OK && got < nz && fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        int i, j;
        double v = 1.0;
        const int k = pattern ? sscanf(line, "%d %d", &i, &j) : sscanf(line, "%d %d %lf", &i, &j, &v);
        if (k != (pattern ? 2 : 3)) continue;
        if (i < 1 || i > A->n || j < 1 || j > A->n) { rc = LUSP_EARG; break; }
        got++;
        if (coo_push(A, i, j, v)) { rc = LUSP_EALLOC; break; }
        if ((sym || skew) && i != j && coo_push(A, j, i, skew ? -v : v)) rc = LUSP_EALLOC;
    }
    fclose(f);
    if (rc == LUSP_OK && got != nz) rc = LUSP_EARG;
    if (rc != LUSP_OK) lusp_coo_free(A);
    return rc;
}

int lusp_read_flt(const char *path, int n, int *rows, int cap, int *count)
{
    if (!path || !count || n <= 0 || cap < 0 || (cap > 0 && !rows)) return LUSP_EARG;
    *count = 0;
    FILE *f = fopen(path, "r");
    if (!f) return LUSP_EARG;
    char line[256];
    int rc = LUSP_OK;
    while (fgets(line, sizeof line, f)) {
        int r;
        if (sscanf(line, "F %d", &r) != 1) continue;
        if (r < 1 || r > n) { rc = LUSP_EARG; break; }
        if (*count < cap) rows[*count] = r - 1;
        ++*count;
    }
    fclose(f);
    if (rc == LUSP_OK && *count > cap) rc = LUSP_EALLOC;
    return rc;
}

int lusp_coo_pin_rows(lusp_coo *A, const int *rows, int count, double pin)
{
    if (!A || count < 0 || (count > 0 && !rows)) return LUSP_EARG;
    if (!(pin > 0.0) || count == 0) return LUSP_OK;
    for (int t = 0; t < count; t++)
        if (rows[t] < 0 || rows[t] >= A->n) return LUSP_EARG;
    /* first stored (i, i) entry of every row, in storage order */
    long long *first = (long long *)malloc((size_t)A->n * sizeof(long long));
    if (!first) return LUSP_EALLOC;
    for (int i = 0; i < A->n; i++) first[i] = -1;
    for (long long p = 0; p < A->nnz; p++) {
        const int i = A->row[p] - 1;
        if (A->row[p] == A->col[p] && first[i] < 0) first[i] = p;
    }
    int rc = LUSP_OK;
    for (int t = 0; t < count && rc == LUSP_OK; t++) {
        const int i = rows[t];
        if (first[i] >= 0) {
            A->val[first[i]] += pin;
        } else {
            if (coo_push(A, i + 1, i + 1, pin)) rc = LUSP_EALLOC;
            else first[i] = A->nnz - 1;
        }
    }
    free(first);
    return rc;
}

int lusp_coo_to_csc(const lusp_coo *A, int *Ap, int *Ai, double *Ax)
{
    if (!A || !Ap || A->n <= 0 || (A->nnz > 0 && (!Ai || !Ax)) || A->nnz > 0x7fffffff) return LUSP_EARG;
    const int n = A->n;
    memset(Ap, 0, (size_t)(n + 1) * sizeof(int));
    for (long long p = 0; p < A->nnz; p++) {
        if (A->row[p] < 1 || A->row[p] > n || A->col[p] < 1 || A->col[p] > n) return LUSP_EARG;
        Ap[A->col[p]]++;
    }
    for (int j = 0; j < n; j++) Ap[j + 1] += Ap[j];
    int *cur = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    if (!cur) return LUSP_EALLOC;
    memcpy(cur, Ap, (size_t)n * sizeof(int));
    /* storage order within a column; duplicates stay separate entries (the
     * pattern analysis sums them) */
    for (long long p = 0; p < A->nnz; p++) {
        const int q = cur[A->col[p] - 1]++;
        Ai[q] = A->row[p] - 1;
        Ax[q] = A->val[p];
    }
    free(cur);
    return LUSP_OK;
}
