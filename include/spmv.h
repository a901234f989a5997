/*
 * spmv.h - sparse matrix-vector product y = A*x on one B200, plus the s0
 * matrix / RHS readers.
 *
 * Drop-in for LUspice src/spmv.h:23-57 (same struct, names, signatures and
 * return conventions: 0 = success, nonzero = failure).  The s0 format
 * (src/spmv.h:9-14): first line "n <n>" (an optional second number is
 * ignored), then lines "A <i> <j> <val>" with 1-based i, j; RHS files: first
 * line "n <n>", then "RHS <i> <val>" lines, 1-based.
 *
 * spmv_launch runs a warp-cooperative fp64 CSR kernel (vectorised index and
 * value loads, fp64 accumulation) on the given stream.  The SELL-C-sigma
 * path the solver uses internally is exposed through luspice_b200.h
 * (lusp_sell_*).
 */
#ifndef RACE7_SOLVER_SPMV_H
#define RACE7_SOLVER_SPMV_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/spmv.h:26-32 */
typedef struct {
    int n;
    long long nnz;
    int* rowptr;
    int* colidx;
    double* values;
} CSRMatrix;

/* src/spmv.h:34 : s0 file -> 0-based CSR, entries of a row in file order
 * (duplicates kept as separate entries, as the file lists them). */
int read_s0_to_csr(const char* path, CSRMatrix* A);

/* src/spmv.h:37 */
void csr_free(CSRMatrix* A);

/* src/spmv.h:40 : returns nonzero when no RHS line was read. */
int read_rhs(const char* path, int n, double* x);

/* src/spmv.h:45 : one full device round trip (alloc, H2D, kernel, D2H,
 * free); time_ms (may be NULL) receives one kernel time after a warm-up. */
int spmv_host(const CSRMatrix* A, const double* x, double* y, double* time_ms);

/* src/spmv.h:49-50 */
int csr_alloc_device(const CSRMatrix* A,
                     int** d_rowptr, int** d_colidx, double** d_values);

/* src/spmv.h:55-57 : stream is a cudaStream_t passed as void* (0 = default). */
void spmv_launch(int n,
                 const int* d_rowptr, const int* d_colidx, const double* d_values,
                 const double* d_x, double* d_y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RACE7_SOLVER_SPMV_H */
