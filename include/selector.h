/*
 * selector.h - SpMV format x precision-path policy.
 *
 * Drop-in for LUspice src/selector.h:5-60: same structs, enums and functions
 * with the same meaning.  Unlike the reference header this one carries an
 * extern "C" guard, so C++ callers need no wrapper (a wrapper they already
 * have stays harmless).
 *
 * Escalation chain (src/selector.c:82-90): P-fast (fp32 factor + fp64 pivot
 * + fp64-residual IR) -> P-safe (fp64 factor + Ruiz + diagonal shift + IR)
 * -> P-hard -> P-sing (terminal).  Escalation is triggered by a failed trial
 * (IR stagnation, pivot degradation) reported by the solver, never by a
 * condition-number threshold.
 */
#ifndef DSH_SELECTOR_H
#define DSH_SELECTOR_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/selector.h:5-14 */
typedef struct {
    int n;
    long nnz;
    double avg_rowlen, max_rowlen, p50_rowlen;
    double row_skew;
    double kappa_ruiz;
    double kappa_est;
    double dyn_range_log10;
    int    singular_flag;
} dsh_matrix_info;

/* src/selector.h:16-21 */
enum {
    DSH_FMT_CSR = 0,
    DSH_FMT_SELL_C_SIGMA = 1,
    DSH_FMT_ELL = 2
};
enum { DSH_PREC_FP32 = 0, DSH_PREC_FP64 = 1 };

/* src/selector.h:30-35 */
enum {
    DSH_MP_PFAST = 0,
    DSH_MP_PSAFE = 1,
    DSH_MP_PHARD = 2,
    DSH_MP_PSING = 3
};

/* src/selector.h:37-50 */
typedef struct {
    int spmv_format;
    int sigma;
    int use_ruiz;
    int use_shift;
    double shift;
    int factor_prec;
    int ir_outer, ir_inner;
    double ir_rtol;
    int mp_path;
    int pre_ruiz_hint;
    int fp16_candidate;
} dsh_config;

/* src/selector.h:52 : row-length statistics from a CSR row pointer. */
void dsh_matrix_analyze(int n, long nnz, const int *rowptr, dsh_matrix_info *info);
/* src/selector.h:53 */
void dsh_format_select(const dsh_matrix_info *info, dsh_config *cfg);
/* src/selector.h:54 */
const char *dsh_fmt_name(int fmt);
/* src/selector.h:57 */
void dsh_mp_initial(const dsh_matrix_info *info, dsh_config *cfg);
/* src/selector.h:59 */
int  dsh_mp_escalate(int cur);
/* src/selector.h:60 */
const char *dsh_mp_name(int p);

#ifdef __cplusplus
}
#endif

#endif /* DSH_SELECTOR_H */
