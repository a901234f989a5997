/* Format x precision-path policy: the reference's decision rules
 * (src/selector.c:26-137) restated.
 *   format : SELL-C-sigma (sigma 32) iff n >= 5000 and row_skew <= 5, else CSR
 *            (src/selector.c:108-114)
 *   path   : always start at P-fast; P-sing when the matrix is flagged
 *            singular; pre_ruiz_hint when kappa_ruiz > 1e12 or the dynamic
 *            range exceeds 1e20; fp16_candidate when 0 < dyn_range_log10 <= 1
 *            and 0 < kappa_ruiz <= 1e6 (src/selector.c:59-80)
 *   IR     : outer 3, inner 50, rtol 1e-9; shift 1e-7 on (src/selector.c:120-126)
 * The median row length uses a counting sort (O(n + max_len)); the reference
 * uses an insertion sort with the same result. */
#include <stdlib.h>
#include <string.h>

#include "selector.h"

void dsh_matrix_analyze(int n, long nnz, const int *rowptr, dsh_matrix_info *info)
{
    memset(info, 0, sizeof(*info));
    info->n = n;
    info->nnz = nnz;
    if (n <= 0 || !rowptr) return;
    long total = 0;
    int longest = 0;
    for (int i = 0; i < n; i++) {
        int len = rowptr[i + 1] - rowptr[i];
        if (len < 0) len = 0;
        total += len;
        if (len > longest) longest = len;
    }
    int *hist = (int *)calloc((size_t)longest + 1, sizeof(int));
    int median = 0;
    if (hist) {
        for (int i = 0; i < n; i++) {
            int len = rowptr[i + 1] - rowptr[i];
            hist[len < 0 ? 0 : len]++;
        }
        /* element n/2 of the ascending order */
        long seen = 0;
        for (int l = 0; l <= longest; l++) {
            seen += hist[l];
            if (seen > n / 2) { median = l; break; }
        }
        free(hist);
    }
    info->avg_rowlen = (double)total / n;
    info->max_rowlen = longest;
    info->p50_rowlen = median;
    info->row_skew = info->avg_rowlen > 0 ? (double)longest / info->avg_rowlen : 0.0;
}

void dsh_mp_initial(const dsh_matrix_info *info, dsh_config *cfg)
{
    cfg->mp_path = DSH_MP_PFAST;
    cfg->pre_ruiz_hint = 0;
    cfg->fp16_candidate = 0;
    if (info->singular_flag) {
        cfg->mp_path = DSH_MP_PSING;
        return;
    }
    if (info->kappa_ruiz > 1e12 || info->dyn_range_log10 > 20.0)
        cfg->pre_ruiz_hint = 1;
    if (info->dyn_range_log10 > 0 && info->dyn_range_log10 <= 1.0 &&
        info->kappa_ruiz > 0 && info->kappa_ruiz <= 1e6)
        cfg->fp16_candidate = 1;
}

int dsh_mp_escalate(int cur)
{
    if (cur == DSH_MP_PFAST) return DSH_MP_PSAFE;
    if (cur == DSH_MP_PSAFE) return DSH_MP_PHARD;
    return DSH_MP_PSING;
}

const char *dsh_mp_name(int p)
{
    static const char *names[] = {"P-fast", "P-safe", "P-hard", "P-sing"};
    return (p >= 0 && p <= 3) ? names[p] : "?";
}

void dsh_format_select(const dsh_matrix_info *info, dsh_config *cfg)
{
    memset(cfg, 0, sizeof(*cfg));
    int sell = info->n >= 5000 && info->row_skew <= 5.0;
    cfg->spmv_format = sell ? DSH_FMT_SELL_C_SIGMA : DSH_FMT_CSR;
    cfg->sigma = sell ? 32 : 0;
    dsh_mp_initial(info, cfg);
    cfg->factor_prec = cfg->mp_path == DSH_MP_PFAST ? DSH_PREC_FP32 : DSH_PREC_FP64;
    cfg->use_ruiz = cfg->pre_ruiz_hint;
    cfg->use_shift = 1;
    cfg->shift = 1e-7;
    cfg->ir_outer = 3;
    cfg->ir_inner = 50;
    cfg->ir_rtol = 1e-9;
}

const char *dsh_fmt_name(int fmt)
{
    switch (fmt) {
    case DSH_FMT_CSR: return "CSR";
    case DSH_FMT_SELL_C_SIGMA: return "SELL-C-sigma32";
    case DSH_FMT_ELL: return "ELL";
    default: return "?";
    }
}
