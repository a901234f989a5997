// dsh_* static-LU handle (lu_static.h) on top of the batched engine: one
// pattern and a one-system batch per handle.  See lu_static.h for the
// ownership and index conventions.
#include "lu_static.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "luspice_b200.h"

namespace {

std::atomic<long> g_symbolic_count{0};

struct DshState {
    int n = 0;
    long cnnz = 0;
    std::vector<int> coo_row, coo_col;     // pattern as given (1-based)
    std::vector<int> Ap, Ai;               // 0-based CSC, rows ascending, unique
    std::vector<int> coo2csc;              // COO entry -> CSC entry
    std::vector<int> diag_slot;            // CSC entry of A(i,i) or -1
    std::vector<int> q;
    lusp_pattern* pat = nullptr;
    lusp_batch* batch = nullptr;
    int batch_m = 0;

    ~DshState() {
        if (batch) lusp_batch_destroy(batch);
        if (pat) lusp_pattern_destroy(pat);
    }
};

DshState* state_of(const dsh_lu_static* F) { return F ? (DshState*)F->factor_cache : nullptr; }

void drop_engine(DshState* S) {
    if (S->batch) lusp_batch_destroy(S->batch);
    if (S->pat) lusp_pattern_destroy(S->pat);
    S->batch = nullptr;
    S->pat = nullptr;
    S->batch_m = 0;
}

int make_batch(DshState* S, int m) {
    lusp_batch_opts o;
    lusp_batch_opts_default(&o);
    o.prec = LUSP_MIXED;
    o.krylov = m;
    o.ctas_per_sm = 1;
    lusp_batch* b = nullptr;
    int rc = lusp_batch_create(1, &S->pat, &o, &b);
    if (rc != LUSP_OK) return rc;
    if (S->batch) lusp_batch_destroy(S->batch);
    S->batch = b;
    S->batch_m = m;
    return LUSP_OK;
}

// Publish the static structure and diagnostics into the C struct.
int publish(dsh_lu_static* F, DshState* S, const std::vector<double>& csc_vals) {
    lusp_pattern_info info;
    lusp_pattern_get_info(S->pat, &info);
    F->lnnz = info.lnnz;
    F->unnz = info.unnz;
    F->cap = info.cap;
    free(F->Ap);
    free(F->Ai);
    free(F->P);
    F->Ap = (int*)malloc(sizeof(int) * ((size_t)S->n + 1));
    F->Ai = (int*)malloc(sizeof(int) * (size_t)std::max<long>(info.cap, 1));
    F->P = (int*)malloc(sizeof(int) * (size_t)S->n);
    if (!F->Ap || !F->Ai || !F->P) return 2;
    lusp_pattern_get_structure(S->pat, F->Ap, F->Ai, nullptr);
    lusp_pattern_get_perm(S->pat, F->P, nullptr);
    void* dptr = nullptr;
    lusp_batch_factor_device_ptr(S->batch, 0, &dptr);
    F->Ax = (float*)dptr;
    F->dev_allocated = 1;
    lusp_sys_stats st;
    if (lusp_batch_stats(S->batch, &st, nullptr) != LUSP_OK) return 2;
    double amax = 0.0;
    for (double v : csc_vals) amax = std::max(amax, std::fabs(v));
    F->min_diag_U = st.min_abs_pivot;
    F->pivot_growth = amax > 0 ? st.max_abs_u / amax : 0.0;
    if (st.status & LUSP_ST_SINGULAR) return 1;
    return 0;
}

}  // namespace

extern "C" {

long dsh_symbolic_count(void) { return g_symbolic_count.load(); }

int dsh_lu_static_init(dsh_lu_static* F) {
    if (!F) return 3;
    memset(F, 0, sizeof(*F));
    return 0;
}

int dsh_lu_static_alloc(dsh_lu_static* F) {
    if (!F || F->n <= 0 || F->cap <= 0) return 3;
    // Device storage is created with the factorization; nothing to add.
    F->dev_allocated = state_of(F) && state_of(F)->batch ? 1 : 0;
    return 0;
}

void dsh_lu_static_free(dsh_lu_static* F) {
    if (!F) return;
    delete state_of(F);
    free(F->Ap);
    free(F->Ai);
    free(F->P);
    free(F->Q);
    F->Ap = F->Ai = F->P = F->Q = nullptr;
    F->Ax = nullptr;
    F->factor_cache = nullptr;
    F->dev_allocated = 0;
}

int dsh_symbolic(int n, long cnnz, const int* coo_row, const int* coo_col, const int* colamd_q,
                 dsh_lu_static* F) {
    if (!F || n <= 0 || cnnz <= 0 || !coo_row || !coo_col) return 3;
    for (long e = 0; e < cnnz; e++)
        if (coo_row[e] < 1 || coo_row[e] > n || coo_col[e] < 1 || coo_col[e] > n) return 3;
    DshState* S = nullptr;
    try {
        S = new DshState();
        S->n = n;
        S->cnnz = cnnz;
        S->coo_row.assign(coo_row, coo_row + cnnz);
        S->coo_col.assign(coo_col, coo_col + cnnz);
        // Column-major order of the entries, rows ascending; duplicates merge.
        std::vector<long> ord(cnnz);
        for (long e = 0; e < cnnz; e++) ord[e] = e;
        std::stable_sort(ord.begin(), ord.end(), [&](long a, long b) {
            if (coo_col[a] != coo_col[b]) return coo_col[a] < coo_col[b];
            return coo_row[a] < coo_row[b];
        });
        S->Ap.assign(n + 1, 0);
        S->coo2csc.assign(cnnz, -1);
        int lastr = -1, lastc = -1;
        for (long t = 0; t < cnnz; t++) {
            const long e = ord[t];
            const int r = coo_row[e] - 1, c = coo_col[e] - 1;
            if (r != lastr || c != lastc) {
                S->Ai.push_back(r);
                S->Ap[c + 1]++;
                lastr = r;
                lastc = c;
            }
            S->coo2csc[e] = (int)S->Ai.size() - 1;
        }
        for (int c = 0; c < n; c++) S->Ap[c + 1] += S->Ap[c];
        S->diag_slot.assign(n, -1);
        for (int c = 0; c < n; c++)
            for (int p = S->Ap[c]; p < S->Ap[c + 1]; p++)
                if (S->Ai[p] == c) S->diag_slot[c] = p;
        S->q.resize(n);
        if (colamd_q) {
            std::vector<char> seen(n, 0);
            for (int k = 0; k < n; k++) {
                if (colamd_q[k] < 0 || colamd_q[k] >= n || seen[colamd_q[k]]) { delete S; return 3; }
                seen[colamd_q[k]] = 1;
                S->q[k] = colamd_q[k];
            }
        } else {
            for (int k = 0; k < n; k++) S->q[k] = k;
        }
    } catch (const std::bad_alloc&) {
        delete S;
        return 2;
    }
    delete state_of(F);
    free(F->Ap);
    free(F->Ai);
    free(F->P);
    free(F->Q);
    F->Ap = F->Ai = F->P = nullptr;
    F->Ax = nullptr;
    F->factor_cache = S;
    F->n = n;
    F->cnnz = cnnz;
    F->lnnz = F->unnz = F->cap = 0;
    F->Q = (int*)malloc(sizeof(int) * (size_t)n);
    if (!F->Q) return 2;
    memcpy(F->Q, S->q.data(), sizeof(int) * (size_t)n);
    g_symbolic_count++;
    return 0;
}

int dsh_numeric(dsh_lu_static* F, const int* coo_row, const int* coo_col, const double* coo_val,
                int nnz) {
    DshState* S = state_of(F);
    if (!S || !coo_row || !coo_col || !coo_val || nnz != S->cnnz) return 3;
    for (long e = 0; e < nnz; e++)
        if (coo_row[e] != S->coo_row[e] || coo_col[e] != S->coo_col[e]) return 3;
    std::vector<double> vals(S->Ai.size(), 0.0);
    for (long e = 0; e < nnz; e++) vals[S->coo2csc[e]] += coo_val[e];
    if (F->pin > 0)
        for (int i = 0; i < S->n; i++)
            if (S->diag_slot[i] >= 0) vals[S->diag_slot[i]] += F->pin;
    std::vector<double> zero_rhs(S->n, 0.0);
    for (int attempt = 0; attempt < 2; attempt++) {
        if (!S->pat) {
            int rc = lusp_pattern_create(S->n, S->Ap.data(), S->Ai.data(), vals.data(), S->q.data(), &S->pat);
            if (rc == LUSP_ESINGULAR) { F->min_diag_U = 0.0; return 1; }
            if (rc != LUSP_OK) return rc == LUSP_EARG ? 3 : 2;
            rc = make_batch(S, 50);
            if (rc != LUSP_OK) { drop_engine(S); return 2; }
        }
        if (lusp_batch_upload(S->batch, vals.data(), zero_rhs.data(), nullptr) != LUSP_OK) return 2;
        if (lusp_batch_run(S->batch, LUSP_RUN_REFACTOR, nullptr) != LUSP_OK) return 2;
        lusp_sys_stats st;
        if (lusp_batch_stats(S->batch, &st, nullptr) != LUSP_OK) return 2;
        // Frozen pivots no longer acceptable for these values: decide them
        // again on the host (same column order), once.
        if ((st.status & (LUSP_ST_PIVOT_WEAK | LUSP_ST_SINGULAR)) && attempt == 0) {
            drop_engine(S);
            continue;
        }
        return publish(F, S, vals);
    }
    return 1;
}

int dsh_trisolve(const dsh_lu_static* F, const double* b, double* x) {
    DshState* S = state_of(F);
    if (!S || !S->batch || !b || !x) return 3;
    if (lusp_batch_upload(S->batch, nullptr, b, nullptr) != LUSP_OK) return 2;
    if (lusp_batch_run(S->batch, LUSP_RUN_SOLVE | LUSP_RUN_DIRECT, nullptr) != LUSP_OK) return 2;
    if (lusp_batch_download(S->batch, x, nullptr) != LUSP_OK) return 2;
    lusp_sys_stats st;
    if (lusp_batch_stats(S->batch, &st, nullptr) != LUSP_OK) return 2;
    return 0;
}

int dsh_gmres_ir(dsh_lu_static* F, const double* b, double* x, int max_outer, int max_inner,
                 double rtol, double* residual_seq, int* iters) {
    DshState* S = state_of(F);
    if (!S || !S->batch || !b || !x) return 3;
    const int m = max_inner <= 0 ? 50 : std::min(max_inner, 64);
    if (m != S->batch_m) {
        // The Krylov dimension sizes the workspace: rebuild the batch and
        // refactor into it.
        lusp_batch* old = S->batch;
        S->batch = nullptr;
        int rc = make_batch(S, m);
        if (rc != LUSP_OK) { S->batch = old; return 2; }
        rc = lusp_batch_copy_values(S->batch, old, nullptr);
        lusp_batch_destroy(old);
        if (rc != LUSP_OK) return 2;
        if (lusp_batch_run(S->batch, LUSP_RUN_REFACTOR, nullptr) != LUSP_OK) return 2;
    }
    lusp_batch_opts o;
    lusp_batch_opts_default(&o);
    o.max_outer = max_outer <= 0 ? 3 : max_outer;
    o.rtol = rtol > 0 ? rtol : 1e-10;
    lusp_batch_set_params(S->batch, &o);
    if (lusp_batch_upload(S->batch, nullptr, b, nullptr) != LUSP_OK) return 2;
    if (lusp_batch_run(S->batch, LUSP_RUN_SOLVE, nullptr) != LUSP_OK) return 2;
    if (lusp_batch_download(S->batch, x, nullptr) != LUSP_OK) return 2;
    lusp_sys_stats st;
    if (lusp_batch_stats(S->batch, &st, nullptr) != LUSP_OK) return 2;
    if (residual_seq)
        for (int t = 0; t < st.nres && t <= o.max_outer; t++) residual_seq[t] = st.res[t];
    if (iters) *iters = st.inner_iters;
    if (st.status & LUSP_ST_SINGULAR) return 1;
    if (st.status & (LUSP_ST_STAGNATED | LUSP_ST_NOT_CONVERGED | LUSP_ST_NONFINITE)) return 4;
    return 0;
}

const char* dsh_lu_status_str(int rc) {
    switch (rc) {
    case 0: return "OK";
    case 1: return "SINGULAR";
    case 2: return "ALLOC";
    case 3: return "ARG/NOT_IMPL";
    case 4: return "IR_STAGNATED";
    default: return "UNKNOWN";
    }
}

}  // extern "C"
