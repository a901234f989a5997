// lusp_* C-ABI: thin, exception-free wrappers over the engine objects.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "luspice_b200.h"
#include "engine_internal.h"

using lusp::BatchObj;
using lusp::PatternObj;

namespace lusp {
const char* last_error_cstr();
}

static PatternObj* PO(lusp_pattern* h) { return reinterpret_cast<PatternObj*>(h); }
static const PatternObj* PO(const lusp_pattern* h) { return reinterpret_cast<const PatternObj*>(h); }
static BatchObj* BO(lusp_batch* h) { return reinterpret_cast<BatchObj*>(h); }
static const BatchObj* BO(const lusp_batch* h) { return reinterpret_cast<const BatchObj*>(h); }

extern "C" {

const char* lusp_last_error(void) { return lusp::last_error_cstr(); }

const char* lusp_version(void) { return "luspice_b200 0.1 (sm_100a)"; }

int lusp_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return c;
}

int lusp_pattern_create(int n, const int* Ap, const int* Ai, const double* Ax, const int* q,
                        lusp_pattern** out) {
    return lusp_pattern_create_ex(n, Ap, Ai, Ax, q, -1, out);
}

int lusp_pattern_create_ex(int n, const int* Ap, const int* Ai, const double* Ax, const int* q,
                           int dense_tail, lusp_pattern** out) {
    if (!out) return LUSP_EARG;
    *out = nullptr;
    if (dense_tail < -1) { lusp::set_error("pattern_create: dense_tail must be >= -1"); return LUSP_EARG; }
    try {
        PatternObj* P = nullptr;
        int rc = lusp::pattern_build(n, Ap, Ai, Ax, q, &P, dense_tail);
        if (rc == LUSP_OK) *out = reinterpret_cast<lusp_pattern*>(P);
        return rc;
    } catch (const std::bad_alloc&) {
        lusp::set_error("pattern_create: host allocation failed");
        return LUSP_EALLOC;
    }
}

void lusp_pattern_destroy(lusp_pattern* p) { lusp::pattern_free(PO(p)); }

int lusp_pattern_get_info(const lusp_pattern* hp, lusp_pattern_info* info) {
    if (!hp || !info) return LUSP_EARG;
    const lusp::StaticPattern& S = PO(hp)->S;
    memset(info, 0, sizeof(*info));
    info->n = S.n;
    info->nnz_a = S.nnz_a;
    info->lnnz = S.lnnz;
    info->unnz = S.unnz;
    info->cap = S.cap;
    info->ncol_levels = S.ncol_levels;
    info->nfwd_levels = S.nfwd_levels;
    info->nbwd_levels = S.nbwd_levels;
    info->max_col = S.max_col;
    info->nslices = S.nslices;
    info->sell_total = S.sell_ptr.empty() ? 0 : S.sell_ptr.back();
    info->flops = S.flops;
    info->gathered = S.gathered;
    info->hash = S.hash;
    info->device_bytes = PO(hp)->bytes;
    info->singular_col = -1;
    info->dense_tail = S.dtail;
    info->tail_start = S.k0;
    return LUSP_OK;
}

int lusp_pattern_get_perm(const lusp_pattern* hp, int* pinv, int* q) {
    if (!hp) return LUSP_EARG;
    const lusp::StaticPattern& S = PO(hp)->S;
    if (pinv) std::copy(S.pinv.begin(), S.pinv.end(), pinv);
    if (q) std::copy(S.q.begin(), S.q.end(), q);
    return LUSP_OK;
}

int lusp_pattern_get_structure(const lusp_pattern* hp, int* cp, int* ri, int* dg) {
    if (!hp) return LUSP_EARG;
    const lusp::StaticPattern& S = PO(hp)->S;
    if (cp) std::copy(S.cp.begin(), S.cp.end(), cp);
    if (ri) std::copy(S.ri.begin(), S.ri.end(), ri);
    if (dg) std::copy(S.dg.begin(), S.dg.end(), dg);
    return LUSP_OK;
}

int lusp_pattern_get_levels(const lusp_pattern* hp, int* col_level) {
    if (!hp || !col_level) return LUSP_EARG;
    const lusp::StaticPattern& S = PO(hp)->S;
    std::copy(S.col_level.begin(), S.col_level.end(), col_level);
    return LUSP_OK;
}

int lusp_colamd(int n_row, int n_col, const int* Ap, const int* Ai, double knob_dense_row,
                double knob_dense_col, int* q) {
    try {
        return lusp::colamd_order(n_row, n_col, Ap, Ai, knob_dense_row, knob_dense_col, q) == 0
                   ? LUSP_OK
                   : LUSP_EARG;
    } catch (const std::bad_alloc&) {
        return LUSP_EALLOC;
    }
}

int lusp_pivot_factor(int n, const int* Ap, const int* Ai, const double* Ax, const int* q,
                      double tol, int* pinv, int* Lp, int* Li, double* Lx, long lcap, int* Up,
                      int* Ui, double* Ux, long ucap, long* lnnz, long* unnz, int* singular_col) {
    if (n <= 0 || !Ap || !Ai || !Ax) return LUSP_EARG;
    try {
        lusp::PivotFactor F;
        const int sc = lusp::pivot_factor(n, Ap, Ai, Ax, q, tol, F);
        if (singular_col) *singular_col = sc;
        if (sc >= 0) return LUSP_ESINGULAR;
        const long ln = F.Lp[n], un = F.Up[n];
        if (lnnz) *lnnz = ln;
        if (unnz) *unnz = un;
        if (ln > lcap || un > ucap) return LUSP_EALLOC;
        if (pinv) std::copy(F.pinv.begin(), F.pinv.end(), pinv);
        if (Lp) std::copy(F.Lp.begin(), F.Lp.end(), Lp);
        if (Up) std::copy(F.Up.begin(), F.Up.end(), Up);
        if (Li) std::copy(F.Li.begin(), F.Li.end(), Li);
        if (Lx) std::copy(F.Lx.begin(), F.Lx.end(), Lx);
        if (Ui) std::copy(F.Ui.begin(), F.Ui.end(), Ui);
        if (Ux) std::copy(F.Ux.begin(), F.Ux.end(), Ux);
        return LUSP_OK;
    } catch (const std::bad_alloc&) {
        return LUSP_EALLOC;
    }
}

void lusp_batch_opts_default(lusp_batch_opts* o) {
    if (!o) return;
    o->prec = LUSP_MIXED;
    o->krylov = 30;
    o->max_outer = 3;
    o->rtol = 1e-10;
    o->inner_rel = 1e-4;
    o->stag_ratio = 0.5;
    o->pivot_tol = 1e-3;
    o->block_threads = 0;
    o->ctas_per_sm = 0;
    o->solve_sweep = 0;
    o->refactor_mode = 0;
    o->inner_prec = 0;
    o->xtol = 1e-8;
    o->refactor_threads = 0;
    o->refactor_cluster = 0;
    o->refactor_spread = 0;
    o->ladder = 0;
    o->ladder_slots = 0;
    o->factor_shift = 0.0;
    o->hard_shift = 1e-7;
}

int lusp_batch_create(int nsys, lusp_pattern* const* pats, const lusp_batch_opts* opts,
                      lusp_batch** out) {
    if (!out || !pats) return LUSP_EARG;
    *out = nullptr;
    lusp_batch_opts o;
    if (opts) o = *opts; else lusp_batch_opts_default(&o);
    try {
        BatchObj* B = nullptr;
        int rc = lusp::batch_build(nsys, reinterpret_cast<PatternObj* const*>(pats), &o, &B);
        if (rc == LUSP_OK) *out = reinterpret_cast<lusp_batch*>(B);
        return rc;
    } catch (const std::bad_alloc&) {
        lusp::set_error("batch_create: host allocation failed");
        return LUSP_EALLOC;
    }
}

void lusp_batch_destroy(lusp_batch* b) { lusp::batch_free(BO(b)); }

int lusp_batch_device_ptrs(lusp_batch* hb, int sys, double** d_vals, double** d_rhs, double** d_x) {
    BatchObj* B = BO(hb);
    if (!B || sys < 0 || sys >= B->nsys) return LUSP_EARG;
    if (d_vals) *d_vals = const_cast<double*>(B->h_sys[sys].a_val);
    if (d_rhs) *d_rhs = const_cast<double*>(B->h_sys[sys].b);
    if (d_x) *d_x = B->h_sys[sys].x;
    return LUSP_OK;
}

int lusp_batch_upload(lusp_batch* hb, const double* vals, const double* rhs, void* stream) {
    BatchObj* B = BO(hb);
    if (!B) return LUSP_EARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (vals) {
        cudaError_t e = cudaMemcpyAsync(B->d_vals, vals, B->val_off[B->nsys] * 8, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return lusp::cuda_fail(e, "upload values");
    }
    if (rhs) {
        cudaError_t e = cudaMemcpyAsync(B->d_rhs, rhs, B->vec_off[B->nsys] * 8, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return lusp::cuda_fail(e, "upload rhs");
    }
    return LUSP_OK;
}

int lusp_batch_download(lusp_batch* hb, double* x, void* stream) {
    BatchObj* B = BO(hb);
    if (!B || !x) return LUSP_EARG;
    cudaError_t e = cudaMemcpyAsync(x, B->d_x, B->vec_off[B->nsys] * 8, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    return e == cudaSuccess ? LUSP_OK : lusp::cuda_fail(e, "download x");
}

int lusp_batch_run(lusp_batch* hb, int what, void* stream) {
    BatchObj* B = BO(hb);
    if (!B || (what & 3) == 0 || what > 7) return LUSP_EARG;
    return lusp::batch_launch(B, what, (cudaStream_t)stream, true);
}

int lusp_batch_run_graph(lusp_batch* hb, int what, void* stream) {
    BatchObj* B = BO(hb);
    if (!B || (what & 3) == 0 || what > 7) return LUSP_EARG;
    cudaStream_t st = (cudaStream_t)stream;
    auto key = std::make_pair(what, st);
    auto it = B->graphs.find(key);
    if (it == B->graphs.end()) {
        // Capture needs a non-legacy stream: capture on a private stream and
        // replay on the caller's.
        cudaStream_t cap;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return lusp::cuda_fail(e, "graph stream");
        lusp::GraphEntry g;
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { cudaStreamDestroy(cap); return lusp::cuda_fail(e, "begin capture"); }
        int rc = lusp::batch_launch(B, what, cap);
        e = cudaStreamEndCapture(cap, &g.graph);
        cudaStreamDestroy(cap);
        if (rc != LUSP_OK) { if (g.graph) cudaGraphDestroy(g.graph); return rc; }
        if (e != cudaSuccess) return lusp::cuda_fail(e, "end capture");
        e = cudaGraphInstantiate(&g.exec, g.graph, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(g.graph); return lusp::cuda_fail(e, "graph instantiate"); }
        it = B->graphs.emplace(key, g).first;
    }
    cudaError_t e = cudaGraphLaunch(it->second.exec, st);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "graph launch");
    B->launches = lusp::launch_kernel_count(B->launch, what);
    return LUSP_OK;
}

int lusp_batch_stats(lusp_batch* hb, lusp_sys_stats* out, void* stream) {
    BatchObj* B = BO(hb);
    if (!B || !out) return LUSP_EARG;
    static_assert(sizeof(lusp_sys_stats) == sizeof(lusp::SysStats), "stats layout");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(out, B->d_stats, sizeof(lusp::SysStats) * B->nsys, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "stats copy");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "stats sync");
    return LUSP_OK;
}

int lusp_batch_factor_values(lusp_batch* hb, int sys, void* out, void* stream) {
    BatchObj* B = BO(hb);
    if (!B || !out || sys < 0 || sys >= B->nsys) return LUSP_EARG;
    const size_t vs = B->prec == LUSP_FP64 ? 8 : 4;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = lusp::batch_merge_factor(B, sys, st);
    if (rc != LUSP_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(out, B->h_sys[sys].lu, B->pats[sys]->S.cap * vs, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "factor copy");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "factor sync");
    return LUSP_OK;
}

int lusp_batch_copy_values(lusp_batch* hd, const lusp_batch* hs, void* stream) {
    BatchObj* D = BO(hd);
    const BatchObj* S = BO(hs);
    if (!D || !S || D->nsys != S->nsys) return LUSP_EARG;
    for (int s = 0; s < D->nsys; s++)
        if (D->pats[s] != S->pats[s]) return LUSP_EARG;
    cudaError_t e = cudaMemcpyAsync(D->d_vals, S->d_vals, D->val_off[D->nsys] * 8,
                                    cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    return e == cudaSuccess ? LUSP_OK : lusp::cuda_fail(e, "copy values");
}

int lusp_batch_factor_device_ptr(lusp_batch* hb, int sys, void** d_values) {
    BatchObj* B = BO(hb);
    if (!B || !d_values || sys < 0 || sys >= B->nsys) return LUSP_EARG;
    // Complete the merged array (default stream: ordered after the caller's
    // earlier runs on it, and before its later work).
    int rc = lusp::batch_merge_factor(B, sys, nullptr);
    if (rc != LUSP_OK) return rc;
    *d_values = B->h_sys[sys].lu;
    return LUSP_OK;
}

int lusp_batch_set_params(lusp_batch* hb, const lusp_batch_opts* o) {
    BatchObj* B = BO(hb);
    if (!B || !o) return LUSP_EARG;
    B->prm.max_outer = o->max_outer > 0 ? o->max_outer : 0;
    B->prm.rtol = o->rtol;
    B->prm.inner_rel = o->inner_rel;
    B->prm.stag_ratio = o->stag_ratio;
    B->prm.pivot_tol = o->pivot_tol;
    B->prm.xtol = o->xtol > 0 ? o->xtol : 1e-8;
    if (o->factor_shift >= 0.0) B->prm.shift = o->factor_shift;
    B->launch.prm = B->prm;
    if (B->launch.rungs) {
        lusp::SolveParams& x = B->launch.xprm;
        const double keep_shift = x.shift;
        x = B->prm;
        x.shift = keep_shift;
        B->launch.esc.rtol = o->rtol;
        if (o->hard_shift > 0) B->launch.hard_shift = o->hard_shift;
    }
    // Captured graphs hold the old parameters by value.
    for (auto& kv : B->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    B->graphs.clear();
    return LUSP_OK;
}

int lusp_batch_launch_count(const lusp_batch* hb) {
    const BatchObj* B = BO(hb);
    return B ? B->launches : 0;
}

int lusp_batch_launch_shape(const lusp_batch* hb, int* shape) {
    const BatchObj* B = BO(hb);
    if (!B || !shape) return LUSP_EARG;
    const lusp::LaunchArgs& a = B->launch;
    shape[0] = a.rgrid;
    shape[1] = a.rblock;
    shape[2] = a.rcluster;
    shape[3] = a.rspread.group;
    shape[4] = a.dgrid;
    shape[5] = a.dblock;
    shape[6] = a.grid;
    shape[7] = a.block;
    shape[8] = a.plan.flow || a.plan.sc_ent == 0 ? 1 : 2;
    shape[9] = a.dcluster;
    return LUSP_OK;
}

int lusp_batch_time_kernels(lusp_batch* hb, int on) {
    BatchObj* B = BO(hb);
    if (!B) return LUSP_EARG;
    if (on && !B->kev[0]) {
        for (cudaEvent_t& ev : B->kev) {
            cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return lusp::cuda_fail(e, "timing events");
        }
    } else if (!on && B->kev[0]) {
        for (cudaEvent_t& ev : B->kev) {
            cudaEventDestroy(ev);
            ev = nullptr;
        }
    }
    return LUSP_OK;
}

int lusp_batch_kernel_ms(lusp_batch* hb, float* ms) {
    BatchObj* B = BO(hb);
    if (!B || !ms || !B->kev[0]) return LUSP_EARG;
    cudaError_t e = cudaEventSynchronize(B->kev[3]);
    for (int k = 0; k < 3 && e == cudaSuccess; k++) e = cudaEventElapsedTime(ms + k, B->kev[k], B->kev[k + 1]);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "kernel times");
    return LUSP_OK;
}

}  // extern "C"
