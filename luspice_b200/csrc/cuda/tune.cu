// Measuring autotuner: times candidate configurations of the engine on the
// caller's own matrix on this GPU and returns the fastest.  The launch
// rules and the dense-block cost model choose well for the matrices they
// were fitted on; the tuner settles a new pattern class by measurement.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

#include "luspice_b200.h"
#include "engine_internal.h"

namespace {

// Device time of one call of fn (best of reps after one warm-up call).
template <typename F>
int time_best(F fn, cudaStream_t st, int reps, double* best_ms) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return lusp::cuda_fail(cudaGetLastError(), "tune event");
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return lusp::cuda_fail(cudaGetLastError(), "tune event");
    }
    int rc = fn();
    double best = 1e300;
    if (rc == LUSP_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = lusp::cuda_fail(cudaGetLastError(), "tune run");
    for (int r = 0; r < reps && rc == LUSP_OK; r++) {
        cudaEventRecord(a, st);
        rc = fn();
        cudaEventRecord(b, st);
        if (rc == LUSP_OK && cudaEventSynchronize(b) != cudaSuccess) rc = lusp::cuda_fail(cudaGetLastError(), "tune run");
        float ms = 0.f;
        if (rc == LUSP_OK) {
            cudaEventElapsedTime(&ms, a, b);
            best = std::min(best, (double)ms);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *best_ms = best;
    return rc;
}

}  // namespace

extern "C" {

int lusp_tune(int n, const int* Ap, const int* Ai, const double* Ax, const double* b, int nsys,
              lusp_batch_opts* opts, int* dense_tail, double* best_ms) {
    if (n <= 0 || !Ap || !Ai || !Ax || !b || nsys <= 0 || !opts || !dense_tail) return LUSP_EARG;
    cudaStream_t st;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "tune stream");
    std::vector<double> vals((size_t)Ap[n] * nsys), rhs((size_t)n * nsys);
    for (int s = 0; s < nsys; s++) {
        std::memcpy(vals.data() + (size_t)s * Ap[n], Ax, sizeof(double) * Ap[n]);
        std::memcpy(rhs.data() + (size_t)s * n, b, sizeof(double) * n);
    }
    // Dense-block candidates around the cost model's choice.
    std::vector<int> tails;
    {
        lusp_pattern* P = nullptr;
        int rc = lusp_pattern_create(n, Ap, Ai, Ax, nullptr, &P);
        if (rc != LUSP_OK) {
            cudaStreamDestroy(st);
            return rc;
        }
        lusp_pattern_info info;
        lusp_pattern_get_info(P, &info);
        lusp_pattern_destroy(P);
        const int d0 = info.dense_tail;
        const int cap = std::min(n, lusp::kMaxDenseTail);
        for (int d : {0, d0, (d0 / 2) & ~31, std::min(cap, d0 > 0 ? d0 + 128 : 64)})
            if (d >= 0 && d <= cap && std::find(tails.begin(), tails.end(), d) == tails.end()) tails.push_back(d);
    }
    double best = 1e300;
    lusp_batch_opts best_o = *opts;
    int best_d = -1, rc_all = LUSP_OK;
    for (int d : tails) {
        lusp_pattern* P = nullptr;
        if (lusp_pattern_create_ex(n, Ap, Ai, Ax, nullptr, d, &P) != LUSP_OK) continue;
        std::vector<lusp_pattern*> pats(nsys, P);
        // Refactor shape: the engine's own rules (0, 0: which also choose
        // spread mode for a batch of medium systems, at most one per SM),
        // then explicit CTA sizes (the automatic one and its neighbour: one
        // CTA per SM when every system has an SM, else two per SM) on lone
        // CTAs and 2-CTA clusters.
        const bool few = nsys <= lusp::sm_count();
        const int rts[2] = {few ? 768 : 512, few ? 1024 : 768};
        std::vector<std::pair<int, int>> shapes{{0, 0}};
        for (int rt : rts)
            for (int rcl : {1, 2}) shapes.push_back({rt, rcl});
        for (const auto& shp : shapes)
            for (int bt : {256, 512})
                for (int sw : {0, 1}) {
                    lusp_batch_opts o = *opts;
                    o.refactor_threads = shp.first;
                    o.refactor_cluster = shp.second;
                    o.block_threads = bt;
                    o.ctas_per_sm = bt == 512 ? 1 : 2;
                    o.solve_sweep = sw;
                    lusp_batch* B = nullptr;
                    if (lusp_batch_create(nsys, pats.data(), &o, &B) != LUSP_OK) continue;
                    double ms = 1e300;
                    int rc = lusp_batch_upload(B, vals.data(), rhs.data(), st);
                    if (rc == LUSP_OK)
                        rc = time_best([&] { return lusp_batch_run(B, LUSP_RUN_BOTH, st); }, st, 3, &ms);
                    lusp_batch_destroy(B);
                    if (rc != LUSP_OK) {
                        rc_all = rc;
                        continue;
                    }
                    if (ms < best) {
                        best = ms;
                        best_o = o;
                        best_d = d;
                    }
                }
        lusp_pattern_destroy(P);
    }
    cudaStreamDestroy(st);
    if (best_d < 0) return rc_all != LUSP_OK ? rc_all : LUSP_EARG;
    *opts = best_o;
    *dense_tail = best_d;
    if (best_ms) *best_ms = best;
    return LUSP_OK;
}

int lusp_sell_tune(int n, const int* rowptr, const int* colidx, const double* vals, int value_kind,
                   int* C_out, int* sigma_out, double* best_us) {
    if (n <= 0 || !rowptr || !colidx || !vals || !C_out || !sigma_out) return LUSP_EARG;
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * 2 * (size_t)n);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "sell tune alloc");
    e = cudaMemset(d, 0, sizeof(double) * 2 * (size_t)n);
    cudaStream_t st;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaFree(d);
        return lusp::cuda_fail(e, "sell tune setup");
    }
    double best = 1e300;
    int bc = -1, bs = -1, rc_last = LUSP_OK;
    for (int C : {8, 16, 32})
        for (int sigma : {32, 256, 1024}) {
            lusp_sell* S = nullptr;
            int rc = lusp_sell_create(n, rowptr, colidx, vals, C, sigma, value_kind, &S);
            if (rc != LUSP_OK) {
                rc_last = rc;
                continue;
            }
            double ms = 1e300;
            rc = time_best([&] { return lusp_sell_spmv(S, d, d + n, st); }, st, 5, &ms);
            lusp_sell_destroy(S);
            if (rc == LUSP_OK && ms < best) {
                best = ms;
                bc = C;
                bs = sigma;
            }
        }
    cudaStreamDestroy(st);
    cudaFree(d);
    if (bc < 0) return rc_last != LUSP_OK ? rc_last : LUSP_EARG;
    *C_out = bc;
    *sigma_out = bs;
    if (best_us) *best_us = best * 1000.0;
    return LUSP_OK;
}

}  // extern "C"
