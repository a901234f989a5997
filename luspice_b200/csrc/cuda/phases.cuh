// Per-CTA phases: refactorization of one system with frozen pivots, the
// level-scheduled triangular solves, SELL SpMV, Arnoldi and the GMRES-IR
// driver.  Every function here is called by all threads of the CTA.
#pragma once
#include "engine.cuh"

namespace lusp {

// Shared-memory map of one CTA (byte offsets inside the dynamic region).
struct Smem {
    int* ctl;            // [0] claim counter, [1] status bits, [2] singular col,
                         // [3] wait-abort flag
    unsigned* ready;     // ready bits
    double* red;         // 40 doubles of reduction scratch
    char* uni;           // phase-specific area

    __device__ Smem(char* base, const SmemPlan& plan) {
        ctl = (int*)base;
        ready = (unsigned*)(base + 64);
        size_t off = 64 + (((size_t)plan.nwords * 4 + 15) & ~(size_t)15);
        red = (double*)(base + off);
        uni = base + off + 40 * sizeof(double);
    }
};

// Status bits that describe a solve (cleared when a new solve starts).
constexpr int kSolveBits = ST_STAGNATED | ST_NOT_CONVERGED | ST_NONFINITE | ST_WAIT_TIMEOUT;

// Slot of row i among rows[lo, hi) (ascending), or -1.
__device__ __forceinline__ int find_slot(const int* rows, int lo, int hi, int i) {
    const int end = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (rows[mid] < i) lo = mid + 1; else hi = mid;
    }
    return (lo < end && rows[lo] == i) ? lo : -1;
}

// Slot of row i through the column's row -> slot map, or -1.
__device__ __forceinline__ int map_slot(const unsigned short* map, const int* rows, int len, int i) {
    const int s = map[i];
    return (s < len && rows[s] == i) ? s : -1;
}

// Non-blocking test of a ready bit.
__device__ __forceinline__ bool is_ready(const unsigned* bits, int j) {
    return (*((const volatile unsigned*)bits + (j >> 5)) >> (j & 31)) & 1u;
}

// Asynchronous global->shared copies (sm_80+ cp.async, L1-allocating):
// issued without waiting, completed by cp_async_wait_all().
__device__ __forceinline__ void cp_async_4(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_val(float* sdst, const float* gsrc) { cp_async_4(sdst, gsrc); }
__device__ __forceinline__ void cp_async_val(double* sdst, const double* gsrc) { cp_async_8(sdst, gsrc); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ int warp_claim(int* counter) {
    int idx = 0;
    if ((threadIdx.x & 31) == 0) idx = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, idx, 0);
}

// ---------------------------------------------------------------------------
// Refactorization with the pivot order and pattern frozen.
//
// Column k (one warp): x = A(:,k) scattered into the column's own slots
// (duplicates summed in input order); for each U(:,k) row j ascending, once
// column j is ready: x[i] -= L(i,j) * x[j] for the rows i of L(:,j), the
// slot of i found by binary search in column k's sorted rows; U(:,k) =
// x[rows < k], U(k,k) = x[k], L(:,k) = x[rows > k] / U(k,k).  The work
// vector is fp64; multiply and subtract are separately rounded so the result
// is bitwise reproducible on the host.  Values are stored as VT (fp32 for
// the mixed path, fp64 for the plain path) in the merged column layout and
// in the row-major copies used by the solves.
// ---------------------------------------------------------------------------
template <typename VT>
__device__ void refactor_phase(const SysDev& S, const SmemPlan& plan, char* smem_base,
                               const SolveParams& prm) {
    const PatternDev& P = *S.pat;
    const int n = P.n;
    Smem sm(smem_base, plan);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // Per warp: work vector x[wcap] (fp64), staged values sval[scap] (VT),
    // column rows wr[wcap], staged rows srow[scap].
    double* wx = (double*)sm.uni + (size_t)warp * plan.wcap;
    VT* sval_all = (VT*)((double*)sm.uni + (size_t)nw * plan.wcap);
    VT* sval = sval_all + (size_t)warp * plan.scap;
    int* wr = (int*)(sval_all + (size_t)nw * plan.scap) + (size_t)warp * plan.wcap;
    int* srow = (int*)(sval_all + (size_t)nw * plan.scap) + (size_t)nw * plan.wcap + (size_t)warp * plan.scap;
    // Optional per-warp row -> slot map (n entries, 16 bit).
    unsigned short* wmap = (unsigned short*)((int*)(sval_all + (size_t)nw * plan.scap) +
                                             (size_t)nw * (plan.wcap + plan.scap)) +
                           (size_t)warp * plan.mcap;
    const bool use_map = plan.mcap >= n;

    for (int t = threadIdx.x; t < (n + 31) / 32; t += blockDim.x) sm.ready[t] = 0u;
    if (threadIdx.x == 0) {
        sm.ctl[0] = 0;
        sm.ctl[1] = 0;
        sm.ctl[2] = 0x7fffffff;
        sm.ctl[3] = 0;
    }
    // A in SELL order for the solves: fp64 (outer residual) and fp32 (inner).
    for (int t = threadIdx.x; t < P.sell_total; t += blockDim.x) {
        const int s = P.sell_src[t];
        const double v = s >= 0 ? S.a_val[s] : 0.0;
        S.sell64[t] = v;
        S.sell32[t] = (float)v;
    }
    __syncthreads();

    VT* lu = (VT*)S.lu;
    VT* lval = (VT*)S.lval;
    VT* uval = (VT*)S.uval;
    VT* udiag = (VT*)S.udiag;
    double minpiv = INFINITY, minratio = INFINITY, maxu = 0.0;
    int bad = 0;
    long long c_wait = 0, c_gather = 0, c_update = 0;
    const long long t_begin = clock64();
    if (threadIdx.x == 0) {
        S.stats->cyc_wait = 0;
        S.stats->cyc_gather = 0;
        S.stats->cyc_update = 0;
    }
    __syncthreads();

    while (true) {
        const int idx = warp_claim(&sm.ctl[0]);
        if (idx >= n) break;
        const int k = P.col_order[idx];
        const int c0 = P.cp[k], c1 = P.cp[k + 1];
        const int d = P.dg[k] - c0, len = c1 - c0;
        double* x;
        const int* rows;
        if (len <= plan.wcap) {
            x = wx;
            for (int t = lane; t < len; t += 32) wr[t] = P.ri[c0 + t];
            rows = wr;
        } else if (S.scratch) {
            x = S.scratch + ((size_t)blockIdx.x * nw + warp) * P.max_col;
            rows = P.ri + c0;
        } else {
            bad |= ST_CAPACITY;
            __syncwarp();
            if (lane == 0) set_ready(sm.ready, k);
            continue;
        }
        for (int t = lane; t < len; t += 32) x[t] = 0.0;
        __syncwarp();
        const int a0 = P.a_ptr[k], a1 = P.a_ptr[k + 1];
        for (int t = a0 + lane; t < a1; t += 32) {
            const int dst = P.a_dst[t];
            if (t == a0 || P.a_dst[t - 1] != dst) {
                double s = S.a_val[P.a_src[t]];
                for (int u = t + 1; u < a1 && P.a_dst[u] == dst; u++)
                    s = __dadd_rn(s, S.a_val[P.a_src[u]]);
                x[dst] = s;
            }
        }
        // Row -> slot map of this column (when the plan has room for one):
        // entries of other rows are stale, but only rows of this column's
        // pattern are looked up (the static pattern is closed under the
        // updates), and map_slot verifies the hit.
        const bool cmap = use_map && rows == wr;
        if (cmap)
            for (int t = lane; t < len; t += 32) wmap[rows[t]] = (unsigned short)t;
        __syncwarp();
        long long tc = clock64();
        // Apply the dependency columns in ascending order.  Each round takes
        // the next run of dependencies that are already complete (blocking
        // only when the very next one is not, so the older dependencies of a
        // column overlap with the computation of its most recent ones), up to
        // plan.scap gathered entries; their L parts are copied to shared
        // memory with all copies in flight together, then applied.
        for (int u0 = 0; u0 < d;) {
            const int u = u0 + lane;
            int beg = 0, cnt = 0;
            bool rdy = true;
            if (u < d) {
                const int jj = rows[u];
                beg = P.dg[jj] + 1;
                cnt = P.cp[jj + 1] - beg;
                rdy = is_ready(sm.ready, jj);
            }
            int nready = __ffs(~__ballot_sync(0xffffffffu, rdy)) - 1;
            if (nready < 0) nready = 32;
            if (nready == 0) {
                if (!wait_ready(sm.ready, rows[u0], &sm.ctl[3])) bad |= ST_WAIT_TIMEOUT;
                __syncwarp();
                nready = 1;
            }
            __threadfence_block();
            {
                const long long t2 = clock64();
                c_wait += t2 - tc;
                tc = t2;
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - cnt;
            int nfit = prm.refactor_mode == 1
                           ? 0
                           : __popc(__ballot_sync(0xffffffffu, u < d && incl <= plan.scap));
            nfit = min(nfit, nready);
            if (nfit == 0) {
                // One dependency longer than the stage: apply it from global.
                const double xj = x[u0];
                const int p0 = __shfl_sync(0xffffffffu, beg, 0);
                const int p1 = p0 + __shfl_sync(0xffffffffu, cnt, 0);
                if (xj != 0.0) {
                    for (int p = p0 + lane; p < p1; p += 32) {
                        const int i = P.ri[p];
                        const double l = ValTraits<VT>::load(lu + p);
                        const int s = cmap ? map_slot(wmap, rows, len, i) : find_slot(rows, u0 + 1, len, i);
                        if (s >= 0) x[s] = __dsub_rn(x[s], __dmul_rn(l, xj));
                        else bad |= ST_CAPACITY;
                    }
                }
                __syncwarp();
                u0 += 1;
                continue;
            }
            for (int t = 0; t < nfit; t++) {
                const int b_t = __shfl_sync(0xffffffffu, beg, t);
                const int c_t = __shfl_sync(0xffffffffu, cnt, t);
                const int o_t = __shfl_sync(0xffffffffu, excl, t);
                for (int e = lane; e < c_t; e += 32) {
                    cp_async_4(srow + o_t + e, P.ri + b_t + e);
                    cp_async_val(sval + o_t + e, lu + b_t + e);
                }
            }
            cp_async_wait_all();
            __syncwarp();
            {
                const long long t2 = clock64();
                c_gather += t2 - tc;
                tc = t2;
            }
            for (int t = 0; t < nfit; t++) {
                const int c_t = __shfl_sync(0xffffffffu, cnt, t);
                const int o_t = __shfl_sync(0xffffffffu, excl, t);
                const int uu = u0 + t;
                const double xj = x[uu];
                if (xj != 0.0) {
                    for (int e = lane; e < c_t; e += 32) {
                        const int i = srow[o_t + e];
                        const double l = ValTraits<VT>::load(sval + o_t + e);
                        const int s = cmap ? map_slot(wmap, rows, len, i) : find_slot(rows, uu + 1, len, i);
                        if (s >= 0) x[s] = __dsub_rn(x[s], __dmul_rn(l, xj));
                        else bad |= ST_CAPACITY;
                    }
                }
                __syncwarp();
            }
            {
                const long long t2 = clock64();
                c_update += t2 - tc;
                tc = t2;
            }
            u0 += nfit;
        }
        const double piv = x[d];
        double amax = 0.0;
        for (int t = d + 1 + lane; t < len; t += 32) amax = fmax(amax, fabs(x[t]));
        amax = warp_max(amax);
        const double ap = fabs(piv);
        if (!(ap > 0.0) || !isfinite(piv)) {
            bad |= ST_SINGULAR;
            if (lane == 0) atomicMin(&sm.ctl[2], k);
        }
        minpiv = fmin(minpiv, ap);
        const double ratio = amax > ap ? ap / amax : 1.0;
        minratio = fmin(minratio, ratio);
        if (ratio < prm.pivot_tol) bad |= ST_PIVOT_WEAK;
        for (int t = lane; t < len; t += 32) {
            const int slot = c0 + t;
            double v = x[t];
            if (t > d) v = __ddiv_rn(v, piv);
            else maxu = fmax(maxu, fabs(v));
            const VT sv = ValTraits<VT>::to(v);
            lu[slot] = sv;
            const int dst = P.slot_dst[slot];
            if (t < d) uval[dst] = sv;
            else if (t == d) udiag[k] = sv;
            else lval[dst] = sv;
        }
        __threadfence_block();
        __syncwarp();
        if (lane == 0) set_ready(sm.ready, k);
    }

    if (lane == 0) {
        atomicAdd((unsigned long long*)&S.stats->cyc_wait, (unsigned long long)c_wait);
        atomicAdd((unsigned long long*)&S.stats->cyc_gather, (unsigned long long)c_gather);
        atomicAdd((unsigned long long*)&S.stats->cyc_update, (unsigned long long)c_update);
    }
    if (threadIdx.x == 0) S.stats->cyc_refactor = clock64() - t_begin;
    // Statistics: warp reductions, then per-warp partials combined in order.
    minpiv = warp_min(minpiv);
    minratio = warp_min(minratio);
    maxu = warp_max(maxu);
    bad = __reduce_or_sync(0xffffffffu, bad);
    __syncthreads();
    if (lane == 0) {
        sm.red[warp] = minpiv;
        atomicOr(&sm.ctl[1], bad);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = INFINITY;
        for (int w = 0; w < nw; w++) a = fmin(a, sm.red[w]);
        S.stats->min_abs_pivot = a;
    }
    __syncthreads();
    if (lane == 0) sm.red[warp] = minratio;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = INFINITY;
        for (int w = 0; w < nw; w++) a = fmin(a, sm.red[w]);
        S.stats->min_pivot_ratio = a;
    }
    __syncthreads();
    if (lane == 0) sm.red[warp] = maxu;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < nw; w++) a = fmax(a, sm.red[w]);
        S.stats->max_abs_u = a;
        S.stats->status = sm.ctl[1];
        S.stats->singular_col = sm.ctl[2] == 0x7fffffff ? -1 : sm.ctl[2];
        S.stats->nres = 0;
        S.stats->inner_iters = 0;
        S.stats->outer_iters = 0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// y := U^-1 L^-1 rhs in pivot-position space (level-scheduled, warp per row,
// factors read as VT, accumulation in fp64).  y may be shared or global
// memory; rhs must not alias y.
// ---------------------------------------------------------------------------
template <typename VT>
__device__ void cta_lu_apply(const PatternDev& P, const VT* lval, const VT* uval,
                             const VT* udiag, const double* rhs, double* y, Smem& sm,
                             int& bad) {
    const int n = P.n;
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = rhs[i];
    for (int t = threadIdx.x; t < (n + 31) / 32; t += blockDim.x) sm.ready[t] = 0u;
    if (threadIdx.x == 0) {
        sm.ctl[0] = 0;
        sm.ctl[3] = 0;
    }
    __syncthreads();
    volatile double* vy = y;
    while (true) {
        const int idx = warp_claim(&sm.ctl[0]);
        if (idx >= n) break;
        const int i = P.fwd_order[idx];
        const int p0 = P.lrp[idx], p1 = P.lrp[idx + 1];
        double acc = 0.0;
        for (int p = p0 + lane; p < p1; p += 32) {
            const int j = P.lci[p];
            const double v = ValTraits<VT>::load(lval + p);
            if (!wait_ready(sm.ready, j, &sm.ctl[3])) bad |= ST_WAIT_TIMEOUT;
            __threadfence_block();
            acc = fma(v, vy[j], acc);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            vy[i] = vy[i] - acc;
            __threadfence_block();
            set_ready(sm.ready, i);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < (n + 31) / 32; t += blockDim.x) sm.ready[t] = 0u;
    if (threadIdx.x == 0) sm.ctl[0] = 0;
    __syncthreads();
    while (true) {
        const int idx = warp_claim(&sm.ctl[0]);
        if (idx >= n) break;
        const int i = P.bwd_order[idx];
        const int p0 = P.urp[idx], p1 = P.urp[idx + 1];
        double acc = 0.0;
        for (int p = p0 + lane; p < p1; p += 32) {
            const int j = P.uci[p];
            const double v = ValTraits<VT>::load(uval + p);
            if (!wait_ready(sm.ready, j, &sm.ctl[3])) bad |= ST_WAIT_TIMEOUT;
            __threadfence_block();
            acc = fma(v, vy[j], acc);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            vy[i] = (vy[i] - acc) / ValTraits<VT>::load(udiag + i);
            __threadfence_block();
            set_ready(sm.ready, i);
        }
    }
    __syncthreads();
}

// One triangular sweep, level-synchronous: the rows of a level are spread
// over the warps (one warp per row, lanes over the row's entries), one
// barrier per level.  Row order, row pointers and level bounds come from
// shared memory; each warp keeps the first 32 entries (one per lane) of its
// next two rows in registers (sets A and B, used alternately so a pending
// load is never copied), loaded while earlier rows and barriers complete.
// UPPER: y[i] = (y[i] - sum) / diag[i] (U sweep), else y[i] -= sum.
template <typename VT, bool UPPER>
__device__ void level_sweep(int nlev, const int* lev, const int* order, const int* rp,
                            const int* ci, const VT* val, const VT* diag, double* y) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int gl = 0, gidx = warp;
    while (gl < nlev && gidx >= lev[gl + 1]) {
        gl++;
        if (gl < nlev) gidx = lev[gl] + warp;
    }
    int a_idx = -1, a_lvl = nlev, a_col = -1, b_idx = -1, b_lvl = nlev, b_col = -1;
    double a_v = 0.0, a_d = 1.0, b_v = 0.0, b_d = 1.0;
#define LUSP_FETCH(IDX, LVL, COL, V, D)                                            \
    if (gl < nlev) {                                                              \
        IDX = gidx;                                                               \
        LVL = gl;                                                                 \
        const int pp = rp[gidx] + lane;                                           \
        COL = -1;                                                                 \
        V = 0.0;                                                                  \
        if (pp < rp[gidx + 1]) {                                                  \
            COL = ci[pp];                                                         \
            V = ValTraits<VT>::load(val + pp);                                    \
        }                                                                         \
        if (UPPER) D = ValTraits<VT>::load(diag + order[gidx]);                   \
        gidx += nw;                                                               \
        while (gl < nlev && gidx >= lev[gl + 1]) {                                \
            gl++;                                                                 \
            if (gl < nlev) gidx = lev[gl] + warp;                                 \
        }                                                                         \
    } else {                                                                      \
        IDX = -1;                                                                 \
        LVL = nlev;                                                               \
    }
#define LUSP_ROW(IDX, COL, V, D)                                                   \
    {                                                                             \
        const int i = order[IDX];                                                 \
        const int p1 = rp[IDX + 1];                                               \
        double acc = COL >= 0 ? V * y[COL] : 0.0;                                 \
        for (int p = rp[IDX] + 32 + lane; p < p1; p += 32)                        \
            acc = fma(ValTraits<VT>::load(val + p), y[ci[p]], acc);               \
        acc = warp_sum(acc);                                                      \
        if (lane == 0) y[i] = UPPER ? (y[i] - acc) / D : y[i] - acc;              \
    }
    LUSP_FETCH(a_idx, a_lvl, a_col, a_v, a_d)
    LUSP_FETCH(b_idx, b_lvl, b_col, b_v, b_d)
    int passed = 0;   // barriers passed = levels known complete
    while (true) {
        if (a_idx < 0) break;
        while (passed < a_lvl) { __syncthreads(); passed++; }
        LUSP_ROW(a_idx, a_col, a_v, a_d)
        LUSP_FETCH(a_idx, a_lvl, a_col, a_v, a_d)
        if (b_idx < 0) break;
        while (passed < b_lvl) { __syncthreads(); passed++; }
        LUSP_ROW(b_idx, b_col, b_v, b_d)
        LUSP_FETCH(b_idx, b_lvl, b_col, b_v, b_d)
    }
    while (passed < nlev) { __syncthreads(); passed++; }
#undef LUSP_FETCH
#undef LUSP_ROW
}

// Shared-memory sweep descriptors of one system: [fwd_order n][fwd rp n+1]
// [fwd_lev nfl+1][bwd_order n][bwd rp n+1][bwd_lev nbl+1].
__device__ __forceinline__ bool sweep_desc_fits(const PatternDev& P, const SmemPlan& plan) {
    return P.n <= plan.ycap && 4 * P.n + P.nfwd_levels + P.nbwd_levels + 4 <= plan.dcap;
}

__device__ __forceinline__ int* sweep_desc_base(const SmemPlan& plan, Smem& sm) {
    return (int*)((double*)sm.uni + plan.ycap + (size_t)(plan.m + 1) * plan.m + 6 * (size_t)(plan.m + 1));
}

__device__ void load_sweep_desc(const PatternDev& P, int* d) {
    const int n = P.n, nfl = P.nfwd_levels, nbl = P.nbwd_levels;
    int* f_ord = d;
    int* f_rp = f_ord + n;
    int* f_lev = f_rp + n + 1;
    int* b_ord = f_lev + nfl + 1;
    int* b_rp = b_ord + n;
    int* b_lev = b_rp + n + 1;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        f_ord[t] = P.fwd_order[t];
        b_ord[t] = P.bwd_order[t];
    }
    for (int t = threadIdx.x; t <= n; t += blockDim.x) {
        f_rp[t] = P.lrp[t];
        b_rp[t] = P.urp[t];
    }
    for (int t = threadIdx.x; t <= nfl; t += blockDim.x) f_lev[t] = P.fwd_lev[t];
    for (int t = threadIdx.x; t <= nbl; t += blockDim.x) b_lev[t] = P.bwd_lev[t];
}

// y := U^-1 L^-1 rhs with the level-synchronous sweeps (descriptors already
// in shared memory at d).
template <typename VT>
__device__ void cta_lu_apply_levels(const PatternDev& P, const VT* lval, const VT* uval,
                                    const VT* udiag, const double* rhs, double* y, const int* d) {
    const int n = P.n, nfl = P.nfwd_levels, nbl = P.nbwd_levels;
    const int* f_ord = d;
    const int* f_rp = f_ord + n;
    const int* f_lev = f_rp + n + 1;
    const int* b_ord = f_lev + nfl + 1;
    const int* b_rp = b_ord + n;
    const int* b_lev = b_rp + n + 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = rhs[i];
    __syncthreads();
    level_sweep<VT, false>(nfl, f_lev, f_ord, f_rp, P.lci, lval, udiag, y);
    level_sweep<VT, true>(nbl, b_lev, b_ord, b_rp, P.uci, uval, udiag, y);
}

// Dispatch: level-synchronous sweeps when their descriptors sit in shared
// memory (desc != nullptr), else the dataflow version.
template <typename VT>
__device__ __forceinline__ void lu_apply(const PatternDev& P, const VT* lval, const VT* uval,
                                         const VT* udiag, const double* rhs, double* y,
                                         Smem& sm, const int* desc, int& bad) {
    if (desc) cta_lu_apply_levels<VT>(P, lval, uval, udiag, rhs, y, desc);
    else cta_lu_apply<VT>(P, lval, uval, udiag, rhs, y, sm, bad);
}

// out = A x (RESID: out = bt - A x) with A in SELL-C-sigma, C = 32, values AT.
template <typename AT, bool RESID>
__device__ void cta_spmv(const PatternDev& P, const AT* vals, const double* xin,
                         const double* bt, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int s = warp; s < P.nslices; s += nw) {
        const int base = P.sell_ptr[s];
        const int L = (P.sell_ptr[s + 1] - base) >> 5;
        double acc = 0.0;
        for (int t = 0; t < L; t++) {
            const int e = base + (t << 5) + lane;
            acc = fma((double)vals[e], xin[P.sell_col[e]], acc);
        }
        const int row = P.sell_perm[(s << 5) + lane];
        if (row >= 0) out[row] = RESID ? bt[row] - acc : acc;
    }
}

__device__ __forceinline__ double cta_dot(const double* a, const double* b, int n, Smem& sm) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(a[i], b[i], s);
    return block_sum(s, sm.red);
}

// Direct solve x = Q U^-1 L^-1 P b with the stored factors, then the fp64
// residual of the result.
template <typename VT>
__device__ void direct_phase(const SysDev& S, const SmemPlan& plan, char* smem_base) {
    const PatternDev& P = *S.pat;
    const int n = P.n;
    Smem sm(smem_base, plan);
    double* bt = S.work;
    double* xt = bt + n;
    double* r = xt + n;
    double* yg = r + 3 * n;
    double* y = (n <= plan.ycap) ? (double*)sm.uni : yg;
    int bad = 0;
    if (threadIdx.x == 0) S.stats->status &= ~kSolveBits;
    for (int i = threadIdx.x; i < n; i += blockDim.x) bt[i] = S.b[P.rowat[i]];
    __syncthreads();
    const int* desc = nullptr;
    if (sweep_desc_fits(P, plan)) {
        int* d = sweep_desc_base(plan, sm);
        load_sweep_desc(P, d);
        desc = d;
    }
    const double nb = sqrt(cta_dot(bt, bt, n, sm));
    lu_apply<VT>(P, (const VT*)S.lval, (const VT*)S.uval, (const VT*)S.udiag, bt, y, sm, desc, bad);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        xt[i] = y[i];
        S.x[P.q[i]] = y[i];
    }
    __syncthreads();
    cta_spmv<double, true>(P, S.sell64, xt, bt, r);
    __syncthreads();
    const double rn = sqrt(cta_dot(r, r, n, sm));
    bad = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(&S.stats->status, bad);
    if (threadIdx.x == 0) {
        const double res = nb > 0 ? rn / nb : rn;
        S.stats->res[0] = res;
        S.stats->nres = 1;
        S.stats->outer_iters = 0;
        S.stats->inner_iters = 0;
        if (!isfinite(res)) atomicOr(&S.stats->status, (int)ST_NONFINITE);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// GMRES-IR: restarted, right-preconditioned GMRES on P A Q with the stored
// factors as preconditioner (VT), inner products A z with AT values; outer
// residual b - A x, Arnoldi (classical Gram-Schmidt, two passes), Givens
// rotations, least-squares update and solution update in fp64.
// Workspace (doubles): bt, xt, r, z, w, yg (n each), V ((m+1) n), xprev (n).
// ---------------------------------------------------------------------------
template <typename VT, typename AT>
__device__ void gmres_phase(const SysDev& S, const SmemPlan& plan, char* smem_base,
                            const SolveParams& prm) {
    const PatternDev& P = *S.pat;
    const int n = P.n;
    const int m = prm.m;
    Smem sm(smem_base, plan);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double* bt = S.work;
    double* xt = bt + n;
    double* r = xt + n;
    double* z = r + n;
    double* w = z + n;
    double* yg = w + n;
    double* V = yg + n;
    double* xprev = V + (size_t)(m + 1) * n;   // iterate before the last correction
    // Shared: y (optional) | H[(m+1) x m] | g, cs, sn, h, h2, yc
    double* ys = (double*)sm.uni;
    double* H = ys + plan.ycap;
    double* g = H + (size_t)(m + 1) * m;
    double* cs = g + (m + 1);
    double* sn = cs + m;
    double* h = sn + m;
    double* yc = h + (m + 1);
    double* y = (n <= plan.ycap) ? ys : yg;
    const VT* lval = (const VT*)S.lval;
    const VT* uval = (const VT*)S.uval;
    const VT* udiag = (const VT*)S.udiag;
    const AT* ainner = (const AT*)(sizeof(AT) == 8 ? (const void*)S.sell64 : (const void*)S.sell32);
    int bad = 0;
    int status = 0;
    int inner_total = 0, outer_done = 0, nres = 0;
    if (threadIdx.x == 0) S.stats->status &= ~kSolveBits;

    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        bt[i] = S.b[P.rowat[i]];
        xt[i] = 0.0;
    }
    const int* desc = nullptr;
    if (sweep_desc_fits(P, plan)) {
        int* d = sweep_desc_base(plan, sm);
        load_sweep_desc(P, d);
        desc = d;
    }
    __syncthreads();
    const double nb = sqrt(cta_dot(bt, bt, n, sm));
    if (!(nb > 0.0)) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) S.x[i] = 0.0;
        if (threadIdx.x == 0) {
            S.stats->res[0] = 0.0;
            S.stats->nres = 1;
            if (!isfinite(nb)) atomicOr(&S.stats->status, (int)ST_NONFINITE);
        }
        __syncthreads();
        return;
    }
    double res_prev = INFINITY;
    // Forward-error estimate of the current iterate from the last two
    // corrections: contraction rho = |dx_k| / |dx_k-1|, remaining error
    // ~ |dx_k| rho / (1 - rho) relative to |x|.
    double dx_prev = 0.0, err_est = INFINITY;
    for (int outer = 0;; outer++) {
        if (outer == 0) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) r[i] = bt[i];
        } else {
            cta_spmv<double, true>(P, S.sell64, xt, bt, r);
        }
        __syncthreads();
        const double beta = sqrt(cta_dot(r, r, n, sm));
        const double res = beta / nb;
        if (nres < 16) {
            if (threadIdx.x == 0) S.stats->res[nres] = res;
            nres++;
        }
        // A correction that made the residual worse (or non-finite) is
        // undone: the result is the best iterate, the status says why.
        if (outer > 0 && !(res <= res_prev)) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) xt[i] = xprev[i];
            __syncthreads();
            status |= isfinite(res) ? ST_STAGNATED : ST_NONFINITE;
            break;
        }
        if (!isfinite(res)) { status |= ST_NONFINITE; break; }
        // Converged when the residual is small and the iterate has stopped
        // moving (or the residual is at fp64 round-off, nothing left to gain).
        if (res <= prm.rtol && (err_est <= prm.xtol || res <= 1e-15)) break;
        if (outer >= prm.max_outer) { status |= ST_NOT_CONVERGED; break; }
        if (outer > 0 && res > prm.stag_ratio * res_prev) { status |= ST_STAGNATED; break; }
        res_prev = res;
        const double inv_beta = 1.0 / beta;
        for (int i = threadIdx.x; i < n; i += blockDim.x) V[i] = r[i] * inv_beta;
        if (threadIdx.x == 0) {
            for (int t = 0; t <= m; t++) g[t] = 0.0;
            g[0] = beta;
        }
        // Inner solve: reduce the current residual by inner_rel (a cap at
        // rtol * |b| would stall the outer loop right above rtol).
        const double inner_stop = prm.inner_rel * beta;
        int jj = 0;
        for (int j = 0; j < m; j++) {
            const double* vj = V + (size_t)j * n;
            lu_apply<VT>(P, lval, uval, udiag, vj, y, sm, desc, bad);
            cta_spmv<AT, false>(P, ainner, y, nullptr, w);
            __syncthreads();
            const double wn0 = sqrt(cta_dot(w, w, n, sm));
            for (int pass = 0; pass < 2; pass++) {
                for (int i = warp; i <= j; i += nw) {
                    const double* vi = V + (size_t)i * n;
                    double s = 0.0;
                    for (int e = lane; e < n; e += 32) s = fma(vi[e], w[e], s);
                    s = warp_sum(s);
                    if (lane == 0) {
                        yc[i] = s;
                        if (pass == 0) h[i] = s;
                        else H[(size_t)i * m + j] = h[i] + s;
                    }
                }
                __syncthreads();
                for (int e = threadIdx.x; e < n; e += blockDim.x) {
                    double acc = w[e];
                    for (int i = 0; i <= j; i++) acc = fma(-yc[i], V[(size_t)i * n + e], acc);
                    w[e] = acc;
                }
                __syncthreads();
            }
            const double hn = sqrt(cta_dot(w, w, n, sm));
            inner_total++;
            jj = j + 1;
            const bool breakdown = !(hn > 1e-14 * wn0) || hn == 0.0;
            if (threadIdx.x == 0) {
                for (int i = 0; i < j; i++) {
                    const double t1 = H[(size_t)i * m + j], t2 = H[(size_t)(i + 1) * m + j];
                    H[(size_t)i * m + j] = cs[i] * t1 + sn[i] * t2;
                    H[(size_t)(i + 1) * m + j] = -sn[i] * t1 + cs[i] * t2;
                }
                const double a = H[(size_t)j * m + j];
                const double bb = breakdown ? 0.0 : hn;
                const double rr = sqrt(a * a + bb * bb);
                const double c = rr > 0.0 ? a / rr : 1.0;
                const double s_ = rr > 0.0 ? bb / rr : 0.0;
                cs[j] = c;
                sn[j] = s_;
                H[(size_t)j * m + j] = rr;
                g[j + 1] = -s_ * g[j];
                g[j] = c * g[j];
                sm.red[34] = g[j + 1];
            }
            __syncthreads();
            const double gres = fabs(sm.red[34]);
            if (breakdown || gres <= inner_stop || !isfinite(gres)) break;
            const double inv_hn = 1.0 / hn;
            double* vn = V + (size_t)(j + 1) * n;
            for (int e = threadIdx.x; e < n; e += blockDim.x) vn[e] = w[e] * inv_hn;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            for (int i = jj - 1; i >= 0; i--) {
                double s = g[i];
                for (int t = i + 1; t < jj; t++) s -= H[(size_t)i * m + t] * yc[t];
                const double dgv = H[(size_t)i * m + i];
                yc[i] = dgv != 0.0 ? s / dgv : 0.0;
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            double acc = 0.0;
            for (int i = 0; i < jj; i++) acc = fma(yc[i], V[(size_t)i * n + e], acc);
            z[e] = acc;
        }
        __syncthreads();
        lu_apply<VT>(P, lval, uval, udiag, z, y, sm, desc, bad);
        double sy = 0.0, sx = 0.0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            xprev[e] = xt[e];
            const double xn = xt[e] + y[e];
            xt[e] = xn;
            sy = fma(y[e], y[e], sy);
            sx = fma(xn, xn, sx);
        }
        const double ny = sqrt(block_sum(sy, sm.red));
        const double nx = sqrt(block_sum(sx, sm.red));
        const double dx = nx > 0.0 ? ny / nx : ny;
        if (dx_prev > 0.0) {
            const double rho = fmin(dx / dx_prev, 0.99);
            err_est = dx * rho / (1.0 - rho);
        }
        dx_prev = dx;
        outer_done++;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) S.x[P.q[i]] = xt[i];
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicOr(&S.stats->status, bad);
    if (threadIdx.x == 0) {
        if (status) atomicOr(&S.stats->status, status);
        S.stats->nres = nres < 16 ? nres : 16;
        S.stats->inner_iters = inner_total;
        S.stats->outer_iters = outer_done;
    }
    __syncthreads();
}

}  // namespace lusp
