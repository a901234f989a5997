// Per-CTA phases: refactorization of one system with frozen pivots, the
// level-scheduled triangular solves, SELL SpMV, Arnoldi and the GMRES-IR
// driver.  Every function here is called by all threads of the CTA.
#pragma once
#include <cooperative_groups.h>

#include <type_traits>

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
constexpr int kSolveBits = ST_STAGNATED | ST_NOT_CONVERGED | ST_NONFINITE | ST_WAIT_TIMEOUT | ST_FP16_OFF;

// Slot of row i among rows[lo, hi) (ascending), or -1.
__device__ __forceinline__ int find_slot(const int* rows, int lo, int hi, int i) {
    const int end = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (rows[mid] < i) lo = mid + 1; else hi = mid;
    }
    return (lo < end && rows[lo] == i) ? lo : -1;
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

// Orders this thread's memory operations for the other CTAs sharing a
// system: block scope for a lone CTA, cluster scope when the system's
// columns are spread over a thread-block cluster (release before publishing
// a ready bit, acquire after observing one).
__device__ __forceinline__ void share_fence(unsigned csize) {
    if (csize > 1) asm volatile("fence.acq_rel.cluster;\n" ::: "memory");
    else __threadfence_block();
}
// GPU scope: CTAs on any SM share the system (spread mode).  The release
// pattern (column values, then its ready bit) needs only a release fence
// before the relaxed atomic that sets the bit, and the acquire pattern (a
// ready bit read, then the column's values) only an acquire fence after the
// read; neither has to wait the way a full acq_rel or sequentially
// consistent fence does (grid refactor 1.68 -> 1.55 ms).
template <bool SPREAD>
__device__ __forceinline__ void share_release_t(unsigned csize) {
    if (SPREAD) asm volatile("fence.release.gpu;\n" ::: "memory");
    else share_fence(csize);
}
__device__ __forceinline__ void spread_acquire() { asm volatile("fence.acquire.gpu;\n" ::: "memory"); }

__device__ __forceinline__ int warp_claim(int* counter) {
    int idx = 0;
    if ((threadIdx.x & 31) == 0) idx = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, idx, 0);
}

// Pivot statistics of a CTA: warp reductions, then per-warp partials
// combined in order by thread 0.  first: overwrite the system's statistics
// (refactor kernel), else merge into them (dense trailing-block kernel).
// Status bits go through ctl[1], the singular column through ctl[2] (the
// CTA's own control words, or those of the cluster's rank 0).
__device__ void cta_store_pivot_stats(SysStats* st, Smem& sm, double minpiv, double minratio, double maxu,
                                      int bad, bool first, int* ctl) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    minpiv = warp_min(minpiv);
    minratio = warp_min(minratio);
    maxu = warp_max(maxu);
    bad = __reduce_or_sync(0xffffffffu, bad);
    __syncthreads();
    if (lane == 0) {
        sm.red[warp] = minpiv;
        atomicOr(&ctl[1], bad);
    }
    __syncthreads();
    double a = INFINITY;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; w++) a = fmin(a, sm.red[w]);
    __syncthreads();
    if (lane == 0) sm.red[warp] = minratio;
    __syncthreads();
    double b = INFINITY;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; w++) b = fmin(b, sm.red[w]);
    __syncthreads();
    if (lane == 0) sm.red[warp] = maxu;
    __syncthreads();
    if (threadIdx.x == 0) {
        double c = 0.0;
        for (int w = 0; w < nw; w++) c = fmax(c, sm.red[w]);
        const int c2 = *(volatile int*)&ctl[2];
        const int sc = c2 == 0x7fffffff ? -1 : c2;
        if (first) {
            st->min_abs_pivot = a;
            st->min_pivot_ratio = b;
            st->max_abs_u = c;
            st->status = *(volatile int*)&ctl[1];
            st->singular_col = sc;
            st->nres = 0;
            st->inner_iters = 0;
            st->outer_iters = 0;
        } else {
            st->min_abs_pivot = fmin(st->min_abs_pivot, a);
            st->min_pivot_ratio = fmin(st->min_pivot_ratio, b);
            st->max_abs_u = fmax(st->max_abs_u, c);
            st->status |= *(volatile int*)&ctl[1];
            if (sc >= 0 && (st->singular_col < 0 || sc < st->singular_col)) st->singular_col = sc;
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Dense trailing block of the refactorization (rows and columns [k0, n)),
// in place in W (fp64, row-major, leading dimension ld).  On entry W holds
// the block after the updates from the columns before k0; on exit its strict
// lower part holds the stored (VT-rounded) multipliers and its upper part
// the fp64 U values.  Right-looking with panels of nb columns (the panel in
// shared memory): entry (i, c) still receives its updates in ascending order
// of the pivot column, each a separately rounded multiply and subtract with
// the stored multiplier and the fp64 U value, so the factor equals the
// column engine's bit for bit.  Pivot statistics as in the column engine.
// ---------------------------------------------------------------------------
// Entry (r, c) of the dense trailing block W, or 0 when it is outside the
// block's pattern (first panel step only: the refactor wrote the pattern
// entries alone, the rest of W holds whatever an earlier launch left).
// Split thread-block cluster barrier (every thread of both CTAs arrives,
// then waits; release / acquire at cluster scope).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

template <bool CG = false>
__device__ __forceinline__ double tail_entry(const double* W, int ld, const unsigned* mask, int r, int c,
                                             bool masked) {
    if (masked && !((__ldg(mask + (size_t)r * (ld >> 5) + (c >> 5)) >> (c & 31)) & 1u)) return 0.0;
    return CG ? __ldcg(W + (size_t)r * ld + c) : W[(size_t)r * ld + c];
}

// CL: the block is shared by the two CTAs of a thread-block cluster.  Rank
// 0 factors each panel alone, one step ahead (look-ahead); rank 1 copies it
// from rank 0's shared memory.  In each step rank 0 takes the U rows and the
// trailing update of the next panel's columns, rank 1 those of all other
// columns, so each column of W is written by one CTA between two cluster
// barriers.  W is then read through L2 (ld.cg), where the other CTA's writes
// are, never from a stale L1 line.
template <typename VT, bool CL = false>
__device__ void dense_tail_factor(const PatternDev& P, double* W, Smem& sm, const SmemPlan& plan,
                                  const SolveParams& prm, double& minpiv, double& minratio, int& bad,
                                  SysStats* st) {
    namespace cgr = cooperative_groups;
    const int crank = CL ? (int)cgr::this_cluster().block_rank() : 0;
    const bool lead = crank == 0;
    const int D = P.dtail, ld = P.tail_ld, k0 = P.k0, nb = plan.tnb;
    const int ps = nb + 1;   // panel row stride: odd, so a lane per row hits distinct banks
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    double* pan = (double*)sm.uni;                                           // [D][ps]
    double* ut = pan + (size_t)D * ps;                                       // [nb][128]
    // Per column of the panel, each warp's maximum |L| before scaling (the
    // pivot statistics' denominator): a slot per warp, reduced after the
    // panel, so the panel's column chain carries no atomics.
    double* wmax = ut + (size_t)nb * 128;                                    // [nb][32]
    long long* ctr = (long long*)(wmax + (size_t)nb * 32);   // [4] stage cycles (thread 0)
    if (tid == 0) {
        ctr[0] = ctr[1] = ctr[2] = 0;
        ctr[3] = clock64();
    }
    const unsigned* mask = P.tail_mask;
    auto wld = [W](size_t i) { return CL ? __ldcg(W + i) : W[i]; };
    const int warp = tid >> 5, nw = nt >> 5;
    // Panel jb: loaded into shared memory, factored, its pivot statistics
    // taken and written back to W (rank 0 alone in a cluster).
    auto panel = [&](int jb) {
        const int w = min(nb, D - jb), R = D - jb;
        const bool first = jb == 0;
        for (int t = tid; t < R * nb; t += nt) {
            const int r = t / nb, c = t - r * nb;
            pan[r * ps + c] = c < w ? tail_entry<CL>(W, ld, mask, jb + r, jb + c, first) : 0.0;
        }
        __syncthreads();
        // Panel: unblocked elimination, a lane per row and a warp per 32
        // rows, so a row's multiplier and its update stay inside one warp:
        // one CTA barrier per column (the pivot row must be final for all).
        for (int c = 0; c < w; c++) {
            const double piv = pan[c * ps + c];
            const double* urow = pan + (size_t)c * ps;
            double lm = 0.0;
            for (int r0 = c + 1 + warp * 32; r0 < R; r0 += nw * 32) {
                const int r = r0 + lane;
                if (r < R) {
                    double* row = pan + (size_t)r * ps;
                    const double v = row[c];
                    lm = fmax(lm, fabs(v));
                    const double l = (double)ValTraits<VT>::to(__ddiv_rn(v, piv));
                    row[c] = l;
                    // Eight entries and their pivot-row values are loaded
                    // before any is stored (the stores could alias the loads).
                    for (int j0 = c + 1; j0 < w; j0 += 8) {
                        double a[8], u[8];
#pragma unroll
                        for (int q = 0; q < 8; q++) {
                            a[q] = j0 + q < w ? row[j0 + q] : 0.0;
                            u[q] = j0 + q < w ? urow[j0 + q] : 0.0;
                        }
#pragma unroll
                        for (int q = 0; q < 8; q++)
                            if (j0 + q < w) row[j0 + q] = __dsub_rn(a[q], __dmul_rn(l, u[q]));
                    }
                }
            }
            lm = warp_max(lm);
            if (lane == 0) wmax[c * 32 + warp] = lm;
            __syncthreads();
        }
        if (tid < w) {
            const int c = tid;
            const double piv = pan[c * ps + c];
            const double ap = fabs(piv);
            double amax = 0.0;
            for (int q = 0; q < nw; q++) amax = fmax(amax, wmax[c * 32 + q]);
            if (!(ap > 0.0) || !isfinite(piv)) {
                bad |= ST_SINGULAR;
                atomicMin(&sm.ctl[2], k0 + jb + c);
            }
            minpiv = fmin(minpiv, ap);
            const double ratio = amax > ap ? ap / amax : 1.0;
            minratio = fmin(minratio, ratio);
            if (ratio < prm.pivot_tol) bad |= ST_PIVOT_WEAK;
        }
        for (int t = tid; t < R * nb; t += nt) {
            const int r = t / nb, c = t - r * nb;
            if (c < w) W[(size_t)(jb + r) * ld + jb + c] = pan[r * ps + c];
        }
        __syncthreads();
    };
    // A cluster factors panel 0 before the loop and each later panel one
    // step ahead: rank 0 owns the next panel's 32 columns in the trailing
    // update of the current step and factors that panel right after them,
    // while rank 1 updates every other column (so the panel chain overlaps
    // the bulk of the update).
    if (CL && lead) panel(0);
    for (int jb = 0; jb < D; jb += nb) {
        const int w = min(nb, D - jb), R = D - jb;
        const bool first = jb == 0;
        if (!CL) panel(jb);
        if (CL) {
            // The panel is final in rank 0's shared memory and in W (first
            // cluster barrier); rank 1 copies its multipliers, and rank 0
            // overwrites them with the next panel only after the second
            // (split: rank 0 arrives at once and waits just before that).
            cluster_arrive();
            cluster_wait();
            if (!lead) {
                const double* pan0 = cgr::this_cluster().map_shared_rank(pan, 0);
                for (int t = tid; t < R * ps; t += nt) pan[t] = pan0[t];
            }
            cluster_arrive();
            if (!lead) {
                cluster_wait();
                __syncthreads();
            }
        }
        if (tid == 0) {
            const long long t2 = clock64();
            ctr[0] += t2 - ctr[3];
            ctr[3] = t2;
        }
        const int c1 = jb + w, ncols = D - c1;
        if (ncols <= 0) {
            if (CL && lead) cluster_wait();
            break;
        }
        // This CTA's columns of the trailing part, colof(t) the t-th: all of
        // them, or (CL) the next panel's nb columns for rank 0 and the rest
        // for rank 1.
        const int cown = CL && !lead ? c1 + nb : c1;
        const int nown = CL ? (lead ? min(nb, ncols) : max(0, ncols - nb)) : ncols;
        const int cend = cown + nown;   // this CTA's columns: [cown, cend)
        auto colof = [&](int t) { return cown + t; };
        // U rows of the panel (triangular solve with the unit-L diagonal
        // block), one thread per column, in groups of 8 rows so the column
        // stays in registers.
        for (int t = tid; t < nown; t += nt) {
            const int colc = colof(t);
            if (colc >= cend) continue;
            const size_t col = (size_t)colc;
            for (int g = 0; g < w; g += 8) {
                double u[8];
#pragma unroll
                for (int r = 0; r < 8; r++) u[r] = g + r < w ? tail_entry<CL>(W, ld, mask, jb + g + r, (int)col, first) : 0.0;
                for (int g2 = 0; g2 < g; g2 += 8) {
                    double v[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) v[c] = wld((size_t)(jb + g2 + c) * ld + col);
#pragma unroll
                    for (int c = 0; c < 8; c++)
#pragma unroll
                        for (int r = 0; r < 8; r++)
                            if (g + r < w) u[r] = __dsub_rn(u[r], __dmul_rn(pan[(g + r) * ps + g2 + c], v[c]));
                }
#pragma unroll
                for (int c = 0; c < 8; c++)
#pragma unroll
                    for (int r = c + 1; r < 8; r++)
                        if (g + r < w) u[r] = __dsub_rn(u[r], __dmul_rn(pan[(g + r) * ps + g + c], u[c]));
#pragma unroll
                for (int r = 0; r < 8; r++)
                    if (g + r < w) W[(size_t)(jb + g + r) * ld + col] = u[r];
            }
        }
        __syncthreads();
        if (tid == 0) {
            const long long t2 = clock64();
            ctr[1] += t2 - ctr[3];
            ctr[3] = t2;
        }
        // Trailing update W22 -= L21 U12, tiles of (4 * nw) rows x 128
        // columns: a thread owns four rows (one per warp stride) and four
        // columns (lane + 32 j); multipliers from the panel in shared memory
        // (broadcast within a warp), U12 staged per tile.
        if (CL && lead) {
            // Rank 0's single panel-wide chunk (at most 32 columns): tiles
            // of 16 nw rows x 32 columns, a thread owning one column and 16
            // rows (one per warp stride), so no lane idles.
            const int TRn = 16 * nw;
            for (int r0 = c1; r0 < D; r0 += TRn) {
                for (int t = tid; t < w * 32; t += nt) {
                    const int c = t >> 5, x = t & 31;
                    const int col = cown + x;
                    ut[c * 128 + x] = col < cend ? wld((size_t)(jb + c) * ld + col) : 0.0;
                }
                __syncthreads();
                const int rw = r0 + warp, col = cown + lane;
                if (rw < D) {
                    double acc[16];
                    int lo[16];
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int row = rw + k * nw;
                        lo[k] = row < D ? k * nw * ps : 0;   // rows past the block reuse rw's multipliers
                        acc[k] = (row < D && col < cend) ? tail_entry<CL>(W, ld, mask, row, col, first) : 0.0;
                    }
                    const double* l0 = pan + (size_t)(rw - jb) * ps;
                    for (int c = 0; c < w; c++) {
                        const double u = ut[c * 128 + lane];
#pragma unroll
                        for (int k = 0; k < 16; k++) acc[k] = __dsub_rn(acc[k], __dmul_rn(l0[lo[k] + c], u));
                    }
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int row = rw + k * nw;
                        if (row < D && col < cend) W[(size_t)row * ld + col] = acc[k];
                    }
                }
                __syncthreads();
            }
        }
        const int TR = 4 * nw;
        const int nrt = (ncols + TR - 1) / TR, nct = CL && lead ? 0 : (nown + 127) / 128;
        for (int tile = 0; tile < nrt * nct; tile++) {
            const int r0 = c1 + (tile / nct) * TR, tq = (tile % nct) * 128;
            for (int t = tid; t < w * 128; t += nt) {
                const int c = t >> 7, x = t & 127;
                const int col = colof(tq + x);
                ut[t] = col < cend ? wld((size_t)(jb + c) * ld + col) : 0.0;
            }
            __syncthreads();
            const int rw = r0 + warp;
            if (rw < D) {
                double acc[4][4];
                int lo[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int row = rw + q * nw;
                    lo[q] = row < D ? q * nw * ps : 0;   // rows past the block reuse rw's multipliers
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int col = colof(tq + lane + 32 * j);
                        acc[q][j] = (row < D && col < cend) ? tail_entry<CL>(W, ld, mask, row, col, first) : 0.0;
                    }
                }
                const double* l0 = pan + (size_t)(rw - jb) * ps;
                for (int c = 0; c < w; c++) {
                    double u[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) u[j] = ut[c * 128 + lane + 32 * j];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double l = l0[lo[q] + c];
#pragma unroll
                        for (int j = 0; j < 4; j++) acc[q][j] = __dsub_rn(acc[q][j], __dmul_rn(l, u[j]));
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int row = rw + q * nw;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int col = colof(tq + lane + 32 * j);
                        if (row < D && col < cend) W[(size_t)row * ld + col] = acc[q][j];
                    }
                }
            }
            __syncthreads();
        }
        if (tid == 0) {
            const long long t2 = clock64();
            ctr[2] += t2 - ctr[3];
            ctr[3] = t2;
        }
        if (CL && lead) {
            // The next panel's columns are final (this CTA's own update):
            // make them visible at L2, where the panel load reads; rank 1
            // is done copying this panel.
            __threadfence();
            __syncthreads();
            cluster_wait();
            panel(c1);
            if (tid == 0) {
                const long long t2 = clock64();
                ctr[0] += t2 - ctr[3];
                ctr[3] = t2;
            }
        }
    }
    if (tid == 0 && lead) {
        st->cyc_tpanel = ctr[0];
        st->cyc_ttrsm = ctr[1];
        st->cyc_tupdate = ctr[2];
    }
}

// Dense trailing block -> VT storage for the solves (unit L below the
// diagonal, U on and above).  The block's entries live only there (the
// merged slot array gets them from merge_factor_kernel when a caller asks).
template <typename VT, bool CG = false>
__device__ void dense_tail_store(const SysDev& S, const PatternDev& P, const double* W, double& maxu,
                                 char* smem_tail_tiles, int ttw) {
    const int D = P.dtail, ld = P.tail_ld, k0 = P.k0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    VT* T = (VT*)S.tail;
    // T is column-major (element (i, c) at T[c * ld + i]) so the solves'
    // block-column products read consecutive rows per warp.  Transpose in
    // 32 x 32 tiles through shared memory (a warp per tile, ttw warps,
    // each with a padded 32 x 33 fp64 tile).
    {
        double* tile = (double*)smem_tail_tiles + (size_t)warp * 32 * 33;
        const int nt32 = ld / 32, twarps = min(nw, ttw);
        if (warp < twarps) {
            for (int tt = warp; tt < nt32 * nt32; tt += twarps) {
                const int ti = tt / nt32, tc = tt - ti * nt32;
                for (int r = 0; r < 32; r++) {
                    const int i = ti * 32 + r, c = tc * 32 + lane;
                    double v = 0.0;
                    if (i < D && c < D) {
                        v = CG ? __ldcg(W + (size_t)i * ld + c) : W[(size_t)i * ld + c];
                        if (i <= c) maxu = fmax(maxu, fabs(v));
                    }
                    tile[r * 33 + lane] = v;
                }
                __syncwarp();
                for (int c = 0; c < 32 && tc * 32 + c < D; c++)
                    T[(size_t)(tc * 32 + c) * ld + ti * 32 + lane] = ValTraits<VT>::to(tile[lane * 33 + c]);
                __syncwarp();
            }
        }
    }
    __syncthreads();
    (void)k0;
}

// The dense trailing block of one system (its own kernel: few warps, many
// registers each): factor, store, merge the pivot statistics.
// Inverses of the 32 x 32 diagonal blocks of the dense block's factor, for
// the solves (a block's triangular solve becomes a matrix-vector product
// instead of a 32-step dependent chain), from the factored fp64 block W
// rounded to VT exactly as the stored factor is: a warp per block and
// factor (nwork warps, each with a 32 x 33 block tile and a 32 x 33 tile of
// the inverse at work + warp * 2 * 32 * 33 doubles), lane c computing column
// c in fp64 by substitution; stored as VT with element (i, c) at c * 32 + i.
// Rows and columns past a partial last block are the identity.  W read
// through L2 (another CTA of a cluster may have written it).
template <typename VT>
__device__ void dense_tail_inverses(const SysDev& S, const PatternDev& P, double* work, int nwork) {
    const int D = P.dtail, ld = P.tail_ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double* W = S.tailw;
    VT* out = (VT*)S.tinv;
    const int nbk = (D + 31) / 32;
    double* Bs = work + (size_t)warp * 2 * 32 * 33;   // block: row r at r * 33
    double* Xs = Bs + 32 * 33;                        // inverse: X[k][c] at k * 33 + c
    if (warp < nwork) {
        for (int task = warp; task < 2 * nbk; task += nwork) {
            const int b = task >> 1, upper = task & 1, jb = b * 32, w = min(32, D - jb);
            for (int r = 0; r < 32; r++)
                Bs[r * 33 + lane] = (r < w && lane < w)
                                        ? (double)ValTraits<VT>::to(__ldcg(W + (size_t)(jb + r) * ld + jb + lane))
                                        : 0.0;
            __syncwarp();
            const int c = lane;
            if (!upper) {
                // X = L^-1 (unit lower): X[r][c] = -sum_{c<=k<r} L[r][k] X[k][c].
                for (int r = 0; r < 32; r++) {
                    double s0 = 0.0, s1 = 0.0;
                    int k = 0;
                    for (; k + 1 < r; k += 2) {
                        s0 = fma(Bs[r * 33 + k], Xs[k * 33 + c], s0);
                        s1 = fma(Bs[r * 33 + k + 1], Xs[(k + 1) * 33 + c], s1);
                    }
                    if (k < r) s0 = fma(Bs[r * 33 + k], Xs[k * 33 + c], s0);
                    Xs[r * 33 + c] = r < c ? 0.0 : r == c ? 1.0 : r >= w ? 0.0 : -(s0 + s1);
                    __syncwarp();
                }
            } else {
                // X = U^-1: X[r][c] = -(sum_{r<k<=c} U[r][k] X[k][c]) / U[r][r].
                for (int r = 31; r >= 0; r--) {
                    double s0 = 0.0, s1 = 0.0;
                    int k = r + 1;
                    for (; k + 1 < 32; k += 2) {
                        s0 = fma(Bs[r * 33 + k], Xs[k * 33 + c], s0);
                        s1 = fma(Bs[r * 33 + k + 1], Xs[(k + 1) * 33 + c], s1);
                    }
                    if (k < 32) s0 = fma(Bs[r * 33 + k], Xs[k * 33 + c], s0);
                    const double dg = r < w ? Bs[r * 33 + r] : 1.0;
                    Xs[r * 33 + c] = r > c ? 0.0 : r == c ? 1.0 / dg : r >= w ? 0.0 : -(s0 + s1) / dg;
                    __syncwarp();
                }
            }
            VT* dst = out + (size_t)b * 2048 + (size_t)upper * 1024;
            for (int cc = 0; cc < 32; cc++) dst[cc * 32 + lane] = ValTraits<VT>::to(Xs[lane * 33 + cc]);
            __syncwarp();
        }
    }
}

// CL: the two CTAs of a thread-block cluster share the system (see
// dense_tail_factor); rank 0 stores the factor and the statistics.
template <typename VT, bool CL = false>
__device__ void dense_phase(const SysDev& S, const SmemPlan& plan, char* smem_base, const SolveParams& prm) {
    const PatternDev& P = *S.pat;
    if (P.dtail <= 0) return;
    Smem sm(smem_base, plan);
    if (threadIdx.x == 0) {
        sm.ctl[1] = 0;
        sm.ctl[2] = 0x7fffffff;
    }
    __syncthreads();
    double minpiv = INFINITY, minratio = INFINITY, maxu = 0.0;
    int bad = 0;
    dense_tail_factor<VT, CL>(P, S.tailw, sm, plan, prm, minpiv, minratio, bad, S.stats);
    __syncthreads();
    // Warps that fit a block tile and an inverse tile in this CTA's area.
    const size_t uoff = (size_t)(sm.uni - smem_base);
    const int nwork = (int)min((size_t)(blockDim.x >> 5),
                               (plan.bytes > uoff ? plan.bytes - uoff : 0) / (2 * 32 * 33 * sizeof(double)));
    if (CL && cooperative_groups::this_cluster().block_rank() != 0) {
        // Rank 1 computes the inverses while rank 0 stores the factor.
        dense_tail_inverses<VT>(S, P, (double*)sm.uni, nwork);
        return;
    }
    dense_tail_store<VT, CL>(S, P, S.tailw, maxu, sm.uni, plan.ttw);
    if (!CL) dense_tail_inverses<VT>(S, P, (double*)sm.uni, nwork);
    cta_store_pivot_stats(S.stats, sm, minpiv, minratio, maxu, bad, false, sm.ctl);
}

// ---------------------------------------------------------------------------
// Refactorization with the pivot order and pattern frozen.
//
// Column k (one warp): x = A(:,k) scattered into the column's own slots
// (duplicates summed in input order); for each U(:,k) row j ascending, once
// column j is ready: x[s] -= L(i,j) * x[j] for the strict-L entries (i, j),
// s = slot of row i in column k (precomputed relative slots; a binary search
// in column k's rows when the pattern has none); U(:,k) = x[rows < k],
// U(k,k) = x[k], L(:,k) = x[rows > k] / U(k,k).  The work vector is fp64;
// multiply and subtract are separately rounded so the result is bitwise
// reproducible on the host.  Values are stored as VT (fp32 for the mixed
// path, fp64 for the plain path) in the merged column layout and in the
// row-major copies used by the solves.
//
// Shared memory per warp: x[wcap] (fp64), a stage of scap L values (VT) and
// scap + 16 relative slots.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_16(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// Spread mode: the pivot statistics and cycle counters of one CTA merged
// into the system's sync area; the last CTA to finish writes the system's
// statistics (pivot minima through the bit patterns of non-negative doubles:
// a larger complement is a smaller value, so 0 means none yet).
__device__ void spread_finish(const SysDev& S, unsigned* sync, int group, Smem& sm, double minpiv,
                              double minratio, double maxu, int bad, long long cw, long long cg, long long cu,
                              long long t_begin) {
    const int lane = threadIdx.x & 31;
    int* ctl = (int*)sync;
    unsigned long long* acc = (unsigned long long*)(sync + kSyncAcc);
    minpiv = warp_min(minpiv);
    minratio = warp_min(minratio);
    maxu = warp_max(maxu);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0) {
        if (bad) atomicOr(&ctl[kSyncStatus], bad);
        if (minpiv < INFINITY) atomicMax(&acc[0], ~(unsigned long long)__double_as_longlong(minpiv));
        if (minratio < INFINITY) atomicMax(&acc[1], ~(unsigned long long)__double_as_longlong(minratio));
        atomicMax(&acc[2], (unsigned long long)__double_as_longlong(maxu));
        atomicAdd(&acc[3], (unsigned long long)cw);
        atomicAdd(&acc[4], (unsigned long long)cg);
        atomicAdd(&acc[5], (unsigned long long)cu);
    }
    __threadfence();
    __syncthreads();
    (void)sm;
    if (threadIdx.x == 0 && atomicAdd(&ctl[kSyncDone], 1) == group - 1) {
        __threadfence();
        const volatile unsigned long long* va = acc;
        const volatile int* vc = ctl;
        SysStats* st = S.stats;
        const unsigned long long a0 = va[0], a1 = va[1];
        st->min_abs_pivot = a0 ? __longlong_as_double((long long)~a0) : INFINITY;
        st->min_pivot_ratio = a1 ? __longlong_as_double((long long)~a1) : INFINITY;
        st->max_abs_u = __longlong_as_double((long long)va[2]);
        st->status = vc[kSyncStatus];
        const int sc = vc[kSyncSingular];
        st->singular_col = sc > 0 ? 0x7fffffff - sc : -1;
        st->nres = 0;
        st->inner_iters = 0;
        st->outer_iters = 0;
        st->cyc_wait = (long long)va[3];
        st->cyc_gather = (long long)va[4];
        st->cyc_update = (long long)va[5];
        st->cyc_refactor = clock64() - t_begin;
    }
}

// Cycle split of the refactor (waits for dependency columns, gathers of
// their L parts, updates) into SysStats::cyc_wait / cyc_gather / cyc_update.
// Reading the SM clock three times per dependency round costs ~3 % of the
// grid refactor, so the split is a build option (-DLUSP_REFACTOR_PHASE_CYCLES=1);
// without it the three fields stay 0 (cyc_refactor is always written).
#ifndef LUSP_REFACTOR_PHASE_CYCLES
#define LUSP_REFACTOR_PHASE_CYCLES 0
#endif
__device__ __forceinline__ long long phase_clock() {
    if constexpr (LUSP_REFACTOR_PHASE_CYCLES != 0) return clock64();
    else return 0;
}

// SPREAD: the system's columns are shared by `group` CTAs anywhere on the
// GPU (CTA `member` of them) through the sync area in global memory; else
// by the CTAs of this thread-block cluster through rank 0's shared memory.
template <typename VT, bool SPREAD = false>
__device__ void refactor_phase(const SysDev& S, const SmemPlan& plan, char* smem_base,
                               const SolveParams& prm, unsigned* sync = nullptr, int member = 0,
                               int group = 1) {
    const PatternDev& P = *S.pat;
    const int n = P.n;
    Smem sm(smem_base, plan);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const size_t per_warp = (size_t)plan.wcap * 8 + (size_t)plan.scap * sizeof(VT) + ((size_t)plan.scap + 16) * 2;
    char* wbase = sm.uni + (size_t)warp * per_warp;
    double* wx = (double*)wbase;
    VT* sval = (VT*)(wbase + (size_t)plan.wcap * 8);
    unsigned short* srel = (unsigned short*)(wbase + (size_t)plan.wcap * 8 + (size_t)plan.scap * sizeof(VT));
    const bool have_rel = P.rel != nullptr && prm.refactor_mode == 0;
    // The CTAs of a thread-block cluster share one system: the claim
    // counter, status, singular column, abort flag and ready bits live in
    // rank 0's shared memory (distributed shared memory for the others).
    namespace cgr = cooperative_groups;
    cgr::cluster_group cl = cgr::this_cluster();
    const unsigned crank = SPREAD ? (unsigned)member : cl.block_rank();
    const unsigned csize = SPREAD ? (unsigned)group : cl.num_blocks();
    unsigned* ready = SPREAD ? sync + kSyncReady : cl.map_shared_rank(sm.ready, 0);
    int* ctl = SPREAD ? (int*)sync : cl.map_shared_rank(sm.ctl, 0);

    if (!SPREAD && crank == 0) {
        for (int t = threadIdx.x; t < (n + 31) / 32; t += blockDim.x) sm.ready[t] = 0u;
        if (threadIdx.x == 0) {
            sm.ctl[0] = 0;
            sm.ctl[1] = 0;
            sm.ctl[2] = 0x7fffffff;
            sm.ctl[3] = 0;
        }
    }
    // The system's dense trailing block: the tail columns scatter their
    // pattern's entries into it (the dense kernel reads the others as 0).
    double* W = P.dtail > 0 ? S.tailw : nullptr;

    VT* lu = (VT*)S.lu;
    VT* lval = (VT*)S.lval;
    VT* uval = (VT*)S.uval;
    VT* udiag = (VT*)S.udiag;
    double minpiv = INFINITY, minratio = INFINITY, maxu = 0.0;
    int bad = 0;
    long long c_wait = 0, c_gather = 0, c_update = 0;
    const long long t_begin = clock64();
    if (!SPREAD) {
        if (crank == 0 && threadIdx.x == 0) {
            S.stats->cyc_wait = 0;
            S.stats->cyc_gather = 0;
            S.stats->cyc_update = 0;
        }
        cl.sync();
    }

    while (true) {
        const int idx = warp_claim(&ctl[0]);
        if (idx >= n) break;
        // The column's record (one broadcast load of three 16-byte words),
        // then, all in flight together: this lane's first input entry, its
        // first dependency, the destination of its first slot, and the input
        // value.  The later entries (columns longer than a warp) load as
        // they are reached.
        const int4 ra = P.crec[3 * idx], rb = P.crec[3 * idx + 1], rc = P.crec[3 * idx + 2];
        const int k = ra.x, c0 = ra.y, len = ra.z, d = ra.w;
        const int a0 = rb.x, a1 = rb.y, dsp = rb.z, bpos = rb.w;
        const int* rows = P.ri + c0;
        const int ta = a0 + lane;
        const int adst = ta < a1 ? P.a_dst[ta] : -1;
        const int asrc = ta < a1 ? P.a_src[ta] : -1;
        const int aprev = (ta < a1 && ta > a0) ? P.a_dst[ta - 1] : -1;
        const int jj0 = lane < dsp ? rows[lane] : 0;
        const int2 bc0 = lane < dsp ? P.dep_bc[c0 + lane] : make_int2(0, 0);
        const int sdst0 = lane < len ? P.slot_dst[c0 + lane] : -1;
        const double av0 = asrc >= 0 ? S.a_val[asrc] : 0.0;
        double* x;
        if (len <= plan.wcap) {
            x = wx;
        } else if (S.scratch) {
            x = S.scratch + ((size_t)blockIdx.x * nw + warp) * P.max_col;
        } else {
            bad |= ST_CAPACITY;
            __syncwarp();
            if (lane == 0) set_ready(ready, k);
            continue;
        }
        // A column of the dense trailing block applies only its dependencies
        // before k0 here (they come first: rows ascending; dsp of them).
        const bool tailcol = k >= P.k0;
        for (int t = lane; t < len; t += 32) x[t] = 0.0;
        __syncwarp();
        // The factor of A + shift diag|A(i,i)|: the input's diagonal entry
        // (duplicates summed first) gains shift times its magnitude.
        const int adg = prm.shift != 0.0 ? rc.z : -1;
        if (ta < a1 && (ta == a0 || aprev != adst)) {
            double s = av0;
            for (int u = ta + 1; u < a1 && P.a_dst[u] == adst; u++) s = __dadd_rn(s, S.a_val[P.a_src[u]]);
            if (adst == adg) s = __dadd_rn(s, __dmul_rn(prm.shift, fabs(s)));
            x[adst] = s;
        }
        for (int t = a0 + 32 + lane; t < a1; t += 32) {
            const int dst = P.a_dst[t];
            if (t == a0 || P.a_dst[t - 1] != dst) {
                double s = S.a_val[P.a_src[t]];
                for (int u = t + 1; u < a1 && P.a_dst[u] == dst; u++)
                    s = __dadd_rn(s, S.a_val[P.a_src[u]]);
                if (dst == adg) s = __dadd_rn(s, __dmul_rn(prm.shift, fabs(s)));
                x[dst] = s;
            }
        }
        __syncwarp();
        long long tc = phase_clock();
        // Apply the dependency columns in ascending order.  Each round takes
        // the next run of dependencies that are already complete (blocking
        // only when the very next one is not, so the older dependencies of a
        // column overlap with the computation of its most recent ones), up to
        // plan.scap gathered entries; their L values and relative slots are
        // copied to shared memory with all copies in flight together, then
        // applied.
        // rel index of dependency u0
        long long roff = have_rel ? (long long)(((unsigned long long)(unsigned)rc.y << 32) | (unsigned)rc.x) : 0;
        // Dependency metadata of the round starting at pf_u0, loaded while
        // the previous round's copies and updates ran.
        int pf_u0 = 0, pf_jj = jj0;
        int2 pf_bc = bc0;
        for (int u0 = 0; u0 < dsp;) {
            const int u = u0 + lane;
            int beg = 0, cnt = 0;
            bool rdy = true;
            if (u < dsp) {
                const bool pre = u0 == pf_u0;
                const int jj = pre ? pf_jj : rows[u];
                const int2 bc = pre ? pf_bc : P.dep_bc[c0 + u];
                beg = bc.x;
                cnt = bc.y;
                rdy = is_ready(ready, jj);
            }
            // Acquire (spread mode): each lane orders what follows after its
            // own ready-bit read; the warp's ballot then orders the other
            // lanes' reads of that dependency's values after it.
            if (SPREAD) spread_acquire();
            int nready = __ffs(~__ballot_sync(0xffffffffu, rdy)) - 1;
            if (nready < 0) nready = 32;
            if (nready == 0) {
                // Wait for the next dependency, then re-scan: others may
                // have completed meanwhile and join the same round.
                const bool ok = __all_sync(0xffffffffu, wait_ready(ready, rows[u0], &ctl[3]));
                if (ok) continue;
                bad |= ST_WAIT_TIMEOUT;
                nready = 1;
            }
            // Acquire (cluster): the dependency columns' values (written by
            // any CTA of the cluster) are read after their ready bits.
            if (!SPREAD) share_fence(csize);
            {
                const long long t2 = phase_clock();
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
            // Value stage layout: each dependency's run starts at the 16-byte
            // boundary at or below its first value (copied in whole 16-byte
            // pieces that bypass L1, so values written by another SM are never
            // read from a stale L1 line).
            constexpr int VPK = 16 / (int)sizeof(VT);
            const int vsh = beg & (VPK - 1);
            const int vlen = u < dsp ? ((vsh + cnt + VPK - 1) / VPK) * VPK : 0;
            int vincl = vlen;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, vincl, o);
                if (lane >= o) vincl += v;
            }
            const int vexcl = vincl - vlen;
            int nfit = have_rel ? __popc(__ballot_sync(0xffffffffu, u < dsp && incl <= plan.scap &&
                                                                        vincl <= plan.scap))
                                : 0;
            nfit = min(nfit, nready);
            if (nfit == 0) {
                // One dependency applied straight from global memory (longer
                // than the stage, or no relative slots).
                const double xj = x[u0];
                const int p0 = __shfl_sync(0xffffffffu, beg, 0);
                const int c = __shfl_sync(0xffffffffu, cnt, 0);
                if (xj != 0.0) {
                    for (int e = lane; e < c; e += 32) {
                        const double l = (double)__ldcg(lu + p0 + e);
                        const int s = have_rel ? (int)P.rel[roff + e]
                                               : find_slot(rows, u0 + 1, len, P.ri[p0 + e]);
                        if (s >= 0) x[s] = __dsub_rn(x[s], __dmul_rn(l, xj));
                        else bad |= ST_CAPACITY;
                    }
                }
                __syncwarp();
                roff += c;
                u0 += 1;
                continue;
            }
            // Stage: relative slots of the round (one contiguous run of rel,
            // copied in aligned 16-byte pieces) and each dependency's values.
            const int tot = __shfl_sync(0xffffffffu, incl, nfit - 1);
            const long long g0 = roff & ~7LL;
            const int sh = (int)(roff - g0);
            const int pieces = (sh + tot + 7) >> 3;
            for (int e = lane; e < pieces; e += 32) cp_async_16(srel + 8 * e, P.rel + g0 + 8 * e);
            for (int t = 0; t < nfit; t++) {
                const int a_t = __shfl_sync(0xffffffffu, beg - vsh, t);
                const int p_t = __shfl_sync(0xffffffffu, vlen, t) / VPK;
                const int o_t = __shfl_sync(0xffffffffu, vexcl, t);
                for (int e = lane; e < p_t; e += 32) cp_async_16(sval + o_t + e * VPK, lu + a_t + e * VPK);
            }
            // The next round's metadata, in flight with the copies.
            pf_u0 = u0 + nfit;
            if (pf_u0 + lane < dsp) {
                pf_jj = __ldg(rows + pf_u0 + lane);
                pf_bc = __ldg(P.dep_bc + c0 + pf_u0 + lane);
            }
            cp_async_wait_all();
            __syncwarp();
            {
                const long long t2 = phase_clock();
                c_gather += t2 - tc;
                tc = t2;
            }
            for (int t = 0; t < nfit; t++) {
                const int c_t = __shfl_sync(0xffffffffu, cnt, t);
                const int o_t = __shfl_sync(0xffffffffu, excl, t);
                const int vo_t = __shfl_sync(0xffffffffu, vexcl + vsh, t);
                const double xj = x[u0 + t];
                if (xj != 0.0 && c_t <= 32) {
                    // A short dependency column: one entry per lane.
                    if (lane < c_t) {
                        const int s = (int)srel[sh + o_t + lane];
                        const double l = ValTraits<VT>::load(sval + vo_t + lane);
                        x[s] = __dsub_rn(x[s], __dmul_rn(l, xj));
                    }
                } else if (xj != 0.0 && c_t <= 64) {
                    // Two entries per lane, both loaded before either store
                    // (rows of one dependency are distinct).
                    const bool h = lane + 32 < c_t;
                    const int s0 = (int)srel[sh + o_t + lane];
                    const int s1 = h ? (int)srel[sh + o_t + lane + 32] : s0;
                    const double l0 = ValTraits<VT>::load(sval + vo_t + lane);
                    const double l1 = h ? ValTraits<VT>::load(sval + vo_t + lane + 32) : 0.0;
                    const double x0 = x[s0], x1 = x[s1];
                    x[s0] = __dsub_rn(x0, __dmul_rn(l0, xj));
                    if (h) x[s1] = __dsub_rn(x1, __dmul_rn(l1, xj));
                } else if (xj != 0.0) {
                    // Rows of one dependency are distinct: four entries per
                    // lane are loaded before any is written back.
                    for (int e = lane; e < c_t; e += 128) {
                        int s[4];
                        double l[4], xv[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int ee = e + 32 * q;
                            s[q] = ee < c_t ? (int)srel[sh + o_t + ee] : -1;
                            l[q] = ee < c_t ? ValTraits<VT>::load(sval + vo_t + ee) : 0.0;
                        }
#pragma unroll
                        for (int q = 0; q < 4; q++) xv[q] = s[q] >= 0 ? x[s[q]] : 0.0;
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            if (s[q] >= 0) x[s[q]] = __dsub_rn(xv[q], __dmul_rn(l[q], xj));
                    }
                }
                __syncwarp();
            }
            {
                const long long t2 = phase_clock();
                c_update += t2 - tc;
                tc = t2;
            }
            roff += tot;
            u0 += nfit;
        }
        if (tailcol) {
            // U rows before k0 are final; the rest goes to the dense block
            // (destinations of four slots per lane loaded first).
            for (int t0 = lane; t0 < len; t0 += 128) {
                int dst[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int t = t0 + 32 * q;
                    dst[q] = t >= len ? 0 : t < dsp ? (t < 32 ? sdst0 : __ldg(P.slot_dst + c0 + t))
                                                    : __ldg(rows + t);
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int t = t0 + 32 * q;
                    if (t >= len) break;
                    const double v = x[t];
                    if (t < dsp) {
                        maxu = fmax(maxu, fabs(v));
                        uval[dst[q]] = ValTraits<VT>::to(v);
                    } else {
                        W[(size_t)(dst[q] - P.k0) * P.tail_ld + (k - P.k0)] = v;
                    }
                }
            }
            __syncwarp();
            continue;
        }
        const double piv = x[d];
        double amax = 0.0;
        for (int t = d + 1 + lane; t < len; t += 32) amax = fmax(amax, fabs(x[t]));
        amax = warp_max(amax);
        const double ap = fabs(piv);
        if (!(ap > 0.0) || !isfinite(piv)) {
            bad |= ST_SINGULAR;
            // The first singular column: a minimum (spread mode: the sync
            // area starts at 0, so the maximum of INT_MAX - k).
            if (lane == 0) {
                if (SPREAD) atomicMax(&ctl[kSyncSingular], 0x7fffffff - k);
                else atomicMin(&ctl[2], k);
            }
        }
        minpiv = fmin(minpiv, ap);
        const double ratio = amax > ap ? ap / amax : 1.0;
        minratio = fmin(minratio, ratio);
        if (ratio < prm.pivot_tol) bad |= ST_PIVOT_WEAK;
        // Each value is stored once where the solves read it (U rows, the
        // diagonal, L rows); the strict-L part also goes to the merged
        // columns, which the later columns' gathers read.  The destinations
        // of four slots per lane are loaded before any of their stores (the
        // loads could not move above the stores of an earlier slot).
        for (int t0 = lane; t0 < len; t0 += 128) {
            int dst[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int t = t0 + 32 * q;
                dst[q] = t < len ? (t < 32 ? sdst0 : __ldg(P.slot_dst + c0 + t)) : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int t = t0 + 32 * q;
                if (t >= len) break;
                double v = x[t];
                if (t > d) v = __ddiv_rn(v, piv);
                else maxu = fmax(maxu, fabs(v));
                const VT sv = ValTraits<VT>::to(v);
                if (t < d) uval[dst[q]] = sv;
                else if (t == d) {
                    udiag[k] = sv;
                    ((VT*)S.udiag_bwd)[bpos] = ValTraits<VT>::to(1.0 / piv);
                } else {
                    lu[c0 + t] = sv;
                    lval[dst[q]] = sv;
                }
            }
        }
        // Release: the column's values before its ready bit.
        share_release_t<SPREAD>(csize);
        __syncwarp();
        if (lane == 0) set_ready(ready, k);
    }

    if (SPREAD) {
        spread_finish(S, sync, group, sm, minpiv, minratio, maxu, bad, c_wait, c_gather, c_update, t_begin);
        return;
    }
    if (lane == 0) {
        atomicAdd((unsigned long long*)&S.stats->cyc_wait, (unsigned long long)c_wait);
        atomicAdd((unsigned long long*)&S.stats->cyc_gather, (unsigned long long)c_gather);
        atomicAdd((unsigned long long*)&S.stats->cyc_update, (unsigned long long)c_update);
    }
    if (threadIdx.x == 0) S.stats->cyc_refactor = clock64() - t_begin;
    // Statistics: rank 0 writes, the others merge, one after another; the
    // last cluster barrier also keeps rank 0's shared state alive until every
    // CTA of the cluster is done with it.
    cl.sync();
    for (unsigned r = 0; r < csize; r++) {
        if (crank == r) cta_store_pivot_stats(S.stats, sm, minpiv, minratio, maxu, bad, r == 0, ctl);
        cl.sync();
    }
}

// ---------------------------------------------------------------------------
// Triangular solves of the dense trailing block (rows [k0, n), factor T in
// VT with leading dimension ld): 32-row blocks, the diagonal block by one
// warp through shuffles, the rest of the block's columns as one
// multiply-add per row and thread.  fp64 accumulation.
// ---------------------------------------------------------------------------
// sum_{c < w} row[c * stride] * y[c] for one 32-column block of a tail row
// (column-major factor): all loads issued before the multiply-adds.
template <typename VT>
__device__ __forceinline__ double tail_row_dot(const VT* row, size_t stride, const double* y, int w) {
    // Unconditional loads from clamped (in-bounds) addresses, so all 32 are
    // in flight before the first multiply-add.
    VT v[32];
#pragma unroll
    for (int c = 0; c < 32; c++) v[c] = row[(size_t)min(c, w - 1) * stride];
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 32; c++) acc = fma(c < w ? (double)v[c] : 0.0, y[min(c, w - 1)], acc);
    return acc;
}

// The 32 factor values of one tail row's 32-column block (clamped
// addresses, all loads in flight), and their dot product with y.
template <typename VT>
__device__ __forceinline__ void tail_load_regs(const VT* row, size_t stride, int w, VT* v) {
#pragma unroll
    for (int c = 0; c < 32; c++) v[c] = row[(size_t)min(c, w - 1) * stride];
}
// tail_row_dot as a call (rows past the ones a thread preloads: D above the
// CTA size; keeps its 32 loads out of the caller's registers).
template <typename VT>
__device__ __noinline__ double tail_row_dot_call(const VT* row, size_t stride, const double* y, int w) {
    return tail_row_dot<VT>(row, stride, y, w);
}
template <typename VT>
__device__ __forceinline__ double tail_dot_regs(const VT* v, const double* y, int w) {
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 32; c++) acc = fma(c < w ? (double)v[c] : 0.0, y[min(c, w - 1)], acc);
    return acc;
}

// y[k0..n) := L_tt^-1 y[k0..n) (unit lower; the tail rows' entries in the
// columns before k0 were applied by the forward sweep's last level).
template <typename VT>
__device__ __noinline__ void tail_forward(const PatternDev& P, const VT* T, const VT* Ti, double* y, SysStats* st) {
    const int k0 = P.k0, D = P.dtail, ld = P.tail_ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long c_diag = 0, c_gemv = 0;
    double* yt = y + k0;
    // Every thread loads 32 values before the diagonal block: warp 0 its
    // row of the block's inverse (L^-1, from the dense kernel), the other
    // warps their first row of the block's 32 columns below it (so those
    // loads overlap the diagonal product).
    const int nt = (int)blockDim.x - 32, t = (int)threadIdx.x - 32;
    for (int jb = 0; jb < D; jb += 32) {
        const int w = min(32, D - jb);
        const long long ta = clock64();
        const int i0 = jb + w + t;
        const bool pre = t >= 0 && i0 < D;
        VT v[32];
        if (warp == 0) tail_load_regs<VT>(Ti + (size_t)(jb >> 5) * 2048 + lane, 32, 32, v);
        else if (pre) tail_load_regs<VT>(T + (size_t)jb * ld + i0, ld, w, v);
        if (warp == 0) {
            // y_b := L_bb^-1 y_b: lane i's row of the inverse against the
            // block of y (all lanes read it before any writes).
            const double yr = lane < w ? tail_dot_regs<VT>(v, yt + jb, w) : 0.0;
            __syncwarp();
            if (lane < w) yt[jb + lane] = yr;
        }
        __syncthreads();
        const long long tb = clock64();
        if (pre) yt[i0] -= tail_dot_regs<VT>(v, yt + jb, w);
        for (int i = i0 + nt; t >= 0 && i < D; i += nt)
            yt[i] -= tail_row_dot_call<VT>(T + (size_t)jb * ld + i, ld, yt + jb, w);
        __syncthreads();
        const long long tc = clock64();
        c_diag += tb - ta;
        c_gemv += tc - tb;
    }
    if (threadIdx.x == 0) {
        st->cyc_tdiag += c_diag;
        st->cyc_tgemv += c_gemv;
    }
}

// y[k0..n) := U_tt^-1 y[k0..n) (upper with diagonal).
template <typename VT>
__device__ __noinline__ void tail_backward(const PatternDev& P, const VT* T, const VT* Ti, double* y, SysStats* st) {
    const int k0 = P.k0, D = P.dtail, ld = P.tail_ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long c_diag = 0, c_gemv = 0;
    double* yt = y + k0;
    // As tail_forward: warp 0 applies the block's U^-1, the other warps
    // update the rows above it, their first row loaded before that product.
    const int nt = (int)blockDim.x - 32, t = (int)threadIdx.x - 32;
    for (int jb = ((D - 1) / 32) * 32; jb >= 0; jb -= 32) {
        const int w = min(32, D - jb);
        const long long ta = clock64();
        const bool pre = t >= 0 && t < jb;
        VT v[32];
        if (warp == 0) tail_load_regs<VT>(Ti + (size_t)(jb >> 5) * 2048 + 1024 + lane, 32, 32, v);
        else if (pre) tail_load_regs<VT>(T + (size_t)jb * ld + t, ld, w, v);
        if (warp == 0) {
            const double yr = lane < w ? tail_dot_regs<VT>(v, yt + jb, w) : 0.0;
            __syncwarp();
            if (lane < w) yt[jb + lane] = yr;
        }
        __syncthreads();
        const long long tb = clock64();
        if (pre) yt[t] -= tail_dot_regs<VT>(v, yt + jb, w);
        for (int i = t + nt; t >= 0 && i < jb; i += nt)
            yt[i] -= tail_row_dot_call<VT>(T + (size_t)jb * ld + i, ld, yt + jb, w);
        __syncthreads();
        const long long tc = clock64();
        c_diag += tb - ta;
        c_gemv += tc - tb;
    }
    if (threadIdx.x == 0) {
        st->cyc_tdiag += c_diag;
        st->cyc_tgemv += c_gemv;
    }
}

// ---------------------------------------------------------------------------
// y := U^-1 L^-1 rhs in pivot-position space (level-scheduled, warp per row,
// factors read as VT, accumulation in fp64).  y may be shared or global
// memory; rhs must not alias y.
// ---------------------------------------------------------------------------
template <typename VT>
__device__ void cta_lu_apply(const PatternDev& P, const VT* lval, const VT* uval,
                             const VT* udiag, const VT* tail, const VT* tinv, const double* rhs, double* y,
                             Smem& sm, int& bad, SysStats* st) {
    const long long t0 = clock64();
    const int n = P.n, k0 = P.k0;
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
    const long long t1 = clock64();
    if (P.dtail > 0) {
        tail_forward<VT>(P, tail, tinv, y, st);
        tail_backward<VT>(P, tail, tinv, y, st);
    }
    const long long t2 = clock64();
    // Rows of the dense tail are complete before the sparse U sweep starts.
    for (int t = threadIdx.x; t < (n + 31) / 32; t += blockDim.x) {
        const int lo = t * 32;
        unsigned bits = 0u;
        for (int b = 0; b < 32; b++)
            if (lo + b >= k0 && lo + b < n) bits |= 1u << b;
        sm.ready[t] = bits;
    }
    if (threadIdx.x == 0) sm.ctl[0] = 0;
    __syncthreads();
    while (true) {
        const int idx = warp_claim(&sm.ctl[0]);
        if (idx >= k0) break;
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
    if (threadIdx.x == 0 && st) {
        st->cyc_lsolve += t1 - t0;
        st->cyc_tail += t2 - t1;
        st->cyc_usolve += clock64() - t2;
    }
}

// cp.async group control (sm_80+).
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One triangular sweep, level-synchronous (one barrier per level).  Each
// level's entries (column positions, values and, for U, the diagonal of its
// rows in sweep order) are copied by cp.async into a ring of kStages
// shared-memory stages, kStages - 1 levels ahead of the level being
// computed, so a level's work reads shared memory only.  A level's rows are
// spread over groups of g lanes, g the power of two at or above its mean
// row length (1..32): wide levels of short rows run a row per thread,
// narrow levels of long rows a row per warp, or, for a level of a few very
// long rows, several warps per row whose partial sums are added in warp
// order (part: NT / 32 doubles of shared memory).  Levels larger than a
// stage read global memory directly.
// UPPER: y[i] = (y[i] - sum) / diag (U sweep), else y[i] -= sum.
constexpr int kStages = 4;

// Bulk asynchronous copies (TMA, untiled) with completion on an mbarrier in
// shared memory: 16-byte aligned addresses, sizes a multiple of 16 bytes.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// The barriers' initialization, visible to the asynchronous proxy.
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// Earlier generic-proxy accesses to shared memory ordered before later
// asynchronous-proxy (bulk copy) writes.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of bar: false (and the status bit set)
// when it does not complete within kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* status) {
    for (long long it = 0; !mbar_try_wait(bar, parity); it++) {
        if (it > kSpinLimit) {
            if (status) atomicOr(status, ST_WAIT_TIMEOUT);
            return false;
        }
    }
    return true;
}

// sum over e = e0, e0 + g, ... < pe of val[e] * y[col[e]]: four partial
// sums, so a lane has four loads of y in flight when y lives in global
// memory (a row with fewer than four entries per lane keeps one sum).
template <typename VT>
__device__ __forceinline__ double row_dot(const VT* vv, const int* cc, const double* y, int e0, int pe, int g) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int e = e0;
    for (; e + 3 * g < pe; e += 4 * g) {
        const int c0 = cc[e], c1 = cc[e + g], c2 = cc[e + 2 * g], c3 = cc[e + 3 * g];
        a0 = fma(ValTraits<VT>::load(vv + e), y[c0], a0);
        a1 = fma(ValTraits<VT>::load(vv + e + g), y[c1], a1);
        a2 = fma(ValTraits<VT>::load(vv + e + 2 * g), y[c2], a2);
        a3 = fma(ValTraits<VT>::load(vv + e + 3 * g), y[c3], a3);
    }
    for (; e < pe; e += g) a0 = fma(ValTraits<VT>::load(vv + e), y[cc[e]], a0);
    return (a0 + a1) + (a2 + a3);
}

__host__ __device__ inline size_t stage_bytes(int cap_e, int cap_r, int vsize) {
    return (size_t)(cap_e + 8) * (4 + vsize) + (size_t)(cap_r + 8) * vsize;
}

// The sweeps run on the first kSweepThreads threads (named barrier 1); the
// other warps of the CTA, if any, wait at the closing CTA barrier.
constexpr int kSweepThreads = 1024;

__device__ __forceinline__ void sweep_barrier(int nthreads) {
    asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

// The rows [r0, r1) of one level, 2^LG lanes per row (a compile-time group
// width, so the row reduction is unrolled), in rounds of NT / 2^LG rows.
template <typename VT, bool UPPER, bool GY, int LG>
__device__ __forceinline__ void sweep_rows(int r0, int r1, int NT, const int* order, const int* rp, const int* cc,
                                           const VT* vv, const VT* dd, int eb, int rb, double* y) {
    constexpr int g = 1 << LG;
    const int lig = threadIdx.x & (g - 1);
    const int warp = threadIdx.x >> 5;
    const int ngr = NT >> LG;
    for (int rbase = r0; rbase < r1; rbase += ngr) {
        if (rbase + ((warp * 32) >> LG) >= r1) break;   // nothing left for this warp
        const int r = rbase + ((int)threadIdx.x >> LG);
        double acc = 0.0, yi = 0.0, di = 1.0;
        int i = 0;
        if (r < r1) {
            // The row's own right-hand side and diagonal, loaded beside the
            // dot product instead of after its reduction (no other thread
            // writes y[i] in this level).
            if (lig == 0) {
                i = order[r];
                yi = y[i];
                if (UPPER) di = ValTraits<VT>::load(dd + (r - rb));
            }
            if (GY) {
                acc = row_dot<VT>(vv, cc, y, rp[r] - eb + lig, rp[r + 1] - eb, g);
            } else {
                // Two entries per lane in flight.
                const int pe = rp[r + 1] - eb;
                int e = rp[r] - eb + lig;
                double a1 = 0.0;
                for (; e + g < pe; e += 2 * g) {
                    const int c0 = cc[e], c1 = cc[e + g];
                    const double v0 = ValTraits<VT>::load(vv + e), v1 = ValTraits<VT>::load(vv + e + g);
                    acc = fma(v0, y[c0], acc);
                    a1 = fma(v1, y[c1], a1);
                }
                if (e < pe) acc = fma(ValTraits<VT>::load(vv + e), y[cc[e]], acc);
                acc += a1;
            }
        }
#pragma unroll
        for (int o = g >> 1; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, g);
        if (r < r1 && lig == 0) y[i] = UPPER ? (yi - acc) * di : yi - acc;
    }
}

// GY: y lives in global memory (large systems): levels of a few long rows
// (64 entries or more on average) get several warps per row, and long rows
// four partial sums per lane; with y in shared memory a lane keeps one sum
// and a row at most one warp.
template <typename VT, bool UPPER, bool GY>
__device__ __noinline__ void staged_sweep(int nlev, const int4* ld4, const int* lgl, const int* order, const int* rp,
                             const int* ci, const VT* val, const VT* dgo, double* y,
                             char* stage, int cap_e, int cap_r, double* part, int* status) {
    const int NT = min((int)blockDim.x, kSweepThreads);
    if ((int)threadIdx.x >= NT) {
        __syncthreads();
        return;
    }
    const int CE = cap_e + 8;
    const size_t sb = stage_bytes(cap_e, cap_r, sizeof(VT));
    const int warp = threadIdx.x >> 5;
    // Each staged level is three bulk copies (column indices, values and,
    // for U, the reciprocal diagonal: contiguous runs in sweep order, rounded
    // out to 16-byte boundaries; every array has slack past its end for the
    // rounding) issued by one thread, the last one (rows go to the lowest
    // warps), completing on the slot's mbarrier; every thread waits on that
    // barrier's phase before the level's CTA barrier.
    __shared__ unsigned long long mbar[kStages];
    const bool issuer = (int)threadIdx.x == NT - 1;
    auto staged = [&](const int4& d) { return d.w - d.z <= cap_e && d.y - d.x <= cap_r; };
    // Every level arrives on its slot's barrier (a level too large for a
    // stage with no bytes), so the k-th use of a slot is its phase k.
    auto issue = [&](int L) {
        if (!issuer || L >= nlev) return;
        const int4 d = ld4[L];
        if (!staged(d)) {
            mbar_expect_tx(&mbar[L % kStages], 0u);
            return;
        }
        char* base = stage + (size_t)(L % kStages) * sb;
        int* sc = (int*)base;
        VT* sv = (VT*)(base + (size_t)CE * 4);
        VT* sd = (VT*)(base + (size_t)CE * (4 + sizeof(VT)));
        const int a0 = d.z & ~3, n4 = ((d.w + 3) & ~3) - a0;
        const int b0 = d.x & ~3, m4 = UPPER ? ((d.y + 3) & ~3) - b0 : 0;
        unsigned long long* bar = &mbar[L % kStages];
        fence_proxy_async();
        mbar_expect_tx(bar, (unsigned)((size_t)n4 * (4 + sizeof(VT)) + (size_t)m4 * sizeof(VT)));
        if (n4 > 0) {
            bulk_g2s(sc, ci + a0, (unsigned)n4 * 4u, bar);
            bulk_g2s(sv, val + a0, (unsigned)(n4 * sizeof(VT)), bar);
        }
        if (UPPER && m4 > 0) bulk_g2s(sd, dgo + b0, (unsigned)(m4 * sizeof(VT)), bar);
    };
    if (threadIdx.x == 0) {
        for (int k = 0; k < kStages; k++) mbar_init(&mbar[k], 1);
        fence_mbar_init();
    }
    sweep_barrier(NT);
    for (int L = 0; L < kStages - 1; L++) issue(L);
    for (int L = 0; L < nlev; L++) {
        mbar_wait(&mbar[L % kStages], (unsigned)(L / kStages) & 1u, status);
        sweep_barrier(NT);
        issue(L + kStages - 1);
        const int4 d = ld4[L];
        const int r0 = d.x, r1 = d.y, nr = r1 - r0;
        const bool st = d.w - d.z <= cap_e && nr <= cap_r;
        char* base = stage + (size_t)(L % kStages) * sb;
        const int* cc = st ? (const int*)base : ci;
        const VT* vv = st ? (const VT*)(base + (size_t)CE * 4) : val;
        const VT* dd = st ? (const VT*)(base + (size_t)CE * (4 + sizeof(VT))) : dgo;
        const int eb = st ? (d.z & ~3) : 0, rb = st ? (r0 & ~3) : 0;
        const int lgd = lgl[L];
        if (lgd < 0) {
            // A run of narrow levels: one warp, its rows in level order (a
            // row's result is visible to the warp's next rows after the warp
            // barrier), no CTA barrier until the run ends.
            if (warp == 0) {
                const int lane = threadIdx.x & 31;
                for (int r = r0; r < r1; r++) {
                    // Four loads per lane in flight (a run too large for a
                    // stage reads global memory).
                    double acc = row_dot<VT>(vv, cc, y, rp[r] - eb + lane, rp[r + 1] - eb, 32);
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                    if (lane == 0) {
                        const int i = order[r];
                        if (UPPER) y[i] = (y[i] - acc) * ValTraits<VT>::load(dd + (r - rb));
                        else y[i] = y[i] - acc;
                    }
                    __syncwarp();
                }
            }
            continue;
        }
        // Several warps per row only for rows long enough to pay for the two
        // extra barriers.
        if (GY && lgd > 5 && d.w - d.z >= 64 * nr) {
            // Threads per row: the largest power of two (32 .. 2^lgd) that
            // still gives every row of the level its own group in one pass.
            int gw = 32;
            while (gw * 2 <= (1 << lgd) && gw * 2 * nr <= NT) gw *= 2;
            if (gw > 32) {
                const int rpp = NT / gw, wpr = gw >> 5;
                const int lane = threadIdx.x & 31;
                for (int rp0 = r0; rp0 < r1; rp0 += rpp) {
                    const int r = rp0 + (int)threadIdx.x / gw;
                    const int lig = (int)threadIdx.x & (gw - 1);
                    double acc = 0.0;
                    if (r < r1) acc = row_dot<VT>(vv, cc, y, rp[r] - eb + lig, rp[r + 1] - eb, gw);
                    acc = warp_sum(acc);
                    if (lane == 0) part[warp] = acc;
                    sweep_barrier(NT);
                    if ((int)threadIdx.x < rpp) {
                        const int rr = rp0 + (int)threadIdx.x;
                        if (rr < r1) {
                            double sum = 0.0;
                            for (int w = 0; w < wpr; w++) sum += part[threadIdx.x * wpr + w];
                            const int i = order[rr];
                            if (UPPER) y[i] = (y[i] - sum) * ValTraits<VT>::load(dd + (rr - rb));
                            else y[i] = y[i] - sum;
                        }
                    }
                    sweep_barrier(NT);
                }
                continue;
            }
        }
        switch (min(lgd, 5)) {
            case 0: sweep_rows<VT, UPPER, GY, 0>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
            case 1: sweep_rows<VT, UPPER, GY, 1>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
            case 2: sweep_rows<VT, UPPER, GY, 2>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
            case 3: sweep_rows<VT, UPPER, GY, 3>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
            case 4: sweep_rows<VT, UPPER, GY, 4>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
            default: sweep_rows<VT, UPPER, GY, 5>(r0, r1, NT, order, rp, cc, vv, dd, eb, rb, y); break;
        }
    }
    // Every staged level's copies were waited for; the barriers are free.
    sweep_barrier(NT);
    if (threadIdx.x == 0)
        for (int k = 0; k < kStages; k++) mbar_inval(&mbar[k]);
    __syncthreads();
}

// Shared-memory sweep descriptors of one system: [fwd level descriptors
// nfl x int4][bwd level descriptors nbl x int4][fwd lanes nfl][bwd lanes
// nbl][fwd_order n][fwd rp n+1][bwd_order n][bwd rp n+1].
__device__ __forceinline__ bool sweep_desc_fits(const PatternDev& P, const SmemPlan& plan) {
    return P.n <= plan.ycap && 4 * P.n + 5 * (P.nfwd_levels + P.nbwd_levels) + 4 <= plan.dcap &&
           (plan.sc_ent > 0 || plan.flow);
}

// Byte offset (16-byte aligned) of the sweep descriptors in the solve
// area: after the solve vector (ycap doubles) and the Hessenberg block.
__host__ __device__ inline size_t sweep_desc_offset(int ycap, int m) {
    const size_t b = ((size_t)ycap + (size_t)(m + 1) * m + 6 * (size_t)(m + 1)) * sizeof(double);
    return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ int* sweep_desc_base(const SmemPlan& plan, Smem& sm) {
    return (int*)(sm.uni + sweep_desc_offset(plan.ycap, plan.m));
}

struct SweepDesc {
    const int4 *f_ld, *b_ld;
    const int *f_lg, *b_lg, *f_ord, *f_rp, *b_ord, *b_rp;
    // The pattern's own arrays in global memory (systems whose solve vector
    // or descriptors do not fit shared memory).
    __device__ explicit SweepDesc(const PatternDev& P) {
        const int nfl = P.nfwd_levels, nbl = P.nbwd_levels;
        f_ld = (const int4*)P.fwd_ldesc;
        b_ld = (const int4*)P.bwd_ldesc;
        f_lg = P.fwd_ldesc + 4 * nfl;
        b_lg = P.bwd_ldesc + 4 * nbl;
        f_ord = P.fwd_order;
        f_rp = P.lrp;
        b_ord = P.bwd_order;
        b_rp = P.urp;
    }
    // The packed copy load_sweep_desc wrote to shared memory at d.
    __device__ SweepDesc(const PatternDev& P, const int* d) {
        const int n = P.n, nfl = P.nfwd_levels, nbl = P.nbwd_levels;
        f_ld = (const int4*)d;
        b_ld = f_ld + nfl;
        f_lg = (const int*)(b_ld + nbl);
        b_lg = f_lg + nfl;
        f_ord = b_lg + nbl;
        f_rp = f_ord + n;
        b_ord = f_rp + n + 1;
        b_rp = b_ord + n;
    }
};

__device__ void load_sweep_desc(const PatternDev& P, int* d) {
    const int n = P.n, nfl = P.nfwd_levels, nbl = P.nbwd_levels;
    const SweepDesc sd(P, d);
    int* f_ld = (int*)sd.f_ld;
    int* b_ld = (int*)sd.b_ld;
    int* f_lg = (int*)sd.f_lg;
    int* b_lg = (int*)sd.b_lg;
    int* f_ord = (int*)sd.f_ord;
    int* f_rp = (int*)sd.f_rp;
    int* b_ord = (int*)sd.b_ord;
    int* b_rp = (int*)sd.b_rp;
    for (int t = threadIdx.x; t < 4 * nfl; t += blockDim.x) f_ld[t] = P.fwd_ldesc[t];
    for (int t = threadIdx.x; t < 4 * nbl; t += blockDim.x) b_ld[t] = P.bwd_ldesc[t];
    for (int t = threadIdx.x; t < nfl; t += blockDim.x) f_lg[t] = P.fwd_ldesc[4 * nfl + t];
    for (int t = threadIdx.x; t < nbl; t += blockDim.x) b_lg[t] = P.bwd_ldesc[4 * nbl + t];
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        f_ord[t] = P.fwd_order[t];
        b_ord[t] = P.bwd_order[t];
    }
    for (int t = threadIdx.x; t <= n; t += blockDim.x) {
        f_rp[t] = P.lrp[t];
        b_rp[t] = P.urp[t];
    }
}

// Stage ring of the level-synchronous sweeps, after the descriptors.
__device__ __forceinline__ char* sweep_stage_base(const SmemPlan& plan, Smem& sm) {
    return (char*)(sweep_desc_base(plan, sm) + ((plan.dcap + 3) & ~3));
}

// y := U^-1 L^-1 rhs with the level-synchronous sweeps (descriptors sd in
// shared or global memory, stage ring at stage).  y may be global memory:
// the sweep barriers order its writes and reads inside the CTA.
template <typename VT>
__device__ void cta_lu_apply_levels(const SysDev& S, const PatternDev& P, const SmemPlan& plan,
                                    const double* rhs, double* y, const SweepDesc& sd, char* stage,
                                    double* part) {
    const int n = P.n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = rhs[i];
    __syncthreads();
    const long long t0 = clock64();
    const bool gy = P.n > plan.ycap;
    if (gy)
        staged_sweep<VT, false, true>(P.nfwd_levels, sd.f_ld, sd.f_lg, sd.f_ord, sd.f_rp, P.lci, (const VT*)S.lval,
                                      nullptr, y, stage, plan.sc_ent, plan.sc_rows, part, &S.stats->status);
    else
        staged_sweep<VT, false, false>(P.nfwd_levels, sd.f_ld, sd.f_lg, sd.f_ord, sd.f_rp, P.lci,
                                       (const VT*)S.lval, nullptr, y, stage, plan.sc_ent, plan.sc_rows, part, &S.stats->status);
    const long long t1 = clock64();
    if (P.dtail > 0) {
        tail_forward<VT>(P, (const VT*)S.tail, (const VT*)S.tinv, y, S.stats);
        tail_backward<VT>(P, (const VT*)S.tail, (const VT*)S.tinv, y, S.stats);
    }
    const long long t2 = clock64();
    if (gy)
        staged_sweep<VT, true, true>(P.nbwd_levels, sd.b_ld, sd.b_lg, sd.b_ord, sd.b_rp, P.uci, (const VT*)S.uval,
                                     (const VT*)S.udiag_bwd, y, stage, plan.sc_ent, plan.sc_rows, part, &S.stats->status);
    else
        staged_sweep<VT, true, false>(P.nbwd_levels, sd.b_ld, sd.b_lg, sd.b_ord, sd.b_rp, P.uci, (const VT*)S.uval,
                                      (const VT*)S.udiag_bwd, y, stage, plan.sc_ent, plan.sc_rows, part, &S.stats->status);
    if (threadIdx.x == 0) {
        S.stats->cyc_lsolve += t1 - t0;
        S.stats->cyc_tail += t2 - t1;
        S.stats->cyc_usolve += clock64() - t2;
    }
}

// ---------------------------------------------------------------------------
// Dataflow triangular sweeps with the solve vector in shared memory.  Warp w
// takes the rows w, w + NW, w + 2 NW, ... of a sweep order.  The order is
// level-sorted, so every dependency of a row comes before it; the smallest
// unfinished row therefore always has its dependencies done and its warp at
// it (a warp's earlier rows are smaller), and the sweep cannot deadlock.
// There is no CTA barrier inside a sweep and no ready flag: every output
// slot starts as a signalling-NaN bit pattern, which arithmetic never
// produces, a row's result is one 8-byte store, and a reader polls the value
// it needs.  Each warp stages its own rows in a private ring of
// kFlowSlots shared-memory slots, kFlowSlots - 1 rows ahead, by cp.async
// (column indices, values, the right-hand side and the reciprocal
// diagonal; a row's entries past kFlowCap are read from global memory, four
// chunks of 32 in flight), so a row waits only for its dependencies.
// ---------------------------------------------------------------------------
constexpr long long kFlowSentinel = 0x7ff00000deadbeefll;   // signalling NaN
constexpr int kFlowSlots = 3, kFlowCap = 128;

// One ring slot: kFlowCap column indices, kFlowCap values, the row's
// right-hand side (fp64) and its reciprocal diagonal (VT).
__host__ __device__ inline size_t flow_slot_bytes(int vsize) { return (size_t)kFlowCap * (4 + vsize) + 16; }
__host__ __device__ inline size_t flow_ring_bytes(int nwarps, int vsize) {
    return (size_t)nwarps * kFlowSlots * flow_slot_bytes(vsize);
}

// out[j] once written (bounded wait: after kSpinLimit polls, or at once when
// *abort is set, the wait gives up, sets ST_WAIT_TIMEOUT and returns the
// sentinel, a NaN).
__device__ __noinline__ double flow_wait(const double* out, int j, int* abort, int& bad) {
    const volatile long long* w = (const volatile long long*)out + j;
    const volatile int* ab = abort;
    long long v, it = 0;
    while ((v = *w) == kFlowSentinel) {
        if (++it > 32) {
            if (*ab) break;
            if (it > kSpinLimit) {
                atomicExch(abort, 1);
                break;
            }
            __nanosleep(32);
        }
    }
    if (v == kFlowSentinel) bad |= ST_WAIT_TIMEOUT;
    return __longlong_as_double(v);
}

__device__ __forceinline__ double flow_take(const double* out, int j, long long raw, int* abort, int& bad) {
    return raw != kFlowSentinel ? __longlong_as_double(raw) : flow_wait(out, j, abort, bad);
}

// Four entries per lane: sum into a[0..3] of v * out[j] (j < 0: none).
__device__ __forceinline__ void flow_acc4(const int* jj, const double* vv, const double* out, int* abort, int& bad,
                                          double* a) {
    const volatile long long* vo = (const volatile long long*)out;
    long long raw[4];
#pragma unroll
    for (int q = 0; q < 4; q++) raw[q] = jj[q] >= 0 ? vo[jj[q]] : 0ll;
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (jj[q] >= 0) a[q] = fma(vv[q], flow_take(out, jj[q], raw[q], abort, bad), a[q]);
}

// out[order[r]] := (rhs[order[r]] - sum_e val[e] out[ci[e]]) (* rdg[r] for
// U) over the rows r < nrows of a sweep order, entries e in [rp[r], rp[r+1]).
// ring: this CTA's staging area (flow_ring_bytes).  rhs may be global or
// shared memory.
template <typename VT, bool UPPER>
__device__ __noinline__ void flow_sweep(int nrows, const int* order, const int* rp, const int* ci, const VT* val,
                                        const VT* rdg, const double* rhs, double* out, char* ring, int* abort,
                                        int& bad) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const size_t sb = flow_slot_bytes(sizeof(VT));
    char* my = ring + (size_t)warp * kFlowSlots * sb;
    const bool rglob = __isGlobal(rhs);
    auto issue = [&](int k) {
        const int idx = warp + k * nw;
        if (idx < nrows) {
            const int b = rp[idx], m = min(rp[idx + 1] - b, kFlowCap);
            char* s = my + (size_t)(k % kFlowSlots) * sb;
            int* sc = (int*)s;
            VT* sv = (VT*)(s + (size_t)kFlowCap * 4);
            double* sx = (double*)(s + (size_t)kFlowCap * (4 + sizeof(VT)));
            for (int t = lane; t < m; t += 32) {
                cp_async_4(sc + t, ci + b + t);
                cp_async_val(sv + t, val + b + t);
            }
            if (lane == 0 && rglob) cp_async_8(sx, rhs + order[idx]);
            if (UPPER && lane == 1) cp_async_val((VT*)(sx + 1), rdg + idx);
        }
        cp_async_commit();
    };
    for (int k = 0; k < kFlowSlots - 1; k++) issue(k);
    for (int k = 0, idx = warp; idx < nrows; k++, idx += nw) {
        issue(k + kFlowSlots - 1);
        cp_async_wait_group<kFlowSlots - 1>();
        __syncwarp();
        const char* s = my + (size_t)(k % kFlowSlots) * sb;
        const int* sc = (const int*)s;
        const VT* sv = (const VT*)(s + (size_t)kFlowCap * 4);
        const double* sx = (const double*)(s + (size_t)kFlowCap * (4 + sizeof(VT)));
        const int i = order[idx], b = rp[idx], e = rp[idx + 1];
        const int m = min(e - b, kFlowCap);
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        for (int t0 = lane; t0 < m; t0 += 128) {
            int jj[4];
            double vv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int t = t0 + 32 * q;
                jj[q] = t < m ? sc[t] : -1;
                vv[q] = t < m ? ValTraits<VT>::load(sv + t) : 0.0;
            }
            flow_acc4(jj, vv, out, abort, bad, a);
        }
        for (int p0 = b + kFlowCap + lane; p0 < e; p0 += 128) {
            int jj[4];
            double vv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int p = p0 + 32 * q;
                jj[q] = p < e ? ci[p] : -1;
                vv[q] = p < e ? ValTraits<VT>::load(val + p) : 0.0;
            }
            flow_acc4(jj, vv, out, abort, bad, a);
        }
        const double acc = warp_sum((a[0] + a[1]) + (a[2] + a[3]));
        if (lane == 0) {
            const double r = (rglob ? sx[0] : rhs[i]) - acc;
            ((volatile double*)out)[i] = UPPER ? r * ValTraits<VT>::load((const VT*)(sx + 1)) : r;
        }
        __syncwarp();   // the slot is staged again by the next issue
    }
    cp_async_wait_all();
    __syncwarp();
}

// y := U^-1 L^-1 rhs with the dataflow sweeps: forward into y, the dense
// trailing block in place, backward into y2 (n doubles of shared memory),
// copied back to y.  ring: the staging area of flow_sweep.
template <typename VT>
__device__ void cta_lu_apply_flow(const SysDev& S, const PatternDev& P, const SweepDesc& sd, const double* rhs,
                                  double* y, double* y2, char* ring, Smem& sm, int& bad) {
    const int n = P.n, k0 = P.k0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) ((long long*)y)[i] = kFlowSentinel;
    if (threadIdx.x == 0) sm.ctl[3] = 0;
    __syncthreads();
    const long long t0 = clock64();
    flow_sweep<VT, false>(n, sd.f_ord, sd.f_rp, P.lci, (const VT*)S.lval, (const VT*)nullptr, rhs, y, ring,
                          &sm.ctl[3], bad);
    __syncthreads();
    const long long t1 = clock64();
    if (P.dtail > 0) {
        tail_forward<VT>(P, (const VT*)S.tail, (const VT*)S.tinv, y, S.stats);
        tail_backward<VT>(P, (const VT*)S.tail, (const VT*)S.tinv, y, S.stats);
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        ((long long*)y2)[i] = i < k0 ? kFlowSentinel : __double_as_longlong(y[i]);
    __syncthreads();
    const long long t2 = clock64();
    flow_sweep<VT, true>(k0, sd.b_ord, sd.b_rp, P.uci, (const VT*)S.uval, (const VT*)S.udiag_bwd, y, y2, ring,
                         &sm.ctl[3], bad);
    __syncthreads();
    for (int i = threadIdx.x; i < k0; i += blockDim.x) y[i] = y2[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        S.stats->cyc_lsolve += t1 - t0;
        S.stats->cyc_tail += t2 - t1;
        S.stats->cyc_usolve += clock64() - t2;
    }
}

// Second solve vector and staging ring of the dataflow sweeps, where the
// level sweeps' stage ring would be.
__device__ __forceinline__ double* flow_y2_base(const SmemPlan& plan, Smem& sm) {
    return (double*)sweep_stage_base(plan, sm);
}
__device__ __forceinline__ char* flow_ring_base(const SmemPlan& plan, Smem& sm) {
    return (char*)sweep_stage_base(plan, sm) + (((size_t)plan.ycap * 8 + 15) & ~(size_t)15);
}

// Dispatch: the dataflow sweeps of shared-memory solve vectors when the
// plan chose them (the second vector where the stage ring would be), else
// level-synchronous sweeps when the launch has a stage ring (sd != nullptr:
// descriptors in shared memory when they fit, else read from the pattern in
// global memory), else the per-row dataflow version over global memory.
template <typename VT>
__device__ __forceinline__ void lu_apply(const SysDev& S, const SmemPlan& plan, const double* rhs,
                                         double* y, Smem& sm, const SweepDesc* sd, int& bad) {
    const PatternDev& P = *S.pat;
    if (plan.flow && sd && P.n <= plan.ycap)
        cta_lu_apply_flow<VT>(S, P, *sd, rhs, y, flow_y2_base(plan, sm), flow_ring_base(plan, sm), sm, bad);
    else if (sd) cta_lu_apply_levels<VT>(S, P, plan, rhs, y, *sd, sweep_stage_base(plan, sm), sm.red);
    else cta_lu_apply<VT>(P, (const VT*)S.lval, (const VT*)S.uval, (const VT*)S.udiag, (const VT*)S.tail,
                          (const VT*)S.tinv, rhs, y, sm, bad, S.stats);
}

// The sweep descriptors of a solve: loaded into shared memory when they fit
// (returns the packed copy), else the pattern's global arrays when the
// launch has a stage ring, else none (dataflow sweeps).  Ends with a CTA
// barrier.
__device__ const SweepDesc* prepare_sweeps(const PatternDev& P, const SmemPlan& plan, Smem& sm, SweepDesc* buf) {
    const SweepDesc* sd = nullptr;
    if (sweep_desc_fits(P, plan)) {
        int* d = sweep_desc_base(plan, sm);
        load_sweep_desc(P, d);
        *buf = SweepDesc(P, d);
        sd = buf;
    } else if (plan.sc_ent > 0 || plan.flow) {
        *buf = SweepDesc(P);
        sd = buf;
    }
    __syncthreads();
    return sd;
}

// out = A x (RESID: out = bt - A x) with A in SELL-C-sigma, C = 32, values AT.
template <typename AT, bool RESID>
__device__ void cta_spmv(const PatternDev& P, const AT* vals, const double* xin,
                         const double* bt, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int s = warp; s < P.nslices; s += nw) {
        const int base = P.sell_ptr[s];
        const int L = (P.sell_ptr[s + 1] - base) >> 5;
        // Four independent partial sums: four loads per lane in flight.
        double acc = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int t = 0;
        for (; t + 3 < L; t += 4) {
            const int e = base + (t << 5) + lane;
            const int c0 = P.sell_col[e], c1 = P.sell_col[e + 32], c2 = P.sell_col[e + 64], c3 = P.sell_col[e + 96];
            acc = fma((double)vals[e], xin[c0], acc);
            a1 = fma((double)vals[e + 32], xin[c1], a1);
            a2 = fma((double)vals[e + 64], xin[c2], a2);
            a3 = fma((double)vals[e + 96], xin[c3], a3);
        }
        for (; t < L; t++) {
            const int e = base + (t << 5) + lane;
            acc = fma((double)vals[e], xin[P.sell_col[e]], acc);
        }
        acc = (acc + a1) + (a2 + a3);
        const int row = P.sell_perm[(s << 5) + lane];
        if (row >= 0) out[row] = RESID ? bt[row] - acc : acc;
    }
}

// ---------------------------------------------------------------------------
// fp16 inner products.  Ruiz equilibration of A (position space, SELL
// order) gives rs, cs with every row and column maximum of |rs_i a_ij cs_j|
// near 1; the scaled values are stored in fp16 only when every nonzero one
// lies in the fp16 normal range [2^-14, 65504], so no value underflows or
// overflows in storage (else the fp32 values are used and ST_FP16_OFF says
// so).  The scaling is the one lusp_sell_create applies (spmv.cu,
// lusp_ruiz_csr), operation for operation: row maxima of |a| rs_i cs_j,
// rs_i /= sqrt(max), then column maxima, cs_j /= sqrt(max), until every
// maximum is within 1e-6 of 1, at most kRuizSweeps sweeps.  The reference
// equilibrates the same way on the host (bench/test_lu_gpu_par.cu:237-260,
// 30 sweeps, early stop 1e-6).
// ---------------------------------------------------------------------------
constexpr int kRuizSweeps = 30;

// colmax: n doubles of global scratch.  Returns whether fp16 storage fits.
__device__ bool ruiz_sell16(const SysDev& S, const PatternDev& P, double* colmax, Smem& sm) {
    const int n = P.n;
    double* rs = S.rs;
    double* cs = S.cs;
    __half* h = (__half*)S.sell16;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        rs[i] = 1.0;
        cs[i] = 1.0;
    }
    __syncthreads();
    const int nq = 32 * P.nslices;
    for (int it = 0; it < kRuizSweeps; it++) {
        double dev = 0.0;
        // Rows: one thread per SELL row (a row's entries are one lane of its slice).
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            const int r = P.sell_perm[q];
            if (r < 0) continue;
            const int base = P.sell_ptr[q >> 5], L = (P.sell_ptr[(q >> 5) + 1] - base) >> 5;
            const double rr = rs[r];
            double m = 0.0;
            for (int t = 0; t < L; t++) {
                const int e = base + (t << 5) + (q & 31);
                if (P.sell_src[e] >= 0) m = fmax(m, fabs(S.sell64[e]) * rr * cs[P.sell_col[e]]);
            }
            if (m > 0.0) {
                rs[r] = rr / sqrt(m);
                dev = fmax(dev, fabs(1.0 - m));
            }
        }
        for (int j = threadIdx.x; j < n; j += blockDim.x) colmax[j] = 0.0;
        __syncthreads();
        // Columns: maxima by atomic max on the bit patterns (non-negative).
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            const int r = P.sell_perm[q];
            if (r < 0) continue;
            const int base = P.sell_ptr[q >> 5], L = (P.sell_ptr[(q >> 5) + 1] - base) >> 5;
            const double rr = rs[r];
            for (int t = 0; t < L; t++) {
                const int e = base + (t << 5) + (q & 31);
                if (P.sell_src[e] < 0) continue;
                const int c = P.sell_col[e];
                const double a = fabs(S.sell64[e]) * rr * cs[c];
                atomicMax((unsigned long long*)(colmax + c), (unsigned long long)__double_as_longlong(a));
            }
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double m = colmax[j];
            if (m > 0.0) {
                cs[j] = cs[j] / sqrt(m);
                dev = fmax(dev, fabs(1.0 - m));
            }
        }
        dev = block_max(dev, sm.red);
        if (dev < 1e-6) break;
    }
    // fp16 values (padding 0) and the range of the scaled nonzeros.
    double mn = INFINITY, mx = 0.0;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int r = P.sell_perm[q];
        const int base = P.sell_ptr[q >> 5], L = (P.sell_ptr[(q >> 5) + 1] - base) >> 5;
        for (int t = 0; t < L; t++) {
            const int e = base + (t << 5) + (q & 31);
            double a = 0.0;
            if (r >= 0 && P.sell_src[e] >= 0) a = S.sell64[e] * rs[r] * cs[P.sell_col[e]];
            h[e] = __double2half(a);
            const double aa = fabs(a);
            if (aa != 0.0) {
                mn = fmin(mn, aa);
                mx = fmax(mx, aa);
            }
        }
    }
    mn = block_min(mn, sm.red);
    mx = block_max(mx, sm.red);
    return mn >= 6.103515625e-05 && mx <= 65504.0;
}

// out = A x with the fp16 values: out_r = (sum_c h_rc (x_c / cs_c)) / rs_r,
// fp64 accumulation; xc: n doubles of scratch.
__device__ void cta_spmv16(const PatternDev& P, const __half* vals, const double* rs, const double* cs,
                           const double* xin, double* xc, double* out) {
    for (int i = threadIdx.x; i < P.n; i += blockDim.x) xc[i] = xin[i] / cs[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int s = warp; s < P.nslices; s += nw) {
        const int base = P.sell_ptr[s];
        const int L = (P.sell_ptr[s + 1] - base) >> 5;
        double acc = 0.0, a1 = 0.0;
        int t = 0;
        for (; t + 1 < L; t += 2) {
            const int e = base + (t << 5) + lane;
            acc = fma((double)__half2float(vals[e]), xc[P.sell_col[e]], acc);
            a1 = fma((double)__half2float(vals[e + 32]), xc[P.sell_col[e + 32]], a1);
        }
        if (t < L) {
            const int e = base + (t << 5) + lane;
            acc = fma((double)__half2float(vals[e]), xc[P.sell_col[e]], acc);
        }
        const int row = P.sell_perm[(s << 5) + lane];
        if (row >= 0) out[row] = (acc + a1) / rs[row];
    }
}

__device__ __forceinline__ double cta_dot(const double* a, const double* b, int n, Smem& sm) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(a[i], b[i], s);
    return block_sum(s, sm.red);
}

// A in SELL order for the solve's products, from the system's input
// values: fp64 (outer residual, direct-solve residual) and, when the inner
// products use it, fp32.  Ends with a CTA barrier.
__device__ void build_sell_values(const SysDev& S, const PatternDev& P, bool f32) {
    const int total = P.sell_total, nt = blockDim.x;
    // Four entries per thread in flight (the value reads are gathers).
    for (int t0 = threadIdx.x; t0 < total; t0 += 4 * nt) {
        int src[4];
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) src[q] = t0 + q * nt < total ? P.sell_src[t0 + q * nt] : -1;
#pragma unroll
        for (int q = 0; q < 4; q++) v[q] = src[q] >= 0 ? S.a_val[src[q]] : 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int t = t0 + q * nt;
            if (t < total) {
                S.sell64[t] = v[q];
                if (f32) S.sell32[t] = (float)v[q];
            }
        }
    }
    __syncthreads();
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
    build_sell_values(S, P, false);
    SweepDesc sdb(P);
    const SweepDesc* desc = prepare_sweeps(P, plan, sm, &sdb);
    const double nb = sqrt(cta_dot(bt, bt, n, sm));
    lu_apply<VT>(S, plan, bt, y, sm, desc, bad);
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

// Arnoldi orthogonalization of w against the first j + 1 basis vectors
// (V_i at V + i n) for j < kFusedDots, every thread on every dot product.
// Both helpers are calls: inlined into the GMRES loop, their addresses stay
// live across the preconditioner application and the level sweeps it calls
// run out of registers (spill loads in every level step).
constexpr int kFusedDots = 3;

// d[i] = V_i . w (i <= j) and, when wsq is given, |w|^2 from one sweep over
// the vectors; all threads receive the sums.
__device__ __noinline__ void cgs_dots(const double* V, int n, int j, const double* w, double* d, double* wsq,
                                      Smem& sm) {
    double s[kFusedDots + 1];
#pragma unroll
    for (int i = 0; i <= kFusedDots; i++) s[i] = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const double we = w[e];
        if (wsq) s[kFusedDots] = fma(we, we, s[kFusedDots]);
#pragma unroll
        for (int i = 0; i < kFusedDots; i++)
            if (i <= j) s[i] = fma(V[(size_t)i * n + e], we, s[i]);
    }
    block_sum2(s[0], s[kFusedDots], sm.red);
    if (j >= 1) block_sum2(s[1], s[2], sm.red);
#pragma unroll
    for (int i = 0; i < kFusedDots; i++) d[i] = i <= j ? s[i] : 0.0;
    if (wsq) *wsq = s[kFusedDots];
}

// w -= sum_{i <= j} d[i] V_i; returns the new |w|^2 (all threads).
__device__ __noinline__ double cgs_update(const double* V, int n, int j, const double* d, double* w, Smem& sm) {
    double nrm = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        double acc = w[e];
#pragma unroll
        for (int i = 0; i < kFusedDots; i++)
            if (i <= j) acc = fma(-d[i], V[(size_t)i * n + e], acc);
        w[e] = acc;
        nrm = fma(acc, acc, nrm);
    }
    return block_sum(nrm, sm.red);
}

// ---------------------------------------------------------------------------
// GMRES-IR: restarted, right-preconditioned GMRES on P A Q with the stored
// factors as preconditioner (VT), inner products A z with AT values; outer
// residual b - A x, Arnoldi (classical Gram-Schmidt: for the first
// kFusedDots basis vectors a second pass only when the first cancels more
// than half of |w|^2, beyond them always two passes), Givens
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
    double* Zb = xprev + n;                      // [m x n] preconditioned basis z_j = M^-1 v_j
    // Shared: y (optional) | H[(m+1) x m] | g, cs, sn, h, h2, yc
    double* ys = (double*)sm.uni;
    double* H = ys + plan.ycap;
    double* g = H + (size_t)(m + 1) * m;
    double* cs = g + (m + 1);
    double* sn = cs + m;
    double* h = sn + m;
    double* yc = h + (m + 1);
    double* y = (n <= plan.ycap) ? ys : yg;
    const VT* udiag = (const VT*)S.udiag;
    const VT* tail = (const VT*)S.tail;
    constexpr bool kHalf = std::is_same<AT, __half>::value;
    const void* ainner = sizeof(AT) == 8 ? (const void*)S.sell64 : (const void*)S.sell32;
    int bad = 0;
    int status = 0;
    int inner_total = 0, outer_done = 0, nres = 0;
    if (threadIdx.x == 0) S.stats->status &= ~kSolveBits;

    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        bt[i] = S.b[P.rowat[i]];
        xt[i] = 0.0;
    }
    build_sell_values(S, P, sizeof(AT) != 8);
    SweepDesc sdb(P);
    const SweepDesc* desc = prepare_sweeps(P, plan, sm, &sdb);
    bool use16 = false;
    if constexpr (kHalf) {
        // V holds nothing yet: its first n doubles serve the column maxima.
        use16 = ruiz_sell16(S, P, V, sm);
        if (!use16 && threadIdx.x == 0) atomicOr(&S.stats->status, (int)ST_FP16_OFF);
    }
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
            lu_apply<VT>(S, plan, vj, y, sm, desc, bad);
            // Keep z_j: the correction is then sum_i y_i z_i, without
            // another preconditioner application (flexible-GMRES layout).
            double* zj = Zb + (size_t)j * n;
            for (int e = threadIdx.x; e < n; e += blockDim.x) zj[e] = y[e];
            const long long tsp = clock64();
            if constexpr (kHalf) {
                // r is free inside the inner loop: it holds x / cs.
                if (use16) cta_spmv16(P, (const __half*)S.sell16, S.rs, S.cs, y, r, w);
                else cta_spmv<float, false>(P, S.sell32, y, nullptr, w);
            } else {
                cta_spmv<AT, false>(P, (const AT*)ainner, y, nullptr, w);
            }
            __syncthreads();
            if (threadIdx.x == 0) S.stats->cyc_spmv += clock64() - tsp;
            double wn0, hn;
            if (j < kFusedDots) {
                // Classical Gram-Schmidt against V_0..V_j, all threads on
                // every dot product: one sweep for the dots and |w|^2, one
                // for the update and the new |w|^2; the second pass only
                // when the first cancelled more than half of |w|^2 (Daniel,
                // Gragg, Kaufman and Stewart's reorthogonalization test).
                double d[kFusedDots];
                double wsq;
                cgs_dots(V, n, j, w, d, &wsq, sm);
                wn0 = sqrt(wsq);
                double hsq = cgs_update(V, n, j, d, w, sm);
                if (hsq < 0.5 * wsq) {
                    double d2[kFusedDots];
                    cgs_dots(V, n, j, w, d2, nullptr, sm);
                    hsq = cgs_update(V, n, j, d2, w, sm);
#pragma unroll
                    for (int i = 0; i < kFusedDots; i++) d[i] += d2[i];
                }
                if (threadIdx.x == 0) {
#pragma unroll
                    for (int i = 0; i < kFusedDots; i++)
                        if (i <= j) H[(size_t)i * m + j] = d[i];
                }
                hn = sqrt(hsq);
            } else {
                wn0 = sqrt(cta_dot(w, w, n, sm));
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
                hn = sqrt(cta_dot(w, w, n, sm));
            }
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
        // The correction sum_i y_i z_i, applied as it is formed.
        double sy = 0.0, sx = 0.0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            double acc = 0.0;
            for (int i = 0; i < jj; i++) acc = fma(yc[i], Zb[(size_t)i * n + e], acc);
            const double xo = xt[e];
            xprev[e] = xo;
            const double xn = xo + acc;
            xt[e] = xn;
            sy = fma(acc, acc, sy);
            sx = fma(xn, xn, sx);
        }
        block_sum2(sy, sx, sm.red);
        const double ny = sqrt(sy);
        const double nx = sqrt(sx);
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
