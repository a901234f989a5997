// Batched refactor-and-solve engine: pattern objects (host analysis + the
// device-resident static layout), batches of systems, the persistent kernel
// and the lusp_* C-ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "luspice_b200.h"
#include "../host/lusp_host.h"
#include "engine_internal.h"
#include "phases.cuh"

namespace lusp {

// ---------------------------------------------------------------------------
// Error reporting
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

const char* last_error_cstr() { return g_last_error.c_str(); }

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return LUSP_ECUDA;
}

// ---------------------------------------------------------------------------
// The persistent kernels: every CTA takes systems from a device work queue
// until it is empty.  The refactorization runs as its own kernel (many warps
// per CTA, few registers each), the dense trailing blocks as a second (few
// warps, many registers), the triangular solves and GMRES-IR as a third.
// queue[0] feeds the refactor kernel, queue[1] the solve kernel, queue[2]
// the dense kernel.
// ---------------------------------------------------------------------------
// dyn (may be null): the number of systems is min(*dyn, nsys), set by an
// earlier kernel of the launch; list (may be null): work item t is system
// list[t] (the escalation ladder's slots).
__device__ __forceinline__ int item_count(int nsys, const int* dyn) {
    return dyn ? min(*(const volatile int*)dyn, nsys) : nsys;
}

// MAXT: resident threads per SM the instance is compiled for (registers
// per thread = 65536 / MAXT); a launch runs one CTA of MAXT threads per SM,
// or several smaller ones.
template <typename VT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
refactor_kernel(const SysDev* __restrict__ sys, int nsys, int* queue, SmemPlan plan, SolveParams prm,
                const int* dyn, const int* list, SpreadArgs sp) {
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_task;
    const int ns = item_count(nsys, dyn);
    (void)sp;
    // A thread-block cluster (or a lone CTA) takes one system at a time:
    // rank 0 draws it, every CTA reads it through distributed shared memory
    // between two cluster barriers (so rank 0 outlives the read).
    namespace cgr = cooperative_groups;
    cgr::cluster_group cl = cgr::this_cluster();
    const volatile int* task0 = cl.map_shared_rank(&s_task, 0);
    while (true) {
        cl.sync();
        if (cl.block_rank() == 0 && threadIdx.x == 0) s_task = atomicAdd(queue, 1);
        cl.sync();
        const int t = *task0;
        cl.sync();
        if (t >= ns) break;
        const SysDev S = sys[list ? list[t] : t];
        refactor_phase<VT>(S, plan, smem, prm);
    }
}

// Spread mode (its own kernel, so the cluster kernel's register allocation
// is its own): CTAs [t * group, (t + 1) * group) share system t, one CTA
// per SM.
template <typename VT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
refactor_spread_kernel(const SysDev* __restrict__ sys, int nsys, int* queue, SmemPlan plan, SolveParams prm,
                       const int* dyn, const int* list, SpreadArgs sp) {
    extern __shared__ __align__(16) char smem[];
    (void)queue;
    const int ns = item_count(nsys, dyn);
    const int t = (int)blockIdx.x / sp.group;
    if (t >= ns) return;
    const SysDev S = sys[list ? list[t] : t];
    refactor_phase<VT, true>(S, plan, smem, prm, sp.sync + (size_t)t * sp.stride, (int)blockIdx.x % sp.group,
                             sp.group);
}

template <typename VT>
__global__ void __launch_bounds__(512, 1)
dense_kernel(const SysDev* __restrict__ sys, int nsys, int* queue, SmemPlan plan, SolveParams prm,
             const int* dyn, const int* list) {
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_task;
    const int ns = item_count(nsys, dyn);
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_task = atomicAdd(queue + 2, 1);
        __syncthreads();
        const int t = s_task;
        if (t >= ns) break;
        const SysDev S = sys[list ? list[t] : t];
        dense_phase<VT>(S, plan, smem, prm);
    }
}

// The dense trailing blocks with a 2-CTA thread-block cluster per system
// (the two CTAs split the trailing updates): rank 0 draws a system, both
// read it through distributed shared memory between two cluster barriers.
template <typename VT>
__global__ void __launch_bounds__(512, 1)
dense_cluster_kernel(const SysDev* __restrict__ sys, int nsys, int* queue, SmemPlan plan, SolveParams prm,
                     const int* dyn, const int* list) {
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_task;
    const int ns = item_count(nsys, dyn);
    namespace cgr = cooperative_groups;
    cgr::cluster_group cl = cgr::this_cluster();
    const volatile int* task0 = cl.map_shared_rank(&s_task, 0);
    while (true) {
        cl.sync();
        if (cl.block_rank() == 0 && threadIdx.x == 0) s_task = atomicAdd(queue + 2, 1);
        cl.sync();
        const int t = *task0;
        cl.sync();
        if (t >= ns) break;
        const SysDev S = sys[list ? list[t] : t];
        dense_phase<VT, true>(S, plan, smem, prm);
    }
}

// After the solve of one system (thread 0, past the CTA barrier that makes
// the solve's statistics visible): record the rung that produced the
// result and hand a failed system to the next rung of the ladder.
__device__ void ladder_handoff(const SysDev& S, int item, const EscDev& esc, int rung) {
    SysStats* st = S.stats;
    st->rung = rung;
    if (rung > 0) st->status |= ST_ESCALATED | (rung == 2 ? ST_SHIFTED : 0);
    if (esc.cap <= 0 || rung == 2) return;
    const int nres = st->nres;
    const double last = nres > 0 ? st->res[nres - 1] : INFINITY;
    const int bits = rung == 0 ? esc.fail_bits : (esc.fail_bits & ~ST_PIVOT_WEAK);
    const bool failed = (st->status & bits) != 0 || !(last <= esc.rtol);
    if (!failed) return;
    if (rung == 0) {
        // Storage first (a refused reservation takes no slot), then a slot.
        const SysSizes z = sizes_of(*S.pat);
        const size_t need = sys_private_bytes(z, sizeof(double), esc.m);
        const unsigned long long off = atomicAdd((unsigned long long*)(esc.ctl + 2), (unsigned long long)need);
        if (off + need > esc.pool) {
            st->status |= ST_LADDER_FULL;
            return;
        }
        const int slot = atomicAdd(&esc.ctl[0], 1);
        if (slot >= esc.cap) {
            st->status |= ST_LADDER_FULL;
            return;
        }
        SysDev D = S;
        sys_carve(D, esc.base + off, z, sizeof(double), esc.m);
        D.scratch = esc.scratch;
        esc.slots[slot] = D;
    } else if (esc.hard) {
        esc.hard[atomicAdd(&esc.ctl[1], 1)] = item;
    }
}

template <typename VT, typename AT>
__global__ void __launch_bounds__(512)
solve_kernel(const SysDev* __restrict__ sys, int nsys, int* queue, SmemPlan plan,
             SolveParams prm, int direct, const int* dyn, const int* list, EscDev esc, int rung) {
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_task;
    const int ns = item_count(nsys, dyn);
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_task = atomicAdd(queue + 1, 1);
        __syncthreads();
        const int t = s_task;
        if (t >= ns) break;
        const int item = list ? list[t] : t;
        const SysDev S = sys[item];
        const long long ts = clock64();
        if (threadIdx.x == 0) {
            S.stats->cyc_lsolve = 0;
            S.stats->cyc_tail = 0;
            S.stats->cyc_usolve = 0;
            S.stats->cyc_spmv = 0;
            S.stats->cyc_tdiag = 0;
            S.stats->cyc_tgemv = 0;
        }
        __syncthreads();
        if (direct) direct_phase<VT>(S, plan, smem);
        else gmres_phase<VT, AT>(S, plan, smem, prm);
        __syncthreads();
        if (threadIdx.x == 0) {
            S.stats->cyc_solve = clock64() - ts;
            ladder_handoff(S, item, esc, rung);
        }
    }
}

// The merged slot array of one system, completed for callers that read the
// factor in that layout: the engine's refactor stores the strict-L part
// there (the later columns' gathers read it) and the U part, the diagonal
// and the dense trailing block only in the arrays the solves read.  A CTA
// per column (grid-stride).
template <typename VT>
__global__ void merge_factor_kernel(SysDev S) {
    const PatternDev& P = *S.pat;
    const int n = P.n, k0 = P.k0, ld = P.tail_ld;
    VT* lu = (VT*)S.lu;
    const VT* uval = (const VT*)S.uval;
    const VT* udiag = (const VT*)S.udiag;
    const VT* T = (const VT*)S.tail;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int c0 = P.cp[k], c1 = P.cp[k + 1], d = P.dg[k];
        for (int p = c0 + (int)threadIdx.x; p < c1; p += blockDim.x) {
            const int r = P.ri[p];
            if (k >= k0 && r >= k0) lu[p] = T[(size_t)(k - k0) * ld + (r - k0)];
            else if (p < d) lu[p] = uval[P.slot_dst[p]];
            else if (p == d) lu[p] = udiag[k];
        }
    }
}

int batch_merge_factor(BatchObj* B, int sys, cudaStream_t st) {
    const SysDev& S = B->h_sys[sys];
    const int n = B->pats[sys]->S.n;
    const int grid = std::max(1, std::min(n, 4 * sm_count()));
    if (B->prec == LUSP_FP64) merge_factor_kernel<double><<<grid, 128, 0, st>>>(S);
    else merge_factor_kernel<float><<<grid, 128, 0, st>>>(S);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LUSP_OK : cuda_fail(e, "merge factor launch");
}

// ---------------------------------------------------------------------------
// Patterns
// ---------------------------------------------------------------------------
// Synchronous copy from pageable memory: returns when the data is on the
// device, without waiting for kernels on other (non-blocking) streams.
static int upload_ints(const std::vector<int>& v, int* dst, cudaStream_t) {
    if (v.empty()) return 0;
    cudaError_t e = cudaMemcpy(dst, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? 0 : cuda_fail(e, "pattern upload");
}

int pattern_build(int n, const int* Ap, const int* Ai, const double* Ax, const int* q_in,
                  PatternObj** out, int dense_tail) {
    *out = nullptr;
    if (n <= 0 || !Ap || !Ai || !Ax) { set_error("pattern_create: bad arguments"); return LUSP_EARG; }
    const int nnz = Ap[n];
    if (Ap[0] != 0 || nnz < 0) { set_error("pattern_create: bad column pointers"); return LUSP_EARG; }
    for (int c = 0; c < n; c++)
        if (Ap[c + 1] < Ap[c]) { set_error("pattern_create: column pointers decrease at %d", c); return LUSP_EARG; }
    for (int p = 0; p < nnz; p++)
        if (Ai[p] < 0 || Ai[p] >= n) { set_error("pattern_create: row index out of range at %d", p); return LUSP_EARG; }
    if (q_in) {
        std::vector<char> seen(n, 0);
        for (int k = 0; k < n; k++) {
            if (q_in[k] < 0 || q_in[k] >= n || seen[q_in[k]]) { set_error("pattern_create: q is not a permutation"); return LUSP_EARG; }
            seen[q_in[k]] = 1;
        }
    }
    // Column-sorted, duplicate-summed copy for the analysis.
    std::vector<int> Bp(n + 1, 0), Bi;
    std::vector<double> Bx;
    Bi.reserve(nnz);
    Bx.reserve(nnz);
    {
        std::vector<std::pair<int, double>> col;
        for (int c = 0; c < n; c++) {
            col.clear();
            for (int p = Ap[c]; p < Ap[c + 1]; p++) col.emplace_back(Ai[p], Ax[p]);
            std::stable_sort(col.begin(), col.end(),
                             [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
            for (size_t t = 0; t < col.size(); t++) {
                if (t > 0 && col[t].first == col[t - 1].first) Bx.back() += col[t].second;
                else { Bi.push_back(col[t].first); Bx.push_back(col[t].second); }
            }
            Bp[c + 1] = (int)Bi.size();
        }
    }
    std::vector<int> q(n);
    if (q_in) {
        std::copy(q_in, q_in + n, q.begin());
    } else if (colamd_order(n, n, Bp.data(), Bi.data(), 0.0, 0.0, q.data()) != 0) {
        set_error("pattern_create: COLAMD failed");
        return LUSP_EARG;
    }
    PivotFactor F;
    const int sc = pivot_factor(n, Bp.data(), Bi.data(), Bx.data(), q.data(), 1.0, F);
    if (sc >= 0) {
        set_error("pattern_create: singular at column %d", sc);
        return LUSP_ESINGULAR;
    }
    PatternObj* P = new PatternObj();
    build_static_pattern(n, Ap, Ai, q.data(), F, 256, P->S, dense_tail);
    const StaticPattern& S = P->S;
    // Column records of the refactorization (see PatternDev::crec).
    std::vector<int> crec((size_t)12 * n, 0);
    for (int idx = 0; idx < n; idx++) {
        const int k = S.col_order[idx];
        int* r = crec.data() + (size_t)12 * idx;
        const int c0 = S.cp[k], d = S.dg[k] - c0;
        int dsp = d;
        if (k >= S.k0) {
            dsp = 0;
            for (int t = 0; t < d; t++) dsp += S.ri[c0 + t] < S.k0;
        }
        const long long rp = S.rel_ptr.empty() ? 0 : S.rel_ptr[k];
        r[0] = k;
        r[1] = c0;
        r[2] = S.cp[k + 1] - c0;
        r[3] = d;
        r[4] = S.a_ptr[k];
        r[5] = S.a_ptr[k + 1];
        r[6] = dsp;
        r[7] = S.bwd_pos[k];
        r[8] = (int)(unsigned)(rp & 0xffffffffll);
        r[9] = (int)(unsigned)((unsigned long long)rp >> 32);
        r[10] = S.a_diag[k];
    }
    // Bit pattern of the dense trailing block (see PatternDev::tail_mask).
    std::vector<int> tail_mask;
    if (S.dtail > 0) {
        const int ldw = tail_ld(S) / 32;
        tail_mask.assign((size_t)S.dtail * ldw, 0);
        for (int k = S.k0; k < n; k++)
            for (int p = S.cp[k]; p < S.cp[k + 1]; p++) {
                const int r = S.ri[p];
                if (r < S.k0) continue;
                const int c = k - S.k0;
                tail_mask[(size_t)(r - S.k0) * ldw + c / 32] |= (int)(1u << (c & 31));
            }
    }

    // One device block for every int array of the layout.
    const std::vector<int>* arrays[] = {&S.cp, &S.ri, &S.dg, &S.col_order, &S.a_ptr, &S.a_src, &S.a_dst,
                                        &S.lrp, &S.lci, &S.urp, &S.uci, &S.slot_dst, &S.fwd_order,
                                        &S.bwd_order, &S.sell_ptr, &S.sell_col, &S.sell_src,
                                        &S.sell_perm, &S.rowat, &S.q, &S.fwd_lev, &S.bwd_lev, &S.bwd_pos,
                                        &S.fwd_ldesc, &S.bwd_ldesc, &S.dep_bc, &S.a_diag, &tail_mask, &crec};
    const int narr = (int)(sizeof(arrays) / sizeof(arrays[0]));
    std::vector<size_t> off(narr + 1, 0);
    // Each array gets at least 8 ints of slack: the sweeps copy index runs
    // in aligned 16-byte pieces that may end up to 3 entries past a run.
    for (int a = 0; a < narr; a++) off[a + 1] = off[a] + ((arrays[a]->size() + 8 + 31) & ~(size_t)31);
    int* blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, std::max<size_t>(off[narr], 32) * sizeof(int));
    if (e != cudaSuccess) { delete P; return cuda_fail(e, "pattern device alloc"); }
    P->d_block = blk;
    P->bytes = off[narr] * sizeof(int) + sizeof(PatternDev);
    for (int a = 0; a < narr; a++) {
        int rc = upload_ints(*arrays[a], blk + off[a], 0);
        if (rc) { pattern_free(P); return rc; }
    }
    PatternDev& D = P->desc;
    D.n = n;
    D.nnz_a = S.nnz_a;
    D.cap = (int)S.cap;
    D.max_col = S.max_col;
    D.nslices = S.nslices;
    D.sell_total = S.sell_ptr.empty() ? 0 : S.sell_ptr.back();
    D.nnz_l = (int)S.lci.size();
    D.nnz_u = (int)S.uci.size();
    int idx = 0;
    D.cp = blk + off[idx++];
    D.ri = blk + off[idx++];
    D.dg = blk + off[idx++];
    D.col_order = blk + off[idx++];
    D.a_ptr = blk + off[idx++];
    D.a_src = blk + off[idx++];
    D.a_dst = blk + off[idx++];
    D.lrp = blk + off[idx++];
    D.lci = blk + off[idx++];
    D.urp = blk + off[idx++];
    D.uci = blk + off[idx++];
    D.slot_dst = blk + off[idx++];
    D.fwd_order = blk + off[idx++];
    D.bwd_order = blk + off[idx++];
    D.sell_ptr = blk + off[idx++];
    D.sell_col = blk + off[idx++];
    D.sell_src = blk + off[idx++];
    D.sell_perm = blk + off[idx++];
    D.rowat = blk + off[idx++];
    D.q = blk + off[idx++];
    D.fwd_lev = blk + off[idx++];
    D.bwd_lev = blk + off[idx++];
    D.bwd_pos = blk + off[idx++];
    D.fwd_ldesc = blk + off[idx++];
    D.bwd_ldesc = blk + off[idx++];
    D.dep_bc = (const int2*)(blk + off[idx++]);
    D.a_diag = blk + off[idx++];
    D.tail_mask = S.dtail > 0 ? (const unsigned*)(blk + off[idx]) : nullptr;
    idx++;
    D.crec = (const int4*)(blk + off[idx++]);
    D.lev_max_ent = S.lev_max_ent;
    D.lev_max_rows = S.lev_max_rows;
    D.nfwd_levels = S.nfwd_steps;   // the device walks the sweep steps
    D.nbwd_levels = S.nbwd_steps;
    D.k0 = S.k0;
    D.dtail = S.dtail;
    D.tail_ld = tail_ld(S);
    // Relative update slots: rel_ptr (n+1 int64) then rel (16 bit, padded by
    // 16 entries so aligned 16-byte copies never run past the end).
    D.rel = nullptr;
    D.rel_ptr = nullptr;
    if (!S.rel_ptr.empty()) {
        const size_t pbytes = ((S.rel_ptr.size() * sizeof(long long)) + 255) & ~(size_t)255;
        const size_t rbytes = (S.rel.size() + 16) * sizeof(uint16_t);
        e = cudaMalloc(&P->d_rel, pbytes + rbytes);
        if (e != cudaSuccess) { pattern_free(P); return cuda_fail(e, "pattern rel alloc"); }
        char* rb = (char*)P->d_rel;
        e = cudaMemcpy(rb, S.rel_ptr.data(), S.rel_ptr.size() * sizeof(long long), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !S.rel.empty())
            e = cudaMemcpy(rb + pbytes, S.rel.data(), S.rel.size() * sizeof(uint16_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(rb + pbytes + S.rel.size() * sizeof(uint16_t), 0, 16 * sizeof(uint16_t));
        if (e != cudaSuccess) { pattern_free(P); return cuda_fail(e, "pattern rel upload"); }
        D.rel_ptr = (const long long*)rb;
        D.rel = (const unsigned short*)(rb + pbytes);
        P->bytes += pbytes + rbytes;
    }
    e = cudaMalloc(&P->d_desc, sizeof(PatternDev));
    if (e != cudaSuccess) { pattern_free(P); return cuda_fail(e, "pattern descriptor alloc"); }
    e = cudaMemcpy(P->d_desc, &D, sizeof(PatternDev), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { pattern_free(P); return cuda_fail(e, "pattern descriptor upload"); }
    *out = P;
    return LUSP_OK;
}

void pattern_free(PatternObj* P) {
    if (!P) return;
    if (P->d_block) cudaFree(P->d_block);
    if (P->d_rel) cudaFree(P->d_rel);
    if (P->d_desc) cudaFree(P->d_desc);
    delete P;
}

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------
int sm_count() {
    static int cached = 0;
    if (!cached) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) cached = 148;
    }
    return cached;
}

static size_t smem_fixed(int nwords) { return 64 + (((size_t)nwords * 4 + 15) & ~(size_t)15) + 40 * sizeof(double); }

// Dynamic shared memory of one solve CTA when ctas_per_sm share an SM.
static size_t solve_smem_budget(int ctas_per_sm) {
    size_t budget = 228 * 1024 / std::max(1, ctas_per_sm);
    budget = budget > 1024 ? budget - 1024 : budget;
    return std::min<size_t>(budget, 227 * 1024);
}

void make_plan(const std::vector<PatternObj*>& pats, int block, int ctas_per_sm, int m, int vsize,
               SmemPlan& plan) {
    int nmax = 1, levmax = 1, entmax = 4, rowmax = 4;
    for (auto* p : pats) {
        nmax = std::max(nmax, p->S.n);
        levmax = std::max(levmax, p->S.nfwd_steps + p->S.nbwd_steps);
        entmax = std::max(entmax, p->S.lev_max_ent);
        rowmax = std::max(rowmax, p->S.lev_max_rows);
    }
    (void)block;
    const size_t budget = solve_smem_budget(ctas_per_sm);
    plan.nwords = (nmax + 31) / 32;
    plan.m = m;
    plan.wcap = 0;
    plan.scap = 0;
    const size_t fixed = smem_fixed(plan.nwords);
    const size_t hbytes = ((size_t)(m + 1) * m + 6 * (size_t)(m + 1)) * sizeof(double);
    size_t avail = budget > fixed + hbytes ? budget - fixed - hbytes : 0;
    // Solve vector in shared memory when it fits, and the level-sweep
    // descriptors (row order, row pointers, level bounds of both sweeps)
    // when they fit beside it.
    plan.ycap = ((size_t)nmax * 8 <= avail) ? nmax : 0;
    const size_t dneed = 4 * (size_t)nmax + (size_t)levmax + 8 + 5 * (size_t)levmax + 16;
    plan.dcap = (plan.ycap && (size_t)nmax * 8 + dneed * 4 <= avail) ? (int)dneed : 0;
    // Stage ring of the level sweeps: the widest level, or as many entries
    // as fit (at least 256; wider levels then read global memory).  Also
    // when the solve vector or the descriptors stay in global memory (large
    // systems): the sweeps then read the pattern's descriptors from there.
    plan.sc_ent = 0;
    plan.sc_rows = 0;
    {
        const size_t used = sweep_desc_offset(plan.ycap, m) - hbytes + (((size_t)plan.dcap + 3) & ~(size_t)3) * 4;
        const size_t left = avail > used ? avail - used : 0;
        int ce = (entmax + 3) & ~3, cr = (rowmax + 3) & ~3;
        while (ce > 256 && kStages * stage_bytes(ce, cr, vsize) > left) ce = (ce / 2 + 3) & ~3;
        while (cr > 64 && kStages * stage_bytes(ce, cr, vsize) > left) cr = (cr / 2 + 3) & ~3;
        if (kStages * stage_bytes(ce, cr, vsize) <= left) {
            plan.sc_ent = ce;
            plan.sc_rows = cr;
        }
    }
    plan.bytes = fixed + sweep_desc_offset(plan.ycap, m) + (((size_t)plan.dcap + 3) & ~(size_t)3) * 4 +
                 (plan.sc_ent ? kStages * stage_bytes(plan.sc_ent, plan.sc_rows, vsize) : 0);
}

void resolve_solve_shape(lusp_batch_opts& o, int nsys) {
    const bool few = nsys <= sm_count();
    if (o.block_threads <= 0) o.block_threads = few ? 512 : 256;
    if (o.ctas_per_sm <= 0) o.ctas_per_sm = few ? 1 : 2;
}

// One 768-thread CTA per SM (80 registers a thread, no spills in the
// column loop) while every system has an SM or more; two 512-thread CTAs
// per SM for wider batches (measured on B200: 768 is ~4% faster than 1024
// threads on one SM, 512 x 2 ~24% faster than 256 x 4).
int refactor_block(const lusp_batch_opts& o, int nsys) {
    if (o.refactor_threads > 0) return o.refactor_threads;
    return nsys <= sm_count() ? 768 : 512;
}

void make_refactor_plan(const std::vector<PatternObj*>& pats, int threads, int vsize, SmemPlan& plan,
                        int ctas_per_sm) {
    int nmax = 1, colmax = 2;
    for (auto* p : pats) {
        nmax = std::max(nmax, p->S.n);
        colmax = std::max(colmax, p->S.max_col);
    }
    colmax = (colmax + 1) & ~1;
    // Target 32 resident warps per SM: one 1024-thread CTA, or several
    // smaller ones (or the given number of CTAs per SM).
    const int ctas = ctas_per_sm > 0 ? ctas_per_sm : std::max(1, 1024 / threads);
    size_t budget = std::min<size_t>(227 * 1024, 228 * 1024 / ctas - 1024);
    plan.nwords = (nmax + 31) / 32;
    plan.m = 0;
    plan.ycap = 0;
    plan.dcap = 0;
    const size_t fixed = smem_fixed(plan.nwords);
    const int nw = threads / 32;
    const size_t per_warp = budget > fixed ? (budget - fixed) / nw : 0;
    // Per warp: work vector (wcap fp64), stage of scap values and scap + 16
    // relative slots.  Prefer the whole longest column in shared memory,
    // then the largest stage (512 down to 64 entries).
    auto need = [&](int wcap, int scap) {
        return (size_t)wcap * 8 + (size_t)scap * vsize + ((size_t)scap + 16) * 2;
    };
    int scap = 512;
    while (scap > 64 && need(colmax, scap) > per_warp) scap /= 2;
    int wcap = colmax;
    if (need(wcap, scap) > per_warp) {
        const size_t rest = per_warp > need(0, scap) ? per_warp - need(0, scap) : 0;
        wcap = (int)std::min<size_t>((size_t)colmax, rest / 8) & ~1;
    }
    plan.wcap = wcap;
    plan.scap = scap;
    plan.bytes = fixed + (size_t)nw * need(wcap, scap);
}

void make_dense_plan(const std::vector<PatternObj*>& pats, int threads, SmemPlan& plan) {
    int dmax = 0;
    for (auto* p : pats) dmax = std::max(dmax, p->S.dtail);
    plan = SmemPlan{};
    plan.nwords = 1;
    const size_t fixed = smem_fixed(plan.nwords);
    const size_t budget = 227 * 1024;
    plan.bytes = fixed;
    if (dmax == 0) return;
    // Panel [D][nb + 1] (padded rows) + U tile [nb][128] + per-warp column
    // maxima [nb][32] + 4 cycle counters: the widest panel (32, 16, 8) that
    // fits.
    auto dneed = [&](int nb) { return fixed + 8 * ((size_t)dmax * (nb + 1) + (size_t)nb * 128 + (size_t)nb * 32 + 4); };
    int nb = 32;
    while (nb > 8 && dneed(nb) > budget) nb /= 2;
    plan.tnb = nb;
    plan.bytes = dneed(nb);
    // The transpose reuses the area: a padded 32 x 33 fp64 tile per warp.
    const size_t tile_b = 32 * 33 * sizeof(double);
    int ttw = (int)std::min<size_t>({(size_t)threads / 32, 16, (budget - fixed) / tile_b});
    ttw = std::max(1, ttw);
    plan.ttw = ttw;
    plan.bytes = std::max(plan.bytes, fixed + ttw * tile_b);
}

// Raise the dynamic shared-memory limit of one kernel (once per size; not a
// stream operation, so it stays out of captured graphs after the first
// call) and optionally report its occupancy.
template <typename K>
static int prepare_kernel(K kern, size_t smem, int block, int* occ, size_t* granted, std::mutex& mu) {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > *granted) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "kernel smem attribute");
        *granted = smem;
    }
    if (occ) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, block, smem);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    }
    return LUSP_OK;
}

template <typename VT, typename AT>
static int kernel_prepare(size_t smem, int block, int* occ) {
    static std::mutex mu;
    static size_t granted = 0;
    return prepare_kernel(solve_kernel<VT, AT>, smem, block, occ, &granted, mu);
}

using RefactorFn = void (*)(const SysDev*, int, int*, SmemPlan, SolveParams, const int*, const int*, SpreadArgs);

// The refactor instance for a CTA of block threads: one CTA per SM above
// 512 threads (the instance with the most registers that still fits the
// block), else the 1024-thread instance, whose CTAs pack several per SM.
template <typename VT>
static RefactorFn refactor_fn(int block, bool spread = false) {
    if (spread) return block <= 512 ? refactor_spread_kernel<VT, 1024> : refactor_spread_kernel<VT, 768>;
    if (block <= 512) return refactor_kernel<VT, 1024>;
    if (block <= 640) return refactor_kernel<VT, 640>;
    if (block <= 768) return refactor_kernel<VT, 768>;
    return refactor_kernel<VT, 1024>;
}

template <typename VT>
static int refactor_prepare(size_t smem, int block, int* occ, bool spread = false) {
    static std::mutex mu;
    static size_t granted[5] = {0, 0, 0, 0, 0};   // per instance: 1024, 640, 768, spread 1024, spread 768
    const int slot = spread ? (block <= 512 ? 3 : 4) : block <= 512 || block > 768 ? 0 : block <= 640 ? 1 : 2;
    return prepare_kernel(refactor_fn<VT>(block, spread), smem, block, occ, &granted[slot], mu);
}

// Clusters of csize refactor CTAs that can be resident at once.
template <typename VT>
static int refactor_cluster_count(size_t smem, int block, int csize, int* nclusters) {
    int rc = refactor_prepare<VT>(smem, block, nullptr);
    if (rc != LUSP_OK) return rc;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)csize * sm_count());
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaOccupancyMaxActiveClusters(nclusters, refactor_fn<VT>(block), &cfg);
    if (e != cudaSuccess) return cuda_fail(e, "cluster occupancy query");
    return LUSP_OK;
}

template <typename VT>
static int dense_prepare(size_t smem, int block, int* occ, bool cluster = false) {
    static std::mutex mu;
    static size_t granted[2] = {0, 0};
    if (cluster) return prepare_kernel(dense_cluster_kernel<VT>, smem, block, occ, &granted[1], mu);
    return prepare_kernel(dense_kernel<VT>, smem, block, occ, &granted[0], mu);
}

// 2-CTA clusters of the dense-block kernel that can be resident at once.
template <typename VT>
static int dense_cluster_count(size_t smem, int block, int* nclusters) {
    int rc = dense_prepare<VT>(smem, block, nullptr, true);
    if (rc != LUSP_OK) return rc;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2u * sm_count());
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaOccupancyMaxActiveClusters(nclusters, dense_cluster_kernel<VT>, &cfg);
    if (e != cudaSuccess) return cuda_fail(e, "dense cluster occupancy query");
    return LUSP_OK;
}

// Loads every kernel of the engine into the current context (CUDA loads a
// module's functions lazily, at their first use; a long-lived caller such as
// the serving loop pays that once at creation instead of inside a request).
int preload_kernels() {
    const void* fns[] = {
        (const void*)refactor_fn<float>(512), (const void*)refactor_fn<float>(640), (const void*)refactor_fn<float>(768),
        (const void*)refactor_fn<double>(512), (const void*)refactor_fn<double>(640),
        (const void*)refactor_fn<double>(768), (const void*)refactor_fn<float>(768, true),
        (const void*)refactor_fn<float>(512, true), (const void*)refactor_fn<double>(768, true),
        (const void*)refactor_fn<double>(512, true), (const void*)dense_kernel<float>, (const void*)dense_kernel<double>,
        (const void*)dense_cluster_kernel<float>, (const void*)dense_cluster_kernel<double>,
        (const void*)solve_kernel<float, float>, (const void*)solve_kernel<float, double>,
        (const void*)solve_kernel<float, __half>, (const void*)solve_kernel<double, double>};
    for (const void* f : fns) {
        cudaFuncAttributes at;
        cudaError_t e = cudaFuncGetAttributes(&at, f);
        if (e != cudaSuccess) return cuda_fail(e, "kernel load");
    }
    return LUSP_OK;
}

int refactor_occupancy(int prec, size_t smem, int block, int* occ, bool spread) {
    if (prec == LUSP_FP64) return refactor_prepare<double>(smem, block, occ, spread);
    return refactor_prepare<float>(smem, block, occ, spread);
}

int kernel_occupancy(int prec, int inner, size_t smem, int block, int* occ) {
    if (prec == LUSP_FP64) return kernel_prepare<double, double>(smem, block, occ);
    if (inner == 1) return kernel_prepare<float, double>(smem, block, occ);
    if (inner == 2) return kernel_prepare<float, __half>(smem, block, occ);
    return kernel_prepare<float, float>(smem, block, occ);
}

// Launch shapes of the three kernels of one rung.
struct RungShape {
    SmemPlan rplan, dplan, plan;
    int rblock, rgrid, rcluster, dblock, dgrid, block, grid;
    SpreadArgs rspread;
    int dcluster;
};

static RungShape main_shape(const LaunchArgs& a) {
    return RungShape{a.rplan, a.dplan, a.plan, a.rblock, a.rgrid, a.rcluster, a.dblock, a.dgrid, a.block, a.grid,
                     a.rspread, a.dcluster};
}

static RungShape ladder_shape(const LaunchArgs& a) {
    return RungShape{a.xrplan, a.xdplan, a.xplan, a.xrblock, a.xrgrid, a.xrcluster, a.xdblock, a.xdgrid,
                     a.xblock, a.xgrid, a.xrspread, 1};
}

// Refactor, dense-block and solve kernels of one rung over sys[0, nsys) (or
// the dyn / list items) with the work counters q[0..2].
template <typename VT, typename AT>
// kev (may be null): four events recorded on st around the kernels: before
// the refactor kernel, between it and the dense-block kernel, between that
// and the solve kernel, after the solve kernel.
static int launch_rung(const SysDev* sys, int nsys, int* q, const int* dyn, const int* list, int what,
                       const RungShape& r, const SolveParams& prm, int direct, const EscDev& esc, int rung,
                       cudaStream_t st, cudaEvent_t* kev = nullptr) {
    cudaError_t e;
    if (kev && cudaEventRecord(kev[0], st) != cudaSuccess) return cuda_fail(cudaGetLastError(), "timing event");
    if (what & LUSP_RUN_REFACTOR) {
        const bool spread = r.rspread.group > 0;
        int rc = refactor_prepare<VT>(r.rplan.bytes, r.rblock, nullptr, spread);
        if (rc != LUSP_OK) return rc;
        if (r.rspread.group > 0) {
            // The systems' sync areas start at zero (claim counters, status
            // words, accumulators, ready bits).
            e = cudaMemsetAsync(r.rspread.sync, 0, (size_t)nsys * r.rspread.stride * sizeof(unsigned), st);
            if (e != cudaSuccess) return cuda_fail(e, "refactor sync reset");
        }
        if (r.rcluster > 1) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)r.rgrid);
            cfg.blockDim = dim3((unsigned)r.rblock);
            cfg.dynamicSmemBytes = r.rplan.bytes;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)r.rcluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            e = cudaLaunchKernelEx(&cfg, refactor_fn<VT>(r.rblock), sys, nsys, q, r.rplan, prm, dyn, list,
                                   r.rspread);
        } else {
            refactor_fn<VT>(r.rblock, spread)<<<r.rgrid, r.rblock, r.rplan.bytes, st>>>(sys, nsys, q, r.rplan, prm,
                                                                                     dyn, list, r.rspread);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return cuda_fail(e, "refactor kernel launch");
        if (kev && cudaEventRecord(kev[1], st) != cudaSuccess) return cuda_fail(cudaGetLastError(), "timing event");
        if (r.dgrid > 0) {
            rc = dense_prepare<VT>(r.dplan.bytes, r.dblock, nullptr, r.dcluster > 1);
            if (rc != LUSP_OK) return rc;
            if (r.dcluster > 1) {
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)r.dgrid);
                cfg.blockDim = dim3((unsigned)r.dblock);
                cfg.dynamicSmemBytes = r.dplan.bytes;
                cfg.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = 2;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                e = cudaLaunchKernelEx(&cfg, dense_cluster_kernel<VT>, sys, nsys, q, r.dplan, prm, dyn, list);
            } else {
                dense_kernel<VT><<<r.dgrid, r.dblock, r.dplan.bytes, st>>>(sys, nsys, q, r.dplan, prm, dyn, list);
                e = cudaGetLastError();
            }
            if (e != cudaSuccess) return cuda_fail(e, "dense kernel launch");
        }
    } else if (kev && cudaEventRecord(kev[1], st) != cudaSuccess) {
        return cuda_fail(cudaGetLastError(), "timing event");
    }
    if (kev && cudaEventRecord(kev[2], st) != cudaSuccess) return cuda_fail(cudaGetLastError(), "timing event");
    if (what & LUSP_RUN_SOLVE) {
        int rc = kernel_prepare<VT, AT>(r.plan.bytes, r.block, nullptr);
        if (rc != LUSP_OK) return rc;
        solve_kernel<VT, AT><<<r.grid, r.block, r.plan.bytes, st>>>(sys, nsys, q, r.plan, prm, direct, dyn, list,
                                                                  esc, rung);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "solve kernel launch");
    }
    if (kev && cudaEventRecord(kev[3], st) != cudaSuccess) return cuda_fail(cudaGetLastError(), "timing event");
    return LUSP_OK;
}

template <typename VT, typename AT>
static int launch_typed(const LaunchArgs& a, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(a.d_queue, 0, kQueueWords * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "queue reset");
    const int direct = ((a.prec == LUSP_FP64 && !a.ir64) || (a.what & LUSP_RUN_DIRECT)) ? 1 : 0;
    const bool ladder = a.rungs != 0 && a.prec != LUSP_FP64 && !direct && (a.what & LUSP_RUN_SOLVE);
    EscDev none{};
    int rc = launch_rung<VT, AT>(a.d_sys, a.nsys, a.d_queue, nullptr, nullptr, a.what, main_shape(a), a.prm, direct,
                                 ladder ? a.esc : none, 0, st, a.kev);
    if (rc != LUSP_OK || !ladder) return rc;
    // The fp64 rungs: every kernel reads its item count from the slot
    // counters the solve kernels above wrote (no host round trip).
    const RungShape x = ladder_shape(a);
    int* ctl = a.d_queue + kLadderCtl;
    if (a.rungs & 1) {
        EscDev esc = a.esc;
        if (!(a.rungs & 2)) esc.hard = nullptr;
        rc = launch_rung<double, double>(a.esc.slots, a.esc.cap, a.d_queue + 3, ctl, nullptr, LUSP_RUN_BOTH, x,
                                         a.xprm, 0, esc, 1, st);
        if (rc != LUSP_OK) return rc;
    }
    if (a.rungs & 2) {
        SolveParams hp = a.xprm;
        hp.shift = a.hard_shift;
        const bool after_safe = (a.rungs & 1) != 0;
        rc = launch_rung<double, double>(a.esc.slots, a.esc.cap, a.d_queue + 6, after_safe ? ctl + 1 : ctl,
                                         after_safe ? a.esc.hard : nullptr, LUSP_RUN_BOTH, x, hp, 0, a.esc, 2, st);
    }
    return rc;
}

int launch_systems(const LaunchArgs& a, cudaStream_t st) {
    if (a.prec == LUSP_FP64) return launch_typed<double, double>(a, st);
    if (a.inner == 1) return launch_typed<float, double>(a, st);
    if (a.inner == 2) return launch_typed<float, __half>(a, st);
    return launch_typed<float, float>(a, st);
}

int launch_kernel_count(const LaunchArgs& a, int what) {
    int n = ((what & LUSP_RUN_REFACTOR) ? (a.dgrid > 0 ? 2 : 1) : 0) + ((what & LUSP_RUN_SOLVE) ? 1 : 0);
    const bool direct = a.prec == LUSP_FP64 || (what & LUSP_RUN_DIRECT);
    if (a.rungs && !direct && (what & LUSP_RUN_SOLVE))
        n += (((a.rungs & 1) ? 1 : 0) + ((a.rungs & 2) ? 1 : 0)) * (a.xdgrid > 0 ? 3 : 2);
    return n;
}

int batch_launch(BatchObj* B, int what, cudaStream_t st, bool timed) {
    LaunchArgs a = B->launch;
    a.what = what;
    a.kev = timed && B->kev[0] ? B->kev : nullptr;
    int rc = launch_systems(a, st);
    if (rc == LUSP_OK) B->launches = launch_kernel_count(a, what);
    return rc;
}

int tail_ld(const StaticPattern& S) { return (S.dtail + 31) & ~31; }

static SysSizes host_sizes(const StaticPattern& S) {
    return SysSizes{(size_t)S.n, (size_t)S.cap, S.lci.size(), S.uci.size(), (size_t)S.sell_ptr.back(),
                    (size_t)S.dtail, (size_t)tail_ld(S)};
}

size_t system_private_bytes(const StaticPattern& S, size_t vs, int m) {
    return sys_private_bytes(host_sizes(S), vs, m);
}

char* carve_system(SysDev& D, char* p, const StaticPattern& S, size_t vs, int m) {
    return sys_carve(D, p, host_sizes(S), vs, m);
}

size_t spill_bytes(int grid, int block, int colmax, const SmemPlan& rplan) {
    return colmax > rplan.wcap ? al256((size_t)grid * (block / 32) * colmax * 8) : 0;
}

int check_opts(const lusp_batch_opts* o) {
    if (o->prec != LUSP_MIXED && o->prec != LUSP_FP64) { set_error("bad prec"); return LUSP_EARG; }
    if (o->krylov < 1 || o->krylov > kMaxKrylov) { set_error("krylov must be 1..%d", kMaxKrylov); return LUSP_EARG; }
    if (o->block_threads != 0 && (o->block_threads < 64 || o->block_threads > 512 || o->block_threads % 32)) {
        set_error("block_threads must be 0 (auto) or 64..512, a multiple of 32");
        return LUSP_EARG;
    }
    if (o->ctas_per_sm < 0) { set_error("ctas_per_sm must be >= 0"); return LUSP_EARG; }
    if (o->inner_prec < 0 || o->inner_prec > 2) { set_error("bad inner_prec"); return LUSP_EARG; }
    if (o->refactor_cluster < 0 || o->refactor_cluster > 8) {
        set_error("refactor_cluster must be 0 (auto) or 1..8");
        return LUSP_EARG;
    }
    if (o->ladder < 0 || o->ladder > 3) { set_error("ladder must be 0..3"); return LUSP_EARG; }
    if (o->ladder_slots < 0) { set_error("ladder_slots must be >= 0"); return LUSP_EARG; }
    if (!(o->factor_shift >= 0.0) || !(o->hard_shift >= 0.0)) {
        set_error("factor_shift and hard_shift must be >= 0");
        return LUSP_EARG;
    }
    if (o->refactor_threads != 0 &&
        (o->refactor_threads < 64 || o->refactor_threads > 1024 || o->refactor_threads % 32)) {
        set_error("refactor_threads must be 0 (auto) or 64..1024, a multiple of 32");
        return LUSP_EARG;
    }
    return LUSP_OK;
}

void fill_params(SolveParams& prm, const lusp_batch_opts& o) {
    prm.m = o.krylov;
    prm.max_outer = std::max(0, o.max_outer);
    prm.rtol = o.rtol;
    prm.inner_rel = o.inner_rel;
    prm.stag_ratio = o.stag_ratio;
    prm.pivot_tol = o.pivot_tol;
    prm.refactor_mode = o.refactor_mode;
    prm.xtol = o.xtol > 0 ? o.xtol : 1e-8;
    prm.shift = o.factor_shift;
}

// Gathered updates per system above which a batch of few systems spreads
// each system's refactorization over many SMs (the n = 40,000 circuit has
// 227 M; the n = 4050 power grid, refactored faster by one 2-SM cluster,
// has 5.9 M).
constexpr long long kSpreadMinUpdates = 16ll << 20;
// Gathered updates per system above which a batch of at most one system
// per SM spreads each system over up to kSpreadMidGroup 256-thread CTAs.
constexpr long long kSpreadMidUpdates = 1ll << 17;
constexpr int kSpreadMidGroup = 12;

int refactor_setup(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, int nsys, LaunchArgs& a) {
    a.rblock = refactor_block(o, nsys);
    make_refactor_plan(pats, a.rblock, o.prec == LUSP_FP64 ? 8 : 4, a.rplan);
    int occ = 0;
    int rc = refactor_occupancy(o.prec, a.rplan.bytes, a.rblock, &occ);
    if (rc != LUSP_OK) return rc;
    if (occ < 1) { set_error("refactor kernel does not fit one SM (smem %zu)", a.rplan.bytes); return LUSP_EARG; }
    a.rgrid = std::min(nsys, occ * sm_count());
    // Spread a system's columns over a cluster of CTAs when every system of
    // the batch still gets its own cluster at once (the refactor is bound by
    // instruction issue on one SM; the dependency chain leaves room).
    a.rcluster = 1;
    int want = o.refactor_cluster;
    if (want == 0) want = (a.rblock > 512 && 2 * nsys <= sm_count()) ? 2 : 1;
    if (want > 1) {
        int ncl = 0;
        rc = o.prec == LUSP_FP64 ? refactor_cluster_count<double>(a.rplan.bytes, a.rblock, want, &ncl)
                                 : refactor_cluster_count<float>(a.rplan.bytes, a.rblock, want, &ncl);
        if (rc != LUSP_OK) return rc;
        if (ncl >= 1 && (o.refactor_cluster > 1 || ncl >= nsys)) {
            a.rcluster = want;
            a.rgrid = want * std::min(nsys, ncl);
        }
    }
    // Spread mode: a few large systems, each refactored by many CTAs that
    // synchronize through global memory (the sync area is bound by the
    // caller: batch_build).
    a.rspread = SpreadArgs{};
    if (o.refactor_spread >= 0) {
        long long gmin = -1;
        int nmax = 1;
        for (auto* p : pats) {
            gmin = gmin < 0 ? p->S.gathered : std::min<long long>(gmin, p->S.gathered);
            nmax = std::max(nmax, p->S.n);
        }
        const int slots = occ * sm_count();
        int g = 0;
        bool mid = false;
        if (o.refactor_spread > 0) g = std::min(o.refactor_spread, slots / std::max(1, nsys));
        else if (nsys * 8 <= sm_count() && gmin >= kSpreadMinUpdates) g = slots / nsys;
        else if (nsys <= sm_count() && gmin >= kSpreadMidUpdates && o.refactor_threads <= 0 &&
                 o.refactor_cluster <= 0) {
            // Medium systems, at most one per SM: 256-thread CTAs, four per
            // SM, up to kSpreadMidGroup per system (B200, 50 systems: the
            // n = 4050 grid 2.22 -> 1.95 ms, an n = 4000 circuit 0.82 ->
            // 0.70 ms against one 2-CTA cluster each; the n = 989 circuit,
            // 41 k updates, gains nothing).
            SmemPlan pl;
            make_refactor_plan(pats, 256, o.prec == LUSP_FP64 ? 8 : 4, pl);
            int mocc = 0;
            rc = refactor_occupancy(o.prec, pl.bytes, 256, &mocc, true);
            if (rc != LUSP_OK) return rc;
            const int mg = std::min(kSpreadMidGroup, mocc * sm_count() / nsys);
            if (mg >= 4) {
                g = mg;
                mid = true;
                a.rblock = 256;
                a.rplan = pl;
            }
        }
        if (g >= 2 && o.refactor_threads <= 0 && !mid) {
            // One CTA per SM, of the size whose per-warp work area holds the
            // longest column before the dense block (longer ones spill to
            // global memory).
            int colsp = 2;
            for (auto* p : pats)
                for (int k = 0; k < p->S.k0; k++) colsp = std::max(colsp, p->S.cp[k + 1] - p->S.cp[k]);
            const int vs = o.prec == LUSP_FP64 ? 8 : 4;
            for (int t : {768, 512, 384, 256}) {
                SmemPlan pl;
                make_refactor_plan(pats, t, vs, pl, 1);
                if (pl.wcap >= colsp || t == 256) {
                    a.rblock = t;
                    a.rplan = pl;
                    break;
                }
            }
            rc = refactor_occupancy(o.prec, a.rplan.bytes, a.rblock, &occ, true);
            if (rc != LUSP_OK) return rc;
            if (occ < 1) { set_error("refactor kernel does not fit one SM (smem %zu)", a.rplan.bytes); return LUSP_EARG; }
            g = std::max(1, std::min(g, occ * sm_count() / nsys));
        }
        if (g >= 2) {
            a.rspread.group = g;
            a.rspread.stride = sync_stride(nmax);
            a.rcluster = 1;
            a.rgrid = g * nsys;
        }
    }
    // Dense trailing blocks: their own kernel when any system has one.
    int ntail = 0;
    for (auto* p : pats) ntail += p->S.dtail > 0 ? 1 : 0;
    a.dblock = 512;
    a.dgrid = 0;
    if (ntail > 0) {
        make_dense_plan(pats, a.dblock, a.dplan);
        int docc = 0;
        rc = o.prec == LUSP_FP64 ? dense_prepare<double>(a.dplan.bytes, a.dblock, &docc)
                                 : dense_prepare<float>(a.dplan.bytes, a.dblock, &docc);
        if (rc != LUSP_OK) return rc;
        if (docc < 1) { set_error("dense kernel does not fit one SM (smem %zu)", a.dplan.bytes); return LUSP_EARG; }
        a.dgrid = std::min(ntail, docc * sm_count());
        // Two CTAs per block (a 2-CTA cluster that splits the trailing
        // updates) when every system with a block gets its pair of SMs.
        a.dcluster = 1;
        if (a.dplan.tnb == 32 && 2 * ntail <= sm_count()) {
            int ncl = 0;
            rc = o.prec == LUSP_FP64 ? dense_cluster_count<double>(a.dplan.bytes, a.dblock, &ncl)
                                     : dense_cluster_count<float>(a.dplan.bytes, a.dblock, &ncl);
            if (rc != LUSP_OK) return rc;
            if (ncl >= ntail) {
                a.dcluster = 2;
                a.dgrid = 2 * ntail;
            }
        }
    }
    return LUSP_OK;
}

int ladder_setup(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, int cap, LaunchArgs& a,
                 LadderPlan& lp, size_t pool) {
    a.rungs = 0;
    lp = LadderPlan{};
    const int rungs = o.ladder == 1 ? 1 : o.ladder == 2 ? 2 : o.ladder == 3 ? 3 : 0;
    if (rungs == 0 || o.prec != LUSP_MIXED || cap <= 0) return LUSP_OK;
    lusp_batch_opts x = o;
    x.prec = LUSP_FP64;
    x.inner_prec = 0;
    x.refactor_spread = -1;
    x.block_threads = 0;
    x.ctas_per_sm = 0;
    resolve_solve_shape(x, cap);
    int rc = plan_for(pats, x, a.xplan);
    if (rc != LUSP_OK) {
        x.solve_sweep = 0;
        rc = plan_for(pats, x, a.xplan);
        if (rc != LUSP_OK) return rc;
    }
    int occ = 0;
    rc = kernel_occupancy(LUSP_FP64, 0, a.xplan.bytes, x.block_threads, &occ);
    if (rc != LUSP_OK) return rc;
    if (occ < 1) { set_error("ladder solve kernel does not fit one SM (smem %zu)", a.xplan.bytes); return LUSP_EARG; }
    a.xblock = x.block_threads;
    a.xgrid = std::min(cap, occ * sm_count());
    LaunchArgs r;
    rc = refactor_setup(pats, x, cap, r);
    if (rc != LUSP_OK) return rc;
    a.xrplan = r.rplan;
    a.xrblock = r.rblock;
    a.xrgrid = r.rgrid;
    a.xrcluster = r.rcluster;
    a.xdplan = r.dplan;
    a.xdblock = r.dblock;
    a.xdgrid = r.dcluster > 1 ? r.dgrid / r.dcluster : r.dgrid;   // the ladder's dense kernel runs lone CTAs
    fill_params(a.xprm, x);
    a.xprm.shift = 0.0;
    a.hard_shift = o.hard_shift > 0 ? o.hard_shift : 1e-7;
    size_t stride = 0;
    int colmax = 0;
    for (auto* p : pats) {
        stride = std::max(stride, system_private_bytes(p->S, 8, o.krylov));
        colmax = std::max(colmax, p->S.max_col);
    }
    lp.pool = pool > 0 ? al256(pool) : (size_t)cap * stride;
    lp.spill = spill_bytes(a.xrgrid, a.xrblock, colmax, a.xrplan);
    lp.bytes = lp.pool + lp.spill + al256(sizeof(SysDev) * cap) + al256(sizeof(int) * cap);
    a.rungs = rungs;
    a.esc = EscDev{};
    a.esc.cap = cap;
    a.esc.m = o.krylov;
    a.esc.pool = lp.pool;
    a.esc.rtol = o.rtol;
    a.esc.fail_bits = ST_SINGULAR | ST_PIVOT_WEAK | ST_STAGNATED | ST_NOT_CONVERGED | ST_NONFINITE |
                      ST_WAIT_TIMEOUT | ST_CAPACITY;
    return LUSP_OK;
}

void ladder_bind(LaunchArgs& a, const LadderPlan& lp, char* mem, int* queue) {
    if (!a.rungs) return;
    char* p = mem;
    a.esc.base = p;
    p += lp.pool;
    a.esc.scratch = lp.spill ? (double*)p : nullptr;
    p += lp.spill;
    a.esc.slots = (SysDev*)p;
    p += al256(sizeof(SysDev) * a.esc.cap);
    a.esc.hard = (int*)p;
    a.esc.ctl = queue + kLadderCtl;
}

// Triangular sweeps chosen by solve_sweep = 0: the dataflow sweeps whenever
// the solve vectors fit shared memory.
constexpr bool kAutoFlow = false;

// Ladder slots when the options leave them at 0: every system of a batch up
// to 256, else an eighth of them (at least 256).
static int ladder_cap(const lusp_batch_opts& o, int nsys) {
    if (o.ladder_slots > 0) return std::min(o.ladder_slots, nsys);
    return nsys <= 256 ? nsys : std::max(256, nsys / 8);
}

int plan_for(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, SmemPlan& plan) {
    make_plan(pats, o.block_threads, o.ctas_per_sm, o.krylov, o.prec == LUSP_FP64 ? 8 : 4, plan);
    plan.flow = 0;
    if (o.solve_sweep == 1 || (o.solve_sweep == 0 && kAutoFlow)) {
        // Dataflow sweeps when every solve vector lives in shared memory and
        // a second one and the warps' staging rings fit where the level
        // sweeps' stage ring would be (that ring then serves no system).
        if (plan.ycap > 0) {
            const size_t ring = plan.sc_ent ? kStages * stage_bytes(plan.sc_ent, plan.sc_rows, o.prec == LUSP_FP64 ? 8 : 4) : 0;
            const size_t base = plan.bytes - ring;
            const size_t need = (((size_t)plan.ycap * 8 + 15) & ~(size_t)15) +
                                flow_ring_bytes(o.block_threads / 32, o.prec == LUSP_FP64 ? 8 : 4);
            if (base + need <= solve_smem_budget(o.ctas_per_sm)) {
                plan.flow = 1;
                plan.sc_ent = plan.sc_rows = 0;
                plan.bytes = base + need;
            }
        }
        if (!plan.flow && o.solve_sweep == 1) {   // per-row dataflow over global memory
            plan.dcap = 0;
            plan.sc_ent = plan.sc_rows = 0;
        }
    }
    if (o.solve_sweep == 2 && plan.sc_ent == 0) {
        set_error("level-synchronous sweeps need a stage ring in shared memory");
        return LUSP_EARG;
    }
    return LUSP_OK;
}

int batch_build(int nsys, PatternObj* const* pats, const lusp_batch_opts* o, BatchObj** out) {
    *out = nullptr;
    if (nsys <= 0 || !pats || !o) { set_error("batch_create: bad arguments"); return LUSP_EARG; }
    for (int s = 0; s < nsys; s++)
        if (!pats[s]) { set_error("batch_create: null pattern %d", s); return LUSP_EARG; }
    int rc = check_opts(o);
    if (rc != LUSP_OK) return rc;
    lusp_batch_opts oo = *o;
    resolve_solve_shape(oo, nsys);
    o = &oo;
    BatchObj* B = new BatchObj();
    B->nsys = nsys;
    B->prec = o->prec;
    B->opts = *o;
    B->pats.assign(pats, pats + nsys);
    B->block = o->block_threads;
    fill_params(B->prm, *o);
    rc = plan_for(B->pats, *o, B->plan);
    if (rc != LUSP_OK) { delete B; return rc; }

    const size_t vs = B->prec == LUSP_FP64 ? 8 : 4;
    // Inputs and outputs of all systems are contiguous (values, rhs, x) so a
    // batch moves host<->device in one copy each; the rest is per system.
    std::vector<size_t> base(nsys + 1, 0);
    B->val_off.assign(nsys + 1, 0);
    B->vec_off.assign(nsys + 1, 0);
    for (int s = 0; s < nsys; s++) {
        B->val_off[s + 1] = B->val_off[s] + B->pats[s]->S.nnz_a;
        B->vec_off[s + 1] = B->vec_off[s] + B->pats[s]->S.n;
    }
    base[0] = al256(B->val_off[nsys] * 8) + 2 * al256(B->vec_off[nsys] * 8);
    for (int s = 0; s < nsys; s++) base[s + 1] = base[s] + system_private_bytes(B->pats[s]->S, vs, o->krylov);
    int colmax = 0;
    for (auto* p : B->pats) colmax = std::max(colmax, p->S.max_col);
    int occ = 0;
    rc = kernel_occupancy(B->prec, o->inner_prec, B->plan.bytes, B->block, &occ);
    if (rc != LUSP_OK) { delete B; return rc; }
    if (occ < 1) { delete B; set_error("batch_create: kernel does not fit one SM (smem %zu)", B->plan.bytes); return LUSP_EARG; }
    B->grid = std::min(nsys, occ * sm_count());
    LaunchArgs& a = B->launch;
    rc = refactor_setup(B->pats, *o, nsys, a);
    if (rc != LUSP_OK) { delete B; return rc; }
    LadderPlan lp;
    rc = ladder_setup(B->pats, *o, ladder_cap(*o, nsys), a, lp);
    if (rc != LUSP_OK) { delete B; return rc; }
    const size_t spill = spill_bytes(a.rgrid, a.rblock, colmax, a.rplan);
    const size_t syncb = a.rspread.group > 0 ? al256((size_t)nsys * a.rspread.stride * sizeof(unsigned)) : 0;
    const size_t total =
        base[nsys] + spill + al256(sizeof(SysStats) * nsys) + al256(sizeof(SysDev) * nsys) + 256 + syncb;
    char* blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, total);
    if (e != cudaSuccess) { delete B; return cuda_fail(e, "batch device alloc"); }
    B->d_block = blk;
    B->bytes = total;
    e = cudaMemset(blk, 0, total);
    if (e != cudaSuccess) { batch_free(B); return cuda_fail(e, "batch memset"); }
    char* stats_base = blk + base[nsys] + spill;
    B->d_stats = (SysStats*)stats_base;
    B->d_sys = (SysDev*)(stats_base + al256(sizeof(SysStats) * nsys));
    B->d_queue = (int*)((char*)B->d_sys + al256(sizeof(SysDev) * nsys));
    if (syncb) a.rspread.sync = (unsigned*)((char*)B->d_queue + 256);
    double* spill_ptr = spill ? (double*)(blk + base[nsys]) : nullptr;
    B->d_vals = (double*)blk;
    B->d_rhs = (double*)(blk + al256(B->val_off[nsys] * 8));
    B->d_x = (double*)(blk + al256(B->val_off[nsys] * 8) + al256(B->vec_off[nsys] * 8));
    B->h_sys.resize(nsys);
    for (int s = 0; s < nsys; s++) {
        SysDev& D = B->h_sys[s];
        D.pat = B->pats[s]->d_desc;
        D.a_val = B->d_vals + B->val_off[s];
        D.b = B->d_rhs + B->vec_off[s];
        D.x = B->d_x + B->vec_off[s];
        carve_system(D, blk + base[s], B->pats[s]->S, vs, o->krylov);
        D.scratch = spill_ptr;
        D.stats = B->d_stats + s;
    }
    e = cudaMemcpy(B->d_sys, B->h_sys.data(), sizeof(SysDev) * nsys, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { batch_free(B); return cuda_fail(e, "batch descriptor upload"); }
    if (a.rungs) {
        e = cudaMalloc(&B->d_ladder, lp.bytes);
        if (e != cudaSuccess) { batch_free(B); return cuda_fail(e, "ladder device alloc"); }
        B->bytes += lp.bytes;
        ladder_bind(a, lp, B->d_ladder, B->d_queue);
    }
    a.d_sys = B->d_sys;
    a.nsys = nsys;
    a.d_queue = B->d_queue;
    a.plan = B->plan;
    a.prm = B->prm;
    a.prec = B->prec;
    a.inner = o->inner_prec;
    a.what = LUSP_RUN_BOTH;
    a.block = B->block;
    a.grid = B->grid;
    *out = B;
    return LUSP_OK;
}

void batch_free(BatchObj* B) {
    if (!B) return;
    for (auto& kv : B->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    if (B->d_block) cudaFree(B->d_block);
    if (B->d_ladder) cudaFree(B->d_ladder);
    for (cudaEvent_t ev : B->kev)
        if (ev) cudaEventDestroy(ev);
    delete B;
}

}  // namespace lusp
