// Device-side data layout of the refactor-and-solve engine and the per-CTA
// phases that run one linear system each.
//
// One CTA owns one system (a pattern plus one set of values).  Inside it,
// warps claim items of a precomputed level-sorted order (columns for the
// refactorization, rows for the triangular solves) from a shared counter
// and wait for the items they depend on through shared-memory ready bits,
// so the level schedule runs without grid-wide barriers or host round trips.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace lusp {

// Device-resident static pattern (all pointers are device memory).
struct PatternDev {
    int n, nnz_a, cap, max_col, nslices, sell_total;
    int nnz_l, nnz_u;        // strict L and strict U entries
    int nfwd_levels, nbwd_levels;    // sweep steps (descriptors) of each sweep
    const int* cp;           // [n+1] merged column pointers
    const int* ri;           // [cap] row positions, ascending per column
    const int* dg;           // [n]   slot of the diagonal
    const int* col_order;    // [n]   level-sorted columns
    const int* a_ptr;        // [n+1] input entries per column
    const int* a_src;        // [nnz_a] input index
    const int* a_dst;        // [nnz_a] slot offset inside the column
    const int* lrp;          // [n+1] strict-L rows in level order (by idx)
    const int* lci;          // [nnz_l] column positions
    const int* urp;          // [n+1] strict-U rows in level order (by idx)
    const int* uci;          // [nnz_u] column positions
    const int* slot_dst;     // [cap] slot -> L-row / U-row index, diag -> k
    const int* fwd_order;    // [n] idx -> row, level-sorted, for L y = b
    const int* bwd_order;    // [n] idx -> row, level-sorted, for U z = y
    const int* fwd_lev;      // [nfwd_levels+1] first idx of each level
    const int* bwd_lev;      // [nbwd_levels+1]
    const int* sell_ptr;     // [nslices+1]
    const int* sell_col;     // [sell_total] column positions
    const int* sell_src;     // [sell_total] input index or -1
    const int* sell_perm;    // [32*nslices] row position or -1
    const int* rowat;        // [n] position -> original row
    const int* q;            // [n] position -> original column
    const int2* dep_bc;           // [cap] for U slots: {first strict-L slot,
                                  // strict-L length} of the dependency column
    const unsigned short* rel;    // relative update slots (null: search rows)
    const long long* rel_ptr;     // [n+1] column k's list in rel
    // Dense trailing block: rows/columns [k0, n), dtail = n - k0 (0: none),
    // stored row-major with leading dimension tail_ld.
    int k0, dtail, tail_ld;
    // Pattern of the dense trailing block, one bit per entry (row r, column c
    // of the block: bit c & 31 of word r * (tail_ld / 32) + c / 32).  The
    // refactor writes only these entries of the fp64 block; the dense kernel
    // reads every other entry as 0 in its first panel step.
    const unsigned* tail_mask;
    // Column records of the refactorization, three 16-byte words per claim
    // index idx (column k = col_order[idx]): {k, cp[k], column length,
    // diagonal offset}, {first input entry a_ptr[k], a_ptr[k + 1],
    // dependencies before the dense block, bwd_pos[k]}, {rel_ptr[k] low and
    // high words, a_diag[k], 0}.
    const int4* crec;
    const int* a_diag;       // [n] slot offset of A(q_k, q_k) in column k, or -1
    const int* bwd_pos;      // [n] row -> index in bwd_order
    const int* fwd_ldesc;    // [nfwd_levels * 5] level descriptors (see host)
    const int* bwd_ldesc;    // [nbwd_levels * 5]
    int lev_max_ent, lev_max_rows;   // widest sweep level (entries, rows)
};

// Per-system statistics written by the kernels.
struct SysStats {
    double min_abs_pivot;    // min |U(k,k)|
    double min_pivot_ratio;  // min |U(k,k)| / max(|U(k,k)|, max|x_L|)
    double max_abs_u;        // max |U(i,j)| (growth numerator)
    double res[16];          // relative residual history ||b-Ax||/||b||
    int nres;
    int inner_iters;
    int outer_iters;
    int status;
    int singular_col;
    int rung;                // ladder rung of the result: 0 P-fast (the batch's
                             // own precision), 1 P-safe, 2 P-hard
    // SM cycles (summed over warps): refactor waits for dependency columns,
    // gathers of their L parts, updates (0 unless built with
    // LUSP_REFACTOR_PHASE_CYCLES); refactor wall cycles of the CTA.
    long long cyc_wait, cyc_gather, cyc_update, cyc_refactor;
    // SM cycles of the solve (CTA wall time, summed over calls): L sweeps,
    // dense-tail solves, U sweeps, SpMVs, whole solve phase.
    long long cyc_lsolve, cyc_tail, cyc_usolve, cyc_spmv, cyc_solve;
    // Refactor: dense trailing block panels, U-row solves, trailing updates.
    long long cyc_tpanel, cyc_ttrsm, cyc_tupdate;
    // Solve: dense-tail diagonal-block chains and block-column products.
    long long cyc_tdiag, cyc_tgemv;
};

// One system: pattern + values + vectors + workspace.
struct SysDev {
    const PatternDev* pat;
    const double* a_val;     // [nnz_a] input values, fp64
    void* lu;                // [cap] merged factor values (VT)
    void* lval;              // [nnz_l] strict L by rows (VT)
    void* uval;              // [nnz_u] strict U by rows (VT)
    void* udiag;             // [n] U(k,k) (VT)
    void* udiag_bwd;         // [n] U(k,k) (VT) in backward sweep order
    double* sell64;          // [sell_total] A in SELL, fp64
    float* sell32;           // [sell_total] A in SELL, fp32
    void* sell16;            // [sell_total] Ruiz-scaled A in SELL, fp16 (__half)
    double* rs;              // [n] Ruiz row scaling (position space)
    double* cs;              // [n] Ruiz column scaling
    const double* b;         // [n] right-hand side, original row order
    double* x;               // [n] solution, original column order
    double* work;            // workspace (see solve phase)
    double* scratch;         // per-CTA refactor spill (columns longer than
                             // the shared-memory work area), may be null
    void* tail;              // [dtail * tail_ld] dense L\U of the trailing
                             // block (VT, column-major: (i, c) at c * ld + i),
                             // unit L below the diagonal
    double* tailw;           // [dtail * tail_ld] fp64 trailing block (row-major)
                             // between the refactor and dense kernels
    void* tinv;              // [ceil(dtail/32) * 2048] inverses of the dense
                             // block's 32 x 32 diagonal blocks (VT): per block
                             // L^-1 then U^-1, element (i, c) at c * 32 + i
    SysStats* stats;
};

struct SolveParams {
    int m;                   // Krylov dimension per restart (<= kMaxKrylov)
    int max_outer;           // outer corrections
    double rtol;             // target ||b-Ax||/||b||
    double inner_rel;        // inner stop relative to the current residual
    double stag_ratio;       // residual must shrink by this factor per outer
    double pivot_tol;        // frozen-pivot acceptance threshold
    int refactor_mode;       // 0 staged gathers (cp.async), 1 per-dependency loads
    double xtol;             // forward-error target of the refinement
    double shift;            // factor of A + shift * diag|A(i,i)| (0: A itself)
};

constexpr int kMaxKrylov = 64;

// Sizes that fix one system's private device area.
struct SysSizes {
    size_t n, cap, nnz_l, nnz_u, sell, dtail, tail_ld;
};

__host__ __device__ inline SysSizes sizes_of(const PatternDev& P) {
    return SysSizes{(size_t)P.n, (size_t)P.cap, (size_t)P.nnz_l, (size_t)P.nnz_u,
                    (size_t)P.sell_total, (size_t)P.dtail, (size_t)P.tail_ld};
}

__host__ __device__ inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// Private bytes of one system with factor values of vs bytes and Krylov
// dimension m.  The merged and row-major values and the sweep-order
// diagonal get 64 bytes of slack: the kernels copy them in aligned 16-byte
// pieces.
__host__ __device__ inline size_t tinv_bytes(const SysSizes& z, size_t vs) {
    return ((z.dtail + 31) / 32) * 2048 * vs;
}

__host__ __device__ inline size_t sys_private_bytes(const SysSizes& z, size_t vs, int m) {
    return al256(z.cap * vs + 64) + al256(z.nnz_l * vs + 64) + al256(z.nnz_u * vs + 64) + al256(z.n * vs) +
           al256(z.n * vs + 64) + al256(z.sell * 8) + al256(z.sell * 4) + al256((2 * (size_t)m + 8) * z.n * 8) +
           al256(z.dtail * z.tail_ld * vs) + al256(z.dtail * z.tail_ld * 8) + al256(z.sell * 2) +
           2 * al256(z.n * 8) + al256(tinv_bytes(z, vs));
}

// Points the private arrays of D into p (sys_private_bytes of them); returns
// the end.  The same layout on the host (batches, serving arenas) and on the
// device (ladder slots).
__host__ __device__ inline char* sys_carve(SysDev& D, char* p, const SysSizes& z, size_t vs, int m) {
    D.tail = p; p += al256(z.dtail * z.tail_ld * vs);
    D.tailw = z.dtail > 0 ? (double*)p : nullptr;
    p += al256(z.dtail * z.tail_ld * 8);
    D.lu = p; p += al256(z.cap * vs + 64);
    D.lval = p; p += al256(z.nnz_l * vs + 64);
    D.uval = p; p += al256(z.nnz_u * vs + 64);
    D.udiag = p; p += al256(z.n * vs);
    D.udiag_bwd = p; p += al256(z.n * vs + 64);
    D.sell64 = (double*)p; p += al256(z.sell * 8);
    D.sell32 = (float*)p; p += al256(z.sell * 4);
    D.work = (double*)p; p += al256((2 * (size_t)m + 8) * z.n * 8);
    D.sell16 = p; p += al256(z.sell * 2);
    D.rs = (double*)p; p += al256(z.n * 8);
    D.cs = (double*)p; p += al256(z.n * 8);
    D.tinv = p; p += al256(tinv_bytes(z, vs));
    return p;
}

// Device-side escalation ladder of one launch.  A system whose P-fast solve
// (the batch's own fp32 factor and GMRES-IR) fails takes a slot: the solve
// kernel that saw the failure points the slot's private arrays into fp64
// storage taken from a pool, keeping the system's pattern, values,
// right-hand side, solution and statistics, and the P-safe kernels (fp64 factor, GMRES-IR with the
// fp64 factor as preconditioner) run over the taken slots.  A slot whose
// P-safe solve fails again goes on to P-hard: the fp64 factor of
// A + shift diag|A(i,i)| (the residual still uses A).
struct EscDev {
    int* ctl;                // [0] slots taken, [1] slots on the P-hard list,
                             // [2..3] bytes of the storage pool taken (64 bit)
    int* hard;               // [cap] slots escalated to P-hard
    SysDev* slots;           // [cap] fp64 systems, filled by the device
    char* base;              // storage pool: each slot takes its own system's
    size_t pool;             // fp64 private bytes from it
    double* scratch;         // refactor spill of the fp64 kernels (may be null)
    int cap;                 // slots (0: no ladder)
    int m;                   // Krylov dimension of the slots' workspace
    int fail_bits;           // status bits that count as a failure (P-fast;
                             // the fp64 rungs ignore a weak pivot alone)
    double rtol;             // ... as does a final residual above rtol
};

// Several CTAs per system for the refactorization of batches of few large
// systems ("spread" mode): CTAs [s * group, (s + 1) * group) take the
// columns of system s.  The claim counter, status words and ready bits of a
// system live in global memory (its sync area, zeroed before the kernel):
// words [0, 16) control (kSync* below), words [16, 32) eight 64-bit
// accumulators of the pivot statistics and cycle counters, words [32, ...)
// the ready bits.
struct SpreadArgs {
    int group;               // CTAs per system (0: cluster / queue mode)
    unsigned* sync;          // sync areas of the systems
    int stride;              // 32-bit words per system
};
constexpr int kSyncClaim = 0, kSyncStatus = 1, kSyncSingular = 2, kSyncAbort = 3, kSyncDone = 4;
constexpr int kSyncAcc = 16, kSyncReady = 32;
__host__ __device__ inline int sync_stride(int nmax) { return (kSyncReady + (nmax + 31) / 32 + 7) & ~7; }

// Shared-memory plan of one launch (same for every CTA).
struct SmemPlan {
    int nwords;              // ready-bit words (>= ceil(n_max/32))
    int wcap;                // per-warp refactor work slots
    int scap;                // per-warp staged L entries (refactor gathers)
    int tnb;                 // panel width of the dense trailing block
    int ttw;                 // warps transposing the dense block (32x33 fp64 tile each)
    int sc_ent, sc_rows;     // sweep stage capacity (entries, rows; 0: no stages)
    int ycap;                // doubles for a shared-memory solve vector
    int dcap;                // ints for shared-memory sweep descriptors
    int m;                   // Krylov dimension for H
    int flow = 0;            // dataflow sweeps for shared-memory solve vectors
                             // (second vector of ycap doubles in place of the
                             // stage ring)
    size_t bytes;
};

}  // namespace lusp
