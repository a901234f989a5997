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
    int nfwd_levels, nbwd_levels;
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
    int pad_;
    // SM cycles (summed over warps): refactor waits for dependency columns,
    // gathers of their L parts, updates; refactor wall cycles of the CTA.
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
};

constexpr int kMaxKrylov = 64;

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
    size_t bytes;
};

}  // namespace lusp
