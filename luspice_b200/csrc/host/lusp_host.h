// Internal host-side declarations shared by the host analysis code and the
// CUDA engine.  Nothing here crosses the public C-ABI.
#pragma once
#include <cstdint>
#include <vector>

namespace lusp {

// Result of the pivoting fp64 factorization that fixes the row permutation
// and the structural L/U pattern (CSparse cs_lu layout, as the reference's
// splu.h:29-41 stores it).
struct PivotFactor {
    int n = 0;
    int singular_col = -1;          // -1 ok, >= 0 first column with no pivot
    std::vector<int> pinv;          // pinv[orig_row] = pivot position
    std::vector<int> Lp, Li;        // L: unit diagonal first, Li = positions
    std::vector<double> Lx;
    std::vector<int> Up, Ui;        // U: diagonal last, Ui = positions
    std::vector<double> Ux;
};

// fp64 left-looking LU with threshold partial pivoting on the q-permuted
// CSC of A (A given with original row indices, rows in any order, no
// duplicate entries within a column).  Bit-for-bit the decisions of the
// reference (splu.h:151-206): same depth-first reach order, same update
// order, same pivot tie-breaks.  Returns singular_col.
int pivot_factor(int n, const int* Ap, const int* Ai, const double* Ax,
                 const int* q, double tol, PivotFactor& F);

// Static layout of one sparsity pattern on the device, in pivot-position
// space.  Column k of the merged factor is slots [cp[k], cp[k+1]): the
// rows j < k of U(:,k) ascending, the diagonal at slot dg[k], then the rows
// i > k of L(:,k) ascending.
struct StaticPattern {
    int n = 0;
    int nnz_a = 0;                  // entries of the input CSC
    long lnnz = 0, unnz = 0;        // splu-convention counts
    long cap = 0;                   // merged slots = lnnz + unnz - n
    uint64_t hash = 0;              // FNV-1a of (n, Ap, Ai, q)

    std::vector<int> q, invq;       // column order and its inverse
    std::vector<int> pinv, rowat;   // row permutation and its inverse

    std::vector<int> cp, ri, dg;    // merged columns

    // Column schedule: level-sorted column order for the refactorization.
    std::vector<int> col_level, col_order;
    int ncol_levels = 0;

    // Input values -> slots.  For column k, entries [a_ptr[k], a_ptr[k+1])
    // give a_src (index into the input value array) and a_dst (slot offset
    // inside column k), sorted by a_dst (duplicates adjacent).
    std::vector<int> a_ptr, a_src, a_dst;
    // a_diag[k]: slot offset inside column k of the input's diagonal entry
    // A(q[k], q[k]), or -1 when the input has none (the factor shift of the
    // escalation ladder adds to it).
    std::vector<int> a_diag;

    // Row-major copies for the triangular solves, rows stored in level
    // order: strict-L row fwd_order[idx] is [lrp[idx], lrp[idx+1]) of lci
    // (column positions ascending); strict-U row bwd_order[idx] likewise in
    // urp/uci.  fwd_lev / bwd_lev: first idx of each level (+ end).
    std::vector<int> lrp, lci;
    std::vector<int> urp, uci;
    // slot -> destination: L slots -> index in the L rows, U slots -> index
    // in the U rows, diagonal slot -> k; -1 for entries of the dense
    // trailing block (not in the row-major copies).
    std::vector<int> slot_dst;
    std::vector<int> fwd_order, bwd_order;   // level-sorted row orders
    std::vector<int> fwd_lev, bwd_lev;
    int nfwd_levels = 0, nbwd_levels = 0;
    int nfwd_steps = 0, nbwd_steps = 0;      // sweep steps (descriptors): levels,
                                             // with runs of narrow levels merged
    std::vector<int> bwd_pos;                // row -> index in bwd_order
    // Level descriptors of the sweeps: nlev x {first row idx, end row idx,
    // first entry, end entry}, then nlev x log2(lanes per row).
    std::vector<int> fwd_ldesc, bwd_ldesc;
    int lev_max_ent = 0, lev_max_rows = 0;  // widest level of either sweep

    // SELL-C-sigma copy of A in position space (C = 32): slice s covers
    // sorted rows [32 s, 32 s + 32); entry (r, t) of slice s is at
    // sell_ptr[s] + 32 t + r.  sell_perm[32 s + r] = row position (-1 pad),
    // sell_col = column position, sell_src = input index (-1 pad).
    int sell_sigma = 256;
    int nslices = 0;
    std::vector<int> sell_ptr, sell_col, sell_src, sell_perm;

    int max_col = 0;                // longest merged column (slots)
    long flops = 0;                 // multiply-adds of one refactorization
    long gathered = 0;              // sum over deps of |L(:,j)| (entries)

    // Relative slots of the refactorization updates: for column k, for each
    // dependency j (rows of U(:,k) ascending), for each strict-L entry of
    // column j in storage order, the slot offset inside column k that the
    // entry updates.  Column k's list is rel[rel_ptr[k] .. rel_ptr[k+1]).
    // Empty when a column is longer than 65535 slots.
    std::vector<uint16_t> rel;
    std::vector<long long> rel_ptr;
    // For each U slot p of column k (row j): {dg[j] + 1, cp[j+1] - dg[j] - 1},
    // the strict-L part of the dependency column (2 ints per slot, all slots).
    std::vector<int> dep_bc;

    // Dense trailing block: rows and columns [k0, n) are refactored and
    // solved as one dense D x D block (D = dtail = n - k0; 0 = none).  The
    // sweep orders then list the rows < k0 level-sorted, followed by the
    // tail rows in ascending order; the forward sweep has one more level,
    // the tail rows' entries in the columns before k0.
    int k0 = 0, dtail = 0;
};

// Largest dense trailing block.
constexpr int kMaxDenseTail = 768;

// Build the static layout from a pivot factorization.  Ap/Ai is the same
// CSC (original indices) the factorization consumed.
// dense_tail: -1 chooses the trailing block size by a cost model, 0 none,
// > 0 that many trailing columns (at most kMaxDenseTail and n).
void build_static_pattern(int n, const int* Ap, const int* Ai, const int* q,
                          const PivotFactor& F, int sell_sigma, StaticPattern& S,
                          int dense_tail = -1);

// Trailing block size the cost model picks for a merged pattern whose
// columns, levels and update counts are already set.
int choose_dense_tail(const StaticPattern& S);

uint64_t pattern_hash(int n, const int* Ap, const int* Ai, const int* q);

// Column approximate minimum degree ordering (our own implementation of the
// published COLAMD algorithm).  dense_row / dense_col: knob values as in
// COLAMD's knobs[0..1] (0 -> threshold 16).  Returns 0 on success.
int colamd_order(int n_row, int n_col, const int* Ap, const int* Ai,
                 double knob_dense_row, double knob_dense_col, int* q_out);

}  // namespace lusp
