// Column approximate minimum degree ordering, written from the published
// COLAMD algorithm (Davis, Gilbert, Larimore, Ng, "A column approximate
// minimum degree ordering algorithm", ACM TOMS 30(3), 2004).
//
// The ordering is that of the Cholesky factor of A^T A, computed without
// forming A^T A: rows of A are the elements of a quotient graph.  Eliminating
// the pivot column merges every row that contains it into one new "pivot
// row" (an element); column scores are approximate external degrees
// (sum over the column's rows of |row \ pivot row|, plus |pivot row| minus
// the column's own weight); columns of the pivot row with identical row
// sets are merged into supercolumns and ordered together.
//
// Preprocessing follows the published knob semantics the reference relies on
// when it passes zero-initialised knobs (bench/test_lu.c:124,
// src/mp/mp_lu_bench.cu:139): rows with more than max(16, knob_row *
// sqrt(n_col)) entries are ignored, columns with more than max(16, knob_col *
// sqrt(min(n_row, n_col))) entries are ordered last, empty columns after
// them; aggressive row absorption is off.  Tie-breaking inside a score
// bucket is last-in-first-out.
#include "lusp_host.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace lusp {

namespace {

enum ColState : unsigned char { LIVE = 0, ORDERED = 1, MERGED = 2, DENSE = 3, EMPTY = 4 };

struct Buckets {
    std::vector<int> head, nxt, prv, score;
    int minscore = 0;
    explicit Buckets(int n) : head(n + 2, -1), nxt(n, -1), prv(n, -1), score(n, -1) {}
    void insert(int c, int s) {
        score[c] = s;
        prv[c] = -1;
        nxt[c] = head[s];
        if (head[s] >= 0) prv[head[s]] = c;
        head[s] = c;
        if (s < minscore) minscore = s;
    }
    void remove(int c) {
        const int s = score[c];
        if (s < 0) return;
        if (prv[c] >= 0) nxt[prv[c]] = nxt[c]; else head[s] = nxt[c];
        if (nxt[c] >= 0) prv[nxt[c]] = prv[c];
        score[c] = -1;
    }
    int pop_min() {
        const int top = (int)head.size();
        while (minscore < top && head[minscore] < 0) minscore++;
        if (minscore >= top) return -1;
        const int c = head[minscore];
        remove(c);
        return c;
    }
};

}  // namespace

int colamd_order(int n_row, int n_col, const int* Ap, const int* Ai,
                 double knob_dense_row, double knob_dense_col, int* q_out) {
    if (n_row < 0 || n_col < 0 || !Ap || !Ai || !q_out) return -1;
    if (n_col == 0) return 0;
    const int dense_row = std::max(16, (int)(knob_dense_row * std::sqrt((double)n_col)));
    const int dense_col =
        std::max(16, (int)(knob_dense_col * std::sqrt((double)std::min(n_row, n_col))));

    std::vector<std::vector<int>> col_rows(n_col);
    for (int c = 0; c < n_col; c++) {
        auto& v = col_rows[c];
        v.reserve(Ap[c + 1] - Ap[c] + 4);
        for (int p = Ap[c]; p < Ap[c + 1]; p++) {
            const int r = Ai[p];
            if (r < 0 || r >= n_row) return -2;
            v.push_back(r);
        }
        if (!std::is_sorted(v.begin(), v.end())) std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    std::vector<unsigned char> cstate(n_col, LIVE);
    std::vector<int> dense_cols, empty_cols;
    for (int c = 0; c < n_col; c++) {
        if (col_rows[c].empty()) { cstate[c] = EMPTY; empty_cols.push_back(c); }
        else if ((int)col_rows[c].size() > dense_col) { cstate[c] = DENSE; dense_cols.push_back(c); }
    }

    // Rows: one vector per original row plus one per pivot row to come.
    std::vector<std::vector<int>> row_cols;
    row_cols.reserve((size_t)n_row + n_col);
    row_cols.resize(n_row);
    {
        std::vector<int> cnt(n_row, 0);
        for (int c = 0; c < n_col; c++)
            if (cstate[c] == LIVE)
                for (int r : col_rows[c]) cnt[r]++;
        for (int r = 0; r < n_row; r++) row_cols[r].reserve(cnt[r]);
    }
    for (int c = 0; c < n_col; c++)
        if (cstate[c] == LIVE)
            for (int r : col_rows[c]) row_cols[r].push_back(c);
    std::vector<unsigned char> row_alive(n_row, 1);
    for (int r = 0; r < n_row; r++) {
        const int d = (int)row_cols[r].size();
        if (d == 0 || d > dense_row) row_alive[r] = 0;
    }
    for (int c = 0; c < n_col; c++) {
        if (cstate[c] != LIVE) continue;
        auto& v = col_rows[c];
        v.erase(std::remove_if(v.begin(), v.end(), [&](int r) { return !row_alive[r]; }), v.end());
        if (v.empty()) { cstate[c] = EMPTY; empty_cols.push_back(c); }
    }

    std::vector<int> col_w(n_col, 1);
    // Weighted live degree of every row.  It never changes while the row is
    // alive: a column is ordered only together with all its rows (they die
    // into the new pivot row), and merging a supercolumn moves weight
    // between two columns that share all their rows.
    std::vector<int> row_w(n_row);
    for (int r = 0; r < n_row; r++) row_w[r] = (int)row_cols[r].size();
    // Members of each supercolumn, a linked list in merge order.
    std::vector<int> mnext(n_col, -1), mtail(n_col);
    for (int c = 0; c < n_col; c++) mtail[c] = c;
    int remaining = 0;
    for (int c = 0; c < n_col; c++)
        if (cstate[c] == LIVE) remaining++;

    Buckets bk(n_col);
    for (int c = 0; c < n_col; c++) {
        if (cstate[c] != LIVE) continue;
        long s = 0;
        for (int r : col_rows[c]) s += (long)row_cols[r].size() - 1;
        s = std::min<long>(s, remaining - 1);
        bk.insert(c, (int)std::max<long>(s, 0));
    }

    std::vector<int> order;
    order.reserve(n_col);
    std::vector<int> cmark(n_col, 0), pivrow;
    std::vector<std::pair<unsigned long long, int>> hs;
    std::vector<int> rtag(n_row, 0), rdiff(n_row, 0);
    rtag.reserve((size_t)n_row + n_col);
    rdiff.reserve((size_t)n_row + n_col);
    row_alive.reserve((size_t)n_row + n_col);
    row_w.reserve((size_t)n_row + n_col);
    int tag = 0;

    while (remaining > 0) {
        const int c = bk.pop_min();
        if (c < 0) break;
        tag++;
        pivrow.clear();
        for (int r : col_rows[c]) {
            if (!row_alive[r]) continue;
            for (int j : row_cols[r]) {
                if (cstate[j] != LIVE || j == c || cmark[j] == tag) continue;
                cmark[j] = tag;
                pivrow.push_back(j);
            }
            row_alive[r] = 0;
        }
        cstate[c] = ORDERED;
        order.push_back(c);
        remaining -= col_w[c];
        col_rows[c].clear();
        if (pivrow.empty()) continue;

        const int e = (int)row_cols.size();
        row_cols.push_back(pivrow);
        row_alive.push_back(1);
        rtag.push_back(0);
        rdiff.push_back(0);
        int wP = 0;
        for (int j : pivrow) {
            wP += col_w[j];
            auto& v = col_rows[j];
            v.erase(std::remove_if(v.begin(), v.end(), [&](int r) { return !row_alive[r]; }), v.end());
            v.push_back(e);
        }
        row_w.push_back(wP);
        // |r \ pivot row| for every row meeting the pivot row's columns.
        for (int j : pivrow)
            for (int r : col_rows[j]) {
                if (r == e) continue;
                if (rtag[r] != tag) { rtag[r] = tag; rdiff[r] = row_w[r]; }
                rdiff[r] -= col_w[j];
            }
        for (int j : pivrow) {
            long s = wP - col_w[j];
            for (int r : col_rows[j])
                if (r != e) s += std::max(rdiff[r], 0);
            s = std::min<long>(s, (long)remaining - col_w[j]);
            s = std::max<long>(s, 0);
            bk.remove(j);
            bk.insert(j, (int)s);
        }
        // Supercolumns: identical row sets among the pivot row's columns.
        if (pivrow.size() > 1) {
            hs.clear();
            for (int j : pivrow) {
                auto& v = col_rows[j];
                // Already ascending in practice (a new pivot row carries the
                // largest row index so far and erasing keeps the order).
                if (!std::is_sorted(v.begin(), v.end())) std::sort(v.begin(), v.end());
                unsigned long long h = v.size();
                for (int r : v) h = h * 1000003ull + (unsigned)r;
                hs.emplace_back(h, j);
            }
            std::sort(hs.begin(), hs.end());
            for (size_t a = 0; a < hs.size();) {
                size_t b = a + 1;
                while (b < hs.size() && hs[b].first == hs[a].first) b++;
                for (size_t u = a; u < b; u++) {
                    const int j1 = hs[u].second;
                    if (cstate[j1] != LIVE) continue;
                    for (size_t w = u + 1; w < b; w++) {
                        const int j2 = hs[w].second;
                        if (cstate[j2] != LIVE) continue;
                        if (col_rows[j1] != col_rows[j2]) continue;
                        col_w[j1] += col_w[j2];
                        mnext[mtail[j1]] = j2;
                        mtail[j1] = mtail[j2];
                        cstate[j2] = MERGED;
                        bk.remove(j2);
                        col_rows[j2].clear();
                    }
                }
                a = b;
            }
        }
    }

    int pos = 0;
    for (int c : order)
        for (int m = c; m >= 0; m = mnext[m]) q_out[pos++] = m;
    for (int c : dense_cols) q_out[pos++] = c;
    for (int c : empty_cols) q_out[pos++] = c;
    return pos == n_col ? 0 : -3;
}

}  // namespace lusp
