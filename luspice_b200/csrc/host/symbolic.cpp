// Host symbolic analysis: the pivoting fp64 factorization that fixes the row
// permutation and the structural L/U pattern, and the static device layout
// derived from it (merged columns, level schedules, row-major copies, value
// scatter maps, SELL-C-sigma copy of A).
//
// Build with -ffp-contract=off: the pivot decisions compare values, and the
// values must be computed with exactly the reference's operation sequence.
#include "lusp_host.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>

namespace lusp {

namespace {

// Depth-first search from original row j over the graph of L (node v has
// the edges L(:, pinv[v]) when v is pivoted).  Nodes are appended to
// xi[--top] in finishing order, so xi[top..n) is a topological order.  The
// stack lives in xi[0..head] and pstack; a node resumes its edge scan where
// it left off.  Same traversal as splu.h:77-106 (CSparse cs_dfs), which the
// pivot tie-breaks depend on.
int dfs_from(int j, const int* Lp, const int* Li, int top, int* xi,
             int* pstack, const int* pinv, unsigned char* mark) {
    int head = 0;
    xi[0] = j;
    while (head >= 0) {
        const int v = xi[head];
        const int col = pinv[v];
        if (!mark[v]) {
            mark[v] = 1;
            pstack[head] = (col < 0) ? 0 : Lp[col];
        }
        const int pend = (col < 0) ? 0 : Lp[col + 1];
        int pushed = 0;
        for (int p = pstack[head]; p < pend; p++) {
            const int w = Li[p];
            if (mark[w]) continue;
            pstack[head] = p;
            xi[++head] = w;
            pushed = 1;
            break;
        }
        if (!pushed) {
            head--;
            xi[--top] = v;
        }
    }
    return top;
}

}  // namespace

int pivot_factor(int n, const int* Ap, const int* Ai, const double* Ax,
                 const int* q, double tol, PivotFactor& F) {
    F.n = n;
    F.singular_col = -1;
    F.pinv.assign(n, -1);
    F.Lp.assign(n + 1, 0);
    F.Up.assign(n + 1, 0);
    const long nnz = Ap[n];
    long cap = 4 * nnz + n + 16;
    F.Li.resize(cap);
    F.Lx.resize(cap);
    F.Ui.resize(cap);
    F.Ux.resize(cap);
    std::vector<int> xi(2 * (size_t)n + 1);
    std::vector<unsigned char> mark(n, 0);
    std::vector<double> x(n, 0.0);
    int* pinv = F.pinv.data();
    long lnz = 0, unz = 0;

    for (int k = 0; k < n; k++) {
        F.Lp[k] = (int)lnz;
        F.Up[k] = (int)unz;
        if ((long)F.Li.size() < lnz + n + 1) {
            long nc = std::max<long>(2 * (long)F.Li.size(), lnz + n + 1);
            F.Li.resize(nc);
            F.Lx.resize(nc);
        }
        if ((long)F.Ui.size() < unz + n + 1) {
            long nc = std::max<long>(2 * (long)F.Ui.size(), unz + n + 1);
            F.Ui.resize(nc);
            F.Ux.resize(nc);
        }
        const int col = q ? q[k] : k;
        const int* Lp = F.Lp.data();
        const int* Li = F.Li.data();
        const double* Lx = F.Lx.data();

        // Reach of A(:,col) in the graph of L (splu.h:109-123).
        int top = n;
        for (int p = Ap[col]; p < Ap[col + 1]; p++) {
            if (!mark[Ai[p]])
                top = dfs_from(Ai[p], Lp, Li, top, xi.data(), xi.data() + n, pinv, mark.data());
        }
        for (int p = top; p < n; p++) mark[xi[p]] = 0;

        // Sparse triangular solve in topological order (splu.h:126-146).
        for (int p = top; p < n; p++) x[xi[p]] = 0.0;
        for (int p = Ap[col]; p < Ap[col + 1]; p++) x[Ai[p]] = Ax[p];
        for (int px = top; px < n; px++) {
            const int j = xi[px];
            const int J = pinv[j];
            if (J < 0) continue;
            const double xj = x[j];   // L(J,J) == 1: the division is exact
            for (int t = Lp[J] + 1; t < Lp[J + 1]; t++) x[Li[t]] -= Lx[t] * xj;
        }

        // Pivot: first strictly larger |x| in reach order; pivoted rows go
        // to U (splu.h:174-187).
        int ipiv = -1;
        double amax = -1.0;
        for (int p = top; p < n; p++) {
            const int i = xi[p];
            if (pinv[i] < 0) {
                const double t = std::fabs(x[i]);
                if (t > amax) { amax = t; ipiv = i; }
            } else {
                F.Ui[unz] = pinv[i];
                F.Ux[unz++] = x[i];
            }
        }
        if (ipiv == -1 || amax <= 0.0) {
            F.singular_col = k;
            F.Lp[n] = (int)lnz;
            F.Up[n] = (int)unz;
            return k;
        }
        if (pinv[col] < 0 && std::fabs(x[col]) >= amax * tol) ipiv = col;
        const double pivot = x[ipiv];
        F.Ui[unz] = k;
        F.Ux[unz++] = pivot;
        pinv[ipiv] = k;
        F.Li[lnz] = ipiv;
        F.Lx[lnz++] = 1.0;
        for (int p = top; p < n; p++) {
            const int i = xi[p];
            if (pinv[i] < 0) {
                F.Li[lnz] = i;
                F.Lx[lnz++] = x[i] / pivot;
            }
            x[i] = 0.0;
        }
    }
    F.Lp[n] = (int)lnz;
    F.Up[n] = (int)unz;
    for (long p = 0; p < lnz; p++) F.Li[p] = pinv[F.Li[p]];
    F.Li.resize(lnz);
    F.Lx.resize(lnz);
    F.Ui.resize(unz);
    F.Ux.resize(unz);
    return -1;
}

uint64_t pattern_hash(int n, const int* Ap, const int* Ai, const int* q) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](uint32_t v) {
        for (int b = 0; b < 4; b++) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    mix((uint32_t)n);
    for (int i = 0; i <= n; i++) mix((uint32_t)Ap[i]);
    for (int p = 0; p < Ap[n]; p++) mix((uint32_t)Ai[p]);
    mix(q ? 1u : 0u);
    if (q)
        for (int i = 0; i < n; i++) mix((uint32_t)q[i]);
    return h;
}

namespace {

// Level of each item, given its dependency lists (deps all earlier in
// `visit` order), then a stable counting sort by level.
void levels_and_order(int n, const std::vector<int>& visit,
                      const std::vector<int>& ptr, const std::vector<int>& dep,
                      std::vector<int>& level, std::vector<int>& order,
                      int& nlevels, std::vector<int>* level_ptr = nullptr) {
    level.assign(n, 0);
    int maxl = -1;
    for (int idx = 0; idx < n; idx++) {
        const int i = visit[idx];
        int l = 0;
        for (int p = ptr[i]; p < ptr[i + 1]; p++) l = std::max(l, level[dep[p]] + 1);
        level[i] = l;
        maxl = std::max(maxl, l);
    }
    nlevels = maxl + 1;
    std::vector<int> cnt(nlevels + 1, 0);
    for (int i = 0; i < n; i++) cnt[level[i] + 1]++;
    for (int l = 0; l < nlevels; l++) cnt[l + 1] += cnt[l];
    if (level_ptr) level_ptr->assign(cnt.begin(), cnt.end());
    order.assign(n, 0);
    for (int idx = 0; idx < n; idx++) {
        const int i = visit[idx];
        order[cnt[level[i]]++] = i;
    }
}

}  // namespace

// Trailing block size by a cost model in SM cycles of one refactor plus the
// triangular solves of one GMRES-IR solve (about six LU applications),
// fitted to measurements on B200: the sparse engine costs about a cycle per
// gathered update plus a latency per level of the column schedule (the
// solve sweeps have a similar depth and each application pays it twice);
// the dense block costs its multiply-subtract pairs (D^3 / 3; the two CTAs
// of the dense kernel's cluster share them), the solves' reads of the dense
// factor (D^2 per application) and a latency per column (the panel chain
// and the blocked solves).  Measured optima on B200 (50 systems, D in steps
// of 32): the n = 4050 grid 320, the n = 989 and n = 4000 analog circuits
// 96; the model picks those.
int choose_dense_tail(const StaticPattern& S) {
    const int n = S.n;
    if (n < 32) return 0;
    const double c_upd = 1.0, c_lev = 28000.0, c_cube = 0.02, c_sq = 20.0, c_lin = 2500.0;
    // Updates that stay in the sparse engine for a tail starting at k0:
    // those whose dependency column j lies before k0.  Column j feeds
    // |L(:,j)| updates into each of the |U(j,:)| later columns.
    std::vector<long> urow(n, 0);
    for (int k = 0; k < n; k++)
        for (int p = S.cp[k]; p < S.dg[k]; p++) urow[S.ri[p]]++;
    std::vector<double> inside(n + 1, 0.0);   // updates with j >= k0
    for (int j = n - 1; j >= 0; j--)
        inside[j] = inside[j + 1] + (double)(S.cp[j + 1] - S.dg[j] - 1) * (double)urow[j];
    std::vector<int> levmax(n + 1, 0);        // levels of the columns < k0
    for (int k = 0; k < n; k++) levmax[k + 1] = std::max(levmax[k], S.col_level[k] + 1);
    double best = c_upd * (double)S.gathered + c_lev * S.ncol_levels;
    int best_d = 0;
    for (int D = 32; D <= std::min(n, kMaxDenseTail); D += 32) {
        const int k0 = n - D;
        const double d = D;
        const double cost = c_upd * ((double)S.gathered - inside[k0]) + c_lev * levmax[k0] +
                            c_cube * d * d * d + c_sq * d * d + c_lin * d;
        if (cost < best) {
            best = cost;
            best_d = D;
        }
    }
    return best_d;
}

void build_static_pattern(int n, const int* Ap, const int* Ai, const int* q,
                          const PivotFactor& F, int sell_sigma, StaticPattern& S, int dense_tail) {
    S.n = n;
    S.nnz_a = Ap[n];
    S.lnnz = F.Lp[n];
    S.unnz = F.Up[n];
    S.cap = S.lnnz + S.unnz - n;
    S.hash = pattern_hash(n, Ap, Ai, q);
    S.q.resize(n);
    S.invq.resize(n);
    for (int k = 0; k < n; k++) S.q[k] = q ? q[k] : k;
    for (int k = 0; k < n; k++) S.invq[S.q[k]] = k;
    S.pinv = F.pinv;
    S.rowat.assign(n, -1);
    for (int i = 0; i < n; i++) S.rowat[S.pinv[i]] = i;

    // Merged columns, rows ascending.
    S.cp.assign(n + 1, 0);
    S.dg.assign(n, 0);
    S.ri.resize(S.cap);
    S.max_col = 0;
    {
        long pos = 0;
        std::vector<int> tmp;
        for (int k = 0; k < n; k++) {
            S.cp[k] = (int)pos;
            tmp.clear();
            for (int p = F.Up[k]; p < F.Up[k + 1] - 1; p++) tmp.push_back(F.Ui[p]);
            std::sort(tmp.begin(), tmp.end());
            for (int v : tmp) S.ri[pos++] = v;
            S.dg[k] = (int)pos;
            S.ri[pos++] = k;
            tmp.clear();
            for (int p = F.Lp[k] + 1; p < F.Lp[k + 1]; p++) tmp.push_back(F.Li[p]);
            std::sort(tmp.begin(), tmp.end());
            for (int v : tmp) S.ri[pos++] = v;
            S.max_col = std::max(S.max_col, (int)(pos - S.cp[k]));
        }
        S.cp[n] = (int)pos;
    }

    // Refactorization schedule: column k depends on the rows j < k of U(:,k)
    // (level.c:20-38 semantics), positions ascending are a topological order.
    {
        std::vector<int> ptr(n + 1), dep;
        dep.reserve(S.unnz);
        for (int k = 0; k < n; k++) {
            ptr[k] = (int)dep.size();
            for (int p = S.cp[k]; p < S.dg[k]; p++) dep.push_back(S.ri[p]);
        }
        ptr[n] = (int)dep.size();
        std::vector<int> visit(n);
        std::iota(visit.begin(), visit.end(), 0);
        // The claim order of the refactorization is the level order (any
        // topological order is safe: a warp waits only on columns claimed
        // before its own).  Measured on B200 (n = 4050 grid, 48 warps per
        // system): list schedules by longest remaining path, simulated on
        // 24, 48 or 96 warps, and level order with the longest path first
        // inside a level all refactor in the same time (2.22-2.28 ms); a
        // longest-path-first order without regard to time, which hands a
        // dependent chain to consecutive warps, takes 4.0 ms.
        levels_and_order(n, visit, ptr, dep, S.col_level, S.col_order, S.ncol_levels);
        long fl = 0, ga = 0;
        for (int k = 0; k < n; k++)
            for (int p = S.cp[k]; p < S.dg[k]; p++) {
                const int j = S.ri[p];
                const long lj = S.cp[j + 1] - S.dg[j] - 1;
                fl += lj;
                ga += lj;
            }
        S.flops = fl;
        S.gathered = ga;
    }

    // Dependency metadata per U slot.
    S.dep_bc.assign((size_t)S.cap * 2, 0);
    for (int k = 0; k < n; k++)
        for (int p = S.cp[k]; p < S.dg[k]; p++) {
            const int j = S.ri[p];
            S.dep_bc[(size_t)p * 2] = S.dg[j] + 1;
            S.dep_bc[(size_t)p * 2 + 1] = S.cp[j + 1] - S.dg[j] - 1;
        }

    // Relative update slots (16 bit), built through a row -> slot table of
    // the current column.
    S.rel.clear();
    S.rel_ptr.clear();
    if (S.max_col <= 65535) {
        S.rel.reserve((size_t)S.gathered);
        S.rel_ptr.assign(n + 1, 0);
        std::vector<int> at(n, -1);
        bool closed = true;
        for (int k = 0; k < n && closed; k++) {
            S.rel_ptr[k] = (long long)S.rel.size();
            for (int p = S.cp[k]; p < S.cp[k + 1]; p++) at[S.ri[p]] = p - S.cp[k];
            for (int p = S.cp[k]; p < S.dg[k]; p++) {
                const int j = S.ri[p];
                for (int t = S.dg[j] + 1; t < S.cp[j + 1]; t++) {
                    const int s = at[S.ri[t]];
                    if (s < 0) closed = false;   // pattern not closed under the updates
                    S.rel.push_back((uint16_t)s);
                }
            }
            for (int p = S.cp[k]; p < S.cp[k + 1]; p++) at[S.ri[p]] = -1;
        }
        S.rel_ptr[n] = (long long)S.rel.size();
        if (!closed) {
            S.rel.clear();
            S.rel_ptr.clear();
        }
    }

    // Dense trailing block.
    {
        int D = dense_tail < 0 ? choose_dense_tail(S) : dense_tail;
        D = std::max(0, std::min({D, n, kMaxDenseTail}));
        S.dtail = D;
        S.k0 = n - D;
    }

    // Row-major copies of strict L and strict U.  Entries inside the dense
    // trailing block (row and column >= k0) live only in the dense copy.
    {
        const int k0 = S.k0;
        auto kept = [k0](int i, int k) { return i < k0 || k < k0; };
        S.lrp.assign(n + 1, 0);
        S.urp.assign(n + 1, 0);
        for (int k = 0; k < n; k++) {
            for (int p = S.cp[k]; p < S.dg[k]; p++)
                if (kept(S.ri[p], k)) S.urp[S.ri[p] + 1]++;
            for (int p = S.dg[k] + 1; p < S.cp[k + 1]; p++)
                if (kept(S.ri[p], k)) S.lrp[S.ri[p] + 1]++;
        }
        for (int i = 0; i < n; i++) {
            S.lrp[i + 1] += S.lrp[i];
            S.urp[i + 1] += S.urp[i];
        }
        S.lci.resize(S.lrp[n]);
        S.uci.resize(S.urp[n]);
        S.slot_dst.assign(S.cap, -1);
        std::vector<int> lcur(S.lrp.begin(), S.lrp.end() - 1), ucur(S.urp.begin(), S.urp.end() - 1);
        // Columns visited in ascending k: each row's entries come out with
        // ascending column positions.
        for (int k = 0; k < n; k++) {
            for (int p = S.cp[k]; p < S.dg[k]; p++) {
                const int i = S.ri[p];
                if (!kept(i, k)) continue;
                const int d = ucur[i]++;
                S.uci[d] = k;
                S.slot_dst[p] = d;
            }
            S.slot_dst[S.dg[k]] = k;
            for (int p = S.dg[k] + 1; p < S.cp[k + 1]; p++) {
                const int i = S.ri[p];
                if (!kept(i, k)) continue;
                const int d = lcur[i]++;
                S.lci[d] = k;
                S.slot_dst[p] = d;
            }
        }
        // Sweep orders over the rows before the dense tail (all rows when
        // there is none); the tail rows follow in ascending order.
        // Forward levels: row i depends on the columns of its L row (< i).
        std::vector<int> visit(k0);
        std::iota(visit.begin(), visit.end(), 0);
        std::vector<int> lev;
        levels_and_order(k0, visit, S.lrp, S.lci, lev, S.fwd_order, S.nfwd_levels, &S.fwd_lev);
        // Backward levels: row i depends on the columns of its U row (> i)
        // that lie before the tail (the tail is solved first).
        std::vector<int> bptr(k0 + 1, 0), bdep;
        for (int i = 0; i < k0; i++) {
            for (int p = S.urp[i]; p < S.urp[i + 1]; p++)
                if (S.uci[p] < k0) bdep.push_back(S.uci[p]);
            bptr[i + 1] = (int)bdep.size();
        }
        std::vector<int> rvisit(k0);
        for (int i = 0; i < k0; i++) rvisit[i] = k0 - 1 - i;
        levels_and_order(k0, rvisit, bptr, bdep, lev, S.bwd_order, S.nbwd_levels, &S.bwd_lev);
        for (int i = k0; i < n; i++) {
            S.fwd_order.push_back(i);
            S.bwd_order.push_back(i);
        }
        // The tail rows' entries in the columns before k0 form one more
        // forward level (the dense forward solve follows it).
        if (k0 > 0 && k0 < n) {
            S.fwd_lev.push_back(n);
            S.nfwd_levels++;
        }
        // Store the rows contiguously in level order: row fwd_order[idx] of L
        // occupies [lrp[idx], lrp[idx+1]) (U likewise with bwd_order), so a
        // sweep streams through memory in the order it consumes it.
        auto relayout = [n](const std::vector<int>& order, std::vector<int>& rp, std::vector<int>& ci,
                            std::vector<int>& remap) {
            std::vector<int> nrp(n + 1, 0), nci(ci.size());
            remap.assign(ci.size(), -1);
            for (int idx = 0; idx < n; idx++) {
                const int i = order[idx];
                const int len = rp[i + 1] - rp[i];
                nrp[idx + 1] = nrp[idx] + len;
                for (int t = 0; t < len; t++) {
                    nci[nrp[idx] + t] = ci[rp[i] + t];
                    remap[rp[i] + t] = nrp[idx] + t;
                }
            }
            rp.swap(nrp);
            ci.swap(nci);
        };
        std::vector<int> lmap, umap;
        relayout(S.fwd_order, S.lrp, S.lci, lmap);
        relayout(S.bwd_order, S.urp, S.uci, umap);
        for (int k = 0; k < n; k++) {
            for (int p = S.cp[k]; p < S.dg[k]; p++)
                if (S.slot_dst[p] >= 0) S.slot_dst[p] = umap[S.slot_dst[p]];
            for (int p = S.dg[k] + 1; p < S.cp[k + 1]; p++)
                if (S.slot_dst[p] >= 0) S.slot_dst[p] = lmap[S.slot_dst[p]];
        }
        // Sweep steps of both sweeps, one descriptor each: first row, end
        // row, first entry, end entry, and log2 of the lanes per row (the
        // power of two at or above the step's mean row length, at most 512:
        // above 32, several warps share a row when the step has few rows).
        // A run of at least two consecutive levels of at most kChainRows
        // rows each becomes one step processed by a single warp, its rows in
        // level order (lanes log2 = -1): the warp finishes a row before it
        // reads it, so the run costs no CTA barrier per level.  A run stops
        // at kChainMaxRows rows or kChainMaxEnt entries (so it fits a stage).
        constexpr int kChainRows = 3, kChainMaxRows = 128, kChainMaxEnt = 1024;
        auto level_desc = [](int nlev, const std::vector<int>& lev, const std::vector<int>& rp,
                             std::vector<int>& out) {
            std::vector<std::array<int, 5>> steps;
            auto narrow = [&](int l) { return lev[l + 1] - lev[l] <= kChainRows; };
            for (int l = 0; l < nlev;) {
                if (narrow(l)) {
                    int l2 = l;
                    while (l2 < nlev && narrow(l2) && lev[l2 + 1] - lev[l] <= kChainMaxRows &&
                           rp[lev[l2 + 1]] - rp[lev[l]] <= kChainMaxEnt)
                        l2++;
                    if (l2 - l >= 2) {
                        steps.push_back({lev[l], lev[l2], rp[lev[l]], rp[lev[l2]], -1});
                        l = l2;
                        continue;
                    }
                }
                const int r0 = lev[l], r1 = lev[l + 1];
                const int e0 = rp[r0], e1 = rp[r1];
                const int nr = std::max(1, r1 - r0);
                const int mean = (e1 - e0 + nr - 1) / nr;
                int lg = 0;
                while ((1 << lg) < mean && lg < 9) lg++;
                steps.push_back({r0, r1, e0, e1, lg});
                l++;
            }
            const int ns = (int)steps.size();
            out.assign((size_t)ns * 5, 0);
            for (int t = 0; t < ns; t++) {
                for (int j = 0; j < 4; j++) out[(size_t)t * 4 + j] = steps[t][j];
                out[(size_t)ns * 4 + t] = steps[t][4];
            }
            return ns;
        };
        S.nfwd_steps = level_desc(S.nfwd_levels, S.fwd_lev, S.lrp, S.fwd_ldesc);
        S.nbwd_steps = level_desc(S.nbwd_levels, S.bwd_lev, S.urp, S.bwd_ldesc);
        // Position of each row in the backward order, and the widest level
        // of either sweep (entries, rows) for the shared-memory stages.
        S.bwd_pos.assign(n, 0);
        for (int idx = 0; idx < n; idx++) S.bwd_pos[S.bwd_order[idx]] = idx;
        S.lev_max_ent = 0;
        S.lev_max_rows = 0;
        for (int pass = 0; pass < 2; pass++) {
            const std::vector<int>& d = pass ? S.bwd_ldesc : S.fwd_ldesc;
            const int ns = pass ? S.nbwd_steps : S.nfwd_steps;
            for (int t = 0; t < ns; t++) {
                S.lev_max_ent = std::max(S.lev_max_ent, d[(size_t)t * 4 + 3] - d[(size_t)t * 4 + 2]);
                S.lev_max_rows = std::max(S.lev_max_rows, d[(size_t)t * 4 + 1] - d[(size_t)t * 4 + 0]);
            }
        }
    }

    // Input entries -> slots (column k = invq[c], row = pinv[orig row]).
    {
        S.a_ptr.assign(n + 1, 0);
        for (int c = 0; c < n; c++) S.a_ptr[S.invq[c] + 1] += Ap[c + 1] - Ap[c];
        for (int k = 0; k < n; k++) S.a_ptr[k + 1] += S.a_ptr[k];
        S.a_src.resize(S.nnz_a);
        S.a_dst.resize(S.nnz_a);
        S.a_diag.assign(n, -1);
        std::vector<std::pair<int, int>> tmp;
        for (int k = 0; k < n; k++) {
            const int c = S.q[k];
            tmp.clear();
            const int* rb = S.ri.data() + S.cp[k];
            const int len = S.cp[k + 1] - S.cp[k];
            for (int p = Ap[c]; p < Ap[c + 1]; p++) {
                const int r = S.pinv[Ai[p]];
                const int* it = std::lower_bound(rb, rb + len, r);
                tmp.emplace_back((int)(it - rb), p);
                if (Ai[p] == c) S.a_diag[k] = (int)(it - rb);
            }
            // By slot, input order within a slot (the second members are the
            // input positions, ascending as appended, so sorting the pairs is
            // the stable order without a merge buffer).
            std::sort(tmp.begin(), tmp.end());
            int o = S.a_ptr[k];
            for (auto& e : tmp) {
                S.a_dst[o] = e.first;
                S.a_src[o] = e.second;
                o++;
            }
        }
    }

    // SELL-C-sigma (C = 32) copy of A in position space.
    {
        const int C = 32;
        S.sell_sigma = std::max(C, sell_sigma);
        // Row r (position) holds the input entries of original row rowat[r].
        std::vector<int> rlen(n, 0);
        for (int c = 0; c < n; c++)
            for (int p = Ap[c]; p < Ap[c + 1]; p++) rlen[S.pinv[Ai[p]]]++;
        std::vector<int> rptr(n + 1, 0);
        for (int r = 0; r < n; r++) rptr[r + 1] = rptr[r] + rlen[r];
        std::vector<int> rcol(S.nnz_a), rsrc(S.nnz_a);
        {
            std::vector<int> cur(rptr.begin(), rptr.end() - 1);
            for (int k = 0; k < n; k++) {
                const int c = S.q[k];
                for (int p = Ap[c]; p < Ap[c + 1]; p++) {
                    const int r = S.pinv[Ai[p]];
                    const int d = cur[r]++;
                    rcol[d] = k;
                    rsrc[d] = p;
                }
            }
        }
        // Sort rows by descending length inside windows of sigma rows.
        std::vector<int> perm(n);
        std::iota(perm.begin(), perm.end(), 0);
        for (int w0 = 0; w0 < n; w0 += S.sell_sigma) {
            const int w1 = std::min(n, w0 + S.sell_sigma);
            std::stable_sort(perm.begin() + w0, perm.begin() + w1,
                             [&rlen](int a, int b) { return rlen[a] > rlen[b]; });
        }
        S.nslices = (n + C - 1) / C;
        S.sell_ptr.assign(S.nslices + 1, 0);
        S.sell_perm.assign((size_t)S.nslices * C, -1);
        for (int s = 0; s < S.nslices; s++) {
            int ml = 0;
            for (int r = 0; r < C; r++) {
                const int k = s * C + r;
                if (k < n) {
                    S.sell_perm[k] = perm[k];
                    ml = std::max(ml, rlen[perm[k]]);
                }
            }
            S.sell_ptr[s + 1] = S.sell_ptr[s] + ml * C;
        }
        const int total = S.sell_ptr[S.nslices];
        S.sell_col.assign(total, 0);
        S.sell_src.assign(total, -1);
        for (int s = 0; s < S.nslices; s++) {
            for (int r = 0; r < C; r++) {
                const int k = s * C + r;
                if (k >= n) continue;
                const int row = perm[k];
                for (int t = 0; t < rlen[row]; t++) {
                    S.sell_col[S.sell_ptr[s] + t * C + r] = rcol[rptr[row] + t];
                    S.sell_src[S.sell_ptr[s] + t * C + r] = rsrc[rptr[row] + t];
                }
                // Padding points at the row's own position: always a valid x.
                for (int t = rlen[row]; t < (S.sell_ptr[s + 1] - S.sell_ptr[s]) / C; t++)
                    S.sell_col[S.sell_ptr[s] + t * C + r] = row;
            }
        }
    }
}

}  // namespace lusp
