// Supernodal numeric Cholesky factorization of the H1 metric (the reference preconditioner's
// factor, src/SimplicialMesh/H1Metric.hpp:171-257 with the ordering of
// NestedDissectionOrdering.hpp:3-207), shared by the host (threads over the supernodes of a
// level) and the device (one CTA per supernode of a level, rpb_solver.cu).
//
// Symbolic part (host): the elimination tree, the column structures of L, fundamental
// supernodes (column j + 1 continues the supernode of j when parent(j) = j + 1 and the
// structure of j + 1 is that of j without j) of at most max_width columns, and for every
// supernode J the list of supernodes K whose structure reaches J's columns (the updates it
// receives, in ascending K). Supernode J is stored as a dense column-major panel of its
// structure rows R_J (sorted; its own columns first) x its w columns.
//
// Numeric part, per supernode J in an order where every K that updates J is done first
// (levels of the supernodal elimination tree): for every K in J's list, subtract
// L_K(rows >= c0_J) L_K(rows in [c0_J, c1_J))^T from the matching panel entries of J (the
// rows are located by binary search in R_J); then factor the panel column by column
// (square root of the pivot, scale the column, update the later columns). All loops are
// written over a thread index and a thread count with a barrier between dependent phases,
// so the same code runs on one host thread or on a CTA.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "sparse_cholesky.hpp"

#if defined(__CUDACC__)
#define RPB_HD __host__ __device__
#else
#define RPB_HD
#endif

namespace rpb {

struct SupernodalSymbolic {
    int n = 0, nsn = 0;
    std::vector<int> perm;               // perm[new] = old
    std::vector<int> sn_begin;           // nsn + 1 column offsets
    std::vector<int> sn_of;              // column -> supernode
    std::vector<int64_t> rows_rp;        // nsn + 1 offsets into rows
    std::vector<int> rows;               // structure rows of every supernode (its own columns first)
    std::vector<int64_t> panel_off;      // nsn + 1 offsets of the dense panels (rows x w doubles)
    std::vector<int> upd_rp, upd_k;      // supernodes updating each supernode (ascending)
    std::vector<int> level_ptr, level_sn;  // supernodes by level of the supernodal elimination tree
    // entries of C = P A P^T with row <= column (CSC), scattered into the panels as L's lower part
    std::vector<int64_t> Cp;
    std::vector<int> Ci;
    std::vector<double> Cx;
};

std::string supernodal_symbolic(const CsrMatrix& A, const std::vector<int>& perm, int max_width,
                                SupernodalSymbolic& S);

// Host numeric factorization (supernodes of a level over `threads` host threads); panels
// sized panel_off[nsn]. Returns "" or the reason it failed.
std::string supernodal_numeric_host(const SupernodalSymbolic& S, std::vector<double>& panels, int threads);

// The factor in the row and column forms of CholeskyFactor from the panels.
void supernodal_to_factor(const SupernodalSymbolic& S, const std::vector<double>& panels, CholeskyFactor& F);

// Raw view of the symbolic arrays and the panels (host or device pointers).
struct SnView {
    const int* sn_begin;
    const int64_t* rows_rp;
    const int* rows;
    const int64_t* panel_off;
    const int* upd_rp;
    const int* upd_k;
    double* panels;
};

// first position p in [lo, hi) with a[p] >= key (hi when none)
RPB_HD inline int sn_lower_bound(const int* a, int lo, int hi, int key)
{
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Entry k of C (row i <= column j, i.e. L(j, i) of the lower factor) added into its panel.
// Returns false if the row is not in the structure (a broken symbolic analysis).
RPB_HD inline bool sn_scatter_entry(const SnView& v, const int* sn_of, int i, int j, double x)
{
    const int I = sn_of[i];
    const int c0 = v.sn_begin[I];
    const int64_t r0 = v.rows_rp[I];
    const int nr = static_cast<int>(v.rows_rp[I + 1] - r0);
    const int* R = v.rows + r0;
    const int pos = sn_lower_bound(R, i - c0, nr, j);
    if (pos >= nr || R[pos] != j) return false;
    v.panels[v.panel_off[I] + static_cast<int64_t>(i - c0) * nr + pos] += x;
    return true;
}

// Positions of K's structure rows inside J: the rows of K in [c0_J, c1_J) are K's positions
// [p1, p2), all its rows from c0_J on are [p1, nrK).
RPB_HD inline void sn_update_range(const SnView& v, int J, int K, int& p1, int& p2)
{
    const int wK = v.sn_begin[K + 1] - v.sn_begin[K];
    const int64_t q0 = v.rows_rp[K];
    const int nrK = static_cast<int>(v.rows_rp[K + 1] - q0);
    p1 = sn_lower_bound(v.rows + q0, wK, nrK, v.sn_begin[J]);
    p2 = sn_lower_bound(v.rows + q0, p1, nrK, v.sn_begin[J + 1]);
}

// Subtracts L_K(rows >= c0_J) L_K(rows in [c0_J, c1_J))^T from J's panel, one entry per
// (row, column) pair with the pairs strided over the threads. Returns 1 if a row of K is not
// in J's structure.
RPB_HD inline int sn_apply_update(const SnView& v, int J, int K, int tid, int nth)
{
    const int c0 = v.sn_begin[J];
    const int64_t r0 = v.rows_rp[J];
    const int nr = static_cast<int>(v.rows_rp[J + 1] - r0);
    const int* R = v.rows + r0;
    double* P = v.panels + v.panel_off[J];
    const int wK = v.sn_begin[K + 1] - v.sn_begin[K];
    const int64_t q0 = v.rows_rp[K];
    const int nrK = static_cast<int>(v.rows_rp[K + 1] - q0);
    const int* RK = v.rows + q0;
    const double* PK = v.panels + v.panel_off[K];
    int p1, p2;
    sn_update_range(v, J, K, p1, p2);
    const int na = nrK - p1, nb = p2 - p1;
    const int64_t pairs = static_cast<int64_t>(na) * nb;
    int status = 0;
    for (int64_t idx = tid; idx < pairs; idx += nth) {
        const int a = static_cast<int>(idx / nb), b = static_cast<int>(idx - static_cast<int64_t>(a) * nb);
        if (a < b) continue;
        double acc = 0.0;
        for (int t = 0; t < wK; ++t)
            acc += PK[static_cast<int64_t>(t) * nrK + p1 + a] * PK[static_cast<int64_t>(t) * nrK + p1 + b];
        const int col = RK[p1 + b] - c0;
        const int row = sn_lower_bound(R, col, nr, RK[p1 + a]);
        if (row >= nr || R[row] != RK[p1 + a]) {
            status = 1;
            continue;
        }
        P[static_cast<int64_t>(col) * nr + row] -= acc;
    }
    return status;
}

// Factors J's panel after all its updates: column by column, the pivot's square root, the
// column scaled, the later columns updated (each thread owns rows). Returns 0, or 2 for a
// non-positive pivot (every thread returns it together).
template <typename Barrier>
RPB_HD int sn_factor_panel(const SnView& v, int J, int tid, int nth, Barrier bar)
{
    const int c0 = v.sn_begin[J], c1 = v.sn_begin[J + 1], w = c1 - c0;
    const int64_t r0 = v.rows_rp[J];
    const int nr = static_cast<int>(v.rows_rp[J + 1] - r0);
    double* P = v.panels + v.panel_off[J];
    for (int c = 0; c < w; ++c) {
        double* Pc = P + static_cast<int64_t>(c) * nr;
        if (tid == 0) {
            const double d = Pc[c];
            Pc[c] = d > 0.0 ? sqrt(d) : -1.0;
        }
        bar();
        const double d = Pc[c];
        if (!(d > 0.0)) return 2;
        const double inv = 1.0 / d;
        for (int r = c + 1 + tid; r < nr; r += nth) Pc[r] *= inv;
        bar();
        for (int r = c + 1 + tid; r < nr; r += nth) {
            const double lrc = Pc[r];
            const int cmax = r < w ? r : w - 1;
            for (int cc = c + 1; cc <= cmax; ++cc) P[static_cast<int64_t>(cc) * nr + r] -= lrc * Pc[cc];
        }
        bar();
    }
    return 0;
}

// Factor supernode J: its updates in list order, then its panel. Returns 0, 1 (a row not
// found: broken structure) or 2 (a non-positive pivot).
template <typename Barrier>
RPB_HD int sn_factor_one(const SnView& v, int J, int tid, int nth, Barrier bar)
{
    int status = 0;
    for (int u = v.upd_rp[J]; u < v.upd_rp[J + 1]; ++u) {
        status |= sn_apply_update(v, J, v.upd_k[u], tid, nth);
        bar();
    }
    const int st = sn_factor_panel(v, J, tid, nth, bar);
    return st ? st : status;
}

}  // namespace rpb
