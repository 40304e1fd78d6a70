// Supernodal Cholesky of the H1 metric: symbolic analysis, host numeric factorization and
// conversion to the row / column forms of CholeskyFactor (see supernodal_chol.hpp).
#include "supernodal_chol.hpp"

#include <algorithm>
#include <atomic>
#include <thread>

namespace rpb {

std::string supernodal_symbolic(const CsrMatrix& A, const std::vector<int>& perm, int max_width,
                                SupernodalSymbolic& S)
{
    const int n = A.n;
    if (n <= 0 || static_cast<int>(perm.size()) != n) return "supernodal Cholesky: bad matrix or ordering";
    max_width = std::max(1, max_width);
    S = SupernodalSymbolic();
    S.n = n;
    S.perm = perm;
    std::vector<int> pinv(n);
    for (int i = 0; i < n; ++i) pinv[perm[i]] = i;
    // C = P A P^T, entries with row <= column, by columns
    S.Cp.assign(static_cast<size_t>(n) + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int64_t p = A.rp[r]; p < A.rp[r + 1]; ++p)
            if (pinv[r] <= pinv[A.ci[p]]) S.Cp[pinv[A.ci[p]] + 1]++;
    for (int j = 0; j < n; ++j) S.Cp[j + 1] += S.Cp[j];
    S.Ci.resize(static_cast<size_t>(S.Cp[n]));
    S.Cx.resize(static_cast<size_t>(S.Cp[n]));
    {
        std::vector<int64_t> pos(S.Cp.begin(), S.Cp.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int64_t p = A.rp[r]; p < A.rp[r + 1]; ++p) {
                const int i = pinv[r], j = pinv[A.ci[p]];
                if (i <= j) {
                    S.Ci[pos[j]] = i;
                    S.Cx[pos[j]++] = A.val[p];
                }
            }
    }
    const std::vector<int64_t>& Cp = S.Cp;
    const std::vector<int>& Ci = S.Ci;
    // elimination tree (path compression by ancestors)
    std::vector<int> parent(n, -1), ancestor(n, -1);
    for (int k = 0; k < n; ++k)
        for (int64_t p = Cp[k]; p < Cp[k + 1]; ++p) {
            int i = Ci[p];
            while (i != -1 && i < k) {
                const int inext = ancestor[i];
                ancestor[i] = k;
                if (inext == -1) parent[i] = k;
                i = inext;
            }
        }
    // column counts from the row structures (the reach of row k in the elimination tree)
    std::vector<int> mark(n, -1), stack(n);
    std::vector<int> colcount(n, 1);
    for (int k = 0; k < n; ++k) {
        mark[k] = k;
        for (int64_t p = Cp[k]; p < Cp[k + 1]; ++p)
            for (int i = Ci[p]; i < k && mark[i] != k; i = parent[i]) {
                mark[i] = k;
                colcount[i]++;
            }
    }
    // fundamental supernodes of at most max_width columns
    std::vector<int> begin;
    for (int j = 0; j < n; ++j) {
        const bool cont = j > 0 && parent[j - 1] == j && colcount[j - 1] == colcount[j] + 1 &&
                          j - begin.back() < max_width;
        if (!cont) begin.push_back(j);
    }
    begin.push_back(n);
    const int nsn = static_cast<int>(begin.size()) - 1;
    S.nsn = nsn;
    S.sn_begin = begin;
    S.sn_of.resize(n);
    for (int s = 0; s < nsn; ++s)
        for (int j = begin[s]; j < begin[s + 1]; ++j) S.sn_of[j] = s;
    // structure of each supernode = structure of its first column: the rows k whose reach
    // contains that column, ascending
    S.rows_rp.assign(static_cast<size_t>(nsn) + 1, 0);
    for (int s = 0; s < nsn; ++s) S.rows_rp[s + 1] = S.rows_rp[s] + colcount[begin[s]];
    S.rows.assign(static_cast<size_t>(S.rows_rp[nsn]), 0);
    std::vector<int64_t> fill(S.rows_rp.begin(), S.rows_rp.end() - 1);
    std::vector<char> first(n, 0);
    for (int s = 0; s < nsn; ++s) first[begin[s]] = 1;
    std::fill(mark.begin(), mark.end(), -1);
    for (int k = 0; k < n; ++k) {
        mark[k] = k;
        if (first[k]) S.rows[fill[S.sn_of[k]]++] = k;   // the diagonal first
        for (int64_t p = Cp[k]; p < Cp[k + 1]; ++p)
            for (int i = Ci[p]; i < k && mark[i] != k; i = parent[i]) {
                mark[i] = k;
                if (first[i]) S.rows[fill[S.sn_of[i]]++] = k;
            }
    }
    for (int s = 0; s < nsn; ++s) {
        if (fill[s] != S.rows_rp[s + 1]) return "supernodal Cholesky: structure count mismatch";
        // a supernode's own columns lead its structure (fundamental supernodes nest)
        for (int t = 0; t < begin[s + 1] - begin[s]; ++t)
            if (S.rows[S.rows_rp[s] + t] != begin[s] + t) return "supernodal Cholesky: supernode structure does not nest";
    }
    S.panel_off.assign(static_cast<size_t>(nsn) + 1, 0);
    for (int s = 0; s < nsn; ++s)
        S.panel_off[s + 1] = S.panel_off[s] + (S.rows_rp[s + 1] - S.rows_rp[s]) * (begin[s + 1] - begin[s]);
    // updates: K -> every supernode its external rows fall into; levels of the supernodal tree
    std::vector<std::vector<int>> upd(nsn);
    std::vector<int> level(nsn, 0);
    for (int K = 0; K < nsn; ++K) {
        const int w = begin[K + 1] - begin[K];
        int last = -1;
        for (int64_t p = S.rows_rp[K] + w; p < S.rows_rp[K + 1]; ++p) {
            const int J = S.sn_of[S.rows[p]];
            if (J != last) {
                upd[J].push_back(K);
                level[J] = std::max(level[J], level[K] + 1);
                last = J;
            }
        }
    }
    S.upd_rp.assign(static_cast<size_t>(nsn) + 1, 0);
    for (int J = 0; J < nsn; ++J) S.upd_rp[J + 1] = S.upd_rp[J] + static_cast<int>(upd[J].size());
    S.upd_k.reserve(static_cast<size_t>(S.upd_rp[nsn]));
    for (int J = 0; J < nsn; ++J) S.upd_k.insert(S.upd_k.end(), upd[J].begin(), upd[J].end());
    int L = 0;
    for (int s = 0; s < nsn; ++s) L = std::max(L, level[s] + 1);
    S.level_ptr.assign(static_cast<size_t>(L) + 1, 0);
    for (int s = 0; s < nsn; ++s) S.level_ptr[level[s] + 1]++;
    for (int l = 0; l < L; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
    S.level_sn.resize(nsn);
    std::vector<int> pos(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int s = 0; s < nsn; ++s) S.level_sn[pos[level[s]]++] = s;
    return std::string();
}

namespace {
template <typename F>
void run_pool(int n, F&& f)
{
    if (n <= 1) { f(0); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < n; ++t) th.emplace_back([&, t] { f(t); });
    for (auto& x : th) x.join();
}
}  // namespace

std::string supernodal_numeric_host(const SupernodalSymbolic& S, std::vector<double>& panels, int threads)
{
    panels.assign(static_cast<size_t>(S.panel_off[S.nsn]), 0.0);
    SnView v{S.sn_begin.data(), S.rows_rp.data(), S.rows.data(), S.panel_off.data(), S.upd_rp.data(),
             S.upd_k.data(), panels.data()};
    for (int j = 0; j < S.n; ++j)
        for (int64_t p = S.Cp[j]; p < S.Cp[j + 1]; ++p)
            if (!sn_scatter_entry(v, S.sn_of.data(), S.Ci[p], j, S.Cx[p]))
                return "supernodal Cholesky: an entry of H1 outside the structure";
    std::atomic<int> bad{0};
    const int L = static_cast<int>(S.level_ptr.size()) - 1;
    for (int l = 0; l < L && bad.load() == 0; ++l) {
        const int b = S.level_ptr[l], e = S.level_ptr[l + 1];
        std::atomic<int> ticket{b};
        run_pool(std::max(1, std::min(threads, e - b)), [&](int) {
            for (;;) {
                const int q = ticket.fetch_add(1);
                if (q >= e) break;
                const int st = sn_factor_one(v, S.level_sn[q], 0, 1, [] {});
                if (st != 0) bad.store(st);
            }
        });
    }
    if (bad.load() == 1) return "supernodal Cholesky: an update outside the structure";
    if (bad.load() == 2) return "H1 metric is not positive definite";
    return std::string();
}

void supernodal_to_factor(const SupernodalSymbolic& S, const std::vector<double>& panels, CholeskyFactor& F)
{
    const int n = S.n;
    const int threads = static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    F = CholeskyFactor();
    F.n = n;
    F.perm = S.perm;
    // column form (rows of L^T, diagonal first): column c0 + t of supernode s holds R_s[t:]
    F.upper_rp.assign(static_cast<size_t>(n) + 1, 0);
    for (int s = 0; s < S.nsn; ++s) {
        const int nr = static_cast<int>(S.rows_rp[s + 1] - S.rows_rp[s]);
        for (int j = S.sn_begin[s]; j < S.sn_begin[s + 1]; ++j) F.upper_rp[j + 1] = nr - (j - S.sn_begin[s]);
    }
    for (int j = 0; j < n; ++j) F.upper_rp[j + 1] += F.upper_rp[j];
    F.upper_ci.resize(static_cast<size_t>(F.upper_rp[n]));
    F.upper_val.resize(static_cast<size_t>(F.upper_rp[n]));
    {
        std::atomic<int> ticket{0};
        run_pool(threads, [&](int) {
            for (;;) {
                const int s0 = ticket.fetch_add(256);
                if (s0 >= S.nsn) break;
                for (int s = s0; s < std::min(S.nsn, s0 + 256); ++s) {
                    const int c0 = S.sn_begin[s];
                    const int nr = static_cast<int>(S.rows_rp[s + 1] - S.rows_rp[s]);
                    const int* R = S.rows.data() + S.rows_rp[s];
                    const double* P = panels.data() + S.panel_off[s];
                    for (int j = c0; j < S.sn_begin[s + 1]; ++j) {
                        const int t = j - c0;
                        int64_t o = F.upper_rp[j];
                        for (int r = t; r < nr; ++r, ++o) {
                            F.upper_ci[o] = R[r];
                            F.upper_val[o] = P[static_cast<int64_t>(t) * nr + r];
                        }
                    }
                }
            }
        });
    }
    // row form (rows of L, diagonal last): threads take contiguous column ranges, count their
    // entries per row, and write them after the entries of the ranges to their left, so every
    // row stays in ascending column order
    const int64_t nnz = F.upper_rp[n];
    std::vector<int> cut(static_cast<size_t>(threads) + 1, n);
    for (int t = 0; t < threads; ++t) {
        const int64_t target = nnz * t / threads;
        cut[t] = static_cast<int>(std::lower_bound(F.upper_rp.begin(), F.upper_rp.end() - 1, target) - F.upper_rp.begin());
    }
    cut[0] = 0;
    std::vector<std::vector<int64_t>> cnt(threads, std::vector<int64_t>(n, 0));
    run_pool(threads, [&](int t) {
        for (int j = cut[t]; j < cut[t + 1]; ++j)
            for (int64_t p = F.upper_rp[j]; p < F.upper_rp[j + 1]; ++p) cnt[t][F.upper_ci[p]]++;
    });
    F.lower_rp.assign(static_cast<size_t>(n) + 1, 0);
    for (int i = 0; i < n; ++i) {
        int64_t tot = 0;
        for (int t = 0; t < threads; ++t) {
            const int64_t c = cnt[t][i];
            cnt[t][i] = tot;   // offset of thread t's entries inside row i
            tot += c;
        }
        F.lower_rp[i + 1] = F.lower_rp[i] + tot;
    }
    F.lower_ci.resize(static_cast<size_t>(nnz));
    F.lower_val.resize(static_cast<size_t>(nnz));
    run_pool(threads, [&](int t) {
        std::vector<int64_t>& pos = cnt[t];
        for (int j = cut[t]; j < cut[t + 1]; ++j)
            for (int64_t p = F.upper_rp[j]; p < F.upper_rp[j + 1]; ++p) {
                const int i = F.upper_ci[p];
                const int64_t o = F.lower_rp[i] + pos[i]++;
                F.lower_ci[o] = j;
                F.lower_val[o] = F.upper_val[p];
            }
    });
}

}  // namespace rpb
