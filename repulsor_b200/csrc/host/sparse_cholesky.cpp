// H1 metric, nested-dissection ordering and up-looking sparse Cholesky (host).
#include "sparse_cholesky.hpp"
#include "supernodal_chol.hpp"

#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdint>

namespace rpb {

CsrMatrix assemble_h1(int dom, const double* V, int nV, const int* S, int N, double ws, double wm)
{
    const int size = dom + 1;
    const double std_vol = (dom == 1) ? 1.0 : 0.5;       // 1/n!
    const double fact = (dom == 1) ? 6.0 : 24.0;         // (n+2)!
    const double m_factor = wm / (std_vol * fact);
    // triplets per simplex, then a row-wise merge
    std::vector<int64_t> cnt(static_cast<size_t>(nV) + 1, 0);
    for (int64_t k = 0; k < static_cast<int64_t>(N) * size; ++k) cnt[S[k] + 1] += size;
    for (int v = 0; v < nV; ++v) cnt[v + 1] += cnt[v];
    std::vector<int> tj(static_cast<size_t>(cnt[nV]));
    std::vector<double> tv(static_cast<size_t>(cnt[nV]));
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int k = 0; k < N; ++k) {
        const int* s = S + static_cast<int64_t>(size) * k;
        double df[3][2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < dom; ++j) df[i][j] = V[3 * static_cast<int64_t>(s[j + 1]) + i] - V[3 * static_cast<int64_t>(s[0]) + i];
        double g[2][2] = {{0, 0}, {0, 0}};
        for (int a = 0; a < dom; ++a)
            for (int b = 0; b < dom; ++b)
                for (int i = 0; i < 3; ++i) g[a][b] += df[i][a] * df[i][b];
        double a = std_vol, ginv[2][2] = {{0, 0}, {0, 0}};
        if (dom == 1) {
            a *= std::sqrt(g[0][0]);
            ginv[0][0] = 1.0 / g[0][0];
        } else {
            const double det = g[0][0] * g[1][1] - g[0][1] * g[1][0];
            a *= std::sqrt(det);
            ginv[0][0] = g[1][1] / det;
            ginv[1][1] = g[0][0] / det;
            ginv[0][1] = ginv[1][0] = -g[0][1] / det;
        }
        double val[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double lf = a * ws;
        for (int i = 0; i < dom; ++i)
            for (int j = 0; j < dom; ++j) {
                const double aij = lf * ginv[i][j];
                val[0][0] += aij;
                val[i + 1][0] -= aij;
                val[0][j + 1] -= aij;
                val[i + 1][j + 1] = aij;
            }
        for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j) val[i][j] += a * m_factor * (1.0 + (i == j ? 1.0 : 0.0));
        for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j) {
                const int64_t p = pos[s[i]]++;
                tj[p] = s[j];
                tv[p] = val[i][j];
            }
    }
    CsrMatrix A;
    A.n = nV;
    A.rp.assign(static_cast<size_t>(nV) + 1, 0);
    std::vector<std::pair<int, double>> row;
    for (int r = 0; r < nV; ++r) {
        row.clear();
        for (int64_t p = cnt[r]; p < cnt[r + 1]; ++p) row.emplace_back(tj[p], tv[p]);
        std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t q = 0; q < row.size(); ++q) {
            if (!A.ci.empty() && static_cast<int64_t>(A.ci.size()) > A.rp[r] && A.ci.back() == row[q].first) {
                A.val.back() += row[q].second;
            } else {
                A.ci.push_back(row[q].first);
                A.val.push_back(row[q].second);
            }
        }
        A.rp[r + 1] = static_cast<int64_t>(A.ci.size());
    }
    return A;
}

// NestedDissectionOrdering (src/SimplicialMesh/NestedDissectionOrdering.hpp:3-207): at
// each tree level the vertices of a cluster's range are grouped into those touching
// only left-child primitives, only right-child primitives, and both (separator, last).
std::vector<int> nested_dissection_ordering(const HostTree& T, const int* S, int nV)
{
    const int N = T.N, size = T.size;
    std::vector<int> perm0(nV), perm1(nV);
    for (int i = 0; i < nV; ++i) perm0[i] = i;
    std::vector<int> Vb(T.NC, 0), Ve(T.NC, 0);
    Vb[0] = 0;
    Ve[0] = nV;
    std::vector<int> queue0{0}, queue1;
    std::vector<unsigned char> vL(N), vR(N), wL(nV), wR(nV);
    std::vector<signed char> type(nV);
    while (!queue0.empty()) {
        queue1.clear();
        perm1 = perm0;
        std::fill(vL.begin(), vL.end(), 0);
        std::fill(vR.begin(), vR.end(), 0);
        for (int C : queue0) {
            const int L = T.C_left[C], R = T.C_right[C];
            if (L < 0) continue;
            for (int i = T.C_begin[L]; i < T.C_end[L]; ++i) vL[i] = 1;
            for (int i = T.C_begin[R]; i < T.C_end[R]; ++i) vR[i] = 1;
        }
        std::fill(wL.begin(), wL.end(), 0);
        std::fill(wR.begin(), wR.end(), 0);
        for (int i = 0; i < N; ++i) {
            if (!vL[i] && !vR[i]) continue;
            const int* s = S + static_cast<int64_t>(size) * T.perm[i];
            for (int l = 0; l < size; ++l) {
                if (vL[i]) wL[s[l]] = 1;
                if (vR[i]) wR[s[l]] = 1;
            }
        }
        for (int i = 0; i < nV; ++i) {
            const int j = perm0[i];
            type[i] = static_cast<signed char>(-1 + (wL[j] ? 1 : 0) + (wR[j] ? 2 : 0));
        }
        for (int C : queue0) {
            const int L = T.C_left[C], R = T.C_right[C];
            if (L < 0) continue;
            const int ib = Vb[C], ie = Ve[C];
            int ctr[3] = {0, 0, 0};
            for (int i = ib; i < ie; ++i)
                if (type[i] >= 0) ++ctr[type[i]];
            int pos[4];
            pos[0] = ib;
            pos[1] = pos[0] + ctr[0];
            pos[2] = pos[1] + ctr[1];
            pos[3] = pos[2] + ctr[2];
            if (ctr[0] > 0 && ctr[1] > 0 && pos[3] == ie) {
                Vb[L] = pos[0]; Ve[L] = pos[1];
                Vb[R] = pos[1]; Ve[R] = pos[2];
                queue1.push_back(L);
                queue1.push_back(R);
                for (int i = ib; i < ie; ++i) {
                    const int t = type[i];
                    if (t >= 0) perm1[pos[t]++] = perm0[i];
                }
            }
        }
        queue0.swap(queue1);
        perm0.swap(perm1);
    }
    return perm0;
}

std::string cholesky_factor(const CsrMatrix& A, const std::vector<int>& perm, CholeskyFactor& F)
{
    // supernodal factorization on host threads (host/supernodal_chol.hpp)
    SupernodalSymbolic S;
    std::string err = supernodal_symbolic(A, perm, kSupernodalWidth, S);
    if (!err.empty()) return err;
    std::vector<double> panels;
    err = supernodal_numeric_host(S, panels, static_cast<int>(std::max(1u, std::thread::hardware_concurrency())));
    if (!err.empty()) return err;
    supernodal_to_factor(S, panels, F);
    return std::string();
}

namespace {

// groups supernodes by level (levels[s] in 0..L-1) in ascending supernode order
void group_levels(const std::vector<int>& levels, const std::vector<int>& sn_begin, std::vector<int>& ptr,
                  std::vector<int>& sns, std::vector<int>& width)
{
    const int nsn = static_cast<int>(levels.size());
    int L = 0;
    for (int s = 0; s < nsn; ++s) L = std::max(L, levels[s] + 1);
    ptr.assign(static_cast<size_t>(L) + 1, 0);
    width.assign(static_cast<size_t>(L), 0);
    for (int s = 0; s < nsn; ++s) {
        ptr[levels[s] + 1]++;
        width[levels[s]] = std::max(width[levels[s]], sn_begin[s + 1] - sn_begin[s]);
    }
    for (int l = 0; l < L; ++l) ptr[l + 1] += ptr[l];
    sns.resize(static_cast<size_t>(nsn));
    std::vector<int> pos(ptr.begin(), ptr.end() - 1);
    for (int s = 0; s < nsn; ++s) sns[pos[levels[s]]++] = s;
}

}  // namespace

std::string supernodal_schedule(const CholeskyFactor& F, int max_width, SupernodalSchedule& out)
{
    const int n = F.n;
    if (n <= 0) return "empty factor";
    max_width = std::max(1, max_width);
    // elimination tree and column counts from the column form (diagonal first)
    std::vector<int> parent(n, -1), nchild(n, 0), cc(n);
    for (int j = 0; j < n; ++j) {
        cc[j] = static_cast<int>(F.upper_rp[j + 1] - F.upper_rp[j]);
        if (cc[j] > 1) parent[j] = F.upper_ci[F.upper_rp[j] + 1];
    }
    for (int j = 0; j < n; ++j)
        if (parent[j] >= 0) nchild[parent[j]]++;
    // fundamental supernodes
    std::vector<int> fb;
    for (int j = 0; j < n; ++j) {
        const bool merge = j > 0 && parent[j - 1] == j && nchild[j] == 1 && cc[j - 1] == cc[j] + 1;
        if (!merge) fb.push_back(j);
    }
    fb.push_back(n);
    const int nf = static_cast<int>(fb.size()) - 1;
    // single-child chains: supernode s+1 whose only child is s (contiguous in postorder)
    std::vector<int> fsn_of(n);
    for (int s = 0; s < nf; ++s)
        for (int j = fb[s]; j < fb[s + 1]; ++j) fsn_of[j] = s;
    std::vector<int> fparent(nf, -1), fnchild(nf, 0);
    for (int s = 0; s < nf; ++s) {
        const int p = parent[fb[s + 1] - 1];
        if (p >= 0) {
            fparent[s] = fsn_of[p];
            fnchild[fparent[s]]++;
        }
    }
    std::vector<int> sb;
    for (int s = 0; s < nf; ++s) {
        const bool chain = s > 0 && fparent[s - 1] == s && fnchild[s] == 1;
        if (!chain || fb[s + 1] - sb.back() > max_width) sb.push_back(fb[s]);
    }
    sb.push_back(n);
    // split ranges wider than max_width
    std::vector<int> begin;
    for (size_t s = 0; s + 1 < sb.size(); ++s)
        for (int c = sb[s]; c < sb[s + 1]; c += max_width) begin.push_back(c);
    begin.push_back(n);
    const int nsn = static_cast<int>(begin.size()) - 1;
    std::vector<int> sn_of(n);
    int maxw = 0;
    for (int s = 0; s < nsn; ++s) {
        for (int j = begin[s]; j < begin[s + 1]; ++j) sn_of[j] = s;
        maxw = std::max(maxw, begin[s + 1] - begin[s]);
    }
    // levels from the actual dependencies: forward reads columns < c0 of its rows of L,
    // backward reads rows >= c1 of its columns of L
    std::vector<int> lf(nsn, 0), lb(nsn, 0);
    for (int s = 0; s < nsn; ++s)
        for (int r = begin[s]; r < begin[s + 1]; ++r)
            for (int64_t k = F.lower_rp[r]; k < F.lower_rp[r + 1]; ++k) {
                const int j = F.lower_ci[k];
                if (j < begin[s]) lf[s] = std::max(lf[s], lf[sn_of[j]] + 1);
            }
    for (int s = nsn - 1; s >= 0; --s)
        for (int c = begin[s]; c < begin[s + 1]; ++c)
            for (int64_t k = F.upper_rp[c]; k < F.upper_rp[c + 1]; ++k) {
                const int r = F.upper_ci[k];
                if (r >= begin[s + 1]) lb[s] = std::max(lb[s], lb[sn_of[r]] + 1);
            }
    out = SupernodalSchedule();
    out.n = n;
    out.nsn = nsn;
    out.max_width = maxw;
    out.sn_begin = begin;
    group_levels(lf, begin, out.fwd_level_ptr, out.fwd_level_sn, out.fwd_level_width);
    group_levels(lb, begin, out.bwd_level_ptr, out.bwd_level_sn, out.bwd_level_width);
    // inverses of the dense diagonal blocks
    out.dinv_off.assign(static_cast<size_t>(nsn) + 1, 0);
    for (int s = 0; s < nsn; ++s) {
        const int64_t w = begin[s + 1] - begin[s];
        out.dinv_off[s + 1] = out.dinv_off[s] + w * (w + 1) / 2;
    }
    out.dinv.assign(static_cast<size_t>(out.dinv_off[nsn]), 0.0);
    out.dinvT.assign(static_cast<size_t>(out.dinv_off[nsn]), 0.0);
    // the blocks are independent: host threads take supernodes by ticket
    std::atomic<int> ticket{0}, zero_pivot{0};
    const int threads = static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    auto invert = [&](int) {
    std::vector<double> D, X;
    for (;;) {
        const int s = ticket.fetch_add(1);
        if (s >= nsn) break;
        const int c0 = begin[s], w = begin[s + 1] - c0;
        D.assign(static_cast<size_t>(w) * w, 0.0);
        for (int r = 0; r < w; ++r)
            for (int64_t k = F.lower_rp[c0 + r]; k < F.lower_rp[c0 + r + 1]; ++k) {
                const int j = F.lower_ci[k];
                if (j >= c0) D[static_cast<size_t>(r) * w + (j - c0)] = F.lower_val[k];
            }
        // X = D^{-1} by forward substitution, one unit column at a time (X lower triangular)
        X.assign(static_cast<size_t>(w) * w, 0.0);
        for (int c = 0; c < w; ++c) {
            for (int r = c; r < w; ++r) {
                double acc = (r == c) ? 1.0 : 0.0;
                const double* Dr = &D[static_cast<size_t>(r) * w];
                for (int k = c; k < r; ++k) acc -= Dr[k] * X[static_cast<size_t>(k) * w + c];
                if (!(Dr[r] > 0.0)) {
                    zero_pivot.store(1);
                    return;
                }
                X[static_cast<size_t>(r) * w + c] = acc / Dr[r];
            }
        }
        double* Li = &out.dinv[static_cast<size_t>(out.dinv_off[s])];
        double* Ui = &out.dinvT[static_cast<size_t>(out.dinv_off[s])];
        for (int r = 0; r < w; ++r)
            for (int c = 0; c <= r; ++c) Li[static_cast<int64_t>(r) * (r + 1) / 2 + c] = X[static_cast<size_t>(r) * w + c];
        // row c of D^{-T} = column c of D^{-1}: entries r = c .. w-1, starting at c w - c (c-1) / 2
        for (int c = 0; c < w; ++c) {
            const int64_t o = static_cast<int64_t>(c) * w - static_cast<int64_t>(c) * (c - 1) / 2;
            for (int r = c; r < w; ++r) Ui[o + (r - c)] = X[static_cast<size_t>(r) * w + c];
        }
    }
    };
    if (threads <= 1 || nsn < 64) {
        invert(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) th.emplace_back(invert, t);
        for (auto& x : th) x.join();
    }
    if (zero_pivot.load()) return "zero pivot in a supernode diagonal block";
    return std::string();
}

}  // namespace rpb
