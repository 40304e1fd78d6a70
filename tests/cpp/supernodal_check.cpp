// The supernodal Cholesky (host/supernodal_chol.hpp: symbolic analysis, the per-supernode
// numeric code shared with the GPU, conversion to the row and column forms) on seeded random
// sparse symmetric positive definite matrices with random orderings and several supernode
// width caps: the factor's column form must have the diagonal first and ascending rows, the
// row form must be its transpose, and L L^T must reproduce P A P^T to 1e-12 relative.
// Prints "ok" or the first violation.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "host/supernodal_chol.hpp"

using namespace rpb;

static int check(int n, int per_row, int max_width, unsigned seed)
{
    std::mt19937 rng(seed);
    std::uniform_int_distribution<int> col(0, n - 1);
    std::uniform_real_distribution<double> val(-1.0, 1.0);
    std::vector<std::map<int, double>> rows(n);
    for (int i = 0; i < n; ++i)
        for (int t = 0; t < per_row; ++t) {
            const int j = col(rng);
            if (j == i) continue;
            const double x = val(rng);
            rows[i][j] += x;
            rows[j][i] += x;
        }
    for (int i = 0; i < n; ++i) {   // diagonal dominance: positive definite
        double s = 1.0;
        for (auto& e : rows[i]) s += std::fabs(e.second);
        rows[i][i] = s;
    }
    CsrMatrix A;
    A.n = n;
    A.rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (auto& e : rows[i]) {
            A.ci.push_back(e.first);
            A.val.push_back(e.second);
        }
        A.rp[i + 1] = static_cast<int64_t>(A.ci.size());
    }
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::shuffle(perm.begin(), perm.end(), rng);
    SupernodalSymbolic S;
    std::string err = supernodal_symbolic(A, perm, max_width, S);
    if (!err.empty()) { std::printf("symbolic: %s\n", err.c_str()); return 1; }
    for (int s = 0; s < S.nsn; ++s)
        if (S.sn_begin[s + 1] - S.sn_begin[s] > max_width) { std::printf("supernode wider than the cap\n"); return 1; }
    std::vector<double> panels;
    err = supernodal_numeric_host(S, panels, 4);
    if (!err.empty()) { std::printf("numeric: %s\n", err.c_str()); return 1; }
    CholeskyFactor F;
    supernodal_to_factor(S, panels, F);
    // column form: diagonal first, rows ascending; row form: diagonal last, the transpose
    std::vector<std::map<int, double>> L(n);   // L[j][i] = L(i, j)
    for (int j = 0; j < n; ++j) {
        if (F.upper_rp[j + 1] <= F.upper_rp[j] || F.upper_ci[F.upper_rp[j]] != j) { std::printf("diagonal not first\n"); return 1; }
        for (int64_t p = F.upper_rp[j]; p < F.upper_rp[j + 1]; ++p) {
            if (p > F.upper_rp[j] && F.upper_ci[p] <= F.upper_ci[p - 1]) { std::printf("rows not ascending\n"); return 1; }
            L[j][F.upper_ci[p]] = F.upper_val[p];
        }
    }
    int64_t seen = 0;
    for (int i = 0; i < n; ++i) {
        if (F.lower_ci[F.lower_rp[i + 1] - 1] != i) { std::printf("diagonal not last\n"); return 1; }
        for (int64_t p = F.lower_rp[i]; p < F.lower_rp[i + 1]; ++p, ++seen) {
            auto it = L[F.lower_ci[p]].find(i);
            if (it == L[F.lower_ci[p]].end() || it->second != F.lower_val[p]) { std::printf("row form is not the transpose\n"); return 1; }
        }
    }
    if (seen != F.upper_rp[n]) { std::printf("row form size\n"); return 1; }
    // (L L^T)(a, b) = sum_k L(a, k) L(b, k) against C = P A P^T
    std::vector<int> pinv(n);
    for (int i = 0; i < n; ++i) pinv[perm[i]] = i;
    std::vector<std::map<int, double>> C(n);
    for (int r = 0; r < n; ++r)
        for (int64_t p = A.rp[r]; p < A.rp[r + 1]; ++p) C[pinv[r]][pinv[A.ci[p]]] = A.val[p];
    std::vector<std::map<int, double>> LLt(n);
    for (int k = 0; k < n; ++k)
        for (auto& a : L[k])
            for (auto& b : L[k])
                if (b.first <= a.first) LLt[a.first][b.first] += a.second * b.second;
    double scale = 0.0, errmax = 0.0;
    for (int a = 0; a < n; ++a)
        for (auto& e : C[a]) scale = std::max(scale, std::fabs(e.second));
    for (int a = 0; a < n; ++a) {
        for (auto& e : LLt[a]) {
            const auto it = C[a].find(e.first);
            errmax = std::max(errmax, std::fabs(e.second - (it == C[a].end() ? 0.0 : it->second)));
        }
        for (auto& e : C[a])
            if (e.first <= a && LLt[a].find(e.first) == LLt[a].end()) { std::printf("entry of C missing in L L^T\n"); return 1; }
    }
    if (errmax > 1e-12 * scale) { std::printf("L L^T differs from P A P^T: %.3e\n", errmax / scale); return 1; }
    return 0;
}

int main()
{
    const int widths[] = {1, 2, 3, 8, 256};
    unsigned seed = 11;
    for (int n : {1, 2, 17, 120, 300})
        for (int per_row : {1, 3, 6})
            for (int w : widths)
                if (check(n, per_row, w, seed++) != 0) {
                    std::printf("failed at n=%d per_row=%d width=%d\n", n, per_row, w);
                    return 1;
                }
    std::printf("ok\n");
    return 0;
}
