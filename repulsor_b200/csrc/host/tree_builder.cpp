// Host construction of the cluster tree and block cluster tree (see tree_builder.hpp).
#include "tree_builder.hpp"

#include "bct_rules.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <utility>

namespace rpb {
namespace {

constexpr int AMB = 3;

struct Node {
    int begin, end;
    double box[7];
    int left = -1, right = -1;
    int desc = 1;
    int depth = 0;
};

// --- primitives ------------------------------------------------------------
// Serialized polytope: [r2, centre(3), hull((dom+1) x 3)], hull in the simplex's own vertex order.
void serialize_polytope(int size, const double* V, const int* s, double* out)
{
    double* c = out + 1;
    double* h = out + 1 + AMB;
    for (int j = 0; j < size; ++j)
        for (int k = 0; k < AMB; ++k) h[AMB * j + k] = V[AMB * static_cast<int64_t>(s[j]) + k];
    const double w = 1.0 / size;
    for (int k = 0; k < AMB; ++k) {
        double acc = h[k];
        for (int j = 1; j < size; ++j) acc += h[AMB * j + k];
        c[k] = acc * w;
    }
    double r2 = 0;
    for (int j = 0; j < size; ++j) {
        double d = h[AMB * j] - c[0];
        double sq = d * d;
        for (int k = 1; k < AMB; ++k) {
            d = h[AMB * j + k] - c[k];
            sq += d * d;
        }
        r2 = std::max(r2, sq);
    }
    out[0] = r2;
}

void aabb_of_range(int size, int ps, const double* P, int begin, int end, double* box)
{
    double lo[3], hi[3];
    for (int k = 0; k < AMB; ++k) {
        lo[k] = std::numeric_limits<double>::max();
        hi[k] = std::numeric_limits<double>::lowest();
    }
    for (int i = begin; i < end; ++i) {
        const double* h = P + static_cast<int64_t>(ps) * i + 1 + AMB;
        for (int j = 0; j < size; ++j)
            for (int k = 0; k < AMB; ++k) {
                const double x = h[AMB * j + k];
                lo[k] = std::min(lo[k], x);
                hi[k] = std::max(hi[k], x);
            }
    }
    double r2 = 0;
    for (int k = 0; k < AMB; ++k) {
        const double half = 0.5 * (hi[k] - lo[k]);
        r2 += half * half;
        box[1 + k] = lo[k] + half;
        box[1 + AMB + k] = half;
    }
    box[0] = r2;
}

struct Splitter {
    int size, ps;
    std::vector<int>& ord;
    std::vector<double>& P;
    std::vector<double> score;
    std::vector<int> lperm, linv;

    Splitter(int size_, std::vector<int>& ord_, std::vector<double>& P_)
        : size(size_), ps(1 + AMB + size_ * AMB), ord(ord_), P(P_), score(ord_.size()), lperm(ord_.size()),
          linv(ord_.size())
    {}

    void swap_rows(int a, int b)
    {
        if (a == b) return;
        std::swap(ord[a], ord[b]);
        std::swap_ranges(P.begin() + static_cast<int64_t>(ps) * a, P.begin() + static_cast<int64_t>(ps) * (a + 1),
                         P.begin() + static_cast<int64_t>(ps) * b);
    }

    // Returns the split index; reorders [begin,end) in place.
    int split(int begin, int end, const double* box)
    {
        int dir = 0;
        double lmax = box[1 + AMB];
        for (int k = 1; k < AMB; ++k)
            if (box[1 + AMB + k] > lmax) {
                lmax = box[1 + AMB + k];
                dir = k;
            }
        const double mid = box[1 + dir];
        int s = begin;
        for (int i = begin; i < end; ++i) {
            if (P[static_cast<int64_t>(ps) * i + 1 + dir] < mid) {
                swap_rows(s, i);
                ++s;
            }
        }
        if (s == begin || s == end) {
            // median fallback with the same permutation cycle walk as the reference
            s = begin + (end - begin) / 2;
            for (int i = begin; i < end; ++i) {
                score[i] = P[static_cast<int64_t>(ps) * i + 1 + dir];
                lperm[i] = i;
            }
            const double* sc = score.data();
            std::nth_element(lperm.begin() + begin, lperm.begin() + s, lperm.begin() + end,
                             [sc](int a, int b) { return sc[a] < sc[b]; });
            for (int i = begin; i < end; ++i) linv[lperm[i]] = i;
            for (int i = begin; i < end; ++i) {
                int next = i;
                while (linv[next] >= 0) {
                    const int t = linv[next];
                    swap_rows(i, t);
                    linv[next] = -1;
                    next = t;
                }
            }
        }
        return s;
    }
};

// Builds the subtree rooted at nodes[0] (range already set) into `nodes`.
void build_subtree(Splitter& sp, std::vector<Node>& nodes)
{
    // explicit pre-order work list; post-order pass for descendant counts
    std::vector<int> stack{0};
    std::vector<int> order;
    while (!stack.empty()) {
        const int c = stack.back();
        stack.pop_back();
        order.push_back(c);
        const int b = nodes[c].begin, e = nodes[c].end;
        if (e - b <= 1) continue;  // split_threshold = 1
        const int s = sp.split(b, e, nodes[c].box);
        Node L, R;
        L.begin = b; L.end = s; L.depth = nodes[c].depth + 1;
        R.begin = s; R.end = e; R.depth = nodes[c].depth + 1;
        aabb_of_range(sp.size, sp.ps, sp.P.data(), b, s, L.box);
        aabb_of_range(sp.size, sp.ps, sp.P.data(), s, e, R.box);
        const int li = static_cast<int>(nodes.size());
        nodes.push_back(L);
        nodes.push_back(R);
        nodes[c].left = li;
        nodes[c].right = li + 1;
        stack.push_back(li + 1);
        stack.push_back(li);
    }
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
        Node& n = nodes[*it];
        if (n.left >= 0) n.desc = 1 + nodes[n.left].desc + nodes[n.right].desc;
    }
}

// --- exact primitive distances and block decisions: host/bct_rules.hpp -------------------
// --- pair traversal --------------------------------------------------------------
struct PairLists {
    std::vector<std::pair<int, int>> near, far, verynear, inter;
};

struct Traversal {
    const HostTree& T;
    const std::vector<double>& P;   // permuted polytopes
    const int* S;                   // original simplices
    int ps;
    double far_t2, near_t2;

    bool adjacent(int pi, int pj) const
    {
        const int* a = S + static_cast<int64_t>(T.size) * T.perm[pi];
        const int* b = S + static_cast<int64_t>(T.size) * T.perm[pj];
        for (int u = 0; u < T.size; ++u)
            for (int v = 0; v < T.size; ++v)
                if (a[u] == b[v]) return true;
        return false;
    }

    void leaf(int pi, int pj, PairLists& out) const  // pi < pj
    {
        if (adjacent(pi, pj)) { out.near.emplace_back(pi, pj); return; }
        const double* A = P.data() + static_cast<int64_t>(ps) * pi;
        const double* B = P.data() + static_cast<int64_t>(ps) * pj;
        const int cls = bct::classify_leaf(T.dom, A, B, near_t2);
        if (cls == 0) out.near.emplace_back(pi, pj);
        else if (cls == 1) out.verynear.emplace_back(pi, pj);
        else out.inter.emplace_back(pi, pj);
    }

    bool admissible(int i, int j) const
    {
        if (i == j) return false;
        return bct::boxes_admissible(&T.C_box[7 * static_cast<int64_t>(i)], &T.C_box[7 * static_cast<int64_t>(j)], far_t2);
    }

    // Processes one block pair; pushes children (in the reference's push order) to `next`.
    template <typename Push>
    void step(int i, int j, PairLists& out, Push&& push) const
    {
        if (admissible(i, j)) {
            if (i <= j) out.far.emplace_back(i, j); else out.far.emplace_back(j, i);
            return;
        }
        const int Li = T.C_left[i], Lj = T.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const int Ri = T.C_right[i], Rj = T.C_right[j];
            const double si = Li >= 0 ? T.C_box[7 * static_cast<int64_t>(i)] : 0.0;
            const double sj = Lj >= 0 ? T.C_box[7 * static_cast<int64_t>(j)] : 0.0;
            if (si == sj && si > 0) {
                if (i == j) { push(Li, Rj); push(Ri, Rj); push(Li, Lj); }
                else { push(Ri, Rj); push(Li, Rj); push(Ri, Lj); push(Li, Lj); }
            } else if (si > sj) {
                push(Ri, j); push(Li, j);
            } else {
                push(i, Rj); push(i, Lj);
            }
            return;
        }
        if (i == j) return;
        const int ii = T.C_begin[i], jj = T.C_begin[j];
        if (ii < jj) leaf(ii, jj, out); else leaf(jj, ii, out);
    }

    void dfs(int i0, int j0, PairLists& out) const
    {
        std::vector<std::pair<int, int>> stack;
        stack.reserve(1024);
        stack.emplace_back(i0, j0);
        while (!stack.empty()) {
            auto [i, j] = stack.back();
            stack.pop_back();
            step(i, j, out, [&](int a, int b) { stack.emplace_back(a, b); });
        }
    }
};

SymPattern to_pattern(int rows, std::vector<PairLists>& parts, std::vector<std::pair<int, int>> PairLists::*member)
{
    SymPattern P;
    P.rows = rows;
    P.rp.assign(static_cast<size_t>(rows) + 1, 0);
    for (auto& pl : parts)
        for (auto& e : pl.*member) { P.rp[e.first + 1]++; P.rp[e.second + 1]++; }
    for (int i = 0; i < rows; ++i) P.rp[i + 1] += P.rp[i];
    P.ci.resize(static_cast<size_t>(P.rp[rows]));
    std::vector<int64_t> pos(P.rp.begin(), P.rp.end() - 1);
    for (auto& pl : parts)
        for (auto& e : pl.*member) {
            P.ci[pos[e.first]++] = e.second;
            P.ci[pos[e.second]++] = e.first;
        }
    P.diag.resize(rows);
    for (int i = 0; i < rows; ++i) {
        auto b = P.ci.begin() + P.rp[i], e = P.ci.begin() + P.rp[i + 1];
        std::sort(b, e);
        P.diag[i] = std::upper_bound(b, e, i) - P.ci.begin();
    }
    return P;
}

template <typename F>
void run_threads(int n, F&& f)
{
    if (n <= 1) { f(0); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < n; ++t) th.emplace_back([&, t] { f(t); });
    for (auto& x : th) x.join();
}

}  // namespace

std::string build_cluster_tree(int dom, const double* V, int nV, const int* S, int N, const TreeSettings& set,
                               HostTree& T, std::vector<double>& P)
{
    if (dom != 1 && dom != 2) return "domain dimension must be 1 or 2";
    if (nV <= 0 || N <= 0) return "empty mesh";
    const int size = dom + 1;
    for (int64_t k = 0; k < static_cast<int64_t>(N) * size; ++k)
        if (S[k] < 0 || S[k] >= nV) return "simplex vertex index out of range";
    for (int64_t k = 0; k < 3 * static_cast<int64_t>(nV); ++k)
        if (!std::isfinite(V[k])) return "non-finite vertex coordinate";
    const int threads = std::max(1, set.threads);

    T = HostTree();
    T.dom = dom;
    T.size = size;
    T.nV = nV;
    T.N = N;
    const int ps = 1 + AMB + size * AMB;
    P.assign(static_cast<size_t>(N) * ps, 0.0);
    for (int i = 0; i < N; ++i) serialize_polytope(size, V, S + static_cast<int64_t>(size) * i, &P[static_cast<size_t>(ps) * i]);
    std::vector<int> ord(N);
    for (int i = 0; i < N; ++i) ord[i] = i;

    // --- split: top levels breadth-first, then independent subtrees in parallel
    std::vector<Node> top;
    top.reserve(256);
    Node root;
    root.begin = 0; root.end = N; root.depth = 0;
    aabb_of_range(size, ps, P.data(), 0, N, root.box);
    top.push_back(root);
    Splitter sp0(size, ord, P);
    std::vector<int> frontier{0};
    const int want = 8 * threads;
    while (static_cast<int>(frontier.size()) < want) {
        std::vector<int> next;
        bool any = false;
        for (int c : frontier) {
            const int b = top[c].begin, e = top[c].end;
            if (e - b <= 1) { next.push_back(c); continue; }
            any = true;
            const int s = sp0.split(b, e, top[c].box);
            Node L, R;
            L.begin = b; L.end = s; L.depth = top[c].depth + 1;
            R.begin = s; R.end = e; R.depth = top[c].depth + 1;
            aabb_of_range(size, ps, P.data(), b, s, L.box);
            aabb_of_range(size, ps, P.data(), s, e, R.box);
            const int li = static_cast<int>(top.size());
            top.push_back(L);
            top.push_back(R);
            top[c].left = li;
            top[c].right = li + 1;
            next.push_back(li);
            next.push_back(li + 1);
        }
        frontier.swap(next);
        if (!any) break;
    }
    // subtrees of the frontier nodes
    std::vector<std::vector<Node>> sub(frontier.size());
    {
        std::atomic<int> ticket{0};
        run_threads(threads, [&](int) {
            Splitter sp(size, ord, P);
            for (;;) {
                const int f = ticket.fetch_add(1);
                if (f >= static_cast<int>(frontier.size())) break;
                sub[f].push_back(top[frontier[f]]);
                build_subtree(sp, sub[f]);
            }
        });
    }
    // merge into one array: frontier subtree roots replace the frontier nodes
    std::vector<Node> nodes = top;
    for (size_t f = 0; f < frontier.size(); ++f) {
        const int off = static_cast<int>(nodes.size()) - 1;  // local index l>0 -> off + l
        Node& r = nodes[frontier[f]];
        const Node& lr = sub[f][0];
        r.desc = lr.desc;
        if (lr.left >= 0) { r.left = off + lr.left; r.right = off + lr.right; }
        for (size_t l = 1; l < sub[f].size(); ++l) {
            Node n = sub[f][l];
            if (n.left >= 0) { n.left += off; n.right += off; }
            nodes.push_back(n);
        }
    }
    // descendant counts of the top levels (children were appended after parents)
    for (int c = static_cast<int>(top.size()); c-- > 0;) {
        Node& n = nodes[c];
        bool is_frontier = std::find(frontier.begin(), frontier.end(), c) != frontier.end();
        if (!is_frontier && n.left >= 0) n.desc = 1 + nodes[n.left].desc + nodes[n.right].desc;
    }

    // --- depth-first serialization
    const int NC = nodes[0].desc;
    T.NC = NC;
    T.C_begin.assign(NC, 0); T.C_end.assign(NC, 0); T.C_left.assign(NC, -1); T.C_right.assign(NC, -1);
    T.C_parent.assign(NC, -1); T.C_depth.assign(NC, 0);
    T.C_box.assign(static_cast<size_t>(NC) * 7, 0.0);
    {
        std::vector<std::pair<int, int>> stack{{0, 0}};  // (node, global id)
        while (!stack.empty()) {
            auto [c, g] = stack.back();
            stack.pop_back();
            const Node& n = nodes[c];
            T.C_begin[g] = n.begin;
            T.C_end[g] = n.end;
            T.C_depth[g] = n.depth;
            T.depth = std::max(T.depth, n.depth);
            std::memcpy(&T.C_box[7 * static_cast<size_t>(g)], n.box, sizeof(n.box));
            if (n.left >= 0) {
                const int gl = g + 1, gr = g + 1 + nodes[n.left].desc;
                T.C_left[g] = gl;
                T.C_right[g] = gr;
                T.C_parent[gl] = g;
                T.C_parent[gr] = g;
                stack.emplace_back(n.right, gr);
                stack.emplace_back(n.left, gl);
            }
        }
    }
    T.perm = ord;
    T.inv_perm.assign(N, 0);
    for (int i = 0; i < N; ++i) T.inv_perm[ord[i]] = i;
    T.leaf_of.assign(N, -1);
    for (int C = 0; C < NC; ++C)
        if (T.C_left[C] < 0)
            for (int i = T.C_begin[C]; i < T.C_end[C]; ++i) T.leaf_of[i] = C;

    return std::string();
}

void build_block_cluster_tree(HostTree& T, const std::vector<double>& P, const int* S, const TreeSettings& set)
{
    const int threads = std::max(1, set.threads);
    const int ps = 1 + AMB + T.size * AMB;
    const int N = T.N, NC = T.NC;
    // --- block cluster tree
    Traversal tr{T, P, S, ps, set.theta_far * set.theta_far, set.theta_near * set.theta_near};
    std::vector<std::pair<int, int>> tasks{{0, 0}};
    std::vector<PairLists> parts(threads);
    // breadth-first expansion into enough independent tasks
    const size_t task_target = static_cast<size_t>(16) * threads;
    while (!tasks.empty() && tasks.size() < task_target) {
        std::vector<std::pair<int, int>> next;
        for (auto [i, j] : tasks) tr.step(i, j, parts[0], [&](int a, int b) { next.emplace_back(a, b); });
        tasks.swap(next);
    }
    {
        std::atomic<size_t> ticket{0};
        run_threads(threads, [&](int t) {
            for (;;) {
                const size_t k = ticket.fetch_add(1);
                if (k >= tasks.size()) break;
                tr.dfs(tasks[k].first, tasks[k].second, parts[t]);
            }
        });
    }
    T.near = to_pattern(N, parts, &PairLists::near);
    T.far = to_pattern(NC, parts, &PairLists::far);
    T.verynear = to_pattern(N, parts, &PairLists::verynear);
    T.inter = to_pattern(N, parts, &PairLists::inter);
}

std::string build_tree(int dom, const double* V, int nV, const int* S, int N, const TreeSettings& set,
                       HostTree& T)
{
    std::vector<double> P;
    std::string err = build_cluster_tree(dom, V, nV, S, N, set, T, P);
    if (!err.empty()) return err;
    build_block_cluster_tree(T, P, S, set);
    return std::string();
}

namespace {

CrossPattern to_cross(int rows, std::vector<std::vector<std::pair<int, int>>>& parts)
{
    CrossPattern P;
    P.rows = rows;
    P.rp.assign(static_cast<size_t>(rows) + 1, 0);
    for (auto& v : parts)
        for (auto& e : v) P.rp[e.first + 1]++;
    for (int i = 0; i < rows; ++i) P.rp[i + 1] += P.rp[i];
    P.ci.resize(static_cast<size_t>(P.rp[rows]));
    std::vector<int64_t> pos(P.rp.begin(), P.rp.end() - 1);
    for (auto& v : parts)
        for (auto& e : v) P.ci[pos[e.first]++] = e.second;
    for (int i = 0; i < rows; ++i) std::sort(P.ci.begin() + P.rp[i], P.ci.begin() + P.rp[i + 1]);
    return P;
}

std::vector<double> permuted_polytopes(const HostTree& T, const double* V, const int* S)
{
    const int ps = 1 + AMB + T.size * AMB;
    std::vector<double> P(static_cast<size_t>(T.N) * ps);
    for (int i = 0; i < T.N; ++i)
        serialize_polytope(T.size, V, S + static_cast<int64_t>(T.size) * T.perm[i], &P[static_cast<size_t>(ps) * i]);
    return P;
}

struct CrossTraversal {
    const HostTree& A;
    const HostTree& B;
    const std::vector<double>& PA;
    const std::vector<double>& PB;
    int psA, psB;
    double far_t2, near_t2;

    struct Out {
        std::vector<std::pair<int, int>> near, far, verynear, inter;
    };

    void leaf(int pi, int pj, Out& out) const
    {
        const double* X = PA.data() + static_cast<int64_t>(psA) * pi;
        const double* Y = PB.data() + static_cast<int64_t>(psB) * pj;
        const int cls = bct::classify_leaf(A.dom, X, Y, near_t2);
        if (cls == 0) out.near.emplace_back(pi, pj);
        else if (cls == 1) out.verynear.emplace_back(pi, pj);
        else out.inter.emplace_back(pi, pj);
    }

    template <typename Push>
    void step(int i, int j, Out& out, Push&& push) const
    {
        const double* a = &A.C_box[7 * static_cast<int64_t>(i)];
        const double* b = &B.C_box[7 * static_cast<int64_t>(j)];
        double d2 = 0;
        for (int k = 0; k < AMB; ++k) {
            const double lo = std::max(a[1 + k] - a[4 + k], b[1 + k] - b[4 + k]);
            const double hi = std::min(a[1 + k] + a[4 + k], b[1 + k] + b[4 + k]);
            const double x = std::max(0.0, lo - hi);
            d2 += x * x;
        }
        if (std::max(a[0], b[0]) < far_t2 * d2) { out.far.emplace_back(i, j); return; }
        const int Li = A.C_left[i], Lj = B.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const int Ri = A.C_right[i], Rj = B.C_right[j];
            const double si = Li >= 0 ? a[0] : 0.0;
            const double sj = Lj >= 0 ? b[0] : 0.0;
            if (si == sj && si > 0) { push(Ri, Rj); push(Li, Rj); push(Ri, Lj); push(Li, Lj); }
            else if (si > sj) { push(Ri, j); push(Li, j); }
            else { push(i, Rj); push(i, Lj); }
            return;
        }
        leaf(A.C_begin[i], B.C_begin[j], out);
    }
};

}  // namespace

std::string build_cross_lists(const HostTree& S, const double* VS, const int* SS, const HostTree& T,
                              const double* VT, const int* ST, const TreeSettings& set, CrossLists& out)
{
    if (S.dom != T.dom) return "the obstacle's domain dimension differs from the mesh's";
    if (S.NC <= 0 || T.NC <= 0) return "empty tree";
    const std::vector<double> PA = permuted_polytopes(S, VS, SS), PB = permuted_polytopes(T, VT, ST);
    CrossTraversal tr{S, T, PA, PB, 1 + AMB + S.size * AMB, 1 + AMB + T.size * AMB,
                      set.theta_far * set.theta_far, set.theta_near * set.theta_near};
    const int threads = std::max(1, set.threads);
    // expand the root block breadth-first into independent tasks, then depth-first in parallel
    CrossTraversal::Out top;
    std::vector<std::pair<int, int>> tasks{{0, 0}};
    while (!tasks.empty() && static_cast<int>(tasks.size()) < 16 * threads) {
        std::vector<std::pair<int, int>> next;
        for (auto [i, j] : tasks) tr.step(i, j, top, [&](int a, int b) { next.emplace_back(a, b); });
        tasks.swap(next);
    }
    std::vector<CrossTraversal::Out> parts(tasks.size());
    std::atomic<int> ticket{0};
    run_threads(threads, [&](int) {
        std::vector<std::pair<int, int>> stack;
        for (;;) {
            const int t = ticket.fetch_add(1);
            if (t >= static_cast<int>(tasks.size())) break;
            stack.assign(1, tasks[t]);
            while (!stack.empty()) {
                auto [i, j] = stack.back();
                stack.pop_back();
                tr.step(i, j, parts[t], [&](int a, int b) { stack.emplace_back(a, b); });
            }
        }
    });
    auto gather = [&](std::vector<std::pair<int, int>> CrossTraversal::Out::*mem, int rows) {
        std::vector<std::vector<std::pair<int, int>>> v;
        v.push_back(std::move(top.*mem));
        for (auto& p : parts) v.push_back(std::move(p.*mem));
        return to_cross(rows, v);
    };
    out = CrossLists();
    out.near = gather(&CrossTraversal::Out::near, S.N);
    out.far = gather(&CrossTraversal::Out::far, S.NC);
    out.verynear = gather(&CrossTraversal::Out::verynear, S.N);
    out.inter = gather(&CrossTraversal::Out::inter, S.N);
    return std::string();
}

void build_row_tiles(const int64_t* rp, const int* ci, int rows, int ncols, int block_lanes, int64_t target_entries,
                     int max_union, int threads, RowTiles& out)
{
    out = RowTiles();
    max_union = std::min(max_union, 65535);
    if (block_lanes < 1 || block_lanes % 32 != 0) return;
    for (int i = 0; i < rows; ++i)
        if (rp[i + 1] - rp[i] > max_union) return;
    target_entries = std::max<int64_t>(1, target_entries);
    out.block_lanes = block_lanes;
    // tile boundaries (sequential): add rows until the tile holds target_entries entries,
    // block_lanes rows, or the column union would exceed the cap
    {
        std::vector<char> mark(ncols, 0);
        std::vector<int> U;
        int r = 0;
        while (r < rows) {
            const int t0 = r;
            int64_t entries = 0;
            U.clear();
            while (r < rows && entries < target_entries && r - t0 < block_lanes) {
                int fresh = 0;
                for (int64_t k = rp[r]; k < rp[r + 1]; ++k) fresh += !mark[ci[k]];
                if (r > t0 && static_cast<int>(U.size()) + fresh > max_union) break;
                for (int64_t k = rp[r]; k < rp[r + 1]; ++k)
                    if (!mark[ci[k]]) { mark[ci[k]] = 1; U.push_back(ci[k]); }
                entries += rp[r + 1] - rp[r];
                ++r;
            }
            for (int u : U) mark[u] = 0;
            out.row0.push_back(t0);
            out.cols_rp.push_back(static_cast<int>(U.size()));   // sizes for now
        }
        out.row0.push_back(rows);
    }
    const int nt = out.tiles();
    {
        std::vector<int> sizes(out.cols_rp.begin(), out.cols_rp.end());
        out.cols_rp.assign(nt + 1, 0);
        for (int b = 0; b < nt; ++b) {
            out.cols_rp[b + 1] = out.cols_rp[b] + sizes[b];
            out.max_union = std::max(out.max_union, sizes[b]);
        }
    }
    out.cols.assign(out.cols_rp[nt], 0);
    out.slot.assign(static_cast<size_t>(rows > 0 ? rp[rows] : 0), 0);
    out.order.assign(rows, 0);
    out.lane_map.assign(static_cast<size_t>(nt) * block_lanes, -1);
    // per tile (parallel): sorted union, slots, lane groups, row order, lane map
    std::atomic<int> ticket{0};
    run_threads(std::max(1, std::min(threads, nt)), [&](int) {
        std::vector<int> pos(ncols, -1), U, size, idx;
        for (;;) {
            const int b = ticket.fetch_add(1);
            if (b >= nt) break;
            const int t0 = out.row0[b], t1 = out.row0[b + 1], R = t1 - t0;
            U.clear();
            for (int64_t k = rp[t0]; k < rp[t1]; ++k)
                if (pos[ci[k]] < 0) { pos[ci[k]] = 0; U.push_back(ci[k]); }
            std::sort(U.begin(), U.end());
            for (size_t u = 0; u < U.size(); ++u) {
                pos[U[u]] = static_cast<int>(u);
                out.cols[out.cols_rp[b] + u] = U[u];
            }
            for (int64_t k = rp[t0]; k < rp[t1]; ++k) out.slot[k] = static_cast<uint16_t>(pos[ci[k]]);
            for (int u : U) pos[u] = -1;
            // lane groups: every row starts with one lane; the row with the most entries per
            // lane doubles its group while the block has lanes left (groups of at most 32)
            auto len = [&](int q) { return rp[t0 + q + 1] - rp[t0 + q]; };
            auto load = [&](int q) { return (len(q) + size[q] - 1) / size[q]; };
            size.assign(R, 1);
            int used = R;
            auto cmp = [&](int x, int y) { return load(x) < load(y) || (load(x) == load(y) && x > y); };
            std::vector<int> heap(R);
            for (int q = 0; q < R; ++q) heap[q] = q;
            std::make_heap(heap.begin(), heap.end(), cmp);
            while (!heap.empty()) {
                std::pop_heap(heap.begin(), heap.end(), cmp);
                const int q = heap.back();
                if (size[q] >= 32 || used + size[q] > block_lanes || len(q) <= size[q]) break;
                used += size[q];
                size[q] *= 2;
                std::push_heap(heap.begin(), heap.end(), cmp);
            }
            // groups in decreasing size (then decreasing length) start at multiples of their
            // size and never straddle a warp
            idx.resize(R);
            for (int q = 0; q < R; ++q) idx[q] = q;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
                return size[x] > size[y] || (size[x] == size[y] && len(x) > len(y));
            });
            int lane = 0;
            for (int pos_in_tile = 0; pos_in_tile < R; ++pos_in_tile) {
                const int q = idx[pos_in_tile];
                out.order[t0 + pos_in_tile] = t0 + q;
                for (int sub = 0; sub < size[q]; ++sub)
                    out.lane_map[static_cast<size_t>(b) * block_lanes + lane + sub] =
                        (pos_in_tile << 10) | ((size[q] - 1) << 5) | sub;
                lane += size[q];
            }
        }
    });
    out.valid = true;
}

}  // namespace rpb
