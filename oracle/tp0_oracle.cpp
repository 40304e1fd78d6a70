// ============================================================================
// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of Repulsor's multipole-accelerated tangent-point path
// (TangentPointEnergy0 Value/Differential, TangentPointMetric0 MultiplyMetric,
// PseudoLaplacian, H1 metric assembly) used as the checker for the CUDA
// implementation in repulsor_b200/. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load this library. The product never links it.
//
// Parity status: the reference cannot be compiled here (its Tensors submodule is
// absent), so this restatement is pinned by the reference's algebraic identities
// (homogeneity, translation invariance, finite differences, symmetry, all-pairs
// limit) and by golden fixtures generated from it -- see tests/.
//
// Citations are path:line inside the reference project (HenrikSchumacher/Repulsor).
// Scalar types follow the reference examples: Real = double, Int = int,
// LInt = size_t (Example/main.cpp:32-34).
// ============================================================================

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace oracle {

using Int  = int;
using LInt = int64_t;

static constexpr int AMB = 3;
static constexpr int PROJ = 6;   // packed upper triangle of a 3x3 matrix
static constexpr int FAR_DIM = 1 + AMB + PROJ;  // src/SimplicialMesh.hpp:68

static inline int near_dim(int dom) { return 1 + (dom + 1) * AMB + PROJ; }  // src/SimplicialMesh.hpp:69

// Packed upper-triangle index of (i,j), i<=j, row-major over the upper triangle:
// (0,0),(0,1),(0,2),(1,1),(1,2),(2,2)
// (CodeGeneration/SimplicialMesh/Code_DNearFar_to_Hulls.m:60-61, lin_k of Tensors).
static inline int lin_k(int i, int j)
{
    if (i > j) std::swap(i, j);
    static const int tab[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    return tab[i][j];
}

// ----------------------------------------------------------------------------
// Threads: plain std::thread fan-out, the decomposition of Tensors' ParallelDo.
// ----------------------------------------------------------------------------
template <typename F>
static void parallel_do(int thread_count, F&& f)
{
    if (thread_count <= 1) { f(0); return; }
    std::vector<std::thread> th;
    th.reserve(thread_count);
    for (int t = 0; t < thread_count; ++t) th.emplace_back([&, t]() { f(t); });
    for (auto& x : th) x.join();
}

static inline Int job_pointer(Int n, Int threads, Int t)
{
    return static_cast<Int>((static_cast<int64_t>(n) * t) / threads);
}

// ----------------------------------------------------------------------------
// Sparse pattern in CSR with full symmetric storage (BinaryMatrixCSR built with
// symmetrization, src/BlockClusterTree.hpp:306-326).
// ----------------------------------------------------------------------------
struct Pattern {
    Int rows = 0;
    std::vector<LInt> rp;    // rows+1
    std::vector<Int>  ci;    // nnz, sorted within each row
    std::vector<LInt> diag;  // first position in row i with column > i
    LInt nnz() const { return rp.empty() ? 0 : rp.back(); }
};

static Pattern make_symmetric_pattern(Int rows, const std::vector<std::pair<Int, Int>>& upper)
{
    Pattern P;
    P.rows = rows;
    P.rp.assign(rows + 1, 0);
    for (auto& e : upper) { P.rp[e.first + 1]++; P.rp[e.second + 1]++; }
    for (Int i = 0; i < rows; ++i) P.rp[i + 1] += P.rp[i];
    P.ci.resize(P.rp[rows]);
    std::vector<LInt> pos(P.rp.begin(), P.rp.end() - 1);
    for (auto& e : upper) { P.ci[pos[e.first]++] = e.second; P.ci[pos[e.second]++] = e.first; }
    P.diag.resize(rows);
    for (Int i = 0; i < rows; ++i) {
        std::sort(P.ci.begin() + P.rp[i], P.ci.begin() + P.rp[i + 1]);
        LInt k = P.rp[i];
        while (k < P.rp[i + 1] && P.ci[k] <= i) ++k;
        P.diag[i] = k;
    }
    return P;
}

// ----------------------------------------------------------------------------
// Settings (src/Settings.hpp:5-54) with the mesh overrides of
// src/SimplicialMesh.hpp:592-595.
// ----------------------------------------------------------------------------
struct Settings {
    double theta_far  = 0.5;
    double theta_near = 10.0;
    int    max_refinement = 30;
    int    threads = 1;
};

// ----------------------------------------------------------------------------
// Mesh + trees
// ----------------------------------------------------------------------------
struct Mesh {
    int dom = 2;
    int SIZE = 3;
    Int nV = 0, nS = 0;
    Settings set;

    std::vector<double> V;          // current coordinates (nV x 3)
    std::vector<double> V_frozen;   // clustering coordinates (src/SimplicialMesh.hpp:247-251)
    std::vector<Int>    S;          // simplices (nS x SIZE), unsorted
    std::vector<double> charge_v;   // vertex charges (1 by default, src/SimplicialMesh.hpp:180)

    // tree
    std::vector<Int> perm, inv_perm;                 // P_ordering (position -> simplex)
    std::vector<Int> C_begin, C_end, C_left, C_right, C_depth, C_parent;
    std::vector<double> C_box;                       // N_C x 7 : r2, centre, half-lengths
    std::vector<double> P_poly;                      // permuted polytope data: r2, centre, hull
    Int NC = 0;

    // block cluster tree
    Pattern near, far, verynear, inter;

    // primitive / cluster data (permuted order)
    std::vector<double> P_near, P_far, C_far;

    // frozen Pre/Post operators (src/ClusterTree.hpp:410-639): per permuted primitive
    // sorted simplex vertex ids, and 4 x SIZE coefficients (row 0 averaging, rows 1..3 gradient)
    std::vector<Int>    pre_cols;   // N x SIZE
    std::vector<double> pre_vals;   // N x 4 x SIZE

    // derivative buffers (original order, after collection)
    std::vector<double> P_D_near, P_D_far;

    int poly_size() const { return 1 + AMB + SIZE * AMB; }
};

// ----------------------------------------------------------------------------
// Simplex data: src/SimplexDataKernel.hpp:92-203
// ----------------------------------------------------------------------------
struct SimplexData {
    double a;
    double hull[3][3];
    double center[3];
    double P[3][3];
    double Df[3][3];     // derivative operator D_f (AMB x SIZE) in sorted vertex order
    Int    sorted[3];
};

static void read_simplex(const Mesh& M, const double* V, Int i, SimplexData& d)
{
    const int n = M.dom, SIZE = M.SIZE;
    Int simplex[3], s[3];
    for (int l = 0; l < SIZE; ++l) simplex[l] = s[l] = M.S[SIZE * i + l];
    std::sort(s, s + SIZE);
    for (int l = 0; l < SIZE; ++l) d.sorted[l] = s[l];
    for (int l = 0; l < SIZE; ++l)
        for (int k = 0; k < AMB; ++k) d.hull[l][k] = V[AMB * simplex[l] + k];
    const double nth = 1.0 / SIZE;
    double charge = M.charge_v[simplex[0]];
    for (int k = 0; k < AMB; ++k) d.center[k] = d.hull[0][k];
    for (int l = 1; l < SIZE; ++l) {
        for (int k = 0; k < AMB; ++k) d.center[k] += d.hull[l][k];
        charge += M.charge_v[simplex[l]];
    }
    for (int k = 0; k < AMB; ++k) d.center[k] *= nth;
    charge *= nth;
    const double std_vol = (n == 1) ? 1.0 : 0.5;   // StandardSimplexVolume = 1/n!
    d.a = charge * std_vol;

    double df[3][2];
    for (int l = 0; l < n; ++l)
        for (int k = 0; k < AMB; ++k) df[k][l] = V[AMB * s[l + 1] + k] - V[AMB * s[0] + k];
    // g = df^T df, Cholesky in place
    double g[2][2] = {{0, 0}, {0, 0}};
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            for (int k = 0; k < AMB; ++k) g[a][b] += df[k][a] * df[k][b];
    double L[2][2] = {{0, 0}, {0, 0}};
    L[0][0] = std::sqrt(g[0][0]);
    if (n == 2) {
        L[1][0] = g[1][0] / L[0][0];
        L[1][1] = std::sqrt(g[1][1] - L[1][0] * L[1][0]);
    }
    for (int l = 0; l < n; ++l) d.a *= L[l][l];
    // dfdagger = g^{-1} df^T
    double dag[2][3];
    for (int k = 0; k < AMB; ++k) {
        // solve g y = df[k][:]
        double b0 = df[k][0];
        if (n == 1) {
            dag[0][k] = b0 / g[0][0];
        } else {
            double b1 = df[k][1];
            // forward L z = b, backward L^T y = z
            double z0 = b0 / L[0][0];
            double z1 = (b1 - L[1][0] * z0) / L[1][1];
            double y1 = z1 / L[1][1];
            double y0 = (z0 - L[1][0] * y1) / L[0][0];
            dag[0][k] = y0;
            dag[1][k] = y1;
        }
    }
    for (int i2 = 0; i2 < AMB; ++i2)
        for (int j2 = 0; j2 < AMB; ++j2) {
            double acc = 0;
            for (int l = 0; l < n; ++l) acc += df[i2][l] * dag[l][j2];
            d.P[i2][j2] = (i2 == j2 ? 1.0 : 0.0) - acc;
        }
    // D_f (src/SimplexDataKernel.hpp:212-238)
    for (int k = 0; k < AMB; ++k) {
        d.Df[k][0] = 0;
        for (int l = 0; l < n; ++l) {
            d.Df[k][0] -= dag[l][k];
            d.Df[k][l + 1] = dag[l][k];
        }
    }
}

static void write_near(const Mesh& M, const SimplexData& d, double* out)
{
    out[0] = d.a;
    for (int l = 0; l < M.SIZE; ++l)
        for (int k = 0; k < AMB; ++k) out[1 + AMB * l + k] = d.hull[l][k];
    const int base = 1 + AMB * M.SIZE;
    int kk = 0;
    for (int i = 0; i < AMB; ++i)
        for (int j = i; j < AMB; ++j) out[base + kk++] = d.P[i][j];
}

static void write_far(const SimplexData& d, double* out)
{
    out[0] = d.a;
    for (int k = 0; k < AMB; ++k) out[1 + k] = d.center[k];
    int kk = 0;
    for (int i = 0; i < AMB; ++i)
        for (int j = i; j < AMB; ++j) out[1 + AMB + kk++] = d.P[i][j];
}

// ----------------------------------------------------------------------------
// Polytope serialization (src/Primitives/Polytope.hpp:113-160) and AABBs
// (src/BoundingVolumes/AABB.hpp:155-237).
// ----------------------------------------------------------------------------
static void polytope_from_index_list(const Mesh& M, const double* coords, Int i, double* out)
{
    const int SIZE = M.SIZE;
    const double w = 1.0 / SIZE;
    double* r2 = out;
    double* c = out + 1;
    double* h = out + 1 + AMB;
    for (int j = 0; j < SIZE; ++j)
        for (int k = 0; k < AMB; ++k) h[AMB * j + k] = coords[AMB * M.S[SIZE * i + j] + k];
    for (int k = 0; k < AMB; ++k) {
        c[k] = h[k];
        for (int j = 1; j < SIZE; ++j) c[k] += h[AMB * j + k];
        c[k] *= w;
    }
    *r2 = 0;
    for (int j = 0; j < SIZE; ++j) {
        double diff = h[AMB * j] - c[0];
        double sq = diff * diff;
        for (int k = 1; k < AMB; ++k) { diff = h[AMB * j + k] - c[k]; sq += diff * diff; }
        *r2 = std::max(*r2, sq);
    }
}

static void box_from_primitives(const Mesh& M, const double* P_ser, Int begin, Int end, double* box)
{
    const int ps = M.poly_size();
    double lo[3], hi[3];
    for (int k = 0; k < AMB; ++k) { lo[k] = std::numeric_limits<double>::max(); hi[k] = std::numeric_limits<double>::lowest(); }
    for (Int i = begin; i < end; ++i) {
        const double* p = P_ser + ps * i + 1 + AMB;
        for (int j = 0; j < M.SIZE; ++j)
            for (int k = 0; k < AMB; ++k) {
                lo[k] = std::min(lo[k], p[AMB * j + k]);
                hi[k] = std::max(hi[k], p[AMB * j + k]);
            }
    }
    double r2 = 0;
    for (int k = 0; k < AMB; ++k) {
        const double diff = 0.5 * (hi[k] - lo[k]);
        r2 += diff * diff;
        lo[k] += diff;
        hi[k] = diff;
    }
    box[0] = r2;
    for (int k = 0; k < AMB; ++k) { box[1 + k] = lo[k]; box[1 + AMB + k] = hi[k]; }
}

static inline double aabb_sq_dist(const double* P, const double* Q)
{
    double d2 = 0;
    for (int k = 0; k < AMB; ++k) {
        const double x = std::max(0.0, std::max(P[1 + k] - P[4 + k], Q[1 + k] - Q[4 + k]) -
                                           std::min(P[1 + k] + P[4 + k], Q[1 + k] + Q[4 + k]));
        d2 += x * x;
    }
    return d2;
}

// ----------------------------------------------------------------------------
// Cluster tree construction: recursive restatement of Split / Serialize
// (src/ClusterTree/Split_Thread.hpp, src/ClusterTree/Serialize_Thread.hpp,
// src/BoundingVolumes/AABB_LongestAxisSplit.hpp:134-253).
// ----------------------------------------------------------------------------
struct BuildNode {
    Int begin, end;
    double box[7];
    int left = -1, right = -1;
    Int desc = 1;
    int depth = 0;
};

static void swap_poly(double* P_ser, int ps, Int a, Int b)
{
    if (a == b) return;
    for (int k = 0; k < ps; ++k) std::swap(P_ser[ps * a + k], P_ser[ps * b + k]);
}

static Int longest_axis_split(const Mesh& M, std::vector<Int>& ord, double* P_ser, Int begin, Int end,
                              const double* box, std::vector<double>& score, std::vector<Int>& perm,
                              std::vector<Int>& inv_perm)
{
    const int ps = M.poly_size();
    int dir = 0;
    double Lmax = box[1 + AMB + 0];
    for (int k = 1; k < AMB; ++k)
        if (box[1 + AMB + k] > Lmax) { Lmax = box[1 + AMB + k]; dir = k; }
    const double mid = box[1 + dir];
    Int split = begin;
    for (Int i = begin; i < end; ++i) {
        const double x = P_ser[ps * i + 1 + dir];
        if (x < mid) {
            std::swap(ord[split], ord[i]);
            swap_poly(P_ser, ps, split, i);
            ++split;
        }
    }
    if (split == begin || split == end) {
        split = begin + (end - begin) / 2;
        for (Int i = begin; i < end; ++i) { score[i] = P_ser[ps * i + 1 + dir]; perm[i] = i; }
        const double* sc = score.data();
        std::nth_element(perm.begin() + begin, perm.begin() + split, perm.begin() + end,
                         [sc](Int a, Int b) { return sc[a] < sc[b]; });
        for (Int i = begin; i < end; ++i) inv_perm[perm[i]] = i;
        for (Int i = begin; i < end; ++i) {
            Int next = i;
            while (inv_perm[next] >= 0) {
                const Int temp = inv_perm[next];
                std::swap(ord[i], ord[temp]);
                swap_poly(P_ser, ps, i, temp);
                inv_perm[next] = -1;
                next = temp;
            }
        }
    }
    return split;
}

static void build_cluster_tree(Mesh& M)
{
    const Int N = M.nS;
    const int ps = M.poly_size();
    std::vector<double> P_ser(static_cast<size_t>(N) * ps);
    for (Int i = 0; i < N; ++i) polytope_from_index_list(M, M.V_frozen.data(), i, &P_ser[ps * i]);
    std::vector<Int> ord(N);
    for (Int i = 0; i < N; ++i) ord[i] = i;
    std::vector<double> score(N);
    std::vector<Int> lperm(N), linv(N);

    std::vector<BuildNode> nodes;
    nodes.reserve(2 * N);
    nodes.push_back(BuildNode{0, N, {}, -1, -1, 1, 0});
    box_from_primitives(M, P_ser.data(), 0, N, nodes[0].box);

    // recursive split (depth-first; each node's split only touches its own range)
    std::function<void(int)> split = [&](int c) {
        const Int b = nodes[c].begin, e = nodes[c].end;
        if (e - b > 1) {  // split_threshold = 1
            const Int s = longest_axis_split(M, ord, P_ser.data(), b, e, nodes[c].box, score, lperm, linv);
            BuildNode L{b, s, {}, -1, -1, 1, nodes[c].depth + 1};
            BuildNode R{s, e, {}, -1, -1, 1, nodes[c].depth + 1};
            box_from_primitives(M, P_ser.data(), b, s, L.box);
            box_from_primitives(M, P_ser.data(), s, e, R.box);
            const int li = static_cast<int>(nodes.size());
            nodes.push_back(L);
            const int ri = static_cast<int>(nodes.size());
            nodes.push_back(R);
            nodes[c].left = li;
            nodes[c].right = ri;
            split(li);
            split(ri);
            nodes[c].desc = 1 + nodes[li].desc + nodes[ri].desc;
        }
    };
    split(0);

    // depth-first serialization: root 0, left = g+1, right = g+1+desc(left)
    const Int NC = nodes[0].desc;
    M.NC = NC;
    M.C_begin.assign(NC, 0); M.C_end.assign(NC, 0); M.C_left.assign(NC, -1); M.C_right.assign(NC, -1);
    M.C_depth.assign(NC, 0); M.C_parent.assign(NC, -1);
    M.C_box.assign(static_cast<size_t>(NC) * 7, 0.0);
    std::function<void(int, Int, Int)> ser = [&](int c, Int g, Int parent) {
        M.C_begin[g] = nodes[c].begin;
        M.C_end[g] = nodes[c].end;
        M.C_depth[g] = nodes[c].depth;
        M.C_parent[g] = parent;
        std::memcpy(&M.C_box[7 * static_cast<size_t>(g)], nodes[c].box, 7 * sizeof(double));
        if (nodes[c].left >= 0) {
            const Int gl = g + 1;
            const Int gr = g + 1 + nodes[nodes[c].left].desc;
            M.C_left[g] = gl;
            M.C_right[g] = gr;
            ser(nodes[c].left, gl, g);
            ser(nodes[c].right, gr, g);
        }
    };
    ser(0, 0, -1);
    M.perm = ord;
    M.inv_perm.assign(N, 0);
    for (Int i = 0; i < N; ++i) M.inv_perm[ord[i]] = i;
    M.P_poly = std::move(P_ser);
}

// ----------------------------------------------------------------------------
// Exact polytope distances (restating the separation predicate of GJK::Compute
// with collision_only, src/GJK.hpp:618-771, for segments and triangles).
// ----------------------------------------------------------------------------
static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void sub3(const double* a, const double* b, double* c) { c[0] = a[0] - b[0]; c[1] = a[1] - b[1]; c[2] = a[2] - b[2]; }
static inline void cross3(const double* a, const double* b, double* c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static double seg_seg_sqdist(const double* p1, const double* q1, const double* p2, const double* q2)
{
    double d1[3], d2[3], r[3];
    sub3(q1, p1, d1); sub3(q2, p2, d2); sub3(p1, p2, r);
    const double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    double s, t;
    if (a <= 0 && e <= 0) { return dot3(r, r); }
    if (a <= 0) { s = 0; t = std::clamp(f / e, 0.0, 1.0); }
    else {
        const double c = dot3(d1, r);
        if (e <= 0) { t = 0; s = std::clamp(-c / a, 0.0, 1.0); }
        else {
            const double b = dot3(d1, d2);
            const double den = a * e - b * b;
            s = (den > 0) ? std::clamp((b * f - c * e) / den, 0.0, 1.0) : 0.0;
            t = (b * s + f) / e;
            if (t < 0) { t = 0; s = std::clamp(-c / a, 0.0, 1.0); }
            else if (t > 1) { t = 1; s = std::clamp((b - c) / a, 0.0, 1.0); }
        }
    }
    double c1[3], c2[3], w[3];
    for (int k = 0; k < 3; ++k) { c1[k] = p1[k] + d1[k] * s; c2[k] = p2[k] + d2[k] * t; }
    sub3(c1, c2, w);
    return dot3(w, w);
}

static double point_tri_sqdist(const double* p, const double* a, const double* b, const double* c)
{
    double ab[3], ac[3], ap[3];
    sub3(b, a, ab); sub3(c, a, ac); sub3(p, a, ap);
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    double x[3];
    auto dist_to = [&](const double* q) { double w[3]; sub3(p, q, w); return dot3(w, w); };
    if (d1 <= 0 && d2 <= 0) return dist_to(a);
    double bp[3]; sub3(p, b, bp);
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) return dist_to(b);
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double v = d1 / (d1 - d3);
        for (int k = 0; k < 3; ++k) x[k] = a[k] + v * ab[k];
        return dist_to(x);
    }
    double cp[3]; sub3(p, c, cp);
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dist_to(c);
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double w = d2 / (d2 - d6);
        for (int k = 0; k < 3; ++k) x[k] = a[k] + w * ac[k];
        return dist_to(x);
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; ++k) x[k] = b[k] + w * (c[k] - b[k]);
        return dist_to(x);
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    for (int k = 0; k < 3; ++k) x[k] = a[k] + ab[k] * v + ac[k] * w;
    return dist_to(x);
}

// segment p-q against triangle a,b,c: true if they intersect
static bool seg_tri_intersect(const double* p, const double* q, const double* a, const double* b, const double* c)
{
    double ab[3], ac[3], qp[3], n[3], ap[3];
    sub3(b, a, ab); sub3(c, a, ac); sub3(p, q, qp);
    cross3(ab, ac, n);
    const double d = dot3(qp, n);
    if (d == 0) return false;
    sub3(p, a, ap);
    double t = dot3(ap, n);
    double e[3];
    cross3(qp, ap, e);
    double v = dot3(ac, e);
    double w = -dot3(ab, e);
    if (d < 0) { t = -t; v = -v; w = -w; }
    const double ad = std::abs(d);
    if (t < 0 || t > ad) return false;
    if (v < 0 || v > ad) return false;
    if (w < 0 || v + w > ad) return false;
    return true;
}

static double poly_sqdist(int dom, const double* hp, const double* hq)
{
    if (dom == 1) return seg_seg_sqdist(hp, hp + 3, hq, hq + 3);
    // triangles
    for (int e = 0; e < 3; ++e) {
        if (seg_tri_intersect(hp + 3 * e, hp + 3 * ((e + 1) % 3), hq, hq + 3, hq + 6)) return 0.0;
        if (seg_tri_intersect(hq + 3 * e, hq + 3 * ((e + 1) % 3), hp, hp + 3, hp + 6)) return 0.0;
    }
    double best = std::numeric_limits<double>::max();
    for (int v = 0; v < 3; ++v) {
        best = std::min(best, point_tri_sqdist(hp + 3 * v, hq, hq + 3, hq + 6));
        best = std::min(best, point_tri_sqdist(hq + 3 * v, hp, hp + 3, hp + 6));
    }
    for (int e = 0; e < 3; ++e)
        for (int f = 0; f < 3; ++f)
            best = std::min(best, seg_seg_sqdist(hp + 3 * e, hp + 3 * ((e + 1) % 3), hq + 3 * f, hq + 3 * ((f + 1) % 3)));
    return best;
}

// ----------------------------------------------------------------------------
// Block cluster tree: dual-tree traversal
// (src/ClusterTreePairTraversor/Traverse_DepthFirst.hpp:52-258) with the split
// kernel of src/BlockClusterTree/BlockSplit_Kernel.hpp:164-251.
// ----------------------------------------------------------------------------
static void build_block_cluster_tree(Mesh& M)
{
    const double far_t2 = M.set.theta_far * M.set.theta_far;
    const double near_t2 = M.set.theta_near * M.set.theta_near;
    const double eps2 = std::numeric_limits<double>::epsilon();  // GJK eps^2, src/GJK.hpp:79-80
    const int ps = M.poly_size();
    const int SIZE = M.SIZE;

    std::vector<std::pair<Int, Int>> near_l, far_l, vn_l, inter_l;

    auto adjacent = [&](Int pi, Int pj) {
        const Int* a = &M.S[SIZE * M.perm[pi]];
        const Int* b = &M.S[SIZE * M.perm[pj]];
        for (int u = 0; u < SIZE; ++u)
            for (int v = 0; v < SIZE; ++v)
                if (a[u] == b[v]) return true;
        return false;
    };

    auto leaf = [&](Int pi, Int pj) {  // pi < pj
        const double* A = &M.P_poly[ps * static_cast<size_t>(pi)];
        const double* B = &M.P_poly[ps * static_cast<size_t>(pj)];
        if (adjacent(pi, pj)) { near_l.emplace_back(pi, pj); return; }
        const double d2 = poly_sqdist(M.dom, A + 1 + AMB, B + 1 + AMB);
        const double tol = std::max(A[0], B[0]);
        if (near_t2 * d2 > tol) { near_l.emplace_back(pi, pj); return; }
        const double tol_i = eps2 * std::min(A[0], B[0]);
        if (near_t2 * d2 <= tol_i) inter_l.emplace_back(pi, pj);
        else vn_l.emplace_back(pi, pj);
    };

    std::vector<std::pair<Int, Int>> stack;
    stack.emplace_back(0, 0);
    while (!stack.empty()) {
        auto [i, j] = stack.back();
        stack.pop_back();
        const double* Bi = &M.C_box[7 * static_cast<size_t>(i)];
        const double* Bj = &M.C_box[7 * static_cast<size_t>(j)];
        const bool adm = (i != j) && (std::max(Bi[0], Bj[0]) < far_t2 * aabb_sq_dist(Bi, Bj));
        if (adm) {
            if (i <= j) far_l.emplace_back(i, j); else far_l.emplace_back(j, i);
            continue;
        }
        const Int Li = M.C_left[i], Lj = M.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const Int Ri = M.C_right[i], Rj = M.C_right[j];
            const double si = (Li >= 0) ? Bi[0] : 0.0;
            const double sj = (Lj >= 0) ? Bj[0] : 0.0;
            if (si == sj && si > 0) {
                if (i == j) {
                    stack.emplace_back(Li, Rj);
                    stack.emplace_back(Ri, Rj);
                    stack.emplace_back(Li, Lj);
                } else {
                    stack.emplace_back(Ri, Rj);
                    stack.emplace_back(Li, Rj);
                    stack.emplace_back(Ri, Lj);
                    stack.emplace_back(Li, Lj);
                }
            } else if (si > sj) {
                stack.emplace_back(Ri, j);
                stack.emplace_back(Li, j);
            } else {
                stack.emplace_back(i, Rj);
                stack.emplace_back(i, Lj);
            }
        } else {
            if (i == j) continue;  // ComputeLeafDiagonal is a no-op
            const Int ii = M.C_begin[i], jj = M.C_begin[j];
            if (ii < jj) leaf(ii, jj); else leaf(jj, ii);
        }
    }
    M.near = make_symmetric_pattern(M.nS, near_l);
    M.far = make_symmetric_pattern(M.NC, far_l);
    M.verynear = make_symmetric_pattern(M.nS, vn_l);
    M.inter = make_symmetric_pattern(M.nS, inter_l);
}

// ----------------------------------------------------------------------------
// Primitive data, cluster moments (upsweep) and frozen Pre/Post operators
// ----------------------------------------------------------------------------
static void compute_primitive_data(Mesh& M, bool first)
{
    const int nd = near_dim(M.dom);
    std::vector<double> near(static_cast<size_t>(M.nS) * nd), far(static_cast<size_t>(M.nS) * FAR_DIM);
    std::vector<SimplexData> sd(M.nS);
    parallel_do(M.set.threads, [&](int t) {
        const Int b = job_pointer(M.nS, M.set.threads, t), e = job_pointer(M.nS, M.set.threads, t + 1);
        for (Int i = b; i < e; ++i) {
            read_simplex(M, M.V.data(), i, sd[i]);
            write_near(M, sd[i], &near[nd * static_cast<size_t>(i)]);
            write_far(sd[i], &far[FAR_DIM * static_cast<size_t>(i)]);
        }
    });
    M.P_near.resize(near.size());
    M.P_far.resize(far.size());
    for (Int i = 0; i < M.nS; ++i) {
        const Int j = M.perm[i];
        std::memcpy(&M.P_near[nd * static_cast<size_t>(i)], &near[nd * static_cast<size_t>(j)], nd * sizeof(double));
        std::memcpy(&M.P_far[FAR_DIM * static_cast<size_t>(i)], &far[FAR_DIM * static_cast<size_t>(j)], FAR_DIM * sizeof(double));
    }
    if (first) {
        // frozen pre/post (src/ClusterTree.hpp:410-506 scaled by the construction-time a)
        const int SIZE = M.SIZE;
        M.pre_cols.resize(static_cast<size_t>(M.nS) * SIZE);
        M.pre_vals.resize(static_cast<size_t>(M.nS) * 4 * SIZE);
        const double nth = 1.0 / SIZE;
        for (Int i = 0; i < M.nS; ++i) {
            const SimplexData& d = sd[M.perm[i]];
            const double a = M.P_near[nd * static_cast<size_t>(i)];
            for (int l = 0; l < SIZE; ++l) {
                M.pre_cols[SIZE * static_cast<size_t>(i) + l] = d.sorted[l];
                M.pre_vals[(4 * static_cast<size_t>(i) + 0) * SIZE + l] = a * nth;
                for (int k = 0; k < AMB; ++k) M.pre_vals[(4 * static_cast<size_t>(i) + 1 + k) * SIZE + l] = a * d.Df[k][l];
            }
        }
    }
}

// src/ClusterTree/ComputeClusterData_Thread.hpp:50-129 (children before parents:
// reverse DFS order)
static void compute_cluster_data(Mesh& M)
{
    M.C_far.assign(static_cast<size_t>(M.NC) * FAR_DIM, 0.0);
    for (Int C = M.NC; C-- > 0;) {
        double* CC = &M.C_far[FAR_DIM * static_cast<size_t>(C)];
        const Int L = M.C_left[C], R = M.C_right[C];
        if (L >= 0) {
            const double* CL = &M.C_far[FAR_DIM * static_cast<size_t>(L)];
            const double* CR = &M.C_far[FAR_DIM * static_cast<size_t>(R)];
            double Lw = CL[0], Rw = CR[0];
            const double mass = Lw + Rw;
            CC[0] = mass;
            const double inv = 1.0 / mass;
            Lw *= inv; Rw *= inv;
            for (int k = 1; k < FAR_DIM; ++k) CC[k] = Lw * CL[k] + Rw * CR[k];
        } else {
            std::memcpy(CC, &M.P_far[FAR_DIM * static_cast<size_t>(M.C_begin[C])], FAR_DIM * sizeof(double));
        }
    }
}

// ----------------------------------------------------------------------------
// Integer powers (Tensors' Power<Real,Int>: exact repeated multiplication,
// reciprocal for negative exponents).
// ----------------------------------------------------------------------------
template <typename R>
static inline R ipow(R x, int k)
{
    if (k < 0) return R(1.0) / ipow(x, -k);
    R r = R(1.0);
    R b = x;
    bool first = true;
    while (k) {
        if (k & 1) {
            if (first) { r = b; first = false; }   // 1 * b is not an operation
            else r = r * b;
        }
        k >>= 1;
        if (k) b = b * b;
    }
    return r;
}

struct TPParams {
    double q, p;
    int q_half_int, p_half_int;
    bool q_int, p_int;
    double s_exp_metric;   // src/Energies/TangentPointEnergy0/TP0_Kernel_FF.hpp:72-73
    int dom;
    TPParams(double q_, double p_, int dom_) : q(q_), p(p_), dom(dom_)
    {
        q_half_int = static_cast<int>(q / 2); p_half_int = static_cast<int>(p / 2);
        q_int = (q / 2 == static_cast<double>(q_half_int));
        p_int = (p / 2 == static_cast<double>(p_half_int));
        const double s = (p - dom) / q;
        s_exp_metric = -0.5 * (2.0 * (s - 1.0) + dom);
    }
};

// ----------------------------------------------------------------------------
// Operation counting (test infrastructure for the roofline's algorithmic flops): a double
// that counts its arithmetic. add/sub, mul, div, sqrt and pow calls are counted
// separately; abs and comparisons are not arithmetic.
// ----------------------------------------------------------------------------
struct OpCounts { int64_t add = 0, mul = 0, div = 0, sqrt = 0, pow = 0; };
static thread_local OpCounts g_ops;
struct FC {
    double v = 0;
    FC() = default;
    FC(double x) : v(x) {}   // NOLINT: implicit from double, as a Real would be
};
static inline FC operator+(FC a, FC b) { ++g_ops.add; return FC(a.v + b.v); }
static inline FC operator-(FC a, FC b) { ++g_ops.add; return FC(a.v - b.v); }
static inline FC operator*(FC a, FC b) { ++g_ops.mul; return FC(a.v * b.v); }
static inline FC operator/(FC a, FC b) { ++g_ops.div; return FC(a.v / b.v); }
static inline FC operator-(FC a) { return FC(-a.v); }
static inline FC& operator+=(FC& a, FC b) { a = a + b; return a; }
static inline FC& operator-=(FC& a, FC b) { a = a - b; return a; }
static inline FC& operator*=(FC& a, FC b) { a = a * b; return a; }
static inline FC fc_abs(FC a) { return FC(std::fabs(a.v)); }
static inline double fc_abs(double a) { return std::fabs(a); }
static inline FC fc_pow(FC a, double e) { ++g_ops.pow; return FC(std::pow(a.v, e)); }
static inline double fc_pow(double a, double e) { return std::pow(a, e); }

// Power of r2 by (-p/2 - 1), and |c|^(q/2 - 1)
template <typename R>
static inline R pow_r_mp2(const TPParams& T, R r2)
{
    return T.p_int ? ipow(r2, -T.p_half_int - 1) : fc_pow(r2, -T.p / 2 - 1);
}
template <typename R>
static inline R pow_c(const TPParams& T, R c_abs)
{
    return T.q_int ? ipow(c_abs, T.q_half_int - 1) : fc_pow(c_abs, T.q / 2 - 1);
}

// One pair of the TP0 FF/NF kernels (TP0_Kernel_FF.hpp:130-319, TP0_Kernel_NF.hpp:140-338)
// in moment coordinates. x,y centres; P,Q packed projectors; a,b weights.
// Outputs (if non-null): DX/DY in (a, x, P) layout of FF (10 entries). For NF
// the hull slots are filled from the x-slot by the caller.
template <typename R>
struct PairOutT {
    R E;          // energy density E (without a*b)
    R energy;     // a*E*b
    R dens_x;     // density contribution at x: b |Pv|^q / |v|^p (TP0_Kernel_FF.hpp:214-218)
    R dens_y;     // density contribution at y: a |Qv|^q / |v|^p
    R DX[10], DY[10];
    R a0, a1;     // metric block
};
using PairOut = PairOutT<double>;

template <typename R>
static inline void tp0_pair(const TPParams& T, R a, const R* x, const R* P, R b, const R* y, const R* Q, bool diff,
                            bool metric, PairOutT<R>& o)
{
    R v[3], Pv[3], Qv[3], V[6];
    R r2, cphi, cpsi;
    for (int l = 0; l < 3; ++l) {
        v[l] = y[l] - x[l];
        r2 = (l == 0) ? v[l] * v[l] : r2 + v[l] * v[l];
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            const int k = lin_k(i, j);
            Pv[i] = (j == 0) ? P[k] * v[j] : Pv[i] + P[k] * v[j];
            Qv[i] = (j == 0) ? Q[k] * v[j] : Qv[i] + Q[k] * v[j];
            if (j > i) V[k] = R(2.0) * v[i] * v[j];
            else if (j == i) V[k] = v[i] * v[j];
        }
        cphi = (i == 0) ? v[i] * Pv[i] : cphi + v[i] * Pv[i];
        cpsi = (i == 0) ? v[i] * Qv[i] : cpsi + v[i] * Qv[i];
    }
    const R rmp2 = pow_r_mp2(T, r2);
    const R rmp = rmp2 * r2;
    const R cphi_qm2 = pow_c(T, fc_abs(cphi));
    const R cpsi_qm2 = pow_c(T, fc_abs(cpsi));
    const R cphi_q = cphi_qm2 * cphi;
    const R cpsi_q = cpsi_qm2 * cpsi;
    const R Num = cphi_q + cpsi_q;
    const R E = Num * rmp;
    o.E = E;
    o.energy = a * E * b;
    o.dens_x = R(0.0);
    o.dens_y = R(0.0);
    if (!diff && !metric) {   // densities only where an energy alone is asked for
        o.dens_x = b * cphi_q * rmp;
        o.dens_y = a * cpsi_q * rmp;
    }
    if (diff) {
        const R factor = R(T.q) * rmp;
        const R Kxy = factor * cphi_qm2;
        const R Kyx = factor * cpsi_qm2;
        const R H = R(T.p) * rmp2 * Num;
        R dEdvx, dEdvy;
        for (int i = 0; i < 3; ++i) {
            const R dEdv = Kxy * Pv[i] + Kyx * Qv[i] - H * v[i];
            dEdvx = (i == 0) ? dEdv * x[i] : dEdvx + dEdv * x[i];
            dEdvy = (i == 0) ? dEdv * y[i] : dEdvy + dEdv * y[i];
            o.DX[1 + i] = -(b * dEdv);
            o.DY[1 + i] = a * dEdv;
        }
        o.DX[0] = b * (E - R(0.5) * factor * cphi_q + dEdvx);
        o.DY[0] = a * (E - R(0.5) * factor * cpsi_q - dEdvy);
        const R hbK = R(0.5) * b * Kxy, haK = R(0.5) * a * Kyx;
        for (int k = 0; k < 6; ++k) { o.DX[4 + k] = hbK * V[k]; o.DY[4 + k] = haK * V[k]; }
    }
    if (metric) {
        const R r4 = r2 * r2;
        const R a1 = R(-2.0) * fc_pow(r2, T.s_exp_metric);
        const R a0 = R(0.5) * (cphi + cpsi) / r4 * a1;
        o.a0 = a0;
        o.a1 = a1;
    }
}

// Upper-triangular job pointers balanced by nnz (UpperTriangularJobPtr of Tensors)
static std::vector<Int> upper_job_ptr(const Pattern& P, int threads)
{
    std::vector<LInt> cost(P.rows + 1, 0);
    for (Int i = 0; i < P.rows; ++i) cost[i + 1] = cost[i] + (P.rp[i + 1] - P.diag[i]);
    std::vector<Int> jp(threads + 1, 0);
    jp[threads] = P.rows;
    const LInt total = cost[P.rows];
    for (int t = 1; t < threads; ++t) {
        const LInt target = (total * t) / threads;
        jp[t] = static_cast<Int>(std::lower_bound(cost.begin(), cost.end(), target) - cost.begin());
        jp[t] = std::max(jp[t], jp[t - 1]);
    }
    return jp;
}

// ----------------------------------------------------------------------------
// VF adaptive quadrature on very-near pairs
// (src/FMM/FMM_Kernel_VF_Common.hpp:3-116, src/Energies/TangentPointEnergy0/TP0_Kernel_VF.hpp:159-378,
//  src/SimplexHierarchy/SimplexHierarchy_2D.hpp:17-128). Barycentric sub-simplices:
// triangles split 1:4, edges 1:2; a sub-pair is evaluated once the GJK MAC with
// theta_near holds or the level limit is reached, with weight w_S * w_T.
// ----------------------------------------------------------------------------
struct SubSimplex { double bary[3][3]; int level; double w; };

static void sub_corners(int dom, const double* hull, const SubSimplex& s, double* out)
{
    for (int c = 0; c < dom + 1; ++c)
        for (int k = 0; k < 3; ++k) {
            double acc = 0;
            for (int v = 0; v < dom + 1; ++v) acc += s.bary[c][v] * hull[3 * v + k];
            out[3 * c + k] = acc;
        }
}

static void subdivide(int dom, const SubSimplex& s, std::vector<SubSimplex>& out)
{
    if (dom == 1) {
        double m[3];
        for (int v = 0; v < 2; ++v) m[v] = 0.5 * (s.bary[0][v] + s.bary[1][v]);
        m[2] = 0;
        SubSimplex a = s, b = s;
        for (int v = 0; v < 3; ++v) { a.bary[1][v] = m[v]; b.bary[0][v] = m[v]; }
        a.level = b.level = s.level + 1;
        a.w = b.w = 0.5 * s.w;
        out.push_back(a); out.push_back(b);
        return;
    }
    double m01[3], m12[3], m20[3];
    for (int v = 0; v < 3; ++v) {
        m01[v] = 0.5 * (s.bary[0][v] + s.bary[1][v]);
        m12[v] = 0.5 * (s.bary[1][v] + s.bary[2][v]);
        m20[v] = 0.5 * (s.bary[2][v] + s.bary[0][v]);
    }
    auto mk = [&](const double* A, const double* B, const double* C) {
        SubSimplex t;
        for (int v = 0; v < 3; ++v) { t.bary[0][v] = A[v]; t.bary[1][v] = B[v]; t.bary[2][v] = C[v]; }
        t.level = s.level + 1;
        t.w = 0.25 * s.w;
        out.push_back(t);
    };
    mk(s.bary[0], m01, m20);
    mk(m01, s.bary[1], m12);
    mk(m20, m12, s.bary[2]);
    mk(m01, m12, m20);
}

// Evaluates the very-near pair (i,j) by adaptive subdivision
// (FMM_Kernel_VF_Common.hpp:3-116): both simplices are refined together, the
// traversal starts at the level-1 child pairs, and a sub-pair is evaluated once
// the GJK MAC with theta_near holds or the level limit is reached. emit() gets the
// sub-simplex centres, their weights w_S, w_T and barycentric centres.
template <typename Emit>
static void vf_quadrature(const Mesh& M, Int i, const Mesh& O, Int j, Emit&& emit)
{
    const int dom = M.dom, SIZE = M.SIZE;
    const int nd = near_dim(dom);
    const double* X = &M.P_near[nd * static_cast<size_t>(i)];
    const double* Y = &O.P_near[nd * static_cast<size_t>(j)];
    const double near_t2 = M.set.theta_near * M.set.theta_near;
    SubSimplex root{};
    for (int c = 0; c < 3; ++c)
        for (int v = 0; v < 3; ++v) root.bary[c][v] = (c == v && c < SIZE) ? 1.0 : 0.0;
    root.level = 0;
    root.w = 1.0;
    std::vector<std::pair<SubSimplex, SubSimplex>> stack;
    {
        std::vector<SubSimplex> cs, ct;
        subdivide(dom, root, cs);
        subdivide(dom, root, ct);
        for (auto& u : cs) for (auto& w : ct) stack.emplace_back(u, w);
    }
    std::vector<SubSimplex> cs, ct;
    while (!stack.empty()) {
        auto [s, t] = stack.back();
        stack.pop_back();
        double hs[9], ht[9];
        sub_corners(dom, X + 1, s, hs);
        sub_corners(dom, Y + 1, t, ht);
        double cs_[3] = {0, 0, 0}, ct_[3] = {0, 0, 0}, rs = 0, rt = 0;
        for (int c = 0; c < SIZE; ++c)
            for (int k = 0; k < 3; ++k) { cs_[k] += hs[3 * c + k] / SIZE; ct_[k] += ht[3 * c + k] / SIZE; }
        for (int c = 0; c < SIZE; ++c) {
            double ds = 0, dt = 0;
            for (int k = 0; k < 3; ++k) {
                ds += (hs[3 * c + k] - cs_[k]) * (hs[3 * c + k] - cs_[k]);
                dt += (ht[3 * c + k] - ct_[k]) * (ht[3 * c + k] - ct_[k]);
            }
            rs = std::max(rs, ds); rt = std::max(rt, dt);
        }
        bool stop = s.level >= M.set.max_refinement;
        if (!stop) {
            const double d2 = poly_sqdist(dom, hs, ht);
            stop = near_t2 * d2 > std::max(rs, rt);
        }
        if (stop) {
            double bs[3] = {0, 0, 0}, bt[3] = {0, 0, 0};
            for (int c = 0; c < SIZE; ++c)
                for (int v = 0; v < SIZE; ++v) { bs[v] += s.bary[c][v] / SIZE; bt[v] += t.bary[c][v] / SIZE; }
            emit(cs_, ct_, s.w, t.w, bs, bt);
            continue;
        }
        cs.clear(); ct.clear();
        subdivide(dom, s, cs);
        subdivide(dom, t, ct);
        for (auto& u : cs) for (auto& w : ct) stack.emplace_back(u, w);
    }
}

// ----------------------------------------------------------------------------
// Energy / differential traversal (TP0_Traversor::Compute, TP0_Traversor.hpp:129-376)
// ----------------------------------------------------------------------------
struct EvalResult { double energy; };

// CollectFarFieldDerivatives (src/ClusterTree.hpp:1164-1208), PercolateDown and
// ClustersToPrimitives, CollectNearFieldDerivatives (src/ClusterTree.hpp:1115-1161):
// per-thread buffers summed, far field pushed to the primitives, both unpermuted.
static void collect_derivatives(Mesh& M, const std::vector<std::vector<double>>& tDn,
                                const std::vector<std::vector<double>>& tDf, int threads, int nd)
{
        // CollectFarFieldDerivatives (src/ClusterTree.hpp:1164-1208)
    std::vector<double> C_out(static_cast<size_t>(M.NC) * FAR_DIM, 0.0);
    for (int t = 0; t < threads; ++t)
        for (size_t k = 0; k < C_out.size(); ++k) C_out[k] += tDf[t][k];
    for (Int C = 0; C < M.NC; ++C) {  // PercolateDown: parents before children in DFS order
        const Int L = M.C_left[C];
        if (L >= 0) {
            const Int R = M.C_right[C];
            for (int k = 0; k < FAR_DIM; ++k) {
                C_out[FAR_DIM * static_cast<size_t>(L) + k] += C_out[FAR_DIM * static_cast<size_t>(C) + k];
                C_out[FAR_DIM * static_cast<size_t>(R) + k] += C_out[FAR_DIM * static_cast<size_t>(C) + k];
            }
        }
    }
    std::vector<double> P_out(static_cast<size_t>(M.nS) * FAR_DIM, 0.0);
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] < 0)
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i)
                for (int k = 0; k < FAR_DIM; ++k) P_out[FAR_DIM * static_cast<size_t>(i) + k] = C_out[FAR_DIM * static_cast<size_t>(C) + k];
    M.P_D_far.assign(static_cast<size_t>(M.nS) * FAR_DIM, 0.0);
    M.P_D_near.assign(static_cast<size_t>(M.nS) * nd, 0.0);
    for (Int i = 0; i < M.nS; ++i) {
        const Int pi = M.inv_perm[i];
        for (int k = 0; k < FAR_DIM; ++k) M.P_D_far[FAR_DIM * static_cast<size_t>(i) + k] = P_out[FAR_DIM * static_cast<size_t>(pi) + k];
        for (int t = 0; t < threads; ++t)
            for (int k = 0; k < nd; ++k) M.P_D_near[nd * static_cast<size_t>(i) + k] += tDn[t][nd * static_cast<size_t>(pi) + k];
    }
    }

// Full evaluation (only < 0), or the slice of one "thread" of `shards` (only >= 0): the
// upper-triangle rows job_pointer(only)..job_pointer(only + 1) of every list, the way the
// reference splits rows over threads (src/FMM/FMM_Traversor.hpp:65-101); the slice's
// derivatives are left in tDn_out / tDf_out (tree order) instead of being collected.
static double tp0_evaluate(Mesh& M, double q, double p, bool diff, int shards = 0, int only = -1,
                           std::vector<double>* tDn_out = nullptr, std::vector<double>* tDf_out = nullptr)
{
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom);
    const int SIZE = M.SIZE;
    const int threads = shards > 0 ? shards : std::max(1, M.set.threads);
    const double S_scale = 1.0 / SIZE;

    std::vector<std::vector<double>> tDn, tDf;   // thread_P_D_near, thread_C_D_far
    if (diff) {
        tDn.assign(threads, std::vector<double>(static_cast<size_t>(M.nS) * nd, 0.0));
        tDf.assign(threads, std::vector<double>(static_cast<size_t>(M.NC) * FAR_DIM, 0.0));
    }
    double en = 0;

    // VF
    if (M.verynear.nnz() > 0) {
        const Pattern& Pt = M.verynear;
        std::vector<double> part(threads, 0.0);
        auto jp = upper_job_ptr(Pt, threads);
        parallel_do(threads, [&](int t) {
            if (only >= 0 && t != only) return;
            double local = 0;
            for (Int i = jp[t]; i < jp[t + 1]; ++i)
                for (LInt k = Pt.diag[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
                    const double* Yj = &M.P_near[nd * static_cast<size_t>(j)];
                    vf_quadrature(M, i, M, j, [&](const double* x, const double* y, double ws, double wt,
                                               const double* bs, const double* bt) {
                        // sub-pair with weights a*w_S, b*w_T: energy w a E b, derivatives in
                        // (a, a*hull, a*P) coordinates (TP0_Kernel_VF.hpp:159-301)
                        PairOut o;
                        tp0_pair(T, Xi[0] * ws, x, Xi + 1 + AMB * SIZE, Yj[0] * wt, y, Yj + 1 + AMB * SIZE, diff, false, o);
                        local += o.energy;
                        if (diff) {
                            double* DX = &tDn[t][nd * static_cast<size_t>(i)];
                            double* DY = &tDn[t][nd * static_cast<size_t>(j)];
                            DX[0] += ws * o.DX[0];
                            DY[0] += wt * o.DY[0];
                            for (int v = 0; v < SIZE; ++v)
                                for (int kk = 0; kk < 3; ++kk) {
                                    DX[1 + 3 * v + kk] += ws * bs[v] * o.DX[1 + kk];
                                    DY[1 + 3 * v + kk] += wt * bt[v] * o.DY[1 + kk];
                                }
                            for (int kk = 0; kk < 6; ++kk) {
                                DX[1 + AMB * SIZE + kk] += ws * o.DX[4 + kk];
                                DY[1 + AMB * SIZE + kk] += wt * o.DY[4 + kk];
                            }
                        }
                    });
                }
            part[t] = local;
        });
        for (double v : part) en += v;
    }

    // NF
    if (M.near.nnz() > 0) {
        const Pattern& Pt = M.near;
        std::vector<double> part(threads, 0.0);
        auto jp = upper_job_ptr(Pt, threads);
        parallel_do(threads, [&](int t) {
            if (only >= 0 && t != only) return;
            double local = 0;
            for (Int i = jp[t]; i < jp[t + 1]; ++i) {
                if (Pt.rp[i + 1] <= Pt.diag[i]) continue;
                const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
                double x[3];
                for (int k = 0; k < 3; ++k) {
                    x[k] = S_scale * Xi[1 + k];
                    for (int kk = 1; kk < SIZE; ++kk) x[k] += S_scale * Xi[1 + AMB * kk + k];
                }
                double DXs[16] = {0};
                for (LInt k = Pt.diag[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Yj = &M.P_near[nd * static_cast<size_t>(j)];
                    double y[3];
                    for (int kk = 0; kk < 3; ++kk) {
                        y[kk] = S_scale * Yj[1 + kk];
                        for (int v = 1; v < SIZE; ++v) y[kk] += S_scale * Yj[1 + AMB * v + kk];
                    }
                    PairOut o;
                    tp0_pair(T, Xi[0], x, Xi + 1 + AMB * SIZE, Yj[0], y, Yj + 1 + AMB * SIZE, diff, false, o);
                    local += o.energy;
                    if (diff) {
                        double* DY = &tDn[t][nd * static_cast<size_t>(j)];
                        DXs[0] += o.DX[0];
                        DY[0] += o.DY[0];
                        for (int v = 0; v < SIZE; ++v)
                            for (int kk = 0; kk < 3; ++kk) {
                                DXs[1 + 3 * v + kk] += S_scale * o.DX[1 + kk];
                                DY[1 + 3 * v + kk] += S_scale * o.DY[1 + kk];
                            }
                        for (int kk = 0; kk < 6; ++kk) {
                            DXs[1 + AMB * SIZE + kk] += o.DX[4 + kk];
                            DY[1 + AMB * SIZE + kk] += o.DY[4 + kk];
                        }
                    }
                }
                if (diff) {
                    double* DX = &tDn[t][nd * static_cast<size_t>(i)];
                    for (int kk = 0; kk < nd; ++kk) DX[kk] += DXs[kk];
                }
            }
            part[t] = local;
        });
        for (double v : part) en += v;
    }

    // FF
    if (M.far.nnz() > 0) {
        const Pattern& Pt = M.far;
        std::vector<double> part(threads, 0.0);
        auto jp = upper_job_ptr(Pt, threads);
        parallel_do(threads, [&](int t) {
            if (only >= 0 && t != only) return;
            double local = 0;
            for (Int i = jp[t]; i < jp[t + 1]; ++i) {
                if (Pt.rp[i + 1] <= Pt.diag[i]) continue;
                const double* Xi = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
                double DXs[10] = {0};
                for (LInt k = Pt.diag[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Yj = &M.C_far[FAR_DIM * static_cast<size_t>(j)];
                    PairOut o;
                    tp0_pair(T, Xi[0], Xi + 1, Xi + 4, Yj[0], Yj + 1, Yj + 4, diff, false, o);
                    local += o.energy;
                    if (diff) {
                        double* DY = &tDf[t][FAR_DIM * static_cast<size_t>(j)];
                        for (int kk = 0; kk < 10; ++kk) { DXs[kk] += o.DX[kk]; DY[kk] += o.DY[kk]; }
                    }
                }
                if (diff) {
                    double* DX = &tDf[t][FAR_DIM * static_cast<size_t>(i)];
                    for (int kk = 0; kk < 10; ++kk) DX[kk] += DXs[kk];
                }
            }
            part[t] = local;
        });
        for (double v : part) en += v;
    }

    if (diff && only >= 0) {
        if (tDn_out) *tDn_out = tDn[only];
        if (tDf_out) *tDf_out = tDf[only];
    } else if (diff) {
        collect_derivatives(M, tDn, tDf, threads, nd);
    }
    return en;
}

// ----------------------------------------------------------------------------
// DNearFarToHulls by forward-mode differentiation of the moment map
// (CodeGeneration/SimplicialMesh/Code_DNearFar_to_Hulls.m:130-261; generated
// code at src/SimplicialMesh/SimplicialMeshDetails.hpp:529-733 and :1097-1410).
// ----------------------------------------------------------------------------
struct Dual { double v, d; };
static inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
static inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
static inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
static inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
static inline Dual dsqrt(Dual a) { const double s = std::sqrt(a.v); return {s, a.d / (2 * s)}; }

static void moments_dual(int dom, const Dual* h, Dual* nearm, Dual* farm)
{
    const int SIZE = dom + 1;
    Dual vol, pr[3][3];
    if (dom == 1) {
        Dual tau[3];
        for (int k = 0; k < 3; ++k) tau[k] = h[3 + k] - h[k];
        Dual tt = tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2];
        vol = dsqrt(tt);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) pr[i][j] = Dual{i == j ? 1.0 : 0.0, 0.0} - tau[i] * tau[j] / tt;
    } else {
        Dual e1[3], e2[3], nu[3];
        for (int k = 0; k < 3; ++k) { e1[k] = h[3 + k] - h[k]; e2[k] = h[6 + k] - h[k]; }
        nu[0] = e1[1] * e2[2] - e1[2] * e2[1];
        nu[1] = e1[2] * e2[0] - e1[0] * e2[2];
        nu[2] = e1[0] * e2[1] - e1[1] * e2[0];
        Dual nn = nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2];
        vol = Dual{0.5, 0.0} * dsqrt(nn);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) pr[i][j] = nu[i] * nu[j] / nn;
    }
    nearm[0] = vol;
    for (int c = 0; c < SIZE; ++c)
        for (int k = 0; k < 3; ++k) nearm[1 + 3 * c + k] = vol * h[3 * c + k];
    int kk = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) { nearm[1 + 3 * SIZE + kk] = vol * pr[i][j]; farm[4 + kk] = vol * pr[i][j]; ++kk; }
    farm[0] = vol;
    for (int k = 0; k < 3; ++k) {
        Dual m{0, 0};
        for (int c = 0; c < SIZE; ++c) m = m + h[3 * c + k];
        farm[1 + k] = vol * m / Dual{static_cast<double>(SIZE), 0.0};
    }
}

static void dnearfar_to_hulls(const Mesh& M, std::vector<double>& B)
{
    const int SIZE = M.SIZE, nd = near_dim(M.dom);
    B.assign(static_cast<size_t>(M.nS) * SIZE * AMB, 0.0);
    for (Int i = 0; i < M.nS; ++i) {
        double charge = 0;
        for (int c = 0; c < SIZE; ++c) charge += M.charge_v[M.S[SIZE * i + c]];
        charge /= SIZE;
        const double* N = &M.P_D_near[nd * static_cast<size_t>(i)];
        const double* F = &M.P_D_far[FAR_DIM * static_cast<size_t>(i)];
        for (int c = 0; c < SIZE; ++c)
            for (int k = 0; k < 3; ++k) {
                Dual h[9];
                for (int cc = 0; cc < SIZE; ++cc)
                    for (int kk = 0; kk < 3; ++kk)
                        h[3 * cc + kk] = Dual{M.V[3 * static_cast<size_t>(M.S[SIZE * i + cc]) + kk], (cc == c && kk == k) ? 1.0 : 0.0};
                Dual nm[16], fm[10];
                moments_dual(M.dom, h, nm, fm);
                double acc = 0;
                for (int l = 0; l < nd; ++l) acc += N[l] * nm[l].d;
                for (int l = 0; l < FAR_DIM; ++l) acc += F[l] * fm[l].d;
                B[(static_cast<size_t>(i) * SIZE + c) * AMB + k] = charge * acc;
            }
    }
}

// Closed-form DNearFarToHulls (same map as the forward-mode version above, written
// out by hand; this is the fast path used for timing). For triangles
// vol = |nu|/2, P = nu nu^T/|nu|^2; for edges vol = |tau|, P = I - tau tau^T/|tau|^2.
static void dnearfar_to_hulls_closed(const Mesh& M, std::vector<double>& B)
{
    const int SIZE = M.SIZE, nd = near_dim(M.dom);
    B.assign(static_cast<size_t>(M.nS) * SIZE * AMB, 0.0);
    parallel_do(std::max(1, M.set.threads), [&](int t) {
        const Int b0 = job_pointer(M.nS, M.set.threads, t), e0 = job_pointer(M.nS, M.set.threads, t + 1);
        for (Int i = b0; i < e0; ++i) {
            const Int* s = &M.S[SIZE * static_cast<size_t>(i)];
            double h[3][3];
            double charge = 0;
            for (int c = 0; c < SIZE; ++c) {
                charge += M.charge_v[s[c]];
                for (int k = 0; k < 3; ++k) h[c][k] = M.V[3 * static_cast<size_t>(s[c]) + k];
            }
            charge /= SIZE;
            const double* N = &M.P_D_near[nd * static_cast<size_t>(i)];
            const double* F = &M.P_D_far[FAR_DIM * static_cast<size_t>(i)];
            double Gp[6], G[3][3];
            for (int k = 0; k < 6; ++k) Gp[k] = N[1 + 3 * SIZE + k] + F[4 + k];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) G[a][b] = (a == b) ? Gp[lin_k(a, b)] : 0.5 * Gp[lin_k(a, b)];
            double center[3] = {0, 0, 0};
            for (int c = 0; c < SIZE; ++c)
                for (int k = 0; k < 3; ++k) center[k] += h[c][k];
            for (int k = 0; k < 3; ++k) center[k] /= SIZE;
            double vol, P[3][3];
            double gradvol[3][3], gradGP[3][3];
            if (M.dom == 2) {
                double e1[3], e2[3], nu[3];
                sub3(h[1], h[0], e1); sub3(h[2], h[0], e2); cross3(e1, e2, nu);
                const double len = std::sqrt(dot3(nu, nu));
                double n_[3] = {nu[0] / len, nu[1] / len, nu[2] / len};
                vol = 0.5 * len;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) P[a][b] = n_[a] * n_[b];
                double Gn[3] = {0, 0, 0};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) Gn[a] += G[a][b] * n_[b];
                const double nGn = dot3(n_, Gn);
                double w[3];
                for (int a = 0; a < 3; ++a) w[a] = 2.0 * (Gn[a] - nGn * n_[a]) / len;
                for (int c = 0; c < 3; ++c) {
                    double u[3];
                    sub3(h[(c + 1) % 3], h[(c + 2) % 3], u);
                    double un[3], uw[3];
                    cross3(u, n_, un);
                    cross3(u, w, uw);
                    for (int k = 0; k < 3; ++k) { gradvol[c][k] = 0.5 * un[k]; gradGP[c][k] = uw[k]; }
                }
            } else {
                double tau[3];
                sub3(h[1], h[0], tau);
                const double len = std::sqrt(dot3(tau, tau));
                double t_[3] = {tau[0] / len, tau[1] / len, tau[2] / len};
                vol = len;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) P[a][b] = (a == b ? 1.0 : 0.0) - t_[a] * t_[b];
                double Gt[3] = {0, 0, 0};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) Gt[a] += G[a][b] * t_[b];
                const double tGt = dot3(t_, Gt);
                double g[3];
                for (int a = 0; a < 3; ++a) g[a] = -2.0 * (Gt[a] - tGt * t_[a]) / len;
                for (int k = 0; k < 3; ++k) {
                    gradvol[1][k] = t_[k]; gradvol[0][k] = -t_[k];
                    gradGP[1][k] = g[k]; gradGP[0][k] = -g[k];
                }
            }
            double alpha = N[0] + F[0];
            for (int c = 0; c < SIZE; ++c)
                for (int k = 0; k < 3; ++k) alpha += N[1 + 3 * c + k] * h[c][k];
            for (int k = 0; k < 3; ++k) alpha += F[1 + k] * center[k];
            for (int a = 0; a < 3; ++a)
                for (int b = a; b < 3; ++b) alpha += Gp[lin_k(a, b)] * P[a][b];
            for (int c = 0; c < SIZE; ++c)
                for (int k = 0; k < 3; ++k)
                    B[(static_cast<size_t>(i) * SIZE + c) * AMB + k] =
                        charge * (alpha * gradvol[c][k] + vol * (N[1 + 3 * c + k] + F[1 + k] / SIZE) + vol * gradGP[c][k]);
        }
    });
}

static int g_chain_rule_mode = 0;   // 0 closed form, 1 forward-mode differentiation

// SimplicialMesh::Assemble_ClusterTree_Derivatives (src/SimplicialMesh.hpp:651-675)
static void assemble_derivatives(const Mesh& M, double alpha, double beta, double* Y, Int ldY)
{
    std::vector<double> B;
    if (g_chain_rule_mode == 1) dnearfar_to_hulls(M, B); else dnearfar_to_hulls_closed(M, B);
    std::vector<double> acc(static_cast<size_t>(M.nV) * 3, 0.0);
    for (Int i = 0; i < M.nS; ++i)
        for (int c = 0; c < M.SIZE; ++c) {
            const Int v = M.S[M.SIZE * i + c];
            for (int k = 0; k < 3; ++k) acc[3 * static_cast<size_t>(v) + k] += B[(static_cast<size_t>(i) * M.SIZE + c) * 3 + k];
        }
    for (Int v = 0; v < M.nV; ++v)
        for (int k = 0; k < 3; ++k) {
            double& y = Y[static_cast<size_t>(ldY) * v + k];
            y = alpha * acc[3 * static_cast<size_t>(v) + k] + (beta == 0.0 ? 0.0 : beta * y);
        }
}

// ----------------------------------------------------------------------------
// Metric values (TP0 kernels with metric_flag, TP0_Traversor.hpp:297-375) on the
// full symmetric pattern, with row diagonals.
// ----------------------------------------------------------------------------
struct MetricValues {
    std::vector<double> nf, ff, vf;          // 2 per full-pattern nnz
    std::vector<double> nf_diag, ff_diag, vf_diag;  // 2 per row
};

static void tp0_metric_values(const Mesh& M, double q, double p, MetricValues& mv)
{
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom), SIZE = M.SIZE;
    const double S_scale = 1.0 / SIZE;
    auto run = [&](const Pattern& Pt, bool far, std::vector<double>& vals, std::vector<double>& diag) {
        vals.assign(2 * static_cast<size_t>(Pt.nnz()), 0.0);
        diag.assign(2 * static_cast<size_t>(Pt.rows), 0.0);
        auto data = [&](Int i, double* x, double* P, double& a) {
            if (far) {
                const double* X = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
                a = X[0];
                for (int k = 0; k < 3; ++k) x[k] = X[1 + k];
                for (int k = 0; k < 6; ++k) P[k] = X[4 + k];
            } else {
                const double* X = &M.P_near[nd * static_cast<size_t>(i)];
                a = X[0];
                for (int k = 0; k < 3; ++k) {
                    x[k] = S_scale * X[1 + k];
                    for (int v = 1; v < SIZE; ++v) x[k] += S_scale * X[1 + AMB * v + k];
                }
                for (int k = 0; k < 6; ++k) P[k] = X[1 + AMB * SIZE + k];
            }
        };
        for (Int i = 0; i < Pt.rows; ++i) {
            double x[3], P[6], a;
            data(i, x, P, a);
            for (LInt k = Pt.diag[i]; k < Pt.rp[i + 1]; ++k) {
                const Int j = Pt.ci[k];
                double y[3], Q[6], b;
                data(j, y, Q, b);
                PairOut o;
                tp0_pair(T, a, x, P, b, y, Q, false, true, o);
                vals[2 * k] = o.a0;
                vals[2 * k + 1] = o.a1;
                diag[2 * i] -= (b / a) * o.a0;
                diag[2 * i + 1] -= (b / a) * o.a1;
                diag[2 * j] -= (a / b) * o.a0;
                diag[2 * j + 1] -= (a / b) * o.a1;
            }
        }
        // FillLowerTriangleFromUpperTriangle: lower (j,i) gets the block of upper (i,j)
        for (Int i = 0; i < Pt.rows; ++i)
            for (LInt k = Pt.rp[i]; k < Pt.diag[i]; ++k) {
                const Int j = Pt.ci[k];
                LInt kk = std::lower_bound(Pt.ci.begin() + Pt.diag[j], Pt.ci.begin() + Pt.rp[j + 1], i) - Pt.ci.begin();
                vals[2 * k] = vals[2 * kk];
                vals[2 * k + 1] = vals[2 * kk + 1];
            }
    };
    run(M.near, false, mv.nf, mv.nf_diag);
    run(M.far, true, mv.ff, mv.ff_diag);
    mv.vf.clear(); mv.vf_diag.clear();
    if (M.verynear.nnz() > 0) {
        // very-near metric: a single-point evaluation at the barycentres is replaced by
        // the quadrature sum of the same block entries (intended stride-2 semantics)
        const Pattern& Pt = M.verynear;
        mv.vf.assign(2 * static_cast<size_t>(Pt.nnz()), 0.0);
        mv.vf_diag.assign(2 * static_cast<size_t>(Pt.rows), 0.0);
        for (Int i = 0; i < Pt.rows; ++i) {
            const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
            for (LInt k = Pt.diag[i]; k < Pt.rp[i + 1]; ++k) {
                const Int j = Pt.ci[k];
                const double* Yj = &M.P_near[nd * static_cast<size_t>(j)];
                double a0 = 0, a1 = 0;
                vf_quadrature(M, i, M, j, [&](const double* x, const double* y, double ws, double wt, const double*, const double*) {
                    PairOut o;
                    tp0_pair(T, Xi[0], x, Xi + 1 + AMB * SIZE, Yj[0], y, Yj + 1 + AMB * SIZE, false, true, o);
                    a0 += ws * wt * o.a0;
                    a1 += ws * wt * o.a1;
                });
                const double a = Xi[0], b = Yj[0];
                mv.vf[2 * k] = a0; mv.vf[2 * k + 1] = a1;
                mv.vf_diag[2 * i] -= (b / a) * a0; mv.vf_diag[2 * i + 1] -= (b / a) * a1;
                mv.vf_diag[2 * j] -= (a / b) * a0; mv.vf_diag[2 * j + 1] -= (a / b) * a1;
            }
        }
        for (Int i = 0; i < Pt.rows; ++i)
            for (LInt k = Pt.rp[i]; k < Pt.diag[i]; ++k) {
                const Int j = Pt.ci[k];
                LInt kk = std::lower_bound(Pt.ci.begin() + Pt.diag[j], Pt.ci.begin() + Pt.rp[j + 1], i) - Pt.ci.begin();
                mv.vf[2 * k] = mv.vf[2 * kk];
                mv.vf[2 * k + 1] = mv.vf[2 * kk + 1];
            }
    }
}

// ----------------------------------------------------------------------------
// MultiplyMetric = Post . (K_NF + K_VF + K_FF) . Pre with MixedOrder operators
// (src/Metrics/MetricDimRestricted.hpp:109-139, src/ClusterTree.hpp:770-943,
//  TP0_Kernel_MultiplyMetric_Tiny.hpp:89-138).
// ----------------------------------------------------------------------------
static void metric_multiply(const Mesh& M, const MetricValues& mv, double alpha, const double* X, Int ldX,
                            double beta, double* Y, Int ldY, bool VF, bool NF, bool FF)
{
    const int SIZE = M.SIZE;
    const int BD = 12;  // (AMB+1) x nrhs
    std::vector<double> P_in(static_cast<size_t>(M.nS) * BD, 0.0), P_out(static_cast<size_t>(M.nS) * BD, 0.0);
    std::vector<double> C_in(static_cast<size_t>(M.NC) * BD, 0.0), C_out(static_cast<size_t>(M.NC) * BD, 0.0);
    for (Int i = 0; i < M.nS; ++i)
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 3; ++c) {
                double acc = 0;
                for (int l = 0; l < SIZE; ++l)
                    acc += M.pre_vals[(4 * static_cast<size_t>(i) + r) * SIZE + l] * X[static_cast<size_t>(ldX) * M.pre_cols[SIZE * static_cast<size_t>(i) + l] + c];
                P_in[BD * static_cast<size_t>(i) + 3 * r + c] = acc;
            }
    // PrimitivesToClusters + PercolateUp
    for (Int C = M.NC; C-- > 0;) {
        double* cc = &C_in[BD * static_cast<size_t>(C)];
        if (M.C_left[C] >= 0) {
            const double* l = &C_in[BD * static_cast<size_t>(M.C_left[C])];
            const double* r = &C_in[BD * static_cast<size_t>(M.C_right[C])];
            for (int k = 0; k < BD; ++k) cc[k] = l[k] + r[k];
        } else {
            for (int k = 0; k < BD; ++k) cc[k] = 0;
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i)
                for (int k = 0; k < BD; ++k) cc[k] += P_in[BD * static_cast<size_t>(i) + k];
        }
    }
    auto apply = [&](const Pattern& Pt, const std::vector<double>& vals, const std::vector<double>& diag,
                     const std::vector<double>& in, std::vector<double>& out) {
        for (Int i = 0; i < Pt.rows; ++i) {
            double* y = &out[BD * static_cast<size_t>(i)];
            for (LInt k = Pt.rp[i]; k < Pt.rp[i + 1]; ++k) {
                const double* x = &in[BD * static_cast<size_t>(Pt.ci[k])];
                const double a0 = vals[2 * k], a1 = vals[2 * k + 1];
                for (int c = 0; c < 3; ++c) y[c] += a0 * x[c];
                for (int c = 3; c < 12; ++c) y[c] += a1 * x[c];
            }
            const double* x = &in[BD * static_cast<size_t>(i)];
            for (int c = 0; c < 3; ++c) y[c] += diag[2 * i] * x[c];
            for (int c = 3; c < 12; ++c) y[c] += diag[2 * i + 1] * x[c];
        }
    };
    if (NF && M.near.nnz() > 0) apply(M.near, mv.nf, mv.nf_diag, P_in, P_out);
    if (VF && M.verynear.nnz() > 0) apply(M.verynear, mv.vf, mv.vf_diag, P_in, P_out);
    if (FF && M.far.nnz() > 0) apply(M.far, mv.ff, mv.ff_diag, C_in, C_out);
    // Post: PercolateDown, ClustersToPrimitives(add), mi_post
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] >= 0)
            for (int k = 0; k < BD; ++k) {
                C_out[BD * static_cast<size_t>(M.C_left[C]) + k] += C_out[BD * static_cast<size_t>(C) + k];
                C_out[BD * static_cast<size_t>(M.C_right[C]) + k] += C_out[BD * static_cast<size_t>(C) + k];
            }
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] < 0)
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i)
                for (int k = 0; k < BD; ++k) P_out[BD * static_cast<size_t>(i) + k] += C_out[BD * static_cast<size_t>(C) + k];
    std::vector<double> acc(static_cast<size_t>(M.nV) * 3, 0.0);
    for (Int i = 0; i < M.nS; ++i)
        for (int l = 0; l < SIZE; ++l) {
            const Int v = M.pre_cols[SIZE * static_cast<size_t>(i) + l];
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 3; ++c)
                    acc[3 * static_cast<size_t>(v) + c] += M.pre_vals[(4 * static_cast<size_t>(i) + r) * SIZE + l] * P_out[BD * static_cast<size_t>(i) + 3 * r + c];
        }
    for (Int v = 0; v < M.nV; ++v)
        for (int c = 0; c < 3; ++c) {
            double& y = Y[static_cast<size_t>(ldY) * v + c];
            y = alpha * acc[3 * static_cast<size_t>(v) + c] + (beta == 0.0 ? 0.0 : beta * y);
        }
}

// ----------------------------------------------------------------------------
// PseudoLaplacian<Mesh,false> (LowOrder) with exponent s:
// kernel -|x-y|^{2 s_exp}, s_exp = -n/2 - s (PseudoLaplacian_Kernel_NF.hpp, _FF.hpp)
// and lo_pre/lo_post operators.
// ----------------------------------------------------------------------------
static void pseudo_laplacian_multiply(const Mesh& M, double s, double alpha, const double* X, Int ldX, double beta,
                                      double* Y, Int ldY)
{
    const int SIZE = M.SIZE, nd = near_dim(M.dom);
    const double S_scale = 1.0 / SIZE;
    const double s_exp = -M.dom / 2.0 - s;
    const int BD = 3;
    std::vector<double> P_in(static_cast<size_t>(M.nS) * BD, 0.0), P_out(static_cast<size_t>(M.nS) * BD, 0.0);
    std::vector<double> C_in(static_cast<size_t>(M.NC) * BD, 0.0), C_out(static_cast<size_t>(M.NC) * BD, 0.0);
    for (Int i = 0; i < M.nS; ++i)
        for (int c = 0; c < 3; ++c) {
            double acc = 0;
            for (int l = 0; l < SIZE; ++l)
                acc += M.pre_vals[(4 * static_cast<size_t>(i)) * SIZE + l] * X[static_cast<size_t>(ldX) * M.pre_cols[SIZE * static_cast<size_t>(i) + l] + c];
            P_in[BD * static_cast<size_t>(i) + c] = acc;
        }
    for (Int C = M.NC; C-- > 0;) {
        double* cc = &C_in[BD * static_cast<size_t>(C)];
        if (M.C_left[C] >= 0) {
            for (int k = 0; k < BD; ++k) cc[k] = C_in[BD * static_cast<size_t>(M.C_left[C]) + k] + C_in[BD * static_cast<size_t>(M.C_right[C]) + k];
        } else {
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i)
                for (int k = 0; k < BD; ++k) cc[k] += P_in[BD * static_cast<size_t>(i) + k];
        }
    }
    auto centre = [&](bool far, Int i, double* x, double& a) {
        if (far) {
            const double* X2 = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
            a = X2[0];
            for (int k = 0; k < 3; ++k) x[k] = X2[1 + k];
        } else {
            const double* X2 = &M.P_near[nd * static_cast<size_t>(i)];
            a = X2[0];
            for (int k = 0; k < 3; ++k) {
                x[k] = S_scale * X2[1 + k];
                for (int v = 1; v < SIZE; ++v) x[k] += S_scale * X2[1 + AMB * v + k];
            }
        }
    };
    auto apply = [&](const Pattern& Pt, bool far, const std::vector<double>& in, std::vector<double>& out) {
        std::vector<double> diag(Pt.rows, 0.0);
        for (Int i = 0; i < Pt.rows; ++i) {
            double x[3], a;
            centre(far, i, x, a);
            for (LInt k = Pt.rp[i]; k < Pt.rp[i + 1]; ++k) {
                const Int j = Pt.ci[k];
                double y[3], b;
                centre(far, j, y, b);
                double r2 = 0;
                for (int kk = 0; kk < 3; ++kk) r2 += (y[kk] - x[kk]) * (y[kk] - x[kk]);
                const double val = -std::pow(r2, s_exp);
                for (int c = 0; c < BD; ++c) out[BD * static_cast<size_t>(i) + c] += val * in[BD * static_cast<size_t>(j) + c];
                diag[i] -= (b / a) * val;
            }
        }
        for (Int i = 0; i < Pt.rows; ++i)
            for (int c = 0; c < BD; ++c) out[BD * static_cast<size_t>(i) + c] += diag[i] * in[BD * static_cast<size_t>(i) + c];
    };
    if (M.near.nnz() > 0) apply(M.near, false, P_in, P_out);
    if (M.far.nnz() > 0) apply(M.far, true, C_in, C_out);
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] >= 0)
            for (int k = 0; k < BD; ++k) {
                C_out[BD * static_cast<size_t>(M.C_left[C]) + k] += C_out[BD * static_cast<size_t>(C) + k];
                C_out[BD * static_cast<size_t>(M.C_right[C]) + k] += C_out[BD * static_cast<size_t>(C) + k];
            }
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] < 0)
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i)
                for (int k = 0; k < BD; ++k) P_out[BD * static_cast<size_t>(i) + k] += C_out[BD * static_cast<size_t>(C) + k];
    std::vector<double> acc(static_cast<size_t>(M.nV) * 3, 0.0);
    for (Int i = 0; i < M.nS; ++i)
        for (int l = 0; l < SIZE; ++l) {
            const Int v = M.pre_cols[SIZE * static_cast<size_t>(i) + l];
            for (int c = 0; c < 3; ++c)
                acc[3 * static_cast<size_t>(v) + c] += M.pre_vals[(4 * static_cast<size_t>(i)) * SIZE + l] * P_out[BD * static_cast<size_t>(i) + c];
        }
    for (Int v = 0; v < M.nV; ++v)
        for (int c = 0; c < 3; ++c) {
            double& y = Y[static_cast<size_t>(ldY) * v + c];
            y = alpha * acc[3 * static_cast<size_t>(v) + c] + (beta == 0.0 ? 0.0 : beta * y);
        }
}

// ----------------------------------------------------------------------------
// H1 metric triplets (src/SimplicialMesh/H1Metric.hpp:36-169): stiffness + mass
// ----------------------------------------------------------------------------
static void h1_triplets(const Mesh& M, double ws, double wm, Int* I, Int* J, double* A)
{
    const int n = M.dom, SIZE = M.SIZE;
    const double std_vol = (n == 1) ? 1.0 : 0.5;
    const double fact = (n == 1) ? 6.0 : 24.0;     // (n+2)!
    const double m_factor = wm / (std_vol * fact);
    for (Int k = 0; k < M.nS; ++k) {
        const Int* s = &M.S[SIZE * static_cast<size_t>(k)];
        double df[3][2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < n; ++j) df[i][j] = M.V[3 * static_cast<size_t>(s[j + 1]) + i] - M.V[3 * static_cast<size_t>(s[0]) + i];
        double g[2][2] = {{0, 0}, {0, 0}};
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                for (int i = 0; i < 3; ++i) g[a][b] += df[i][a] * df[i][b];
        double a = std_vol, ginv[2][2];
        if (n == 1) { a *= std::sqrt(g[0][0]); ginv[0][0] = 1.0 / g[0][0]; }
        else {
            const double L00 = std::sqrt(g[0][0]);
            const double L10 = g[1][0] / L00;
            const double L11 = std::sqrt(g[1][1] - L10 * L10);
            a *= L00 * L11;
            const double det = g[0][0] * g[1][1] - g[0][1] * g[1][0];
            ginv[0][0] = g[1][1] / det; ginv[1][1] = g[0][0] / det;
            ginv[0][1] = ginv[1][0] = -g[0][1] / det;
        }
        double val[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double lf = a * ws;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const double aij = lf * ginv[i][j];
                val[0][0] += aij;
                val[i + 1][0] -= aij;
                val[0][j + 1] -= aij;
                val[i + 1][j + 1] = aij;
            }
        for (int i = 0; i < SIZE; ++i)
            for (int j = 0; j < SIZE; ++j) val[i][j] += a * m_factor * (1.0 + (i == j ? 1.0 : 0.0));
        for (int i = 0; i < SIZE; ++i)
            for (int j = 0; j < SIZE; ++j) {
                const size_t o = static_cast<size_t>(k) * SIZE * SIZE + i * SIZE + j;
                I[o] = s[i]; J[o] = s[j]; A[o] = val[i][j];
            }
    }
}

// ----------------------------------------------------------------------------
// All-pairs exact sum (TP_AllPairs_Traversor.hpp:144-280): NF kernel on every
// primitive pair i<j at the barycentres.
// ----------------------------------------------------------------------------
static double allpairs_energy(const Mesh& M, double q, double p)
{
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom), SIZE = M.SIZE;
    std::vector<double> part(std::max(1, M.set.threads), 0.0);
    parallel_do(std::max(1, M.set.threads), [&](int t) {
        const Int b = job_pointer(M.nS, M.set.threads, t), e = job_pointer(M.nS, M.set.threads, t + 1);
        double local = 0;
        for (Int i = b; i < e; ++i) {
            const double* X = &M.P_near[nd * static_cast<size_t>(i)];
            double x[3];
            for (int k = 0; k < 3; ++k) { x[k] = 0; for (int v = 0; v < SIZE; ++v) x[k] += X[1 + 3 * v + k] / SIZE; }
            for (Int j = i + 1; j < M.nS; ++j) {
                const double* Y = &M.P_near[nd * static_cast<size_t>(j)];
                double y[3];
                for (int k = 0; k < 3; ++k) { y[k] = 0; for (int v = 0; v < SIZE; ++v) y[k] += Y[1 + 3 * v + k] / SIZE; }
                PairOut o;
                tp0_pair(T, X[0], x, X + 1 + AMB * SIZE, Y[0], y, Y + 1 + AMB * SIZE, false, false, o);
                local += o.energy;
            }
        }
        part[t] = local;
    });
    double en = 0;
    for (double v : part) en += v;
    return en;
}

// ----------------------------------------------------------------------------
// TangentPointObstacleEnergy (src/Energies/TangentPointObstacleEnergy.hpp:62-96): the TP
// energy/differential kernels (src/Energies/TangentPointEnergy/TP_Kernel_FF.hpp:130-260,
// TP_Kernel_NF.hpp, identical to TP0's for energy and differential) over the
// non-symmetric block cluster tree of (mesh tree, obstacle tree)
// (src/SimplicialMesh.hpp:741-756, BlockClusterTree<...,false>; traversal
// src/ClusterTreePairTraversor/Traverse_DepthFirst.hpp:52-258 with symmetricQ = false).
// Every (mesh, obstacle) pair is visited once with the symmetry factor 1/2
// (src/FMM/FMM_Kernel.hpp:43) on energy and derivatives; only the mesh side's derivatives
// are assembled (the obstacle does not move).
// ----------------------------------------------------------------------------
struct CrossPattern {
    Int rows = 0;
    std::vector<LInt> rp;
    std::vector<Int> ci;
    LInt nnz() const { return rp.empty() ? 0 : rp.back(); }
};

static CrossPattern make_cross_pattern(Int rows, std::vector<std::pair<Int, Int>>& pairs)
{
    std::sort(pairs.begin(), pairs.end());
    CrossPattern P;
    P.rows = rows;
    P.rp.assign(static_cast<size_t>(rows) + 1, 0);
    for (auto& e : pairs) P.rp[e.first + 1]++;
    for (Int i = 0; i < rows; ++i) P.rp[i + 1] += P.rp[i];
    P.ci.resize(pairs.size());
    for (size_t k = 0; k < pairs.size(); ++k) P.ci[k] = pairs[k].second;
    return P;
}

struct ObstacleLists {
    CrossPattern near, far, verynear, inter;
};

static void build_obstacle_block_cluster_tree(const Mesh& M, const Mesh& O, ObstacleLists& L)
{
    const double far_t2 = M.set.theta_far * M.set.theta_far;
    const double near_t2 = M.set.theta_near * M.set.theta_near;
    const double eps2 = std::numeric_limits<double>::epsilon();
    const int psM = M.poly_size(), psO = O.poly_size();
    std::vector<std::pair<Int, Int>> near_l, far_l, vn_l, inter_l;
    auto leaf = [&](Int pi, Int pj) {
        const double* A = &M.P_poly[psM * static_cast<size_t>(pi)];
        const double* B = &O.P_poly[psO * static_cast<size_t>(pj)];
        const double d2 = poly_sqdist(M.dom, A + 1 + AMB, B + 1 + AMB);
        const double tol = std::max(A[0], B[0]);
        if (near_t2 * d2 > tol) { near_l.emplace_back(pi, pj); return; }
        const double tol_i = eps2 * std::min(A[0], B[0]);
        if (near_t2 * d2 <= tol_i) inter_l.emplace_back(pi, pj);
        else vn_l.emplace_back(pi, pj);
    };
    std::vector<std::pair<Int, Int>> stack;
    stack.emplace_back(0, 0);
    while (!stack.empty()) {
        auto [i, j] = stack.back();
        stack.pop_back();
        const double* Bi = &M.C_box[7 * static_cast<size_t>(i)];
        const double* Bj = &O.C_box[7 * static_cast<size_t>(j)];
        if (std::max(Bi[0], Bj[0]) < far_t2 * aabb_sq_dist(Bi, Bj)) {
            far_l.emplace_back(i, j);
            continue;
        }
        const Int Li = M.C_left[i], Lj = O.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const Int Ri = M.C_right[i], Rj = O.C_right[j];
            const double si = (Li >= 0) ? Bi[0] : 0.0;
            const double sj = (Lj >= 0) ? Bj[0] : 0.0;
            if (si == sj && si > 0) {
                stack.emplace_back(Ri, Rj);
                stack.emplace_back(Li, Rj);
                stack.emplace_back(Ri, Lj);
                stack.emplace_back(Li, Lj);
            } else if (si > sj) {
                stack.emplace_back(Ri, j);
                stack.emplace_back(Li, j);
            } else {
                stack.emplace_back(i, Rj);
                stack.emplace_back(i, Lj);
            }
        } else {
            leaf(M.C_begin[i], O.C_begin[j]);
        }
    }
    L.near = make_cross_pattern(M.nS, near_l);
    L.far = make_cross_pattern(M.NC, far_l);
    L.verynear = make_cross_pattern(M.nS, vn_l);
    L.inter = make_cross_pattern(M.nS, inter_l);
}

static double obstacle_evaluate(Mesh& M, const Mesh& O, const ObstacleLists& L, double q, double p, bool diff)
{
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom);
    const int SIZE = M.SIZE;
    const int threads = std::max(1, M.set.threads);
    const double S_scale = 1.0 / SIZE;
    const double sf = 0.5;   // symmetry factor of a non-symmetric block cluster tree
    std::vector<std::vector<double>> tDn, tDf;
    if (diff) {
        tDn.assign(threads, std::vector<double>(static_cast<size_t>(M.nS) * nd, 0.0));
        tDf.assign(threads, std::vector<double>(static_cast<size_t>(M.NC) * FAR_DIM, 0.0));
    }
    double en = 0;
    auto center = [&](const Mesh& X, Int i, double* c) {
        const double* D = &X.P_near[near_dim(X.dom) * static_cast<size_t>(i)];
        for (int k = 0; k < 3; ++k) {
            c[k] = 0;
            for (int v = 0; v < X.SIZE; ++v) c[k] += D[1 + AMB * v + k] / X.SIZE;
        }
    };
    {   // VF: the subdivision quadrature of TP0_Kernel_VF / FMM_Kernel_VF_Common on the
        // (mesh, obstacle) very-near pairs, every pair once with the symmetry factor 1/2
        const CrossPattern& Pt = L.verynear;
        std::vector<double> part(threads, 0.0);
        parallel_do(threads, [&](int t) {
            double local = 0;
            for (Int i = job_pointer(M.nS, threads, t); i < job_pointer(M.nS, threads, t + 1); ++i) {
                const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
                for (LInt k = Pt.rp[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Yj = &O.P_near[near_dim(O.dom) * static_cast<size_t>(j)];
                    vf_quadrature(M, i, O, j, [&](const double* x, const double* y, double ws, double wt,
                                                  const double* bs, const double*) {
                        PairOut o;
                        tp0_pair(T, Xi[0] * ws, x, Xi + 1 + AMB * SIZE, Yj[0] * wt, y, Yj + 1 + AMB * O.SIZE, diff,
                                 false, o);
                        local += sf * o.energy;
                        if (diff) {
                            double* DX = &tDn[t][nd * static_cast<size_t>(i)];
                            DX[0] += sf * ws * o.DX[0];
                            for (int v = 0; v < SIZE; ++v)
                                for (int kk = 0; kk < 3; ++kk) DX[1 + 3 * v + kk] += sf * ws * bs[v] * o.DX[1 + kk];
                            for (int kk = 0; kk < 6; ++kk) DX[1 + AMB * SIZE + kk] += sf * ws * o.DX[4 + kk];
                        }
                    });
                }
            }
            part[t] = local;
        });
        for (double v : part) en += v;
    }
    {   // NF
        const CrossPattern& Pt = L.near;
        std::vector<double> part(threads, 0.0);
        parallel_do(threads, [&](int t) {
            double local = 0;
            for (Int i = job_pointer(M.nS, threads, t); i < job_pointer(M.nS, threads, t + 1); ++i) {
                const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
                double x[3];
                center(M, i, x);
                for (LInt k = Pt.rp[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Yj = &O.P_near[near_dim(O.dom) * static_cast<size_t>(j)];
                    double y[3];
                    center(O, j, y);
                    PairOut o;
                    tp0_pair(T, Xi[0], x, Xi + 1 + AMB * SIZE, Yj[0], y, Yj + 1 + AMB * O.SIZE, diff, false, o);
                    local += sf * o.energy;
                    if (diff) {
                        double* DX = &tDn[t][nd * static_cast<size_t>(i)];
                        DX[0] += sf * o.DX[0];
                        for (int v = 0; v < SIZE; ++v)
                            for (int kk = 0; kk < 3; ++kk) DX[1 + 3 * v + kk] += sf * S_scale * o.DX[1 + kk];
                        for (int kk = 0; kk < 6; ++kk) DX[1 + AMB * SIZE + kk] += sf * o.DX[4 + kk];
                    }
                }
            }
            part[t] = local;
        });
        for (double v : part) en += v;
    }
    {   // FF
        const CrossPattern& Pt = L.far;
        std::vector<double> part(threads, 0.0);
        parallel_do(threads, [&](int t) {
            double local = 0;
            for (Int i = job_pointer(M.NC, threads, t); i < job_pointer(M.NC, threads, t + 1); ++i) {
                const double* Xi = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
                for (LInt k = Pt.rp[i]; k < Pt.rp[i + 1]; ++k) {
                    const Int j = Pt.ci[k];
                    const double* Yj = &O.C_far[FAR_DIM * static_cast<size_t>(j)];
                    PairOut o;
                    tp0_pair(T, Xi[0], Xi + 1, Xi + 4, Yj[0], Yj + 1, Yj + 4, diff, false, o);
                    local += sf * o.energy;
                    if (diff) {
                        double* DX = &tDf[t][FAR_DIM * static_cast<size_t>(i)];
                        for (int kk = 0; kk < 10; ++kk) DX[kk] += sf * o.DX[kk];
                    }
                }
            }
            part[t] = local;
        });
        for (double v : part) en += v;
    }
    if (diff) collect_derivatives(M, tDn, tDf, threads, nd);
    return en;
}

// 1/2 sum over all (mesh primitive, obstacle primitive) pairs of a E b at the barycentres
static double obstacle_allpairs_energy(const Mesh& M, const Mesh& O, double q, double p)
{
    const TPParams T(q, p, M.dom);
    const int threads = std::max(1, M.set.threads);
    std::vector<double> part(threads, 0.0);
    parallel_do(threads, [&](int t) {
        double local = 0;
        for (Int i = job_pointer(M.nS, threads, t); i < job_pointer(M.nS, threads, t + 1); ++i) {
            const double* X = &M.P_near[near_dim(M.dom) * static_cast<size_t>(i)];
            double x[3];
            for (int k = 0; k < 3; ++k) { x[k] = 0; for (int v = 0; v < M.SIZE; ++v) x[k] += X[1 + 3 * v + k] / M.SIZE; }
            for (Int j = 0; j < O.nS; ++j) {
                const double* Y = &O.P_near[near_dim(O.dom) * static_cast<size_t>(j)];
                double y[3];
                for (int k = 0; k < 3; ++k) { y[k] = 0; for (int v = 0; v < O.SIZE; ++v) y[k] += Y[1 + 3 * v + k] / O.SIZE; }
                PairOut o;
                tp0_pair(T, X[0], x, X + 1 + AMB * M.SIZE, Y[0], y, Y + 1 + AMB * O.SIZE, false, false, o);
                local += 0.5 * o.energy;
            }
        }
        part[t] = local;
    });
    double en = 0;
    for (double v : part) en += v;
    return en;
}

// Energy densities (EnergyBase::SimplexDensities / VertexDensities,
// src/Energies/EnergyBase.hpp:129-150; CollectPrimitiveDensities / CollectVertexDensities,
// src/ClusterTree/ClusterTreeBase.hpp:601-729): per pair, x receives b |Pv|^q / |v|^p and
// y receives a |Qv|^q / |v|^p; far-field cluster densities are pushed down to the
// primitives (sum over the ancestors). Sum_i a_i rho_i equals the energy. Returns the
// energy; rho in original simplex order. The very-near list must be empty.
static double tp0_densities(const Mesh& M, double q, double p, std::vector<double>& rho)
{
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom), SIZE = M.SIZE;
    std::vector<double> rn(M.nS, 0.0), rf(M.NC, 0.0);
    double en = 0;
    auto center = [&](Int i, double* c) {
        const double* D = &M.P_near[nd * static_cast<size_t>(i)];
        for (int k = 0; k < 3; ++k) {
            c[k] = 0;
            for (int v = 0; v < SIZE; ++v) c[k] += D[1 + AMB * v + k] / SIZE;
        }
    };
    for (Int i = 0; i < M.nS; ++i) {
        const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
        double x[3];
        center(i, x);
        for (LInt k = M.near.diag[i]; k < M.near.rp[i + 1]; ++k) {
            const Int j = M.near.ci[k];
            const double* Yj = &M.P_near[nd * static_cast<size_t>(j)];
            double y[3];
            center(j, y);
            PairOut o;
            tp0_pair(T, Xi[0], x, Xi + 1 + AMB * SIZE, Yj[0], y, Yj + 1 + AMB * SIZE, false, false, o);
            en += o.energy;
            rn[i] += o.dens_x;
            rn[j] += o.dens_y;
        }
    }
    for (Int i = 0; i < M.NC; ++i) {
        const double* Xi = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
        for (LInt k = M.far.diag[i]; k < M.far.rp[i + 1]; ++k) {
            const Int j = M.far.ci[k];
            const double* Yj = &M.C_far[FAR_DIM * static_cast<size_t>(j)];
            PairOut o;
            tp0_pair(T, Xi[0], Xi + 1, Xi + 4, Yj[0], Yj + 1, Yj + 4, false, false, o);
            en += o.energy;
            rf[i] += o.dens_x;
            rf[j] += o.dens_y;
        }
    }
    for (Int C = 0; C < M.NC; ++C)   // PercolateDown (parents precede children)
        if (M.C_left[C] >= 0) {
            rf[M.C_left[C]] += rf[C];
            rf[M.C_right[C]] += rf[C];
        }
    rho.assign(M.nS, 0.0);
    for (Int C = 0; C < M.NC; ++C)
        if (M.C_left[C] < 0)
            for (Int i = M.C_begin[C]; i < M.C_end[C]; ++i) rho[M.perm[i]] = rn[i] + rf[C];
    return en;
}

}  // namespace oracle

// ============================================================================
// C API (ctypes)
// ============================================================================
using namespace oracle;

// ----------------------------------------------------------------------------
// MaximumSafeStepSize (src/SimplicialMesh.hpp:441-468, src/CollisionTree.hpp:175-215):
// the largest t <= max_time for which the mesh moved by t * (vertex velocities) keeps
// all non-adjacent primitive pairs apart, found on the frozen (construction) coordinates
// the cluster tree was built from. Moving simplices as space-time hulls
// (src/Primitives/MovingPolytope.hpp:148-460), a collision-only GJK in 4 dimensions
// (src/GJK.hpp:618-797), bisection with a stack (src/CollisionFinder.hpp:94-200), AABB
// collision time intervals (src/CollisionTree/Compute_AABB_CollisionTimeInterval.hpp)
// and the symmetric dual traversal with the step-size kernel
// (src/CollisionTree/MaximumSafeStepSize_Kernel.hpp).
// ----------------------------------------------------------------------------
static const double kGjkEps = std::sqrt(std::numeric_limits<double>::epsilon());

struct MovingSimplex {
    int n = 3;
    double x[3][3], u[3][3];
    double c[3], cu[3];
    double r = 0, v = 0, w = 0;
    double a = 0, b = 1, T = 1;

    double support(const double d[4], double s[4], bool maximum) const
    {
        double best_a = 0, best_b = 0;
        int ia = 0, ib = 0;
        for (int i = 0; i < n; ++i) {
            double va = x[i][0] * d[0] + a * (u[i][0] * d[0]);
            double vb = x[i][0] * d[0] + b * (u[i][0] * d[0]);
            for (int j = 1; j < 3; ++j) {
                const double px = x[i][j] * d[j], py = u[i][j] * d[j];
                va += px + a * py;
                vb += px + b * py;
            }
            if (i == 0 || (maximum ? va > best_a : va < best_a)) { best_a = va; ia = i; }
            if (i == 0 || (maximum ? vb > best_b : vb < best_b)) { best_b = vb; ib = i; }
        }
        best_a += a * T * d[3];
        best_b += b * T * d[3];
        const bool take_a = maximum ? best_a >= best_b : best_a <= best_b;
        const int i = take_a ? ia : ib;
        const double t = take_a ? a : b;
        for (int j = 0; j < 3; ++j) s[j] = x[i][j] + t * u[i][j];
        s[3] = t * T;
        return take_a ? best_a : best_b;
    }
    void interior(double p[4]) const
    {
        const double t = 0.5 * (a + b);
        for (int k = 0; k < 3; ++k) p[k] = c[k] + t * cu[k];
        p[3] = t * T;
    }
    double sq_radius() const
    {
        const double s = 0.5 * std::fabs(b - a);
        const double X = s * v + r + w * b, Y = s * T;
        return X * X + Y * Y;
    }
};

// Closest point of the convex hull of k <= 5 points in R^4 to the origin: the minimum over
// the faces whose affine closest point has nonnegative barycentric coordinates. Returns
// |v|^2, the point in v and the supporting points (reordered to the front) in their count.
static double closest_on_simplex(double W[5][4], int& k, double v[4])
{
    double best = std::numeric_limits<double>::infinity();
    int best_mask = 0;
    double best_v[4] = {0, 0, 0, 0};
    for (int mask = 1; mask < (1 << k); ++mask) {
        int idx[5], m = 0;
        for (int i = 0; i < k; ++i)
            if (mask & (1 << i)) idx[m++] = i;
        double lam[5];
        if (m == 1) {
            lam[0] = 1.0;
        } else {
            // (w_i - w_0).(w_j - w_0) mu_j = -(w_i - w_0).w_0, i, j = 1..m-1
            const int n = m - 1;
            double G[4][5];
            for (int i = 0; i < n; ++i) {
                for (int j = 0; j < n; ++j) {
                    double g = 0;
                    for (int q = 0; q < 4; ++q) g += (W[idx[i + 1]][q] - W[idx[0]][q]) * (W[idx[j + 1]][q] - W[idx[0]][q]);
                    G[i][j] = g;
                }
                double rhs = 0;
                for (int q = 0; q < 4; ++q) rhs -= (W[idx[i + 1]][q] - W[idx[0]][q]) * W[idx[0]][q];
                G[i][n] = rhs;
            }
            bool singular = false;
            for (int col = 0; col < n && !singular; ++col) {
                int piv = col;
                for (int r = col + 1; r < n; ++r)
                    if (std::fabs(G[r][col]) > std::fabs(G[piv][col])) piv = r;
                double scale = 0;
                for (int r = 0; r < n; ++r) scale = std::max(scale, std::fabs(G[r][r]));
                if (std::fabs(G[piv][col]) <= 1e-14 * std::max(scale, 1e-300)) { singular = true; break; }
                if (piv != col)
                    for (int c2 = 0; c2 <= n; ++c2) std::swap(G[piv][c2], G[col][c2]);
                for (int r = col + 1; r < n; ++r) {
                    const double f = G[r][col] / G[col][col];
                    for (int c2 = col; c2 <= n; ++c2) G[r][c2] -= f * G[col][c2];
                }
            }
            if (singular) continue;
            double mu[4];
            for (int r = n - 1; r >= 0; --r) {
                double acc = G[r][n];
                for (int c2 = r + 1; c2 < n; ++c2) acc -= G[r][c2] * mu[c2];
                mu[r] = acc / G[r][r];
            }
            double s0 = 1.0;
            for (int i = 0; i < n; ++i) { lam[i + 1] = mu[i]; s0 -= mu[i]; }
            lam[0] = s0;
        }
        bool inside = true;
        for (int i = 0; i < m; ++i) inside = inside && lam[i] >= 0.0;
        if (!inside) continue;
        double p[4] = {0, 0, 0, 0};
        for (int i = 0; i < m; ++i)
            for (int q = 0; q < 4; ++q) p[q] += lam[i] * W[idx[i]][q];
        const double d2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
        if (d2 < best) { best = d2; best_mask = mask; for (int q = 0; q < 4; ++q) best_v[q] = p[q]; }
    }
    double keep[5][4];
    int m = 0;
    for (int i = 0; i < k; ++i)
        if (best_mask & (1 << i)) { for (int q = 0; q < 4; ++q) keep[m][q] = W[i][q]; ++m; }
    for (int i = 0; i < m; ++i) for (int q = 0; q < 4; ++q) W[i][q] = keep[i][q];
    k = m;
    for (int q = 0; q < 4; ++q) v[q] = best_v[q];
    return best;
}

// Collision-only GJK: true if the two space-time hulls come closer than
// eps * sqrt(min squared radius) (GJK::IntersectingQ with theta = 1).
static bool gjk_intersecting(const MovingSimplex& P, const MovingSimplex& Q)
{
    const double eps = kGjkEps, eps2 = eps * eps;
    double TOL2 = eps2 * std::min(P.sq_radius(), Q.sq_radius());
    if (TOL2 <= 0) TOL2 = eps2 * std::max(P.sq_radius(), Q.sq_radius());
    double v[4], q4[4];
    P.interior(v);
    Q.interior(q4);
    for (int k = 0; k < 4; ++k) v[k] -= q4[k];
    double W[5][4];
    int k = 0;
    double ps[4], qs[4];
    P.support(v, ps, false);
    Q.support(v, qs, true);
    for (int j = 0; j < 4; ++j) W[0][j] = ps[j] - qs[j];
    k = 1;
    for (int j = 0; j < 4; ++j) v[j] = W[0][j];
    double dotvv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
    bool separated = false;
    int iter = 0;
    while (true) {
        if (dotvv < TOL2) break;
        if (k >= 5) break;
        if (iter >= 100) break;
        ++iter;
        const double a = P.support(v, ps, false);
        const double b = Q.support(v, qs, true);
        const double dotvw = a - b;
        if (dotvw > 0 && dotvw * dotvw > TOL2) { separated = true; break; }
        if (std::fabs(dotvv - dotvw) <= eps * dotvv) break;
        double w[4];
        for (int j = 0; j < 4; ++j) w[j] = ps[j] - qs[j];
        bool dup = false;
        for (int i = 0; i < k && !dup; ++i)
            dup = W[i][0] == w[0] && W[i][1] == w[1] && W[i][2] == w[2] && W[i][3] == w[3];
        if (dup) break;
        for (int j = 0; j < 4; ++j) W[k][j] = w[j];
        ++k;
        const double old = dotvv;
        dotvv = closest_on_simplex(W, k, v);
        if (std::fabs(old - dotvv) <= eps * dotvv) break;
    }
    separated = separated || TOL2 < dotvv;
    return !separated;
}

// CollisionFinder::FindMaximumSafeStepSize (src/CollisionFinder.hpp:94-200)
static double find_max_safe_step(MovingSimplex P, MovingSimplex Q, double tinit, double TOL)
{
    double a = 0.0, b = tinit;
    P.a = Q.a = a; P.b = Q.b = b; P.T = Q.T = 1.0;
    double pi4[4], qi4[4];
    P.interior(pi4);
    Q.interior(qi4);
    double d2 = 0;
    for (int k = 0; k < 4; ++k) d2 += (qi4[k] - pi4[k]) * (qi4[k] - pi4[k]);
    const double T = std::sqrt(d2 + P.sq_radius() + Q.sq_radius()) / tinit;
    P.T = Q.T = T;
    constexpr int max_iter = 126;
    double stack[max_iter + 2];
    int iter = 0, sp = 0;
    stack[0] = 0.0;
    while (b - a > TOL * b && iter < max_iter) {
        ++iter;
        if (!gjk_intersecting(P, Q)) {
            if (sp > 0) {
                a = b; P.a = Q.a = a;
                b = stack[sp--]; P.b = Q.b = b;
            } else {
                return b;
            }
        } else {
            stack[++sp] = b;
            b = 0.5 * (a + b);
            P.b = Q.b = b;
        }
    }
    if (sp >= max_iter || iter >= max_iter) return a;
    return a <= 0.0 ? b : a;
}

static void moving_simplex(const Mesh& M, const double* vel, Int i, MovingSimplex& P)
{
    const int ps = M.poly_size();
    const double* poly = &M.P_poly[ps * static_cast<size_t>(i)];
    const Int* s = &M.S[static_cast<size_t>(M.SIZE) * M.perm[i]];
    P.n = M.SIZE;
    P.r = std::sqrt(poly[0]);
    for (int k = 0; k < 3; ++k) P.c[k] = poly[1 + k];
    for (int j = 0; j < M.SIZE; ++j)
        for (int k = 0; k < 3; ++k) { P.x[j][k] = poly[1 + AMB + AMB * j + k]; P.u[j][k] = vel[AMB * s[j] + k]; }
    for (int k = 0; k < 3; ++k) {
        P.cu[k] = P.u[0][k];
        for (int j = 1; j < M.SIZE; ++j) P.cu[k] += P.u[j][k];
        P.cu[k] *= 1.0 / M.SIZE;
    }
    P.v = std::sqrt(P.cu[0] * P.cu[0] + P.cu[1] * P.cu[1] + P.cu[2] * P.cu[2]);
    double w2 = 0;
    for (int j = 0; j < M.SIZE; ++j) {
        double q = 0;
        for (int k = 0; k < 3; ++k) q += (P.u[j][k] - P.cu[k]) * (P.u[j][k] - P.cu[k]);
        w2 = std::max(w2, q);
    }
    P.w = std::sqrt(w2);
}

// Compute_AABB_CollisionTimeInterval: the first time in [0, 1] at which the boxes moving
// linearly from p0 to p1 and from q0 to q1 ([r2, centre, half]) can intersect (1: never).
static double aabb_collision_start(const double* p0, const double* p1, const double* q0, const double* q1)
{
    double t0 = 0.0, t1 = 1.0;
    for (int k = 0; k < 3; ++k) {
        const int i = 1 + k, j = 4 + k;
        const double Pmin0 = p0[i] - p0[j], Pmax0 = p0[i] + p0[j], Pmin1 = p1[i] - p1[j], Pmax1 = p1[i] + p1[j];
        const double Qmin0 = q0[i] - q0[j], Qmax0 = q0[i] + q0[j], Qmin1 = q1[i] - q1[j], Qmax1 = q1[i] + q1[j];
        const bool init = (Pmin0 <= Qmax0) && (Qmin0 <= Pmax0);
        const double m0 = Qmax0 - Qmax1 - Pmin0 + Pmin1, m1 = Pmax0 - Pmax1 - Qmin0 + Qmin1;
        double A = m0 != 0 ? std::min(1.0, (Qmax0 - Pmin0) / m0) : 1.0;
        double B = m1 != 0 ? std::min(1.0, (Pmax0 - Qmin0) / m1) : 1.0;
        if (A > B) std::swap(A, B);
        double a, b;
        if (init) { a = 0.0; b = A > 0 ? A : (B <= 0 ? 1.0 : B); }
        else if (B < 0) { a = 1.0; b = 1.0; }
        else if (A >= 0) { a = A; b = B; }
        else { a = B; b = 1.0; }
        t0 = std::max(t0, a);
        t1 = std::min(t1, b);
    }
    return t1 < t0 ? 1.0 : t0;
}

static bool primitives_adjacent(const Mesh& M, Int pi, Int pj)
{
    const Int* a = &M.S[static_cast<size_t>(M.SIZE) * M.perm[pi]];
    const Int* b = &M.S[static_cast<size_t>(M.SIZE) * M.perm[pj]];
    for (int x = 0; x < M.SIZE; ++x)
        for (int y = 0; y < M.SIZE; ++y)
            if (a[x] == b[y]) return true;
    return false;
}

// cluster boxes of a tree at max_time: leaves from the moved simplex, internal clusters merged
static std::vector<double> moved_boxes(const Mesh& M, const std::vector<MovingSimplex>& P, double max_time)
{
    const Int NC = M.NC;
    std::vector<double> lo(3 * static_cast<size_t>(NC)), hi(3 * static_cast<size_t>(NC)), C_up(7 * static_cast<size_t>(NC));
    for (Int C = NC - 1; C >= 0; --C) {
        double* l = &lo[3 * static_cast<size_t>(C)];
        double* h = &hi[3 * static_cast<size_t>(C)];
        if (M.C_left[C] < 0) {
            const MovingSimplex& S = P[M.C_begin[C]];
            for (int k = 0; k < 3; ++k) { l[k] = std::numeric_limits<double>::max(); h[k] = std::numeric_limits<double>::lowest(); }
            for (int j = 0; j < S.n; ++j)
                for (int k = 0; k < 3; ++k) {
                    const double x = S.x[j][k] + max_time * S.u[j][k];
                    l[k] = std::min(l[k], x);
                    h[k] = std::max(h[k], x);
                }
        } else {
            const Int L = M.C_left[C], R = M.C_right[C];
            for (int k = 0; k < 3; ++k) {
                l[k] = std::min(lo[3 * static_cast<size_t>(L) + k], lo[3 * static_cast<size_t>(R) + k]);
                h[k] = std::max(hi[3 * static_cast<size_t>(L) + k], hi[3 * static_cast<size_t>(R) + k]);
            }
        }
        double* bx = &C_up[7 * static_cast<size_t>(C)];
        double r2 = 0;
        for (int k = 0; k < 3; ++k) {
            const double half = 0.5 * (h[k] - l[k]);
            bx[1 + k] = l[k] + half;
            bx[4 + k] = half;
            r2 += half * half;
        }
        bx[0] = r2;
    }
    return C_up;
}

static double maximum_safe_step_size(const Mesh& M, const double* vel, double max_time, double TOL,
                                     const Mesh* Ob = nullptr)
{
    const Int N = M.nS;
    std::vector<MovingSimplex> P(N);
    for (Int i = 0; i < N; ++i) moving_simplex(M, vel, i, P[i]);
    const std::vector<double> C_up = moved_boxes(M, P, max_time);
    double t = max_time;
    if (Ob) {
        // the obstacle's collision tree first (src/SimplicialMesh.hpp:453-461): the obstacle at
        // rest, mesh x obstacle block pairs from the roots, every leaf pair evaluated
        std::vector<double> zero(3 * static_cast<size_t>(Ob->nV), 0.0);
        std::vector<MovingSimplex> Q(Ob->nS);
        for (Int i = 0; i < Ob->nS; ++i) moving_simplex(*Ob, zero.data(), i, Q[i]);
        const std::vector<double> O_up = moved_boxes(*Ob, Q, max_time);
        const double t_init = t;
        double t_max = t_init;
        std::vector<std::pair<Int, Int>> st{{0, 0}};
        while (!st.empty()) {
            auto [i, j] = st.back();
            st.pop_back();
            const double a = aabb_collision_start(&M.C_box[7 * static_cast<size_t>(i)], &C_up[7 * static_cast<size_t>(i)],
                                                  &Ob->C_box[7 * static_cast<size_t>(j)], &O_up[7 * static_cast<size_t>(j)]);
            if (a * t_init >= t_max) continue;
            const Int Li = M.C_left[i], Lj = Ob->C_left[j];
            if (Li >= 0 || Lj >= 0) {
                const Int Ri = M.C_right[i], Rj = Ob->C_right[j];
                const double si = Li >= 0 ? M.C_box[7 * static_cast<size_t>(i)] : 0.0;
                const double sj = Lj >= 0 ? Ob->C_box[7 * static_cast<size_t>(j)] : 0.0;
                if (si == sj && si > 0) { st.push_back({Ri, Rj}); st.push_back({Li, Rj}); st.push_back({Ri, Lj}); st.push_back({Li, Lj}); }
                else if (si > sj) { st.push_back({Ri, j}); st.push_back({Li, j}); }
                else { st.push_back({i, Rj}); st.push_back({i, Lj}); }
                continue;
            }
            t_max = find_max_safe_step(P[M.C_begin[i]], Q[Ob->C_begin[j]], t_max, TOL);
        }
        t = std::min(t_max, t_init);
    }
    const double t_init = t;
    double t_max = t_init;
    std::vector<std::pair<Int, Int>> stack{{0, 0}};
    while (!stack.empty()) {
        auto [i, j] = stack.back();
        stack.pop_back();
        if (i != j) {
            const double a = aabb_collision_start(&M.C_box[7 * static_cast<size_t>(i)], &C_up[7 * static_cast<size_t>(i)],
                                                  &M.C_box[7 * static_cast<size_t>(j)], &C_up[7 * static_cast<size_t>(j)]);
            if (a * t_init >= t_max) continue;   // admissible: no contact before t_max
        }
        const Int Li = M.C_left[i], Lj = M.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const Int Ri = M.C_right[i], Rj = M.C_right[j];
            const double si = Li >= 0 ? M.C_box[7 * static_cast<size_t>(i)] : 0.0;
            const double sj = Lj >= 0 ? M.C_box[7 * static_cast<size_t>(j)] : 0.0;
            if (si == sj && si > 0) {
                if (i == j) { stack.push_back({Li, Rj}); stack.push_back({Ri, Rj}); stack.push_back({Li, Lj}); }
                else { stack.push_back({Ri, Rj}); stack.push_back({Li, Rj}); stack.push_back({Ri, Lj}); stack.push_back({Li, Lj}); }
            } else if (si > sj) {
                stack.push_back({Ri, j}); stack.push_back({Li, j});
            } else {
                stack.push_back({i, Rj}); stack.push_back({i, Lj});
            }
            continue;
        }
        if (i == j) continue;
        const Int pi = M.C_begin[i], pj = M.C_begin[j];
        if (primitives_adjacent(M, pi, pj)) continue;
        t_max = find_max_safe_step(P[pi], P[pj], t_max, TOL);
    }
    return std::min(t_max, t_init);
}

struct OracleHandle {
    Mesh M;
    const Mesh* obstacle = nullptr;   // not owned
    ObstacleLists ob;
    MetricValues mv;
    bool mv_valid = false;
    double mv_q = 0, mv_p = 0;
};

extern "C" {

void* oracle_create(int dom, const double* V, int nV, const int* S, int nS, const double* charges,
                    double theta_far, double theta_near, int max_refinement, int threads)
{
    if (dom < 1 || dom > 2 || nV <= 0 || nS <= 0) return nullptr;
    auto* H = new OracleHandle();
    Mesh& M = H->M;
    M.dom = dom;
    M.SIZE = dom + 1;
    M.nV = nV;
    M.nS = nS;
    M.set.theta_far = theta_far;
    M.set.theta_near = theta_near;
    M.set.max_refinement = max_refinement;
    M.set.threads = std::max(1, threads);
    M.V.assign(V, V + 3 * static_cast<size_t>(nV));
    M.V_frozen = M.V;
    M.S.assign(S, S + static_cast<size_t>(M.SIZE) * nS);
    M.charge_v.assign(nV, 1.0);
    if (charges) M.charge_v.assign(charges, charges + nV);
    build_cluster_tree(M);
    compute_primitive_data(M, true);
    compute_cluster_data(M);
    build_block_cluster_tree(M);
    return H;
}

void oracle_destroy(void* h) { delete static_cast<OracleHandle*>(h); }

// 0: closed-form chain rule (default), 1: forward-mode differentiation of the moment map
void oracle_set_chain_rule(int mode) { g_chain_rule_mode = mode; }

void oracle_set_threads(void* h, int threads) { static_cast<OracleHandle*>(h)->M.set.threads = std::max(1, threads); }

// counts: [N, NC, near_nnz, far_nnz, verynear_nnz, inter_nnz, depth]
void oracle_counts(void* h, int64_t* out)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    out[0] = M.nS; out[1] = M.NC;
    out[2] = M.near.nnz(); out[3] = M.far.nnz(); out[4] = M.verynear.nnz(); out[5] = M.inter.nnz();
    int d = 0;
    for (int x : M.C_depth) d = std::max(d, x);
    out[6] = d;
}

void oracle_tree(void* h, int* perm, int* C_begin, int* C_end, int* C_left, int* C_right)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::memcpy(perm, M.perm.data(), sizeof(int) * M.nS);
    std::memcpy(C_begin, M.C_begin.data(), sizeof(int) * M.NC);
    std::memcpy(C_end, M.C_end.data(), sizeof(int) * M.NC);
    std::memcpy(C_left, M.C_left.data(), sizeof(int) * M.NC);
    std::memcpy(C_right, M.C_right.data(), sizeof(int) * M.NC);
}

// which: 0 near, 1 far, 2 verynear, 3 inter
void oracle_pattern(void* h, int which, int64_t* rp, int* ci)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    const Pattern* P = which == 0 ? &M.near : which == 1 ? &M.far : which == 2 ? &M.verynear : &M.inter;
    std::memcpy(rp, P->rp.data(), sizeof(int64_t) * (P->rows + 1));
    if (P->nnz() > 0) std::memcpy(ci, P->ci.data(), sizeof(int) * P->nnz());
}

void oracle_cluster_data(void* h, double* C_far)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::memcpy(C_far, M.C_far.data(), sizeof(double) * M.C_far.size());
}

void oracle_primitive_data(void* h, double* P_near, double* P_far)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    if (P_near) std::memcpy(P_near, M.P_near.data(), sizeof(double) * M.P_near.size());
    if (P_far) std::memcpy(P_far, M.P_far.data(), sizeof(double) * M.P_far.size());
}

void oracle_semistatic_update(void* h, const double* V)
{
    auto* H = static_cast<OracleHandle*>(h);
    Mesh& M = H->M;
    M.V.assign(V, V + 3 * static_cast<size_t>(M.nV));
    compute_primitive_data(M, false);
    compute_cluster_data(M);
    H->mv_valid = false;
}

double oracle_energy(void* h, double q, double p)
{
    return tp0_evaluate(static_cast<OracleHandle*>(h)->M, q, p, false);
}

double oracle_differential(void* h, double q, double p, double alpha, double beta, double* Y, int ldY)
{
    Mesh& M = static_cast<OracleHandle*>(h)->M;
    const double en = tp0_evaluate(M, q, p, true);
    assemble_derivatives(M, alpha, beta, Y, ldY);
    return en;
}

// One row shard of `shards` (the upper-triangle rows split like the reference's threads):
// its thread slice of near derivatives (N x NEAR_DIM) and far derivatives (N_C x FAR_DIM),
// tree order, before collection; returns the shard's energy part.
double oracle_partial_derivatives(void* h, double q, double p, int shard, int shards, double* D_near, double* D_far)
{
    Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::vector<double> dn, df;
    const double en = tp0_evaluate(M, q, p, true, shards, shard, &dn, &df);
    std::memcpy(D_near, dn.data(), sizeof(double) * dn.size());
    std::memcpy(D_far, df.data(), sizeof(double) * df.size());
    return en;
}

// Row-owned slices for a disjoint row partition (the decomposition of the device's row
// shards): rows [near_first, near_last) of the FULL symmetric Near() pattern and rows
// [far_first, far_last) of Far(), every pair evaluated from its row with only the row's
// derivative DX accumulated (no column scatter), the energy of the pairs with j > i. The
// slices of a partition of all rows sum to the upper-triangle traversal's
// (FMM_Traversor.hpp:56-147 visits each pair once and scatters DY to the column instead).
// Meshes with very-near pairs are rejected (returns NaN), as by the device's shards.
double oracle_row_derivatives(void* h, double q, double p, int64_t near_first, int64_t near_last, int64_t far_first,
                              int64_t far_last, double* D_near, double* D_far)
{
    Mesh& M = static_cast<OracleHandle*>(h)->M;
    if (M.verynear.nnz() > 0) return std::numeric_limits<double>::quiet_NaN();
    const TPParams T(q, p, M.dom);
    const int nd = near_dim(M.dom);
    const int SIZE = M.SIZE;
    const double S_scale = 1.0 / SIZE;
    std::fill(D_near, D_near + static_cast<size_t>(M.nS) * nd, 0.0);
    std::fill(D_far, D_far + static_cast<size_t>(M.NC) * FAR_DIM, 0.0);
    double en = 0;
    auto bary = [&](const double* Z, double* x) {
        for (int k = 0; k < 3; ++k) {
            x[k] = S_scale * Z[1 + k];
            for (int v = 1; v < SIZE; ++v) x[k] += S_scale * Z[1 + AMB * v + k];
        }
    };
    for (int64_t i = near_first; i < near_last && M.near.nnz() > 0; ++i) {
        const double* Xi = &M.P_near[nd * static_cast<size_t>(i)];
        double x[3];
        bary(Xi, x);
        double* DX = &D_near[nd * static_cast<size_t>(i)];
        for (LInt k = M.near.rp[i]; k < M.near.rp[i + 1]; ++k) {
            const Int j = M.near.ci[k];
            const double* Yj = &M.P_near[nd * static_cast<size_t>(j)];
            double y[3];
            bary(Yj, y);
            PairOut o;
            tp0_pair(T, Xi[0], x, Xi + 1 + AMB * SIZE, Yj[0], y, Yj + 1 + AMB * SIZE, true, false, o);
            if (j > i) en += o.energy;
            DX[0] += o.DX[0];
            for (int v = 0; v < SIZE; ++v)
                for (int kk = 0; kk < 3; ++kk) DX[1 + 3 * v + kk] += S_scale * o.DX[1 + kk];
            for (int kk = 0; kk < 6; ++kk) DX[1 + AMB * SIZE + kk] += o.DX[4 + kk];
        }
    }
    for (int64_t i = far_first; i < far_last && M.far.nnz() > 0; ++i) {
        const double* Xi = &M.C_far[FAR_DIM * static_cast<size_t>(i)];
        double* DX = &D_far[FAR_DIM * static_cast<size_t>(i)];
        for (LInt k = M.far.rp[i]; k < M.far.rp[i + 1]; ++k) {
            const Int j = M.far.ci[k];
            const double* Yj = &M.C_far[FAR_DIM * static_cast<size_t>(j)];
            PairOut o;
            tp0_pair(T, Xi[0], Xi + 1, Xi + 4, Yj[0], Yj + 1, Yj + 4, true, false, o);
            if (j > i) en += o.energy;
            for (int kk = 0; kk < 10; ++kk) DX[kk] += o.DX[kk];
        }
    }
    return en;
}

// Collection (percolate-down, primitive copy, unpermute), chain rule and vertex scatter
// from summed slices: Y = alpha dE + beta Y.
void oracle_collect(void* h, const double* D_near, const double* D_far, double alpha, double beta, double* Y, int ldY)
{
    Mesh& M = static_cast<OracleHandle*>(h)->M;
    const int nd = near_dim(M.dom);
    std::vector<std::vector<double>> tDn(1, std::vector<double>(D_near, D_near + static_cast<size_t>(M.nS) * nd));
    std::vector<std::vector<double>> tDf(1, std::vector<double>(D_far, D_far + static_cast<size_t>(M.NC) * FAR_DIM));
    collect_derivatives(M, tDn, tDf, 1, nd);
    assemble_derivatives(M, alpha, beta, Y, ldY);
}

// Arithmetic of one unique pair of the energy + differential traversals, counted with
// FC: far = 1 the FF loop body (tp0_pair + accumulation of DX into the row and DY into
// the column, TP0_Kernel_FF.hpp:130-319 with FMM_Kernel_FF.hpp:162-217), far = 0 the NF
// loop body for simplices of dimension dom (column barycentre from the hull, tp0_pair,
// spreading of dE/dx over the hull slots of row and column, TP0_Kernel_NF.hpp:140-338 with
// FMM_Kernel_NF.hpp:169-272). Per-row work (row barycentre, row write) is excluded.
// out: add/sub, mul, div, sqrt, pow.
void oracle_pair_opcounts(int dom, int far, double q, double p, int64_t* out)
{
    const TPParams T(q, p, dom);
    const int SIZE = dom + 1;
    const FC S_scale(1.0 / SIZE);
    FC x[3] = {0.1, 0.2, 0.3}, P[6] = {1, 0, 0, 1, 0, 1}, Q[6] = {1, 0, 0, 1, 0, 1}, hull[9];
    for (int k = 0; k < 9; ++k) hull[k] = FC(0.5 + 0.1 * k);
    FC DXs[16], DY[16];
    for (int k = 0; k < 16; ++k) { DXs[k] = FC(0.0); DY[k] = FC(0.0); }
    g_ops = OpCounts();
    PairOutT<FC> o;
    if (far) {
        const FC y[3] = {1.1, 1.2, 1.3};
        tp0_pair<FC>(T, FC(1.0), x, P, FC(2.0), y, Q, true, false, o);
        for (int k = 0; k < 10; ++k) { DXs[k] += o.DX[k]; DY[k] += o.DY[k]; }
    } else {
        FC y[3];
        for (int k = 0; k < 3; ++k) {
            y[k] = S_scale * hull[k];
            for (int v = 1; v < SIZE; ++v) y[k] += S_scale * hull[3 * v + k];
        }
        tp0_pair<FC>(T, FC(1.0), x, P, FC(2.0), y, Q, true, false, o);
        DXs[0] += o.DX[0];
        DY[0] += o.DY[0];
        for (int v = 0; v < SIZE; ++v)
            for (int k = 0; k < 3; ++k) {
                DXs[1 + 3 * v + k] += S_scale * o.DX[1 + k];
                DY[1 + 3 * v + k] += S_scale * o.DY[1 + k];
            }
        for (int k = 0; k < 6; ++k) {
            DXs[1 + AMB * SIZE + k] += o.DX[4 + k];
            DY[1 + AMB * SIZE + k] += o.DY[4 + k];
        }
    }
    out[0] = g_ops.add; out[1] = g_ops.mul; out[2] = g_ops.div; out[3] = g_ops.sqrt; out[4] = g_ops.pow;
}

// SimplicialMesh::MaximumSafeStepSize(vecs, max_time, TOL), with the loaded obstacle if any; vel: nV x 3
double oracle_maximum_safe_step_size(void* h, const double* vel, double max_time, double tol)
{
    const OracleHandle* H = static_cast<OracleHandle*>(h);
    return maximum_safe_step_size(H->M, vel, max_time, tol, H->obstacle);
}

// moment-coordinate derivatives after collection (original order)
void oracle_moment_derivatives(void* h, double* D_near, double* D_far)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::memcpy(D_near, M.P_D_near.data(), sizeof(double) * M.P_D_near.size());
    std::memcpy(D_far, M.P_D_far.data(), sizeof(double) * M.P_D_far.size());
}

double oracle_allpairs_energy(void* h, double q, double p)
{
    return allpairs_energy(static_cast<OracleHandle*>(h)->M, q, p);
}

static void ensure_metric(OracleHandle* H, double q, double p)
{
    if (!H->mv_valid || H->mv_q != q || H->mv_p != p) {
        tp0_metric_values(H->M, q, p, H->mv);
        H->mv_valid = true;
        H->mv_q = q;
        H->mv_p = p;
    }
}

// values: near full-pattern (2*nnz), far (2*nnz), diag near (2*N), diag far (2*NC)
void oracle_metric_values(void* h, double q, double p, double* nf, double* ff, double* nf_diag, double* ff_diag)
{
    auto* H = static_cast<OracleHandle*>(h);
    ensure_metric(H, q, p);
    if (nf) std::memcpy(nf, H->mv.nf.data(), sizeof(double) * H->mv.nf.size());
    if (ff) std::memcpy(ff, H->mv.ff.data(), sizeof(double) * H->mv.ff.size());
    if (nf_diag) std::memcpy(nf_diag, H->mv.nf_diag.data(), sizeof(double) * H->mv.nf_diag.size());
    if (ff_diag) std::memcpy(ff_diag, H->mv.ff_diag.data(), sizeof(double) * H->mv.ff_diag.size());
}

void oracle_metric_multiply(void* h, double q, double p, double alpha, const double* X, int ldX, double beta,
                            double* Y, int ldY, int flags)
{
    auto* H = static_cast<OracleHandle*>(h);
    ensure_metric(H, q, p);
    metric_multiply(H->M, H->mv, alpha, X, ldX, beta, Y, ldY, flags & 1, flags & 2, flags & 4);
}

void oracle_pseudo_laplacian_multiply(void* h, double s, double alpha, const double* X, int ldX, double beta,
                                      double* Y, int ldY)
{
    pseudo_laplacian_multiply(static_cast<OracleHandle*>(h)->M, s, alpha, X, ldX, beta, Y, ldY);
}

int64_t oracle_h1_triplet_count(void* h)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    return static_cast<int64_t>(M.nS) * M.SIZE * M.SIZE;
}

void oracle_h1_triplets(void* h, double ws, double wm, int* I, int* J, double* A)
{
    h1_triplets(static_cast<OracleHandle*>(h)->M, ws, wm, I, J, A);
}


// Obstacle (the obstacle handle must outlive its use by h). Returns 0, or -1 if the
// domain dimensions differ.
int oracle_load_obstacle(void* h, void* obstacle)
{
    auto* H = static_cast<OracleHandle*>(h);
    const Mesh& O = static_cast<OracleHandle*>(obstacle)->M;
    if (O.dom != H->M.dom) return -1;
    H->obstacle = &O;
    build_obstacle_block_cluster_tree(H->M, O, H->ob);
    return 0;
}

// [near, far, verynear, inter] nnz of the obstacle lists
void oracle_obstacle_counts(void* h, int64_t* out)
{
    const auto* H = static_cast<OracleHandle*>(h);
    out[0] = H->ob.near.nnz(); out[1] = H->ob.far.nnz(); out[2] = H->ob.verynear.nnz(); out[3] = H->ob.inter.nnz();
}

void oracle_obstacle_pattern(void* h, int which, int64_t* rp, int* ci)
{
    const auto* H = static_cast<OracleHandle*>(h);
    const CrossPattern& P = which == 0 ? H->ob.near : which == 1 ? H->ob.far : which == 2 ? H->ob.verynear : H->ob.inter;
    for (size_t k = 0; k < P.rp.size(); ++k) rp[k] = static_cast<int64_t>(P.rp[k]);
    for (size_t k = 0; k < P.ci.size(); ++k) ci[k] = P.ci[k];
}

double oracle_obstacle_energy(void* h, double q, double p)
{
    auto* H = static_cast<OracleHandle*>(h);
    if (!H->obstacle) return 0.0;
    return obstacle_evaluate(H->M, *H->obstacle, H->ob, q, p, false);
}

double oracle_obstacle_differential(void* h, double q, double p, double alpha, double beta, double* Y, int ldY)
{
    auto* H = static_cast<OracleHandle*>(h);
    if (!H->obstacle) return 0.0;
    const double en = obstacle_evaluate(H->M, *H->obstacle, H->ob, q, p, true);
    assemble_derivatives(H->M, alpha, beta, Y, ldY);
    return en;
}

double oracle_obstacle_allpairs_energy(void* h, double q, double p)
{
    auto* H = static_cast<OracleHandle*>(h);
    if (!H->obstacle) return 0.0;
    return obstacle_allpairs_energy(H->M, *H->obstacle, q, p);
}


// SimplexDensities (rho per simplex, original order); returns the energy
double oracle_simplex_densities(void* h, double q, double p, double* out)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::vector<double> rho;
    const double en = tp0_densities(M, q, p, rho);
    std::copy(rho.begin(), rho.end(), out);
    return en;
}

// VertexDensities: sum over the simplices at v of (a_i/(n+1)) rho_i, divided by the same sum
// of a_i/(n+1) (the dual volume); a_i = mean vertex charge * volume
double oracle_vertex_densities(void* h, double q, double p, double* out)
{
    const Mesh& M = static_cast<OracleHandle*>(h)->M;
    std::vector<double> rho;
    const double en = tp0_densities(M, q, p, rho);
    std::vector<double> num(M.nV, 0.0), den(M.nV, 0.0);
    for (Int i = 0; i < M.nS; ++i) {
        const Int pi = M.inv_perm[i];
        const double w = M.pre_vals[4 * static_cast<size_t>(pi) * M.SIZE];   // row 0: a_i / (n+1)
        for (int c = 0; c < M.SIZE; ++c) {
            const Int v = M.S[M.SIZE * static_cast<size_t>(i) + c];
            num[v] += w * rho[i];
            den[v] += w;
        }
    }
    for (Int v = 0; v < M.nV; ++v) out[v] = den[v] > 0 ? num[v] / den[v] : 0.0;
    return en;
}

}  // extern "C"
