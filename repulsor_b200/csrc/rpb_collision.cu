// SimplicialMesh::MaximumSafeStepSize on the B200 (src/SimplicialMesh.hpp:441-468,
// src/CollisionTree.hpp:175-215): the largest step t <= max_time along given vertex
// velocities for which no two non-adjacent primitives of the mesh touch. As in the
// reference, the geometry is the one the cluster tree was built from (construction-time
// coordinates; SemiStaticUpdate does not move the bounding volume hierarchy).
//
//   host   moving cluster boxes at max_time (leaves from the moved simplices, internal
//          clusters merged) and the symmetric dual traversal of the cluster tree, pruned
//          where the boxes' collision time interval (Compute_AABB_CollisionTimeInterval)
//          starts at or after max_time; non-adjacent leaf pairs are the candidates
//   device one thread per candidate pair: the bisection of CollisionFinder::
//          FindMaximumSafeStepSize (src/CollisionFinder.hpp:94-200) over space-time hulls
//          of the two moving simplices (src/Primitives/MovingPolytope.hpp:148-460) with a
//          collision-only GJK in four dimensions (src/GJK.hpp:618-797); the minimum over
//          the pairs by an atomic min on the bit pattern (nonnegative doubles order like
//          their bits), exact and order-independent.
//
// Every pair's bisection starts from [0, max_time]; the reference's sequential traversal
// starts later pairs from the running minimum, so both results are safe steps that can
// differ by up to the relative bisection tolerance.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/repulsor_b200.h"
#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

#define RPB_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);   \
            return e_ == cudaErrorMemoryAllocation ? RPB_ENOMEM : RPB_ECUDA;                  \
        }                                                                                     \
    } while (0)

namespace {

// A simplex moving linearly: vertices x_j + t u_j. 27 doubles.
struct MovingData {
    double x[3][3], u[3][3];
    double c[3], cu[3];      // barycentre and mean velocity
    double r, v, w;          // radius about c, |cu|, max |u_j - cu|
};

struct SpaceTime {
    const MovingData* d;
    int n;
    double a, b, T;

    // max (or min) of dir . (x_j + t u_j, t T) over the vertices and t in {a, b}
    __device__ double support(const double dir[4], double s[4], bool maximum) const
    {
        double best_a = 0, best_b = 0;
        int ia = 0, ib = 0;
        for (int i = 0; i < n; ++i) {
            double va = d->x[i][0] * dir[0] + a * (d->u[i][0] * dir[0]);
            double vb = d->x[i][0] * dir[0] + b * (d->u[i][0] * dir[0]);
            for (int j = 1; j < 3; ++j) {
                const double px = d->x[i][j] * dir[j], py = d->u[i][j] * dir[j];
                va += px + a * py;
                vb += px + b * py;
            }
            if (i == 0 || (maximum ? va > best_a : va < best_a)) { best_a = va; ia = i; }
            if (i == 0 || (maximum ? vb > best_b : vb < best_b)) { best_b = vb; ib = i; }
        }
        best_a += a * T * dir[3];
        best_b += b * T * dir[3];
        const bool take_a = maximum ? best_a >= best_b : best_a <= best_b;
        const int i = take_a ? ia : ib;
        const double t = take_a ? a : b;
        for (int j = 0; j < 3; ++j) s[j] = d->x[i][j] + t * d->u[i][j];
        s[3] = t * T;
        return take_a ? best_a : best_b;
    }
    __device__ void interior(double p[4]) const
    {
        const double t = 0.5 * (a + b);
        for (int k = 0; k < 3; ++k) p[k] = d->c[k] + t * d->cu[k];
        p[3] = t * T;
    }
    __device__ double sq_radius() const
    {
        const double s = 0.5 * fabs(b - a);
        const double X = s * d->v + d->r + d->w * b, Y = s * T;
        return X * X + Y * Y;
    }
};

// Closest point to the origin of the hull of k <= 5 points in R^4 (minimum over the faces
// whose affine closest point has nonnegative barycentric coordinates); keeps the face.
__device__ double closest_on_simplex(double W[5][4], int& k, double v[4])
{
    double best = 1e300;
    int best_mask = 0;
    double bv[4] = {0, 0, 0, 0};
    for (int mask = 1; mask < (1 << k); ++mask) {
        int idx[5], m = 0;
        for (int i = 0; i < k; ++i)
            if (mask & (1 << i)) idx[m++] = i;
        double lam[5];
        lam[0] = 1.0;
        if (m > 1) {
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
                    if (fabs(G[r][col]) > fabs(G[piv][col])) piv = r;
                double scale = 0;
                for (int r = 0; r < n; ++r) scale = fmax(scale, fabs(G[r][r]));
                if (fabs(G[piv][col]) <= 1e-14 * fmax(scale, 1e-300)) { singular = true; break; }
                if (piv != col)
                    for (int c2 = 0; c2 <= n; ++c2) { const double t = G[piv][c2]; G[piv][c2] = G[col][c2]; G[col][c2] = t; }
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
        if (d2 < best) { best = d2; best_mask = mask; for (int q = 0; q < 4; ++q) bv[q] = p[q]; }
    }
    int m = 0;
    for (int i = 0; i < k; ++i)
        if (best_mask & (1 << i)) {
            for (int q = 0; q < 4; ++q) W[m][q] = W[i][q];
            ++m;
        }
    k = m;
    for (int q = 0; q < 4; ++q) v[q] = bv[q];
    return best;
}

// collision-only GJK (GJK::IntersectingQ, theta = 1): true if the hulls come closer than
// sqrt(DBL_EPSILON) times the smaller radius
__device__ bool gjk_intersecting(const SpaceTime& P, const SpaceTime& Q)
{
    const double eps = 1.4901161193847656e-08, eps2 = eps * eps;
    double TOL2 = eps2 * fmin(P.sq_radius(), Q.sq_radius());
    if (TOL2 <= 0) TOL2 = eps2 * fmax(P.sq_radius(), Q.sq_radius());
    double v[4], q4[4];
    P.interior(v);
    Q.interior(q4);
    for (int k = 0; k < 4; ++k) v[k] -= q4[k];
    double W[5][4], ps[4], qs[4];
    P.support(v, ps, false);
    Q.support(v, qs, true);
    for (int j = 0; j < 4; ++j) { W[0][j] = ps[j] - qs[j]; v[j] = W[0][j]; }
    int k = 1;
    double dotvv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
    bool separated = false;
    for (int iter = 0; iter < 100; ++iter) {
        if (dotvv < TOL2 || k >= 5) break;
        const double a = P.support(v, ps, false);
        const double b = Q.support(v, qs, true);
        const double dotvw = a - b;
        if (dotvw > 0 && dotvw * dotvw > TOL2) { separated = true; break; }
        if (fabs(dotvv - dotvw) <= eps * dotvv) break;
        double w[4];
        for (int j = 0; j < 4; ++j) w[j] = ps[j] - qs[j];
        bool dup = false;
        for (int i = 0; i < k && !dup; ++i) dup = W[i][0] == w[0] && W[i][1] == w[1] && W[i][2] == w[2] && W[i][3] == w[3];
        if (dup) break;
        for (int j = 0; j < 4; ++j) W[k][j] = w[j];
        ++k;
        const double old = dotvv;
        dotvv = closest_on_simplex(W, k, v);
        if (fabs(old - dotvv) <= eps * dotvv) break;
    }
    return !(separated || TOL2 < dotvv);
}

constexpr int BISECT_MAX = 126;

// CollisionFinder::FindMaximumSafeStepSize: bisection of [0, tinit] with a stack of
// upper ends; the hulls' time axis is scaled by T so that space and time are comparable
__device__ double max_safe_step(const MovingData* dp, const MovingData* dq, int n, double tinit, double tol)
{
    SpaceTime P{dp, n, 0.0, tinit, 1.0}, Q{dq, n, 0.0, tinit, 1.0};
    double pi4[4], qi4[4];
    P.interior(pi4);
    Q.interior(qi4);
    double d2 = 0;
    for (int k = 0; k < 4; ++k) d2 += (qi4[k] - pi4[k]) * (qi4[k] - pi4[k]);
    const double T = sqrt(d2 + P.sq_radius() + Q.sq_radius()) / tinit;
    P.T = Q.T = T;
    double stack[BISECT_MAX + 2];
    double a = 0.0, b = tinit;
    int iter = 0, sp = 0;
    stack[0] = 0.0;
    while (b - a > tol * b && iter < BISECT_MAX) {
        ++iter;
        if (!gjk_intersecting(P, Q)) {
            if (sp > 0) {
                a = b;
                P.a = Q.a = a;
                b = stack[sp--];
                P.b = Q.b = b;
            } else {
                return b;
            }
        } else {
            stack[++sp] = b;
            b = 0.5 * (a + b);
            P.b = Q.b = b;
        }
    }
    if (sp >= BISECT_MAX || iter >= BISECT_MAX) return a;
    return a <= 0.0 ? b : a;
}

__global__ void __launch_bounds__(128) k_safe_step(int pairs, const int2* pair, const MovingData* data, int n,
                                                   double tinit, double tol, unsigned long long* t_bits)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double t = tinit;
    if (k < pairs) {
        const int2 pq = pair[k];
        t = max_safe_step(data + pq.x, data + pq.y, n, tinit, tol);
    }
    // nonnegative doubles order like their bit patterns
    t = fmax(t, 0.0);
    unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(t));
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = o < bits ? o : bits;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(t_bits, bits);
}

struct Box {
    double r2, c[3], h[3];
};

double aabb_collision_start(const Box& p0, const Box& p1, const Box& q0, const Box& q1)
{
    double t0 = 0.0, t1 = 1.0;
    for (int k = 0; k < 3; ++k) {
        const double Pmin0 = p0.c[k] - p0.h[k], Pmax0 = p0.c[k] + p0.h[k];
        const double Pmin1 = p1.c[k] - p1.h[k], Pmax1 = p1.c[k] + p1.h[k];
        const double Qmin0 = q0.c[k] - q0.h[k], Qmax0 = q0.c[k] + q0.h[k];
        const double Qmin1 = q1.c[k] - q1.h[k], Qmax1 = q1.c[k] + q1.h[k];
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

template <typename F>
void parallel_for(int threads, int n, F&& f)
{
    threads = std::max(1, std::min(threads, n / 4096 + 1));
    if (threads == 1) { f(0, n); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&, t] { f(static_cast<int>(static_cast<int64_t>(n) * t / threads),
                                   static_cast<int>(static_cast<int64_t>(n) * (t + 1) / threads)); });
    for (auto& x : th) x.join();
}

}  // namespace

// Moving data of every primitive of a mesh (tree order) on its construction coordinates;
// vel = nullptr: at rest.
static void moving_data(const rpb_mesh* m, const double* vel, std::vector<MovingData>& data)
{
    const HostTree& T = m->tree;
    const int N = m->N, size = m->size;
    const double* V = m->V_frozen.data();
    data.resize(N);
    parallel_for(std::max(1, m->settings.threads), N, [&](int i0, int i1) {
    for (int i = i0; i < i1; ++i) {
        MovingData& d = data[i];
        const int* s = m->S_host.data() + static_cast<int64_t>(size) * T.perm[i];
        double r2 = 0;
        for (int k = 0; k < 3; ++k) {
            double c = 0, cu = 0;
            for (int j = 0; j < size; ++j) {
                d.x[j][k] = V[3 * static_cast<int64_t>(s[j]) + k];
                d.u[j][k] = vel ? vel[3 * static_cast<int64_t>(s[j]) + k] : 0.0;
                c += d.x[j][k];
                cu += d.u[j][k];
            }
            d.c[k] = c / size;
            d.cu[k] = cu / size;
        }
        double w2 = 0;
        for (int j = 0; j < size; ++j) {
            double q = 0, e = 0;
            for (int k = 0; k < 3; ++k) {
                q += (d.x[j][k] - d.c[k]) * (d.x[j][k] - d.c[k]);
                e += (d.u[j][k] - d.cu[k]) * (d.u[j][k] - d.cu[k]);
            }
            r2 = std::max(r2, q);
            w2 = std::max(w2, e);
        }
        for (int j = size; j < 3; ++j)
            for (int k = 0; k < 3; ++k) d.x[j][k] = d.u[j][k] = 0.0;
        d.r = std::sqrt(r2);
        d.v = std::sqrt(d.cu[0] * d.cu[0] + d.cu[1] * d.cu[1] + d.cu[2] * d.cu[2]);
        d.w = std::sqrt(w2);
    }
    });
}

// Cluster boxes of a mesh's tree now (construction) and at max_time (moved leaves, merged
// upwards).
static void moving_boxes(const rpb_mesh* m, const std::vector<MovingData>& data, double max_time, std::vector<Box>& box,
                         std::vector<Box>& up)
{
    const HostTree& T = m->tree;
    const int NC = m->NC, size = m->size;
    box.resize(NC);
    up.resize(NC);
    std::vector<double> lo(3 * static_cast<size_t>(NC)), hi(3 * static_cast<size_t>(NC));
    for (int C = NC - 1; C >= 0; --C) {
        const double* cb = &T.C_box[7 * static_cast<size_t>(C)];
        box[C].r2 = cb[0];
        for (int k = 0; k < 3; ++k) { box[C].c[k] = cb[1 + k]; box[C].h[k] = cb[4 + k]; }
        double* l = &lo[3 * static_cast<size_t>(C)];
        double* h = &hi[3 * static_cast<size_t>(C)];
        if (T.C_left[C] < 0) {
            const MovingData& d = data[T.C_begin[C]];
            for (int k = 0; k < 3; ++k) { l[k] = 1e300; h[k] = -1e300; }
            for (int j = 0; j < size; ++j)
                for (int k = 0; k < 3; ++k) {
                    const double x = d.x[j][k] + max_time * d.u[j][k];
                    l[k] = std::min(l[k], x);
                    h[k] = std::max(h[k], x);
                }
        } else {
            const int L = T.C_left[C], R = T.C_right[C];
            for (int k = 0; k < 3; ++k) {
                l[k] = std::min(lo[3 * static_cast<size_t>(L) + k], lo[3 * static_cast<size_t>(R) + k]);
                h[k] = std::max(hi[3 * static_cast<size_t>(L) + k], hi[3 * static_cast<size_t>(R) + k]);
            }
        }
        double r2 = 0;
        for (int k = 0; k < 3; ++k) {
            const double half = 0.5 * (h[k] - l[k]);
            up[C].c[k] = l[k] + half;
            up[C].h[k] = half;
            r2 += half * half;
        }
        up[C].r2 = r2;
    }
}

// Candidates and moving data on the host, the bisections on the device.
static rpb_status safe_step(rpb_mesh* m, const double* vel, double max_time, double tol, double* t_out)
{
    const HostTree& T = m->tree;
    const int size = m->size;
    std::vector<MovingData> data;
    std::vector<Box> up, box;
    moving_data(m, vel, data);
    moving_boxes(m, data, max_time, box, up);
    auto adjacent = [&](int pi, int pj) {
        const int* a = m->S_host.data() + static_cast<int64_t>(size) * T.perm[pi];
        const int* b = m->S_host.data() + static_cast<int64_t>(size) * T.perm[pj];
        for (int x = 0; x < size; ++x)
            for (int y = 0; y < size; ++y)
                if (a[x] == b[y]) return true;
        return false;
    };
    // symmetric dual traversal (the reference's split rule), pruned where the moving boxes
    // cannot meet before max_time; the top levels are expanded breadth first into
    // independent block pairs that threads then traverse depth first
    std::vector<int2> cand;
    std::vector<std::pair<int, int>> stack;
    auto step = [&](int i, int j, std::vector<int2>& out, std::vector<std::pair<int, int>>& push) {
        if (i != j && aabb_collision_start(box[i], up[i], box[j], up[j]) >= 1.0) return;
        const int Li = T.C_left[i], Lj = T.C_left[j];
        if (Li >= 0 || Lj >= 0) {
            const int Ri = T.C_right[i], Rj = T.C_right[j];
            const double si = Li >= 0 ? box[i].r2 : 0.0, sj = Lj >= 0 ? box[j].r2 : 0.0;
            if (si == sj && si > 0) {
                if (i == j) { push.push_back({Li, Rj}); push.push_back({Ri, Rj}); push.push_back({Li, Lj}); }
                else { push.push_back({Ri, Rj}); push.push_back({Li, Rj}); push.push_back({Ri, Lj}); push.push_back({Li, Lj}); }
            } else if (si > sj) {
                push.push_back({Ri, j}); push.push_back({Li, j});
            } else {
                push.push_back({i, Rj}); push.push_back({i, Lj});
            }
            return;
        }
        if (i == j) return;
        const int pi = T.C_begin[i], pj = T.C_begin[j];
        if (!adjacent(pi, pj)) out.push_back(make_int2(pi, pj));
    };
    {
        const int threads = std::max(1, m->settings.threads);
        std::vector<std::pair<int, int>> level{{0, 0}}, next;
        while (!level.empty() && static_cast<int>(level.size()) < 64 * threads) {
            next.clear();
            for (const auto& [i, j] : level) step(i, j, cand, next);
            level.swap(next);
        }
        std::vector<std::vector<int2>> part(level.size());
        std::atomic<int> ticket{0};
        auto work = [&] {
            std::vector<std::pair<int, int>> st;
            for (;;) {
                const int k = ticket.fetch_add(1);
                if (k >= static_cast<int>(level.size())) break;
                st.assign(1, level[k]);
                while (!st.empty()) {
                    const auto [i, j] = st.back();
                    st.pop_back();
                    step(i, j, part[k], st);
                }
            }
        };
        std::vector<std::thread> th;
        for (int t = 1; t < threads && !level.empty(); ++t) th.emplace_back(work);
        work();
        for (auto& x : th) x.join();
        for (auto& p : part) cand.insert(cand.end(), p.begin(), p.end());
    }
    // the obstacle at rest (LoadUpdateVectors(nullptr) on the obstacle,
    // src/SimplicialMesh.hpp:455-460): mesh x obstacle block pairs, the larger box split
    // (both when equal), every leaf pair a candidate; obstacle data follow the mesh's
    const rpb_mesh* ob = obstacle_mesh(m);
    if (ob) {
        std::vector<MovingData> odata;
        std::vector<Box> obox, oup;
        moving_data(ob, nullptr, odata);
        moving_boxes(ob, odata, max_time, obox, oup);
        const HostTree& O = ob->tree;
        const int base = static_cast<int>(data.size());
        data.insert(data.end(), odata.begin(), odata.end());
        stack.assign(1, {0, 0});
        while (!stack.empty()) {
            const auto [i, j] = stack.back();
            stack.pop_back();
            if (aabb_collision_start(box[i], up[i], obox[j], oup[j]) >= 1.0) continue;
            const int Li = T.C_left[i], Lj = O.C_left[j];
            if (Li >= 0 || Lj >= 0) {
                const int Ri = T.C_right[i], Rj = O.C_right[j];
                const double si = Li >= 0 ? box[i].r2 : 0.0, sj = Lj >= 0 ? obox[j].r2 : 0.0;
                if (si == sj && si > 0) {
                    stack.push_back({Ri, Rj}); stack.push_back({Li, Rj}); stack.push_back({Ri, Lj}); stack.push_back({Li, Lj});
                } else if (si > sj) {
                    stack.push_back({Ri, j}); stack.push_back({Li, j});
                } else {
                    stack.push_back({i, Rj}); stack.push_back({i, Lj});
                }
                continue;
            }
            cand.push_back(make_int2(T.C_begin[i], base + O.C_begin[j]));
        }
    }
    *t_out = max_time;
    if (cand.empty()) return RPB_OK;
    DevBuf<MovingData> d_data;
    DevBuf<int2> d_pairs;
    DevBuf<unsigned long long> d_t;
    RPB_CUDA(d_data.alloc(data.size()));
    RPB_CUDA(d_pairs.alloc(cand.size()));
    RPB_CUDA(d_t.alloc(1));
    cudaStream_t s = m->stream;
    RPB_CUDA(cudaMemcpyAsync(d_data.ptr, data.data(), d_data.bytes(), cudaMemcpyHostToDevice, s));
    RPB_CUDA(cudaMemcpyAsync(d_pairs.ptr, cand.data(), d_pairs.bytes(), cudaMemcpyHostToDevice, s));
    double t0 = max_time;
    unsigned long long bits0;
    std::memcpy(&bits0, &t0, sizeof(bits0));
    RPB_CUDA(cudaMemcpyAsync(d_t.ptr, &bits0, sizeof(bits0), cudaMemcpyHostToDevice, s));
    const int pairs = static_cast<int>(cand.size());
    k_safe_step<<<(pairs + 127) / 128, 128, 0, s>>>(pairs, d_pairs.ptr, d_data.ptr, size, max_time, tol, d_t.ptr);
    RPB_CUDA(cudaGetLastError());
    unsigned long long bits = 0;
    RPB_CUDA(cudaMemcpyAsync(&bits, d_t.ptr, sizeof(bits), cudaMemcpyDeviceToHost, s));
    RPB_CUDA(cudaStreamSynchronize(s));
    double t;
    std::memcpy(&t, &bits, sizeof(t));
    *t_out = std::min(t, max_time);
    m->last_step_candidates = pairs;
    return RPB_OK;
}

}  // namespace rpb

using namespace rpb;

extern "C" {

rpb_status rpb_mesh_maximum_safe_step_size(rpb_mesh* m, const double* velocities, double max_time, double tol,
                                           double* t)
{
    if (!m || !velocities || !t) { set_error("null argument"); return RPB_EINVAL; }
    if (!(max_time > 0)) { set_error("max_time must be positive"); return RPB_EINVAL; }
    if (!(tol > 0 && tol < 1)) { set_error("tol must lie in (0, 1)"); return RPB_EINVAL; }
    for (int64_t k = 0; k < 3 * static_cast<int64_t>(m->nV); ++k)
        if (!std::isfinite(velocities[k])) { set_error("non-finite velocity"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    return safe_step(m, velocities, max_time, tol, t);
}

}  // extern "C"
