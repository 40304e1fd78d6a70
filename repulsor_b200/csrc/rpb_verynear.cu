// Very-near field: adaptive subdivision quadrature on non-adjacent primitive pairs
// that fail the near-field separation test (FMM_Kernel_VF_Common.hpp:3-116,
// TP0_Kernel_VF.hpp:159-378, SimplexHierarchy_2D.hpp:17-128).
//
// One thread per unordered very-near pair, FP64. Both primitives are refined
// together (1:4 for triangles, 1:2 for edges) starting from the level-1 child
// pairs; a sub-pair is evaluated when the separation test with theta_near holds
// or the level limit is reached. Sub-simplices are stored as child-index paths;
// their barycentric corners are dyadic rationals and are rebuilt exactly.
//
// The quadrature weight w = w_S w_T multiplies the energy, the derivative and the
// metric entries once (the reference applies it to the derivative, omits it from
// the energy and applies it twice to a_0 -- TP0_Kernel_VF.hpp:214,256-301,360-366).
#include <cstring>
#include <string>

#include "geometry.cuh"
#include "kernels_energy.cuh"
#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

constexpr int VF_STACK = 15 * 30 + 16 + 8;

struct VFArgs {
    int dom, N;
    const int64_t* rp;
    const int* ci;
    const double* V;
    const int* S;
    const int* perm;
    const double* charge_v;
    double theta2;
    int max_level;
    TPExp ex;
    // energy / differential mode
    double* D_vf;          // N x 16 (reference layout: a, a*hull, a*P derivatives), zeroed before
    double* energy;        // accumulated with atomics
    bool diff;
    // metric mode
    float2* vals;          // full-pattern values (both triangles written)
    double2* diag;         // row diagonals (accumulated with atomics)
};

struct Prim {
    double h[3][3];
    double a;
    double P[6];
};

__device__ void load_prim(const VFArgs& A, int i, Prim& pr)
{
    const int size = A.dom + 1;
    SimplexGeom g;
    simplex_geometry(A.dom, A.V, A.S + static_cast<int64_t>(size) * A.perm[i], A.charge_v, g);
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) pr.h[c][k] = (c < size) ? g.h[c][k] : 0.0;
    pr.a = g.charge * g.vol;
    projector_packed(A.dom, g.t, pr.P);
}

// Barycentric corners of the sub-simplex reached by `path` at `level`.
__device__ void corners_of(int dom, uint64_t path, int level, double bc[3][3])
{
    for (int c = 0; c < 3; ++c)
        for (int v = 0; v < 3; ++v) bc[c][v] = (c == v) ? 1.0 : 0.0;
    const int bits = (dom == 2) ? 2 : 1;
    for (int l = level - 1; l >= 0; --l) {
        const int k = static_cast<int>((path >> (bits * l)) & ((1u << bits) - 1u));
        double nb[3][3];
        if (dom == 1) {
            for (int v = 0; v < 3; ++v) {
                const double mid = 0.5 * (bc[0][v] + bc[1][v]);
                nb[0][v] = (k == 0) ? bc[0][v] : mid;
                nb[1][v] = (k == 0) ? mid : bc[1][v];
                nb[2][v] = 0.0;
            }
        } else if (k < 3) {
            for (int c = 0; c < 3; ++c)
                for (int v = 0; v < 3; ++v) nb[c][v] = (c == k) ? bc[k][v] : 0.5 * (bc[k][v] + bc[c][v]);
        } else {
            for (int c = 0; c < 3; ++c)
                for (int v = 0; v < 3; ++v) nb[c][v] = 0.5 * (bc[(c + 1) % 3][v] + bc[(c + 2) % 3][v]);
        }
        for (int c = 0; c < 3; ++c)
            for (int v = 0; v < 3; ++v) bc[c][v] = nb[c][v];
    }
}

__device__ void sub_geometry(int dom, const Prim& pr, const double bc[3][3], double pts[9], double cen[3], double& r2,
                             double lam[3])
{
    const int size = dom + 1;
    for (int c = 0; c < size; ++c)
        for (int k = 0; k < 3; ++k) {
            double acc = 0;
            for (int v = 0; v < size; ++v) acc += bc[c][v] * pr.h[v][k];
            pts[3 * c + k] = acc;
        }
    for (int v = 0; v < 3; ++v) {
        double acc = 0;
        for (int c = 0; c < size; ++c) acc += bc[c][v];
        lam[v] = acc / size;
    }
    for (int k = 0; k < 3; ++k) {
        double acc = 0;
        for (int c = 0; c < size; ++c) acc += pts[3 * c + k];
        cen[k] = acc / size;
    }
    r2 = 0;
    for (int c = 0; c < size; ++c) {
        double d = 0;
        for (int k = 0; k < 3; ++k) d += (pts[3 * c + k] - cen[k]) * (pts[3 * c + k] - cen[k]);
        r2 = d > r2 ? d : r2;
    }
}

__device__ void make_proj(const double v[3], const double P[6], const double Q[6], Proj<double>& g)
{
    for (int k = 0; k < 3; ++k) g.v[k] = v[k];
    g.r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    g.Pv[0] = P[0] * v[0] + P[1] * v[1] + P[2] * v[2];
    g.Pv[1] = P[1] * v[0] + P[3] * v[1] + P[4] * v[2];
    g.Pv[2] = P[2] * v[0] + P[4] * v[1] + P[5] * v[2];
    g.Qv[0] = Q[0] * v[0] + Q[1] * v[1] + Q[2] * v[2];
    g.Qv[1] = Q[1] * v[0] + Q[3] * v[1] + Q[4] * v[2];
    g.Qv[2] = Q[2] * v[0] + Q[4] * v[1] + Q[5] * v[2];
    g.cphi = v[0] * g.Pv[0] + v[1] * g.Pv[1] + v[2] * g.Pv[2];
    g.cpsi = v[0] * g.Qv[0] + v[1] * g.Qv[1] + v[2] * g.Qv[2];
}

template <bool METRIC>
__global__ void k_verynear(VFArgs A)
{
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= A.rp[A.N]) return;
    // row of entry k
    int lo = 0, hi = A.N;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (A.rp[mid] <= k) lo = mid; else hi = mid;
    }
    const int i = lo, j = A.ci[k];
    if (j <= i) return;  // each unordered pair once
    Prim X, Y;
    load_prim(A, i, X);
    load_prim(A, j, Y);
    const int size = A.dom + 1;
    const int nch = (A.dom == 2) ? 4 : 2;
    const int bits = (A.dom == 2) ? 2 : 1;
    const double wstep = (A.dom == 2) ? 0.25 : 0.5;

    uint64_t stS[VF_STACK], stT[VF_STACK];
    unsigned char stL[VF_STACK];
    int sp = 0;
    for (int a = 0; a < nch; ++a)
        for (int b = 0; b < nch; ++b) { stS[sp] = a; stT[sp] = b; stL[sp] = 1; ++sp; }

    double e_sum = 0.0, a0_sum = 0.0, a1_sum = 0.0;
    double DX[16], DY[16];
    for (int m = 0; m < 16; ++m) { DX[m] = 0; DY[m] = 0; }
    while (sp > 0) {
        --sp;
        const uint64_t ps = stS[sp], pt = stT[sp];
        const int level = stL[sp];
        double bs[3][3], bt[3][3], xs[9], xt[9], cs[3], ct[3], rs, rt, ls[3], lt[3];
        corners_of(A.dom, ps, level, bs);
        corners_of(A.dom, pt, level, bt);
        sub_geometry(A.dom, X, bs, xs, cs, rs, ls);
        sub_geometry(A.dom, Y, bt, xt, ct, rt, lt);
        bool stop = level >= A.max_level;
        if (!stop) {
            const double d2 = (A.dom == 2) ? tri_tri_d2(xs, xt) : seg_seg_d2(xs, xs + 3, xt, xt + 3);
            stop = A.theta2 * d2 > (rs > rt ? rs : rt);
        }
        if (!stop) {
            if (sp + nch * nch > VF_STACK) continue;  // cannot happen for level <= 30
            for (int a = 0; a < nch; ++a)
                for (int b = 0; b < nch; ++b) {
                    stS[sp] = (ps << bits) | static_cast<uint64_t>(a);
                    stT[sp] = (pt << bits) | static_cast<uint64_t>(b);
                    stL[sp] = static_cast<unsigned char>(level + 1);
                    ++sp;
                }
            continue;
        }
        double w1 = 1.0;
        for (int l = 0; l < level; ++l) w1 *= wstep;
        const double ws = w1, wt = w1;
        double v[3] = {ct[0] - cs[0], ct[1] - cs[1], ct[2] - cs[2]};
        if (METRIC && A.ex.qh == -2) {
            // pseudo-Laplacian kernel -|x-y|^{2 s_exp} (PseudoLaplacian_Kernel_VF.hpp)
            const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            const double val = -pow(r2, A.ex.s_exp_metric);
            a0_sum += ws * wt * val;
            a1_sum += ws * wt * val;
            continue;
        }
        if (METRIC) {
            const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double Pv[3], Qv[3];
            Pv[0] = X.P[0] * v[0] + X.P[1] * v[1] + X.P[2] * v[2];
            Pv[1] = X.P[1] * v[0] + X.P[3] * v[1] + X.P[4] * v[2];
            Pv[2] = X.P[2] * v[0] + X.P[4] * v[1] + X.P[5] * v[2];
            Qv[0] = Y.P[0] * v[0] + Y.P[1] * v[1] + Y.P[2] * v[2];
            Qv[1] = Y.P[1] * v[0] + Y.P[3] * v[1] + Y.P[4] * v[2];
            Qv[2] = Y.P[2] * v[0] + Y.P[4] * v[1] + Y.P[5] * v[2];
            const double cphi = v[0] * Pv[0] + v[1] * Pv[1] + v[2] * Pv[2];
            const double cpsi = v[0] * Qv[0] + v[1] * Qv[1] + v[2] * Qv[2];
            const double a1 = -2.0 * pow(r2, A.ex.s_exp_metric);
            const double a0 = 0.5 * (cphi + cpsi) / (r2 * r2) * a1;
            a0_sum += ws * wt * a0;
            a1_sum += ws * wt * a1;
            continue;
        }
        PairAcc<double> accX = {}, accY = {};
        const double ap = X.a * ws, bp = Y.a * wt;
        Proj<double> gx, gy;
        make_proj(v, X.P, Y.P, gx);
        const double mv[3] = {-v[0], -v[1], -v[2]};
        make_proj(mv, Y.P, X.P, gy);
        double e;
        if (A.ex.qh == 3 && A.ex.ph == 6) {
            e = tp0_core<double, 3, 6, true>(A.ex, gx, ap, bp, accX);
            if (A.diff) tp0_core<double, 3, 6, true>(A.ex, gy, bp, ap, accY);
        } else {
            e = tp0_core<double, -1, -1, true>(A.ex, gx, ap, bp, accX);
            if (A.diff) tp0_core<double, -1, -1, true>(A.ex, gy, bp, ap, accY);
        }
        e_sum += e;
        if (A.diff) {
            // reference layout: DX[0] = ws (d0 - dx . x), hull slot v = ws lambda_v dx, P part ws dP
            DX[0] += ws * (accX.d0 - (accX.dx[0] * cs[0] + accX.dx[1] * cs[1] + accX.dx[2] * cs[2]));
            DY[0] += wt * (accY.d0 - (accY.dx[0] * ct[0] + accY.dx[1] * ct[1] + accY.dx[2] * ct[2]));
            for (int c = 0; c < size; ++c)
                for (int kk = 0; kk < 3; ++kk) {
                    DX[1 + 3 * c + kk] += ws * ls[c] * accX.dx[kk];
                    DY[1 + 3 * c + kk] += wt * lt[c] * accY.dx[kk];
                }
            for (int m = 0; m < 6; ++m) {
                DX[1 + 3 * size + m] += ws * accX.dP[m];
                DY[1 + 3 * size + m] += wt * accY.dP[m];
            }
        }
    }
    if (METRIC) {
        A.vals[k] = make_float2(static_cast<float>(a0_sum), static_cast<float>(a1_sum));
        // transposed entry (j, i)
        int64_t lo2 = A.rp[j], hi2 = A.rp[j + 1];
        while (hi2 - lo2 > 1) {
            const int64_t mid = (lo2 + hi2) >> 1;
            if (A.ci[mid] <= i) lo2 = mid; else hi2 = mid;
        }
        A.vals[lo2] = make_float2(static_cast<float>(a0_sum), static_cast<float>(a1_sum));
        const double bo = Y.a / X.a, ao = X.a / Y.a;
        atomicAdd(&A.diag[i].x, -bo * a0_sum);
        atomicAdd(&A.diag[i].y, -bo * a1_sum);
        atomicAdd(&A.diag[j].x, -ao * a0_sum);
        atomicAdd(&A.diag[j].y, -ao * a1_sum);
        return;
    }
    atomicAdd(A.energy, e_sum);
    if (A.diff) {
        const int nd = 1 + 3 * size + 6;
        for (int m = 0; m < nd; ++m) {
            atomicAdd(&A.D_vf[16 * static_cast<int64_t>(i) + m], DX[m]);
            atomicAdd(&A.D_vf[16 * static_cast<int64_t>(j) + m], DY[m]);
        }
    }
}

static VFArgs make_args(rpb_mesh* m, const TPExp& ex)
{
    VFArgs A;
    std::memset(&A, 0, sizeof(A));
    A.dom = m->dom;
    A.N = m->N;
    A.rp = m->verynear.rp.ptr;
    A.ci = m->verynear.ci.ptr;
    A.V = m->V.ptr;
    A.S = m->S.ptr;
    A.perm = m->perm.ptr;
    A.charge_v = m->charge_v.ptr;
    A.theta2 = m->settings.theta_near * m->settings.theta_near;
    A.max_level = m->settings.max_refinement;
    A.ex = ex;
    return A;
}

rpb_status launch_vf(rpb_mesh* m, const TPExp& ex, bool diff)
{
    if (m->verynear.nnz == 0) return RPB_OK;
    VFArgs A = make_args(m, ex);
    A.D_vf = m->D_vf.ptr;
    A.energy = m->energy.ptr + 2;
    A.diff = diff;
    if (cudaMemsetAsync(m->energy.ptr + 2, 0, sizeof(double), m->stream) != cudaSuccess ||
        (diff && cudaMemsetAsync(m->D_vf.ptr, 0, m->D_vf.bytes(), m->stream) != cudaSuccess)) {
        set_error("memset failed");
        return RPB_ECUDA;
    }
    const int64_t n = m->verynear.nnz;
    k_verynear<false><<<static_cast<unsigned>((n + 63) / 64), 64, 0, m->stream>>>(A);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near kernel launch failed"); return RPB_ECUDA; }
    return RPB_OK;
}

rpb_status launch_vf_metric(rpb_mesh* m, const TPExp& ex, float2* vals, double2* diag)
{
    if (m->verynear.nnz == 0) return RPB_OK;
    VFArgs A = make_args(m, ex);
    A.vals = vals;
    A.diag = diag;
    if (ex.qh == -2) A.max_level = m->settings.max_refinement < 20 ? m->settings.max_refinement : 20;
    const int64_t n = m->verynear.nnz;
    k_verynear<true><<<static_cast<unsigned>((n + 63) / 64), 64, 0, m->stream>>>(A);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near metric kernel launch failed"); return RPB_ECUDA; }
    return RPB_OK;
}

}  // namespace rpb
