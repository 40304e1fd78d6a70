// Tangent-point energy and differential kernels (B200, sm_100a).
//
//   k_geometry_prims,  : SimplicialMesh::SemiStaticUpdate -- simplex data
//   k_cluster_moments    (src/SimplexDataKernel.hpp:92-203) in tree order, plus the
//                        ClusterTree moments (ComputeClusterData_Thread.hpp:50-129) as
//                        prefix-sum range differences.
//   k_tp0_pairs_tiled  : TP0 near-field and far-field pair kernels
//   k_tp0_pairs          (TP0_Kernel_NF.hpp:140-338, TP0_Kernel_FF.hpp:130-319) over the
//                        full symmetric CSR patterns, LANES threads per row; every row
//                        accumulates only its own derivative, so no scatter/atomics. The
//                        tiled form stages each row tile's column data in shared memory;
//                        the gather form reads it through L1/L2.
//   k_collect_chain    : CollectFar/NearFieldDerivatives (src/ClusterTree.hpp:1115-1208),
//                        the percolate-down of the far field and DNearFarToHulls
//                        (SimplicialMeshDetails.hpp:529-733, :1097-1410) per primitive.
//   k_gather_vertices  : DerivativeAssembler().Dot (src/SimplicialMesh.hpp:625-674).
#pragma once

#include <type_traits>

#include "rpb_device.cuh"

namespace rpb {

// ----------------------------------------------------------------------------------------
// Simplex geometry shared by the data, chain-rule and metric kernels.
// ----------------------------------------------------------------------------------------
struct SimplexGeom {
    double h[3][3];      // hull in the simplex's own vertex order
    double c[3];         // barycentre
    double vol;          // |tau| (edges) or |nu|/2 (triangles)
    double t[3];         // unit tangent (edges) or unit normal (triangles)
    double len;          // |tau| or |nu|
    double charge;       // mean vertex charge
    double diam;         // longest edge
};

__device__ __forceinline__ void simplex_geometry(int dom, const double* __restrict__ V, const int* __restrict__ s,
                                                 const double* __restrict__ charge_v, SimplexGeom& g)
{
    const int size = dom + 1;
    g.charge = 0.0;
    for (int j = 0; j < size; ++j) {
        const int v = s[j];
        g.h[j][0] = V[3 * static_cast<int64_t>(v) + 0];
        g.h[j][1] = V[3 * static_cast<int64_t>(v) + 1];
        g.h[j][2] = V[3 * static_cast<int64_t>(v) + 2];
        g.charge += charge_v ? charge_v[v] : 1.0;   // no charges: unit charges
    }
    // multiplications by 1/size and 1/len instead of FP64 divisions (the results differ by at
    // most an ulp; +1 % evals/s)
    const double inv_size = (dom == 1) ? 0.5 : (1.0 / 3.0);
    g.charge *= inv_size;
    for (int k = 0; k < 3; ++k) {
        double acc = g.h[0][k];
        for (int j = 1; j < size; ++j) acc += g.h[j][k];
        g.c[k] = acc * inv_size;
    }
    if (dom == 1) {
        double tau[3] = {g.h[1][0] - g.h[0][0], g.h[1][1] - g.h[0][1], g.h[1][2] - g.h[0][2]};
        g.len = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
        g.vol = g.len;
        const double inv_len = 1.0 / g.len;
        for (int k = 0; k < 3; ++k) g.t[k] = tau[k] * inv_len;
        g.diam = g.len;
    } else {
        double e1[3], e2[3], e3[3];
        for (int k = 0; k < 3; ++k) {
            e1[k] = g.h[1][k] - g.h[0][k];
            e2[k] = g.h[2][k] - g.h[0][k];
            e3[k] = g.h[2][k] - g.h[1][k];
        }
        double nu[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        g.len = sqrt(nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2]);
        g.vol = 0.5 * g.len;
        const double inv_len = 1.0 / g.len;
        for (int k = 0; k < 3; ++k) g.t[k] = nu[k] * inv_len;
        const double l1 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
        const double l2 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
        const double l3 = e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2];
        g.diam = sqrt(fmax(l1, fmax(l2, l3)));
    }
}

// Packed normal projector: triangles n n^T, edges I - t t^T.
__device__ __forceinline__ void projector_packed(int dom, const double* t, double* P6)
{
    const double sgn = (dom == 1) ? -1.0 : 1.0;
    const double id = (dom == 1) ? 1.0 : 0.0;
    P6[0] = id + sgn * t[0] * t[0];
    P6[1] = sgn * t[0] * t[1];
    P6[2] = sgn * t[0] * t[2];
    P6[3] = id + sgn * t[1] * t[1];
    P6[4] = sgn * t[1] * t[2];
    P6[5] = id + sgn * t[2] * t[2];
}

// ----------------------------------------------------------------------------------------
// Block-wide exclusive scan of W doubles per thread (blockDim.x = SCAN_BLOCK).
// ----------------------------------------------------------------------------------------
constexpr int SCAN_BLOCK = 256;

template <int W>
__device__ __forceinline__ void block_exclusive_scan(double (&v)[W], double (&total)[W])
{
    __shared__ double warp_tot[SCAN_BLOCK / 32][W];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double incl[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
        double x = v[k];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        incl[k] = x;
    }
    if (lane == 31) {
#pragma unroll
        for (int k = 0; k < W; ++k) warp_tot[w][k] = incl[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < W; ++k) {
        double before = 0.0, all = 0.0;
        for (int q = 0; q < SCAN_BLOCK / 32; ++q) {
            const double t = warp_tot[q][k];
            if (q < w) before += t;
            all += t;
        }
        v[k] = before + incl[k] - v[k];
        total[k] = all;
    }
    __syncthreads();
}

// Exclusive scan of `n` rows of W doubles (block sums) by one block, in place; row n
// receives the grand total. The rows are read through L2 (they may have been written by
// other blocks of the same launch).
template <int W>
__device__ __forceinline__ void scan_rows_block(double* rows, int n)
{
    __shared__ double carry[W];
    if (threadIdx.x < W) carry[threadIdx.x] = 0.0;
    __syncthreads();
    for (int base = 0; base < n; base += SCAN_BLOCK) {
        const int i = base + threadIdx.x;
        double v[W], tot[W];
#pragma unroll
        for (int k = 0; k < W; ++k) v[k] = (i < n) ? __ldcg(rows + static_cast<int64_t>(W) * i + k) : 0.0;
        block_exclusive_scan<W>(v, tot);
        if (i < n) {
#pragma unroll
            for (int k = 0; k < W; ++k) rows[static_cast<int64_t>(W) * i + k] = carry[k] + v[k];
        }
        __syncthreads();
        if (threadIdx.x < W) carry[threadIdx.x] += tot[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x < W) rows[static_cast<int64_t>(W) * n + threadIdx.x] = carry[threadIdx.x];
}

template <int W>
__global__ void k_scan_rows(double* rows, int n)
{
    pdl_wait();
    pdl_launch_dependents();
    scan_rows_block<W>(rows, n);
}

// The last of a launch's `n` blocks to arrive (counter: zero before the launch, zero again
// after it) scans the rows of W block sums the blocks wrote before arriving. The counter
// only counts; no block waits for another.
template <int W>
__device__ __forceinline__ void last_block_scans_rows(double* rows, int n, unsigned* counter)
{
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == static_cast<unsigned>(n) - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    scan_rows_block<W>(rows, n);
    if (threadIdx.x == 0) *counter = 0u;
}

// Range sums over clusters of a per-primitive W-vector: in-block scans, block scan
// (k_scan_rows), then out_C = S[end] - S[begin].
template <int W>
__global__ void __launch_bounds__(SCAN_BLOCK) k_block_scan_rows(int N, const double* vals, double* local, double* blocks)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[W], tot[W];
#pragma unroll
    for (int k = 0; k < W; ++k) v[k] = (i < N) ? vals[static_cast<int64_t>(W) * i + k] : 0.0;
    block_exclusive_scan<W>(v, tot);
    if (i < N) {
#pragma unroll
        for (int k = 0; k < W; ++k) local[static_cast<int64_t>(W) * i + k] = v[k];
    }
    if (threadIdx.x < W) blocks[static_cast<int64_t>(W) * blockIdx.x + threadIdx.x] = tot[threadIdx.x];
}

template <int W>
__global__ void k_range_sums(int N, int NC, const int* C_begin, const int* C_end, const double* local,
                             const double* blocks, double* out)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= NC) return;
    const int b = C_begin[C], e = C_end[C];
    const int nb = (N + SCAN_BLOCK - 1) / SCAN_BLOCK;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        const double sb = blocks[static_cast<int64_t>(W) * (b / SCAN_BLOCK) + k] + local[static_cast<int64_t>(W) * b + k];
        const double se = (e < N) ? blocks[static_cast<int64_t>(W) * (e / SCAN_BLOCK) + k] + local[static_cast<int64_t>(W) * e + k]
                                  : blocks[static_cast<int64_t>(W) * nb + k];
        out[static_cast<int64_t>(W) * C + k] = se - sb;
    }
}

struct GeomArgs {
    int dom, N, NC;
    const double* V;          // nV x 3
    const int* S;             // N x (dom+1)
    const double* charge_v;   // nV
    const int* perm;          // position -> simplex
    const int* C_begin;
    const int* C_end;
    PrimDatum* P_pair;        // N
    ClusterDatum* C_pair;     // NC
    double* C_mom;            // NC x 10 (a, centre, P) in FP64, or null (not written)
    double* local;            // N x 10: exclusive in-block prefix of the moments (a, a c, a P)
    double* blocks;           // (nblocks + 1) x 10: block sums -> exclusive block prefix
};

__device__ __forceinline__ void store_cluster(ClusterDatum* base, int i, const double* mom)
{
    ClusterDatum d;
    d.c[0] = mom[1]; d.c[1] = mom[2]; d.c[2] = mom[3];
    for (int k = 0; k < 6; ++k) d.P[k] = static_cast<float>(mom[4 + k]);
    d.a = mom[0];
    d.pad[0] = d.pad[1] = 0.0f;
    store_datum(base, i, d);
}

// Simplex data in tree order (SimplexDataKernel::ReadSimplex/WriteFar) and the in-block
// prefix sums of the additive moments (a, a c, a P).
static __global__ void __launch_bounds__(SCAN_BLOCK) k_geometry_prims(GeomArgs g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mom[10];
    for (int k = 0; k < 10; ++k) mom[k] = 0.0;
    if (i < g.N) {
        const int size = g.dom + 1;
        SimplexGeom sg;
        simplex_geometry(g.dom, g.V, g.S + static_cast<int64_t>(size) * g.perm[i], g.charge_v, sg);
        PrimDatum d;
        for (int k = 0; k < 3; ++k) { d.c[k] = sg.c[k]; d.n[k] = sg.t[k]; }
        d.a = sg.charge * sg.vol;
        d.diam = static_cast<float>(sg.diam);
        d.pad = 0.0f;
        store_datum(g.P_pair, i, d);
        double P6[6];
        projector_packed(g.dom, sg.t, P6);
        mom[0] = d.a;
        for (int k = 0; k < 3; ++k) mom[1 + k] = d.a * sg.c[k];
        for (int k = 0; k < 6; ++k) mom[4 + k] = d.a * P6[k];
    }
    double tot[10];
    block_exclusive_scan<10>(mom, tot);
    if (i < g.N)
        for (int k = 0; k < 10; ++k) g.local[10 * static_cast<int64_t>(i) + k] = mom[k];
    if (threadIdx.x < 10) g.blocks[10 * static_cast<int64_t>(blockIdx.x) + threadIdx.x] = tot[threadIdx.x];
}

// ClusterTree moments (ComputeClusterData_Thread.hpp:50-129): a cluster's moments are
// the sums over its contiguous primitive range, A = S[end] - S[begin], centre and
// projector = moment / A.
static __global__ void k_cluster_moments(GeomArgs g)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= g.NC) return;
    const int b = g.C_begin[C], e = g.C_end[C];
    pdl_wait();
    pdl_launch_dependents();
    double m[10];
    const double* lb = g.local + 10 * static_cast<int64_t>(b);
    const double* bb = g.blocks + 10 * static_cast<int64_t>(b / SCAN_BLOCK);
    const double* be = g.blocks + 10 * static_cast<int64_t>(e / SCAN_BLOCK);
    for (int k = 0; k < 10; ++k) {
        const double sb = bb[k] + lb[k];
        const double se = (e < g.N) ? be[k] + g.local[10 * static_cast<int64_t>(e) + k]
                                    : g.blocks[10 * static_cast<int64_t>((g.N + SCAN_BLOCK - 1) / SCAN_BLOCK) + k];
        m[k] = se - sb;
    }
    const double inv = 1.0 / m[0];
    for (int k = 1; k < 10; ++k) m[k] *= inv;
    if (g.C_mom)
        for (int k = 0; k < 10; ++k) g.C_mom[10 * static_cast<int64_t>(C) + k] = m[k];
    store_cluster(g.C_pair, C, m);
}

// ----------------------------------------------------------------------------------------
// TP0 pair kernel, row side. Evaluates one pair (row x, column y) and accumulates the
// row's derivative in moment coordinates in the centred form
//     d0 = sum b (E - q/2 |u|^{q/2-1} u s^{p/2-q/2})   (no dEdv.x term),
//     dx = -sum b dEdv,   dP = sum b/2 K_xy V,
// where u = (v^T P v)/|v|^2, s = 1/|v|^2. The reference's DX[0] equals d0 - dx.x
// (TP0_Kernel_FF.hpp:220-255). Near rows keep the centred d0 and the collection adds
// dx.(x_i - x) with the primitive's own x; far rows store d0 - dx.c_C (the cluster
// centre, in FP64 when the row is written), so that the collection's ancestor walk adds
// dx.x_i without loading the clusters' centres (measured: +2 % evals/s, the FP64 sum
// keeps ~14 digits against the 1e-5 differential tolerance).
// Powers are taken of the bounded ratios u, w and of s, which keeps the FP32 range
// safe for close pairs (r^-p itself would overflow FP32 near r ~ 1e-3).
// ----------------------------------------------------------------------------------------
template <typename R>
struct PairAcc {
    R d0, dx[3], dP[6];
};

// v (row -> column), r2 = |v|^2, cphi = v^T P v, cpsi = v^T Q v, Pv, Qv.
template <typename R>
struct Proj {
    R v[3], r2, cphi, cpsi, Pv[3], Qv[3];
};

template <typename R, int QH, int PH, bool DIFF>
__device__ __forceinline__ R tp0_core(const TPExp& ex, const Proj<R>& g, R a, R b, PairAcc<R>& acc)
{
    const R s = dev_rcp(g.r2);
    const R u = g.cphi * s;
    const R w = g.cpsi * s;
    R uq1, wq1, se;
    if constexpr (QH > 0 && PH >= QH) {
        uq1 = ipow_pos(fabs(u), QH - 1);
        wq1 = ipow_pos(fabs(w), QH - 1);
        se = ipow_pos(s, PH - QH);
    } else {
        const R qh = static_cast<R>(ex.q * 0.5), ph = static_cast<R>(ex.p * 0.5);
        uq1 = (fabs(u) > R(0)) ? dev_pow(fabs(u), qh - R(1)) : R(0);
        wq1 = (fabs(w) > R(0)) ? dev_pow(fabs(w), qh - R(1)) : R(0);
        se = dev_pow(s, ph - qh);
    }
    const R uq = uq1 * u, wq = wq1 * w;
    const R E = (uq + wq) * se;
    if constexpr (DIFF) {
        const R q = static_cast<R>(ex.q), p = static_cast<R>(ex.p);
        const R se1 = se * s;
        const R Kxy = q * uq1 * se1;
        const R Kyx = q * wq1 * se1;
        const R H = p * (uq + wq) * se1;
        acc.d0 += b * (E - R(0.5) * q * uq * se);
#pragma unroll
        for (int k = 0; k < 3; ++k) acc.dx[k] -= b * (Kxy * g.Pv[k] + Kyx * g.Qv[k] - H * g.v[k]);
        const R hb = R(0.5) * b * Kxy;
        acc.dP[0] += hb * g.v[0] * g.v[0];
        acc.dP[1] += hb * R(2) * g.v[0] * g.v[1];
        acc.dP[2] += hb * R(2) * g.v[0] * g.v[2];
        acc.dP[3] += hb * g.v[1] * g.v[1];
        acc.dP[4] += hb * R(2) * g.v[1] * g.v[2];
        acc.dP[5] += hb * g.v[2] * g.v[2];
    }
    return a * E * b;
}

// A primitive's pair data as the tiled near-field kernel keeps it in shared memory: the
// 64-byte PrimDatum plus FP32 copies of the normal and the weight, converted once when the
// tile is staged instead of once per pair (80 bytes: consecutive data start on different
// shared-memory banks).
struct __align__(16) PrimTile {
    double c[3];
    double n[3];
    double a;
    float diam;
    float af;
    float nf[3];
    float pad;
};
static_assert(sizeof(PrimTile) == 80, "PrimTile must be 80 bytes");

template <typename R>
__device__ __forceinline__ R col_normal(const PrimDatum& Y, int k) { return static_cast<R>(Y.n[k]); }
template <typename R>
__device__ __forceinline__ R col_normal(const PrimTile& Y, int k)
{
    if constexpr (std::is_same<R, float>::value) return Y.nf[k];
    else return Y.n[k];
}
__device__ __forceinline__ float weight_f(const PrimDatum& Y) { return static_cast<float>(Y.a); }
__device__ __forceinline__ float weight_f(const PrimTile& Y) { return Y.af; }
__device__ __forceinline__ float weight_f(const ClusterDatum& Y) { return static_cast<float>(Y.a); }

// Projection of v = y - x for two primitives. Triangles: P = n n^T, so only n.v is
// needed (FP64); edges: P v = v - t (t.v) (FP64). Everything downstream of n.v (or of
// P v) is well conditioned and is rounded to R.
template <typename R, typename YD>
__device__ __forceinline__ void project_prims(int dom, const PrimDatum& X, const YD& Y, Proj<R>& g)
{
    const double v0 = Y.c[0] - X.c[0], v1 = Y.c[1] - X.c[1], v2 = Y.c[2] - X.c[2];
    g.v[0] = static_cast<R>(v0); g.v[1] = static_cast<R>(v1); g.v[2] = static_cast<R>(v2);
    g.r2 = g.v[0] * g.v[0] + g.v[1] * g.v[1] + g.v[2] * g.v[2];
    const double xv = X.n[0] * v0 + X.n[1] * v1 + X.n[2] * v2;
    const double yv = Y.n[0] * v0 + Y.n[1] * v1 + Y.n[2] * v2;
    if (dom == 2) {
        const R xf = static_cast<R>(xv), yf = static_cast<R>(yv);
        g.cphi = xf * xf;
        g.cpsi = yf * yf;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            g.Pv[k] = static_cast<R>(X.n[k]) * xf;
            g.Qv[k] = col_normal<R>(Y, k) * yf;
        }
    } else {
        const double p0 = v0 - X.n[0] * xv, p1 = v1 - X.n[1] * xv, p2 = v2 - X.n[2] * xv;
        const double q0 = v0 - Y.n[0] * yv, q1 = v1 - Y.n[1] * yv, q2 = v2 - Y.n[2] * yv;
        g.cphi = static_cast<R>(p0 * p0 + p1 * p1 + p2 * p2);
        g.cpsi = static_cast<R>(q0 * q0 + q1 * q1 + q2 * q2);
        g.Pv[0] = static_cast<R>(p0); g.Pv[1] = static_cast<R>(p1); g.Pv[2] = static_cast<R>(p2);
        g.Qv[0] = static_cast<R>(q0); g.Qv[1] = static_cast<R>(q1); g.Qv[2] = static_cast<R>(q2);
    }
}

// Projection for two clusters with averaged projectors. Far pairs are well separated
// (max radius < theta |v|), so v is formed in FP64 and everything after it in FP32: on the
// level-6 icosphere this moves the energy by 1e-9 relative against FP64 products, while
// the FP64 version cost 15 % of the far kernel's time.
template <typename R>
__device__ __forceinline__ void project_clusters(const ClusterDatum& X, const ClusterDatum& Y, Proj<R>& g)
{
    const R v0 = static_cast<R>(Y.c[0] - X.c[0]), v1 = static_cast<R>(Y.c[1] - X.c[1]),
            v2 = static_cast<R>(Y.c[2] - X.c[2]);
    g.v[0] = v0; g.v[1] = v1; g.v[2] = v2;
    g.r2 = v0 * v0 + v1 * v1 + v2 * v2;
    R P[6], Q[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        P[k] = static_cast<R>(X.P[k]);
        Q[k] = static_cast<R>(Y.P[k]);
    }
    const R p0 = P[0] * v0 + P[1] * v1 + P[2] * v2;
    const R p1 = P[1] * v0 + P[3] * v1 + P[4] * v2;
    const R p2 = P[2] * v0 + P[4] * v1 + P[5] * v2;
    const R q0 = Q[0] * v0 + Q[1] * v1 + Q[2] * v2;
    const R q1 = Q[1] * v0 + Q[3] * v1 + Q[4] * v2;
    const R q2 = Q[2] * v0 + Q[4] * v1 + Q[5] * v2;
    g.cphi = v0 * p0 + v1 * p1 + v2 * p2;
    g.cpsi = v0 * q0 + v1 * q1 + v2 * q2;
    g.Pv[0] = p0; g.Pv[1] = p1; g.Pv[2] = p2;
    g.Qv[0] = q0; g.Qv[1] = q1; g.Qv[2] = q2;
}

struct PairArgs {
    int dom;
    int rows;
    const int64_t* rp;
    const int* ci;
    const int* order;         // rows in processing order (length-sorted within 256-row chunks)
    const void* data;         // PrimDatum* (near) or ClusterDatum* (far)
    const void* col_data;     // CROSS: the obstacle's data the columns index
    double* D;                // rows x 10 (d0, dx[3], dP[6]) moment derivatives (far: d0 - dx.c)
    double* block_energy;     // gridDim.x
    unsigned* done;           // 1 counter, zero between launches
    double* energy_out;       // 1
    TPExp ex;
    float close_factor;       // FP64 path for near pairs with r < close_factor (d_i + d_j)
};

constexpr int PAIR_BLOCK = 256;
constexpr int PAIR_FLUSH = 16;  // FP32 partial sums are carried into FP64 every 16 pairs
// Threads per CSR row: a row's nonzeros are strided over LANES consecutive lanes and the
// partial sums combined by an xor-butterfly of warp shuffles (fixed order, deterministic).
// Near rows (~60 nonzeros at theta = 0.5) take 4 lanes, far rows (~30) take 2, which puts
// enough rows in flight to fill all SMs at the benchmark sizes.
constexpr int NEAR_LANES = 4;
constexpr int FAR_LANES = 2;

constexpr int pair_blocks(int rows, int lanes) { return (rows * lanes + PAIR_BLOCK - 1) / PAIR_BLOCK; }

// Row tiles of the shared-memory kernels: threads per block (two blocks per SM), the mean
// rows per tile the host aims below, and the largest column union a tile may stage. The
// host sizes the tiles so that their count is a whole number of waves of resident blocks.
constexpr int PAIR_TILE_THREADS = 384;
constexpr int NEAR_TILE_ROWS = 384;
constexpr int FAR_TILE_ROWS = 192;
constexpr int NEAR_TILE_UNION = 768;
constexpr int FAR_TILE_UNION = 1536;

// One lane's share of a row: the row's entries t = sub, sub + stride, ... < len (counted
// from the row's first entry) with the column handle u = index(t) and the column datum
// from datum(u, j, Y) (j: the column's tree position). The next entry's handle (PREFETCH:
// and its datum) is requested before the current pair is evaluated. A row accumulates
// only its own derivative. Energy: with COUNT_ALL every pair the row holds (a symmetric
// pattern holds each unordered pair twice and the pair energy is symmetric in its two
// primitives, so the epilogue halves the sum); otherwise each unordered pair from the row
// with the smaller index (j > i), CROSS pairs always (halved for the symmetry factor).
// A close near-field pair evaluated in FP64: energy and the ten derivative components.
// Out of line and with its operands passed by value, so that its FP64 temporaries do not
// count against the registers of the FP32 pair loop that calls it (rarely).
struct Close64 {
    double e;
    double d[10];
};

template <int QH, int PH, bool DIFF, typename Datum, typename ColDatum>
__device__ __noinline__ Close64 close_pair_fp64(TPExp ex, int dom, Datum X, ColDatum Y)
{
    Proj<double> gd;
    project_prims(dom, X, Y, gd);
    PairAcc<double> a64 = {};
    Close64 c;
    c.e = tp0_core<double, QH, PH, DIFF>(ex, gd, X.a, Y.a, a64);
    c.d[0] = a64.d0;
#pragma unroll
    for (int m = 0; m < 3; ++m) c.d[1 + m] = a64.dx[m];
#pragma unroll
    for (int m = 0; m < 6; ++m) c.d[4 + m] = a64.dP[m];
    return c;
}

// SACC: the row's FP64 derivative accumulators live in shared memory at
// Dsm[m * PAIR_TILE_THREADS] (zeroed by the caller) instead of D64, which is then filled
// from them at the end; this keeps 20 registers free inside the loop.
template <bool FAR, int QH, int PH, bool DIFF, bool CROSS, bool PREFETCH, bool SACC, bool COUNT_ALL,
          typename ColDatum, typename Datum, typename Index, typename Fetch>
__device__ __forceinline__ void pair_row(const PairArgs& A, const Datum& X, int i, int len, int sub, int stride,
                                         Index index, Fetch datum, double& e_row, double (&D64)[10], double* Dsm)
{
    auto add64 = [&](int m, double v) {
        if constexpr (SACC) Dsm[m * PAIR_TILE_THREADS] += v;
        else D64[m] += v;
    };
    const float ax = static_cast<float>(X.a);
    PairAcc<float> acc = {};
    float e32 = 0.0f;
    int since_flush = 0;
    int t = sub;
    int un = (t < len) ? index(t) : 0;
    int jn = 0;
    ColDatum Yn;
    if (PREFETCH && t < len) datum(un, jn, Yn);
    for (; t < len; t += stride) {
        int j;
        ColDatum Y;
        if constexpr (PREFETCH) {
            j = jn;
            Y = Yn;
            if (t + stride < len) datum(index(t + stride), jn, Yn);
        } else {
            datum(un, j, Y);
            if (t + stride < len) un = index(t + stride);
        }
        Proj<float> g;
        if constexpr (FAR) project_clusters(X, Y, g);
        else project_prims(A.dom, X, Y, g);
        bool close = false;
        if constexpr (!FAR) {
            const float dd = A.close_factor * (X.diam + Y.diam);
            close = g.r2 < dd * dd;
        }
        if (close) {
            // close near-field pair: the same kernel in FP64, added straight into FP64 (the
            // row datum is read again, so that its weight need not stay in registers)
            if constexpr (!FAR) {
                const Close64 c =
                    close_pair_fp64<QH, PH, DIFF>(A.ex, A.dom, load_datum(static_cast<const Datum*>(A.data), i), Y);
                if (COUNT_ALL || CROSS || j > i) e_row += c.e;
                if (DIFF) {
#pragma unroll
                    for (int m = 0; m < 10; ++m) add64(m, c.d[m]);
                }
            }
        } else {
            const float e = tp0_core<float, QH, PH, DIFF>(A.ex, g, ax, weight_f(Y), acc);
            if (COUNT_ALL || CROSS || j > i) e32 += e;
            if (++since_flush == PAIR_FLUSH) {
                since_flush = 0;
                e_row += e32;
                e32 = 0.0f;
                if (DIFF) {
                    add64(0, acc.d0);
#pragma unroll
                    for (int m = 0; m < 3; ++m) add64(1 + m, acc.dx[m]);
#pragma unroll
                    for (int m = 0; m < 6; ++m) add64(4 + m, acc.dP[m]);
                    acc = PairAcc<float>{};
                }
            }
        }
    }
    e_row += e32;
    if (DIFF) {
        add64(0, acc.d0);
#pragma unroll
        for (int m = 0; m < 3; ++m) add64(1 + m, acc.dx[m]);
#pragma unroll
        for (int m = 0; m < 6; ++m) add64(4 + m, acc.dP[m]);
        if constexpr (SACC)
#pragma unroll
            for (int m = 0; m < 10; ++m) D64[m] = Dsm[m * PAIR_TILE_THREADS];
    }
}

// Combines the partial sums of a row's lane group (size consecutive lanes of one warp, sub
// the lane's place in it) into the group's first lane by a fixed tree — at offset off the
// lanes whose sub is a multiple of 2 off add the partial of lane sub + off when it is in the
// group; every lane of the warp takes part in the shuffles —, writes the row's derivative,
// and reduces the energy deterministically: one partial per block, the last block to
// finish sums the partials in block order.
// bid / nblocks: this block's index among the launch's blocks for this pattern (the
// block energies are summed in that order by the last of them)
template <bool DIFF, bool CROSS, bool COUNT_ALL>
__device__ __forceinline__ void pair_epilogue(const PairArgs& A, bool active, int i, int sub, int size, int warp_size_max,
                                              double e_row, double (&D64)[10], int bid, int nblocks)
{
    if constexpr (COUNT_ALL || CROSS) e_row *= 0.5;
    if constexpr (CROSS) {
#pragma unroll
        for (int m = 0; m < 10; ++m) D64[m] *= 0.5;
    }
    for (int off = 1; off < warp_size_max; off <<= 1) {
        const bool take = (sub & (2 * off - 1)) == 0 && sub + off < size;
        const double e = __shfl_down_sync(0xffffffffu, e_row, off);
        if (take) e_row += e;
        if (DIFF) {
#pragma unroll
            for (int m = 0; m < 10; ++m) {
                const double d = __shfl_down_sync(0xffffffffu, D64[m], off);
                if (take) D64[m] += d;
            }
        }
    }
    if (DIFF && active && sub == 0) {
        double* dst = A.D + 10 * static_cast<int64_t>(i);
#pragma unroll
        for (int m = 0; m < 10; ++m) dst[m] = D64[m];
    }
    if (sub != 0) e_row = 0.0;
    __shared__ double sh[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    e_row = warp_sum_f64(e_row);
    if (lane == 0) sh[wib] = e_row;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += sh[w];
        A.block_energy[bid] = s;
        __threadfence();
        last = (atomicAdd(A.done, 1u) == static_cast<unsigned>(nblocks) - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += __ldcg(A.block_energy + b);
        s = warp_sum_f64(s);
        __syncthreads();
        if (lane == 0) sh[wib] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t2 = 0.0;
            for (int w = 0; w < nw; ++w) t2 += sh[w];
            *A.energy_out = t2;
            *A.done = 0u;
        }
    }
}

// LANES threads per row, column data gathered from global memory (L1/L2). FAR: rows are
// clusters of the Far() pattern; otherwise rows are primitives of the Near() pattern.
// CROSS: rows are the mesh's, columns the obstacle's (a non-symmetric block cluster tree):
// every pair counts, energy and derivatives carry the symmetry factor 1/2
// (src/FMM/FMM_Kernel.hpp:43) and the obstacle's derivatives are not formed.
template <bool FAR, int QH, int PH, bool DIFF, int LANES, bool CROSS = false>
__global__ void __launch_bounds__(PAIR_BLOCK) k_tp0_pairs(PairArgs A)
{
    static_assert(LANES == 1 || LANES == 2 || LANES == 4 || LANES == 8, "LANES must divide a warp");
    using Datum = typename std::conditional<FAR, ClusterDatum, PrimDatum>::type;
    const Datum* base = static_cast<const Datum*>(A.data);
    const Datum* cols = CROSS ? static_cast<const Datum*>(A.col_data) : base;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = t / LANES, sub = t & (LANES - 1);
    const bool active = slot < A.rows;
    double e_row = 0.0;
    double D64[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int i = 0;
    if (active) {
        i = A.order ? A.order[slot] : slot;
        const Datum X = load_datum(base, i);
        const int64_t k0 = A.rp[i];
        const int* crow = A.ci + k0;
        auto index = [&](int t) { return __ldg(crow + t); };
        auto datum = [&](int u, int& j, Datum& Y) {
            j = u;
            Y = load_datum(cols, u);
        };
        pair_row<FAR, QH, PH, DIFF, CROSS, true, false, false, Datum>(A, X, i, static_cast<int>(A.rp[i + 1] - k0), sub,
                                                                     LANES, index, datum, e_row, D64, nullptr);
        if constexpr (FAR && DIFF) D64[0] -= D64[1] * X.c[0] + D64[2] * X.c[1] + D64[3] * X.c[2];
    }
    pair_epilogue<DIFF, CROSS, false>(A, active, i, sub, LANES, LANES, e_row, D64, blockIdx.x, gridDim.x);
}

// Row tiles (build_row_tiles): block b owns the rows order[row0[b] .. row0[b+1]) and
// stages the data of the union of their columns, cols[cols_rp[b] .. cols_rp[b+1]), in
// shared memory; entry k then reads its column datum from shared-memory slot slot[k].
// Far tiles are copied with asynchronous 16-byte copies whose pieces are rotated by the
// slot (the lanes of a warp then spread their reads over all banks); near tiles are
// expanded to PrimTile on the way in. Each thread's row, group size and lane in the
// group come from the tile's lane map, so long rows get more lanes.
struct PairTiles {
    const int* row0;
    const int* cols_rp;
    const int* cols;
    const uint16_t* slot;
    const int* order;
    const int* lane_map;      // tiles x PAIR_TILE_THREADS (RowTiles::lane_map)
    int tile_base;            // block b takes tile tile_base + b (a row shard's first tile)
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ ClusterDatum load_cluster_rot(const float4* sdat, int u)
{
    ClusterDatum d;
    float4* o = reinterpret_cast<float4*>(&d);
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = sdat[4 * u + ((q + u) & 3)];
    return d;
}

// dynamic shared memory per tile of union size n: the data (PrimTile 80 bytes, ClusterDatum
// 64 bytes); far tiles also the union's column ids (their rows count each pair's energy
// from the smaller index; near rows count every pair and halve: measured fastest for each)
__host__ __device__ constexpr size_t pair_tile_union_bytes(int n, bool far)
{
    return (static_cast<size_t>(n) * (far ? sizeof(ClusterDatum) + sizeof(int) : sizeof(PrimTile)) + 15) / 16 * 16;
}

// union; near tiles also the FP64 derivative accumulators of every thread
__host__ __device__ constexpr size_t pair_tile_data_bytes(int n, bool far)
{
    return pair_tile_union_bytes(n, far) + (far ? 0 : sizeof(double) * 10 * PAIR_TILE_THREADS);
}

// Entries of a near tile's slot copy: its entries [e0, e1) extended down to a multiple of
// 8 (16-byte pieces) and up to the next one; the slot array holds PAIR_SLOT_PAD spare
// entries after the last so that the last piece stays inside it. Far tiles read their
// slots from global memory: staged, they measured slower (44.1 against 41.3 us on the
// 160 x 120 torus; near tiles 29.7 against 30.8 us).
constexpr int PAIR_SLOT_PAD = 8;
__host__ __device__ constexpr size_t pair_tile_slot_bytes(int64_t entries)
{
    return static_cast<size_t>((entries + 2 * PAIR_SLOT_PAD - 1) / PAIR_SLOT_PAD * PAIR_SLOT_PAD) * sizeof(uint16_t);
}

// the whole dynamic shared memory of a tile: data, then (near tiles) the tile's slots
__host__ __device__ constexpr size_t pair_tile_smem(int n, bool far, int64_t entries)
{
    return pair_tile_data_bytes(n, far) + (far ? 0 : pair_tile_slot_bytes(entries));
}

template <bool FAR, int QH, int PH, bool DIFF>
__device__ __forceinline__ void pairs_tiled_body(const PairArgs& A, const PairTiles& T, int bid, int nblocks)
{
    using Datum = typename std::conditional<FAR, ClusterDatum, PrimDatum>::type;
    using ColDatum = typename std::conditional<FAR, ClusterDatum, PrimTile>::type;
    extern __shared__ float4 tile_smem[];
    const Datum* base = static_cast<const Datum*>(A.data);
    const int b = T.tile_base + bid;
    const int u0 = T.cols_rp[b], un = T.cols_rp[b + 1] - u0;
    float4* sdat = tile_smem;
    int* sid = reinterpret_cast<int*>(reinterpret_cast<char*>(tile_smem) + sizeof(ColDatum) * static_cast<size_t>(un));
    if constexpr (FAR)
        for (int u = threadIdx.x; u < un; u += blockDim.x) sid[u] = __ldg(T.cols + u0 + u);
    // the tile's lane map first; the primitive / cluster data once the producer has finished
    const int r0 = T.row0[b];
    const int lm = __ldg(T.lane_map + static_cast<int64_t>(b) * PAIR_TILE_THREADS + threadIdx.x);
    const bool active = lm >= 0;
    const int sub = active ? (lm & 31) : 0, size = active ? ((lm >> 5) & 31) + 1 : 1;
    const int i = active ? T.order[r0 + (lm >> 10)] : 0;
    // near tiles: the tile's slots (entries rp[r0] .. rp[row0[b + 1]], contiguous) into
    // shared memory by 16-byte pieces from the 8-entry boundary at or below the first
    int64_t e_lo = 0;
    uint16_t* sslot = nullptr;
    if constexpr (!FAR) {
        e_lo = A.rp[r0] / PAIR_SLOT_PAD * PAIR_SLOT_PAD;
        const int pieces = static_cast<int>((A.rp[T.row0[b + 1]] - e_lo + PAIR_SLOT_PAD - 1) / PAIR_SLOT_PAD);
        sslot = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(tile_smem) + pair_tile_data_bytes(un, false));
        for (int q = threadIdx.x; q < pieces; q += blockDim.x)
            cp_async16(sslot + PAIR_SLOT_PAD * q, T.slot + e_lo + PAIR_SLOT_PAD * static_cast<int64_t>(q));
    }
    pdl_wait();
    pdl_launch_dependents();
    if constexpr (FAR) {
        for (int idx = threadIdx.x; idx < 4 * un; idx += blockDim.x) {
            const int u = idx >> 2, q = idx & 3;
            const float4* src = reinterpret_cast<const float4*>(base + __ldg(T.cols + u0 + u)) + q;
            cp_async16(sdat + 4 * u + ((q + u) & 3), src);
        }
    } else {
        PrimTile* st = reinterpret_cast<PrimTile*>(tile_smem);
        for (int u = threadIdx.x; u < un; u += blockDim.x) {
            const PrimDatum d = load_datum(base, __ldg(T.cols + u0 + u));
            PrimTile t;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                t.c[k] = d.c[k];
                t.n[k] = d.n[k];
                t.nf[k] = static_cast<float>(d.n[k]);
            }
            t.a = d.a;
            t.af = static_cast<float>(d.a);
            t.diam = d.diam;
            t.pad = 0.0f;
            st[u] = t;
        }
    }
    Datum X;
    if (active) X = load_datum(base, i);
    cp_async_wait_all();
    __syncthreads();
    double e_row = 0.0;
    double D64[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    double* Dsm = nullptr;
    if constexpr (!FAR && DIFF) {
        // this thread's accumulators, after the union (pair_tile_smem)
        Dsm = reinterpret_cast<double*>(reinterpret_cast<char*>(tile_smem) + pair_tile_union_bytes(un, false)) +
              threadIdx.x;
#pragma unroll
        for (int m = 0; m < 10; ++m) Dsm[m * PAIR_TILE_THREADS] = 0.0;
    }
    if (active) {
        const int64_t k0 = A.rp[i];
        // near rows: the row's slots by 32-bit shared-memory address (a generic pointer would
        // hold two more registers in the loop); far rows: from global memory
        const unsigned srow = FAR ? 0u
                                  : static_cast<unsigned>(__cvta_generic_to_shared(sslot)) +
                                        2u * static_cast<unsigned>(k0 - e_lo);
        const uint16_t* grow = T.slot + k0;
        auto index = [&](int t) {
            if constexpr (FAR) {
                return static_cast<int>(__ldg(grow + t));
            } else {
                unsigned short v;
                asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(srow + 2u * static_cast<unsigned>(t)));
                return static_cast<int>(v);
            }
        };
        auto datum = [&](int u, int& j, ColDatum& Y) {
            if constexpr (FAR) {
                Y = load_cluster_rot(sdat, u);
                j = sid[u];
            } else {
                Y = reinterpret_cast<const PrimTile*>(tile_smem)[u];
                j = 0;
            }
        };
        pair_row<FAR, QH, PH, DIFF, false, false, !FAR && DIFF, !FAR, ColDatum>(
            A, X, i, static_cast<int>(A.rp[i + 1] - k0), sub, size, index, datum, e_row, D64, Dsm);
        if constexpr (FAR && DIFF) D64[0] -= D64[1] * X.c[0] + D64[2] * X.c[1] + D64[3] * X.c[2];
    }
    pair_epilogue<DIFF, false, !FAR>(A, active, i, sub, size, __reduce_max_sync(0xffffffffu, size), e_row, D64, bid, nblocks);
}

template <bool FAR, int QH, int PH, bool DIFF>
__global__ void __launch_bounds__(PAIR_TILE_THREADS, 2) k_tp0_pairs_tiled(PairArgs A, PairTiles T)
{
    pairs_tiled_body<FAR, QH, PH, DIFF>(A, T, blockIdx.x, gridDim.x);
}

// Both patterns in one launch: blocks [0, nfar) take the far tiles, the others the near
// tiles, so the far and near tiles share the waves instead of draining and refilling
// the GPU between two launches. Each part keeps its own block indices, energy partials
// and last-block sum, so the results equal those of the two separate launches.
template <int QH, int PH, bool DIFF>
__global__ void __launch_bounds__(PAIR_TILE_THREADS, 2)
    k_tp0_pairs_tiled_both(PairArgs An, PairTiles Tn, PairArgs Af, PairTiles Tf, int nfar)
{
    if (static_cast<int>(blockIdx.x) < nfar) pairs_tiled_body<true, QH, PH, DIFF>(Af, Tf, blockIdx.x, nfar);
    else pairs_tiled_body<false, QH, PH, DIFF>(An, Tn, blockIdx.x - nfar, gridDim.x - nfar);
}

// energy = near-field part + far-field part (the order evaluate() uses on the host)
static __global__ void k_add_pair(const double* e2, double* out) { *out = e2[0] + e2[1]; }

// ----------------------------------------------------------------------------------------
// Collection + chain rule. One thread per primitive (tree order).
// ----------------------------------------------------------------------------------------
// Visits every ancestor of cluster C (C itself included) once, in a fixed order. The chain
// is cut into segments of four clusters by the jump pointers up4 (the fourth ancestor, -1
// when the root is nearer): the first ANC_SEG - 1 segments are walked interleaved, so their
// parent loads overlap while the jump pointers are followed, and the last segment walks on
// to the root. Dependent loads: about ANC_SEG - 1 + max(4, depth - 4 (ANC_SEG - 1)) instead
// of the depth.
constexpr int ANC_SEG = 5;
template <typename Visit>
__device__ __forceinline__ void ancestor_walk(int C, const int* __restrict__ parent, const int* __restrict__ up4,
                                              Visit visit)
{
    int s[ANC_SEG];
    s[0] = C;
#pragma unroll
    for (int k = 1; k < ANC_SEG; ++k) s[k] = s[k - 1] >= 0 ? __ldg(up4 + s[k - 1]) : -1;
    int node[ANC_SEG - 1];
#pragma unroll
    for (int k = 0; k < ANC_SEG - 1; ++k) node[k] = s[k];
#pragma unroll
    for (int step = 0; step < 4; ++step) {
#pragma unroll
        for (int k = 0; k < ANC_SEG - 1; ++k) {
            if (node[k] >= 0) {
                visit(node[k]);
                node[k] = __ldg(parent + node[k]);
            }
        }
    }
    for (int c = s[ANC_SEG - 1]; c >= 0; c = __ldg(parent + c)) visit(c);
}

struct CollectArgs {
    int dom, N;
    const double* V;
    const int* S;
    const double* charge_v;
    const int* perm;
    const int* leaf_of;
    const int* C_parent;
    const int* C_up4;
    const ClusterDatum* C_pair;
    const double* D_near;      // N x 10 centred
    const double* D_far;       // NC x 10, d0 - dx.c_C in the first entry
    const double* D_vf;        // N x 16 very-near derivatives (reference layout) or nullptr
    double* B;                 // N x (dom+1) x 3, original simplex order
};

static __global__ void k_collect_chain(CollectArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.N) return;
    const int size = A.dom + 1;
    const int j = A.perm[i];
    SimplexGeom g;
    // the coordinates were written before the pair kernels that precede this launch
    simplex_geometry(A.dom, A.V, A.S + static_cast<int64_t>(size) * j, A.charge_v, g);
    pdl_wait();
    pdl_launch_dependents();

    // near field (centred at the primitive barycentre)
    const double* dn = A.D_near + 10 * static_cast<int64_t>(i);
    double alpha = dn[0];
    double gx[3] = {dn[1], dn[2], dn[3]};
    double G6[6];
    for (int k = 0; k < 6; ++k) G6[k] = dn[4 + k];
    // far field: percolate down = sum over all ancestors of the leaf (d0 - dx.c_C + dx.x_i)
    ancestor_walk(A.leaf_of[i], A.C_parent, A.C_up4, [&](int C) {
        const double* df = A.D_far + 10 * static_cast<int64_t>(C);
        const double dx0 = df[1], dx1 = df[2], dx2 = df[3];
        alpha += df[0] + dx0 * g.c[0] + dx1 * g.c[1] + dx2 * g.c[2];
        gx[0] += dx0; gx[1] += dx1; gx[2] += dx2;
        for (int k = 0; k < 6; ++k) G6[k] += df[4 + k];
    });
    double hull_extra[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (A.D_vf) {
        const double* dv = A.D_vf + 16 * static_cast<int64_t>(i);
        alpha += dv[0];
        for (int c = 0; c < size; ++c)
            for (int k = 0; k < 3; ++k) {
                alpha += dv[1 + 3 * c + k] * g.h[c][k];
                hull_extra[c][k] = dv[1 + 3 * c + k];
            }
        for (int k = 0; k < 6; ++k) G6[k] += dv[1 + 3 * size + k];
    }
    double P6[6];
    projector_packed(A.dom, g.t, P6);
    for (int k = 0; k < 6; ++k) alpha += G6[k] * P6[k];
    // symmetric G with halved off-diagonals: G_ab = d/dP_ab of sum_{a<=b} G6 P_ab
    const double G[3][3] = {{G6[0], 0.5 * G6[1], 0.5 * G6[2]},
                            {0.5 * G6[1], G6[3], 0.5 * G6[4]},
                            {0.5 * G6[2], 0.5 * G6[4], G6[5]}};
    double Gt[3];
    for (int a = 0; a < 3; ++a) Gt[a] = G[a][0] * g.t[0] + G[a][1] * g.t[1] + G[a][2] * g.t[2];
    const double tGt = g.t[0] * Gt[0] + g.t[1] * Gt[1] + g.t[2] * Gt[2];
    double Bc[3][3];
    if (A.dom == 2) {
        double w[3];
        for (int a = 0; a < 3; ++a) w[a] = 2.0 * (Gt[a] - tGt * g.t[a]) * (1.0 / g.len);
        for (int c = 0; c < 3; ++c) {
            const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
            const double u[3] = {g.h[c1][0] - g.h[c2][0], g.h[c1][1] - g.h[c2][1], g.h[c1][2] - g.h[c2][2]};
            const double un[3] = {u[1] * g.t[2] - u[2] * g.t[1], u[2] * g.t[0] - u[0] * g.t[2], u[0] * g.t[1] - u[1] * g.t[0]};
            const double uw[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
            for (int k = 0; k < 3; ++k)
                Bc[c][k] = g.charge * (alpha * 0.5 * un[k] + g.vol * (gx[k] * (1.0 / 3.0) + hull_extra[c][k]) + g.vol * uw[k]);
        }
    } else {
        double gg[3];
        for (int a = 0; a < 3; ++a) gg[a] = -2.0 * (Gt[a] - tGt * g.t[a]) / g.len;
        for (int c = 0; c < 2; ++c) {
            const double sgn = (c == 1) ? 1.0 : -1.0;
            for (int k = 0; k < 3; ++k)
                Bc[c][k] = g.charge * (alpha * sgn * g.t[k] + g.vol * (gx[k] * 0.5 + hull_extra[c][k]) + g.vol * sgn * gg[k]);
        }
    }
    double* dst = A.B + static_cast<int64_t>(size) * 3 * j;
    for (int c = 0; c < size; ++c)
        for (int k = 0; k < 3; ++k) dst[3 * c + k] = Bc[c][k];
}

struct GatherArgs {
    int nV;
    const int* v_rp;     // nV + 1
    const int* v_slot;   // slot = simplex * (dom+1) + corner
    const double* B;     // slots x 3
    double alpha, beta;
    double* Y;
    int ldY;
};

// GATHER_LANES consecutive lanes per vertex, each summing every GATHER_LANES-th of the
// vertex's slots; an xor butterfly combines them and lane k < 3 writes component k.
constexpr int GATHER_LANES = 4;

static __global__ void k_gather_vertices(GatherArgs A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = t / GATHER_LANES, lane = t % GATHER_LANES;
    const bool active = v < A.nV;
    int k0 = 0, k1 = 0;
    if (active) {
        k0 = A.v_rp[v];
        k1 = A.v_rp[v + 1];
    }
    pdl_wait();
    pdl_launch_dependents();
    double acc[3] = {0, 0, 0};
    for (int k = k0 + lane; k < k1; k += GATHER_LANES) {
        const double* b = A.B + 3 * static_cast<int64_t>(A.v_slot[k]);
        acc[0] += b[0]; acc[1] += b[1]; acc[2] += b[2];
    }
#pragma unroll
    for (int off = 1; off < GATHER_LANES; off <<= 1)
#pragma unroll
        for (int m = 0; m < 3; ++m) acc[m] += __shfl_xor_sync(0xffffffffu, acc[m], off);
    if (!active || lane >= 3) return;
    const double a = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : acc[2]);
    double* y = A.Y + static_cast<int64_t>(A.ldY) * v + lane;
    *y = A.alpha * a + (A.beta == 0.0 ? 0.0 : A.beta * *y);
}

}  // namespace rpb
