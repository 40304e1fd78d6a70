// MetricBase::Solve and MultiplyPreconditioner on the B200
// (src/Metrics/MetricDimRestricted.hpp:232-289, src/Metrics/TangentPointMetric0.hpp:88-126).
//
// The reference runs left-preconditioned GMRES with P = H1^{-1} L_{2-s} H1^{-1}. Here the
// metric (symmetric, positive semi-definite; its kernel is the translations) is solved by
// conjugate gradients with FP64 inner products and residual recurrence, one independent CG
// per right-hand-side column, with
//   RPB_PRECOND_NONE       identity,
//   RPB_PRECOND_REFERENCE  H1^{-1} L_{2-s} H1^{-1}: host Cholesky of the H1 metric (nested-
//                          dissection order from the cluster tree), GPU triangular solves
//                          level-scheduled by supernodes, GPU pseudo-Laplacian,
//   RPB_PRECOND_LEARNED    per-cluster MLP (rpb_learned.cu) inside flexible CG, falling back
//                          to REFERENCE when the flexible iteration stalls.
// Convergence is decided on the true relative residual ||B - A X|| / ||B|| per column.
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "host/sparse_cholesky.hpp"
#include "host/supernodal_chol.hpp"
#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"
#include "rpb_solver.cuh"

namespace rpb {

#define RPB_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);   \
            return e_ == cudaErrorMemoryAllocation ? RPB_ENOMEM : RPB_ECUDA;                  \
        }                                                                                     \
    } while (0)

// ------------------------------------------------------------------------------------------
// Level-scheduled supernodal triangular solves with 3 right-hand sides. A supernode c0..c1-1
// is solved as t = b - (its rows' entries outside the supernode) . y, then y = D^{-1} t with
// the inverse of its dense diagonal block. Forward: rows of L, external columns < c0,
// D^{-1} packed lower by rows. Backward: rows of L^T, external columns >= c1, D^{-T} packed
// upper by rows. The external entries are stored apart from the diagonal blocks (ext_*),
// so the gathers run without a branch. Every level of the supernode schedule
// (host/sparse_cholesky.cpp) is either
//   a warp level (all supernodes at most 32 wide, short external rows): one launch, one
//     warp per supernode, g = 32 / pow2ceil(w) lanes per row, t passed by shuffles;
//   a split level: two launches over the level's rows, G lanes per row (G a power of two,
//     4..256, chosen by the host from the level's longest row): external part into t,
//     then y = D^{-1} t.
// No inter-CTA waits of any kind.
// ------------------------------------------------------------------------------------------
struct SnTri {
    const int* sn_begin;
    const int* sn_of;         // row -> supernode
    const int64_t* ext_rp;    // row -> its entries outside its supernode
    const int* ext_ci;
    const double* ext_val;
    const int64_t* dinv_off;
    const double* dinv;
    const double* b;          // right-hand side, n x 3
    const int* perm_in;       // if set, row i reads b[perm_in[i]]
    double* t;                // split levels: n x 3 scratch
    double* y;                // solution in factor order, n x 3
    double* out;              // if set, out[perm_out[i]] = y_i
    const int* perm_out;
};

constexpr int SN_BLOCK = 256;
// widest supernode
constexpr int kMaxSupernodeWidth = 1024;
// a level runs as a warp level when every external row takes at most this many
// iterations of its lane group
constexpr int kWarpExtIters = 8;

// row r of the packed inverse diagonal block of a w-wide supernode: offset, first column, length
template <bool LOWER>
__device__ __forceinline__ void dense_row(int r, int w, int64_t& o, int& cb, int& len)
{
    o = LOWER ? static_cast<int64_t>(r) * (r + 1) / 2 : static_cast<int64_t>(r) * w - static_cast<int64_t>(r) * (r - 1) / 2;
    cb = LOWER ? 0 : r;
    len = LOWER ? r + 1 : w - r;
}

__device__ __forceinline__ void ext_dot(const SnTri& A, int64_t k0, int64_t k1, int step, double& s0, double& s1,
                                        double& s2)
{
#pragma unroll 4
    for (int64_t k = k0; k < k1; k += step) {
        const int j = __ldg(A.ext_ci + k);
        const double v = __ldg(A.ext_val + k);
        const double* yj = A.y + 3 * static_cast<int64_t>(j);
        s0 += v * yj[0];
        s1 += v * yj[1];
        s2 += v * yj[2];
    }
}

// The first PRE external entries k0, k0 + step, ... < k1 of a row, loaded before pdl_wait()
// (pattern and values are fixed during a solve); only the gathers of y wait for the
// predecessor.
template <int PRE>
struct ExtPre {
    int j[PRE];
    double v[PRE];
};

template <int PRE>
__device__ __forceinline__ void ext_preload(const SnTri& A, int64_t k0, int64_t k1, int step, ExtPre<PRE>& e)
{
#pragma unroll
    for (int i = 0; i < PRE; ++i) {
        const int64_t k = k0 + static_cast<int64_t>(i) * step;
        const bool in = k < k1;
        e.j[i] = in ? __ldg(A.ext_ci + k) : -1;
        e.v[i] = in ? __ldg(A.ext_val + k) : 0.0;
    }
}

template <int PRE>
__device__ __forceinline__ void ext_finish(const SnTri& A, const ExtPre<PRE>& e, int64_t k0, int64_t k1, int step,
                                           double& s0, double& s1, double& s2)
{
#pragma unroll
    for (int i = 0; i < PRE; ++i)
        if (e.j[i] >= 0) {
            const double* yj = A.y + 3 * static_cast<int64_t>(e.j[i]);
            s0 += e.v[i] * yj[0];
            s1 += e.v[i] * yj[1];
            s2 += e.v[i] * yj[2];
        }
    ext_dot(A, k0 + static_cast<int64_t>(PRE) * step, k1, step, s0, s1, s2);
}

// sum over aligned groups of g lanes (g a power of two, at most 32, uniform in the warp)
__device__ __forceinline__ double lane_group_sum(double v, int g)
{
    for (int o = g >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum over aligned groups of G threads (G a power of two up to the block size, uniform in
// the block; every thread of the block calls it); valid in the group's first thread
__device__ __forceinline__ void block_group_sum3(double& s0, double& s1, double& s2, int G, double (*sh)[3])
{
    if (G <= 32) {
        s0 = lane_group_sum(s0, G);
        s1 = lane_group_sum(s1, G);
        s2 = lane_group_sum(s2, G);
        return;
    }
    s0 = warp_sum_f64(s0);
    s1 = warp_sum_f64(s1);
    s2 = warp_sum_f64(s2);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[warp][0] = s0;
        sh[warp][1] = s1;
        sh[warp][2] = s2;
    }
    __syncthreads();
    if ((threadIdx.x & (G - 1)) == 0) {
        s0 = s1 = s2 = 0;
        for (int q = warp; q < warp + G / 32; ++q) {
            s0 += sh[q][0];
            s1 += sh[q][1];
            s2 += sh[q][2];
        }
    }
}

__device__ __forceinline__ void store_solution(const SnTri& A, int row, double s0, double s1, double s2)
{
    A.y[3 * static_cast<int64_t>(row) + 0] = s0;
    A.y[3 * static_cast<int64_t>(row) + 1] = s1;
    A.y[3 * static_cast<int64_t>(row) + 2] = s2;
    if (A.out) {
        const int dst = A.perm_out[row];
        A.out[3 * static_cast<int64_t>(dst) + 0] = s0;
        A.out[3 * static_cast<int64_t>(dst) + 1] = s1;
        A.out[3 * static_cast<int64_t>(dst) + 2] = s2;
    }
}

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_warp(SnTri A, const int* sn_list, int nsn)
{
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= nsn) return;   // whole warps
    const int s = sn_list[wid];
    const int c0 = A.sn_begin[s], w = A.sn_begin[s + 1] - c0;
    int p2 = 1;
    while (p2 < w) p2 <<= 1;
    const int g = 32 / p2, r = lane / g, sl = lane - r * g;
    const bool live = r < w;
    const int rr = live ? r : 0, row = c0 + rr;
    const int64_t k0 = A.ext_rp[row] + sl, k1 = live ? A.ext_rp[row + 1] : k0;
    ExtPre<kWarpExtIters> e;
    ext_preload(A, k0, k1, g, e);
    // the first kDensePre entries of this lane's part of row r of the inverse diagonal block
    constexpr int kDensePre = 8;
    const double* D = A.dinv + A.dinv_off[s];
    int64_t o;
    int cb, len;
    dense_row<LOWER>(rr, w, o, cb, len);
    double dp[kDensePre];
#pragma unroll
    for (int i = 0; i < kDensePre; ++i) {
        const int c = i * g + sl;
        dp[i] = (live && c < len) ? __ldg(D + o + c) : 0.0;
    }
    pdl_wait();
    pdl_launch_dependents();
    double s0 = 0, s1 = 0, s2 = 0;
    ext_finish(A, e, k0, k1, g, s0, s1, s2);
    s0 = lane_group_sum(s0, g);
    s1 = lane_group_sum(s1, g);
    s2 = lane_group_sum(s2, g);
    double t0 = 0, t1 = 0, t2 = 0;
    if (live) {
        const int src = A.perm_in ? A.perm_in[row] : row;
        t0 = A.b[3 * static_cast<int64_t>(src) + 0] - s0;
        t1 = A.b[3 * static_cast<int64_t>(src) + 1] - s1;
        t2 = A.b[3 * static_cast<int64_t>(src) + 2] - s2;
    }
    // y_r = sum_c Dinv[r][c] t_c; t_c lives in the lanes of row c's group
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
    for (int i = 0; i < kDensePre; ++i) {
        if (i * g >= p2) break;   // warp-uniform
        const int col = cb + i * g + sl;
        const int src = (col < w ? col : 0) * g;
        const double u0 = __shfl_sync(0xffffffffu, t0, src);
        const double u1 = __shfl_sync(0xffffffffu, t1, src);
        const double u2 = __shfl_sync(0xffffffffu, t2, src);
        a0 += dp[i] * u0;
        a1 += dp[i] * u1;
        a2 += dp[i] * u2;
    }
    for (int it = kDensePre * g; it < p2; it += g) {
        const int c = it + sl, col = cb + c;
        const int src = (col < w ? col : 0) * g;
        const double u0 = __shfl_sync(0xffffffffu, t0, src);
        const double u1 = __shfl_sync(0xffffffffu, t1, src);
        const double u2 = __shfl_sync(0xffffffffu, t2, src);
        if (live && c < len) {
            const double d = D[o + c];
            a0 += d * u0;
            a1 += d * u1;
            a2 += d * u2;
        }
    }
    a0 = lane_group_sum(a0, g);
    a1 = lane_group_sum(a1, g);
    a2 = lane_group_sum(a2, g);
    if (live && sl == 0) store_solution(A, row, a0, a1, a2);
}

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_split_ext(SnTri A, const int* rows, int nrows, int G)
{
    __shared__ double sh[SN_BLOCK / 32][3];
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) / G, sl = threadIdx.x & (G - 1);
    const bool live = q < nrows;
    const int row = live ? rows[q] : 0;
    const int64_t k0 = A.ext_rp[row] + sl, k1 = live ? A.ext_rp[row + 1] : k0;
    ExtPre<4> e;
    ext_preload(A, k0, k1, G, e);
    pdl_wait();
    pdl_launch_dependents();
    double s0 = 0, s1 = 0, s2 = 0;
    ext_finish(A, e, k0, k1, G, s0, s1, s2);
    block_group_sum3(s0, s1, s2, G, sh);
    if (live && sl == 0) {
        const int src = A.perm_in ? A.perm_in[row] : row;
        A.t[3 * static_cast<int64_t>(row) + 0] = A.b[3 * static_cast<int64_t>(src) + 0] - s0;
        A.t[3 * static_cast<int64_t>(row) + 1] = A.b[3 * static_cast<int64_t>(src) + 1] - s1;
        A.t[3 * static_cast<int64_t>(row) + 2] = A.b[3 * static_cast<int64_t>(src) + 2] - s2;
    }
}

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_split_dense(SnTri A, const int* rows, int nrows, int G)
{
    __shared__ double sh[SN_BLOCK / 32][3];
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) / G, sl = threadIdx.x & (G - 1);
    const bool live = q < nrows;
    const int row = live ? rows[q] : 0;
    const int s = A.sn_of[row];
    const int c0 = A.sn_begin[s], w = A.sn_begin[s + 1] - c0;
    int64_t o;
    int cb, len;
    dense_row<LOWER>(row - c0, w, o, cb, len);
    const double* D = A.dinv + A.dinv_off[s] + o;
    constexpr int kPre = 4;
    double dp[kPre];
#pragma unroll
    for (int i = 0; i < kPre; ++i) {
        const int c = i * G + sl;
        dp[i] = (live && c < len) ? __ldg(D + c) : 0.0;
    }
    pdl_wait();
    pdl_launch_dependents();
    double s0 = 0, s1 = 0, s2 = 0;
    if (live) {
        const double* t = A.t + 3 * static_cast<int64_t>(c0 + cb);
#pragma unroll
        for (int i = 0; i < kPre; ++i) {
            const int c = i * G + sl;
            if (c < len) {
                s0 += dp[i] * t[3 * c + 0];
                s1 += dp[i] * t[3 * c + 1];
                s2 += dp[i] * t[3 * c + 2];
            }
        }
#pragma unroll 4
        for (int c = kPre * G + sl; c < len; c += G) {
            const double d = D[c];
            s0 += d * t[3 * c + 0];
            s1 += d * t[3 * c + 1];
            s2 += d * t[3 * c + 2];
        }
    }
    block_group_sum3(s0, s1, s2, G, sh);
    if (live && sl == 0) store_solution(A, row, s0, s1, s2);
}

// ------------------------------------------------------------------------------------------
// CG vector kernels (FP64). Scalars live on the device; per column c:
//   S_RZ rz, S_RZOLD previous rz, S_PAP (p,Ap), S_RR (r,r), S_ZR_OLD (z, r_old)
// ------------------------------------------------------------------------------------------
enum { S_RZ = 0, S_RZOLD = 3, S_PAP = 6, S_RR = 9, S_ZROLD = 12, S_ACTIVE = 15, S_BB = 18, S_CONV_IT = 21, S_IT = 24,
       S_HYB_W = 25, S_COUNT = 26 };

struct DotArgs {
    int n;                    // rows (n x 3)
    const double* a;
    const double* b;
    const double* c;          // optional: accumulate (a, b - c) in the second slot
    double* partials;         // gridDim.x x 6
    unsigned* done;
    double* out0;             // 3 results (a, b)
    double* out1;             // 3 results (a, b - c) if c
};

__global__ void __launch_bounds__(256) k_dot3(DotArgs A)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = tid; i < A.n; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            const double a = A.a[3 * static_cast<int64_t>(i) + c];
            const double b = A.b[3 * static_cast<int64_t>(i) + c];
            s[c] += a * b;
            if (A.c) s[3 + c] += a * (b - A.c[3 * static_cast<int64_t>(i) + c]);
        }
    }
    __shared__ double sh[8][6];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 6; ++k) {
        const double v = warp_sum_f64(s[k]);
        if (lane == 0) sh[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0;
        for (int q = 0; q < (blockDim.x >> 5); ++q) v += sh[q][threadIdx.x];
        A.partials[6 * blockIdx.x + threadIdx.x] = v;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(A.done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        // every thread adds the partials of blocks t, t + blockDim.x, ..., then a fixed
        // tree over warps: deterministic, and no serial chain over the blocks
        __threadfence();
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
            for (int k = 0; k < 6; ++k) v[k] += __ldcg(A.partials + 6 * b + k);
        for (int k = 0; k < 6; ++k) {
            const double t = warp_sum_f64(v[k]);
            if (lane == 0) sh[w][k] = t;
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            double t = 0;
            for (int q = 0; q < (blockDim.x >> 5); ++q) t += sh[q][threadIdx.x];
            if (threadIdx.x < 3) A.out0[threadIdx.x] = t;
            else if (A.out1) A.out1[threadIdx.x - 3] = t;
        }
        if (threadIdx.x == 0) *A.done = 0u;
    }
}

// x += alpha p, r -= alpha Ap with alpha = rz / (p, Ap) per active column, fused with the
// copy r_old = r (flexible CG) and the inner products (r, r) per column: grid-stride over the rows, per-block partials, the last block adds them in
// block order (deterministic) into S[S_RR..].
__global__ void __launch_bounds__(256) k_cg_update_rr(int n, double* S, double* x, double* r, const double* p,
                                                      const double* Ap, double* rold, double* partials, unsigned* done)
{
    double alpha[3];
    bool act[3];
    for (int c = 0; c < 3; ++c) {
        act[c] = S[S_ACTIVE + c] != 0.0;
        const double pap = S[S_PAP + c];
        alpha[c] = pap != 0.0 ? S[S_RZ + c] / pap : 0.0;
    }
    double s3[3] = {0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const int64_t k = 3 * static_cast<int64_t>(i) + c;
            double rk = r[k];
            if (rold) rold[k] = rk;
            if (act[c]) {
                x[k] += alpha[c] * p[k];
                rk -= alpha[c] * Ap[k];
                r[k] = rk;
            }
            s3[c] += rk * rk;
        }
    __shared__ double sh[8][3];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = 0; c < 3; ++c) {
        const double v = warp_sum_f64(s3[c]);
        if (lane == 0) sh[w][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int q = 0; q < (blockDim.x >> 5); ++q) v += sh[q][threadIdx.x];
        partials[3 * blockIdx.x + threadIdx.x] = v;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double v[3] = {0, 0, 0};
        for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
            for (int c = 0; c < 3; ++c) v[c] += __ldcg(partials + 3 * b + c);
        for (int c = 0; c < 3; ++c) {
            const double t = warp_sum_f64(v[c]);
            if (lane == 0) sh[w][c] = t;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double t = 0;
            for (int q = 0; q < (blockDim.x >> 5); ++q) t += sh[q][threadIdx.x];
            S[S_RR + threadIdx.x] = t;
        }
        if (threadIdx.x == 0) *done = 0u;
    }
}

// p = z + beta p; beta = rz_new / rz_old (fixed preconditioner) or (z, r - r_old) / rz_old
// (flexible CG, Polak-Ribiere form).
__global__ void k_cg_direction(int n, const double* S, bool flexible, const double* z, double* p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) {
        if (S[S_ACTIVE + c] == 0.0) continue;
        const double old = S[S_RZOLD + c];
        const double num = flexible ? S[S_ZROLD + c] : S[S_RZ + c];
        const double beta = old != 0.0 ? num / old : 0.0;
        const int64_t k = 3 * static_cast<int64_t>(i) + c;
        p[k] = z[k] + beta * p[k];
    }
}

// After an iteration: count it, and freeze the columns whose recurrence residual met the
// tolerance (||r_c||^2 <= tol^2 ||b_c||^2), recording the iteration at which they did.
// Also keeps rz as rz_old for the next direction update.
// rz_is_rr: no preconditioner (z = r), so the new rz is the (r, r) just computed.
__global__ void k_cg_check(double* S, double tol2, bool rz_is_rr)
{
    S[S_IT] += 1.0;
    for (int c = 0; c < 3; ++c) {
        if (S[S_ACTIVE + c] != 0.0 && S[S_RR + c] <= tol2 * S[S_BB + c]) {
            S[S_ACTIVE + c] = 0.0;
            S[S_CONV_IT + c] = S[S_IT];
        }
        S[S_RZOLD + c] = S[S_RZ + c];
        if (rz_is_rr) S[S_RZ + c] = S[S_RR + c];
    }
}

// y += w x over n x 3 values, w read from the device (the hybrid preconditioner's weight,
// fixed for a solve, so that captured iterations replay with it)
__global__ void k_add_weighted3(int n, const double* w, const double* x, double* y)
{
    const double a = *w;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < 3 * static_cast<int64_t>(n);
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] += a * x[i];
}

__global__ void k_axpby3(int n, double alpha, const double* x, double beta, double* y, int ldy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) {
        double& t = y[static_cast<int64_t>(ldy) * i + c];
        t = alpha * x[3 * static_cast<int64_t>(i) + c] + (beta == 0.0 ? 0.0 : beta * t);
    }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
Solver::~Solver() {}

static rpb_status ensure_solver(rpb_mesh* m)
{
    if (!m->solver) m->solver = new Solver();
    Solver& s = *m->solver;
    if (!s.vec.ptr) {
        const size_t n3 = 3 * static_cast<size_t>(m->nV);
        RPB_CUDA(s.vec.alloc(Solver::NVEC * n3));
        RPB_CUDA(s.scal.alloc(S_COUNT));
        RPB_CUDA(s.partials.alloc(6 * 1024));
        RPB_CUDA(s.done.alloc(1));
        RPB_CUDA(cudaMemsetAsync(s.done.ptr, 0, s.done.bytes(), m->stream));
        RPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s.host_scal), sizeof(double) * S_COUNT));
    }
    return RPB_OK;
}

void solver_free(rpb_mesh* m)
{
    if (m->solver) {
        if (m->solver->host_scal) cudaFreeHost(m->solver->host_scal);
        delete m->solver;
        m->solver = nullptr;
    }
}

// ------------------------------------------------------------------------------------------
// Numeric supernodal Cholesky of H1 on the device (host/supernodal_chol.hpp). The entries of
// H1 are scattered into the dense supernode panels (one thread per column); then, level by
// level of the supernodal elimination tree, two launches:
//   k_chol_update: the updates a supernode J receives from the supernodes K below it, cut
//     into regions of J's panel (blocks of CHOL_REGION_ROWS structure rows x CHOL_TILE
//     columns, one CTA each, regions entirely above the diagonal skipped); a CTA walks J's
//     update list in order and subtracts, for each K, the part of L_K L_K^T that lands in
//     its region (a 64 x 64-tiled product with the inner dimension staged in shared memory,
//     or a direct loop for small parts). Every panel entry belongs to one region, so the
//     sums are formed in a fixed order without atomics;
//   k_chol_panel: one CTA per supernode factors its updated panel, right-looking in blocks
//     of 16 columns (the host fallback runs the unblocked sn_factor_panel on one thread).
// The symbolic analysis stays on the host.
// ------------------------------------------------------------------------------------------
struct CtaBarrier {
    __host__ __device__ void operator()() const
    {
#if defined(__CUDA_ARCH__)
        __syncthreads();
#endif
    }
};

__global__ void k_chol_scatter(int n, const int64_t* __restrict__ Cp, const int* __restrict__ Ci,
                               const double* __restrict__ Cx, const int* __restrict__ sn_of, SnView v, unsigned* error)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int64_t p = Cp[j]; p < Cp[j + 1]; ++p)
        if (!sn_scatter_entry(v, sn_of, Ci[p], j, Cx[p])) atomicOr(error, 1u);
}

constexpr int CHOL_BLOCK = 256;
constexpr int CHOL_TILE = 64;          // rows x columns of an update tile (4 x 4 per thread)
constexpr int CHOL_KCHUNK = 16;        // inner-dimension chunk staged in shared memory
constexpr int CHOL_REGION_ROWS = 128;  // structure rows of a panel region
constexpr int64_t CHOL_DIRECT_PAIRS = 2048;   // smaller parts of an update take the direct loop
static_assert(CHOL_BLOCK == 256 && CHOL_TILE == 64, "the update tiles map 16 x 16 threads onto 64 x 64 entries");

// Part of the update of J by K: rows a in [alo, ahi) and columns b in [blo, bhi) of K's
// structure positions (a >= b), subtracted from J's panel. Tiled: 64 x 64 tiles, the inner
// dimension in chunks of 16 staged in shared memory, thread (ty, tx) accumulating rows
// ty + 16 i and columns tx + 16 j of a tile.
__device__ int chol_update_part(const SnView& v, int J, int K, int alo, int ahi, int blo, int bhi,
                                double (*As)[CHOL_TILE], double (*Bs)[CHOL_TILE])
{
    const int tid = threadIdx.x;
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
    const int na = ahi - alo, nb = bhi - blo;
    int status = 0;
    if (static_cast<int64_t>(na) * nb <= CHOL_DIRECT_PAIRS) {
        for (int idx = tid; idx < na * nb; idx += CHOL_BLOCK) {
            const int a = alo + idx / nb, b = blo + idx % nb;
            if (a < b) continue;
            double acc = 0.0;
            for (int t = 0; t < wK; ++t)
                acc += PK[static_cast<int64_t>(t) * nrK + a] * PK[static_cast<int64_t>(t) * nrK + b];
            const int row = sn_lower_bound(R, 0, nr, RK[a]);
            if (row >= nr || R[row] != RK[a]) {
                status = 1;
                continue;
            }
            P[static_cast<int64_t>(RK[b] - c0) * nr + row] -= acc;
        }
        return status;
    }
    const int tx = tid & 15, ty = tid >> 4;
    for (int ta = alo; ta < ahi; ta += CHOL_TILE)
        for (int tb = blo; tb < bhi && tb < ta + CHOL_TILE; tb += CHOL_TILE) {
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int t0 = 0; t0 < wK; t0 += CHOL_KCHUNK) {
                for (int e = tid; e < CHOL_KCHUNK * CHOL_TILE; e += CHOL_BLOCK) {
                    const int tt = e / CHOL_TILE, q = e - tt * CHOL_TILE, t = t0 + tt;
                    const int64_t base = static_cast<int64_t>(t) * nrK;
                    As[tt][q] = (t < wK && ta + q < ahi) ? PK[base + ta + q] : 0.0;
                    Bs[tt][q] = (t < wK && tb + q < bhi) ? PK[base + tb + q] : 0.0;
                }
                __syncthreads();
#pragma unroll 4
                for (int tt = 0; tt < CHOL_KCHUNK; ++tt) {
                    double x[4], y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) x[i] = As[tt][ty + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; ++j) y[j] = Bs[tt][tx + 16 * j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] += x[i] * y[j];
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int a = ta + ty + 16 * i;
                if (a >= ahi) continue;
                int row = -1;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int b = tb + tx + 16 * j;
                    if (b >= bhi || a < b) continue;
                    if (row < 0) {
                        row = sn_lower_bound(R, 0, nr, RK[a]);
                        if (row >= nr || R[row] != RK[a]) {
                            status = 1;
                            break;
                        }
                    }
                    P[static_cast<int64_t>(RK[b] - c0) * nr + row] -= acc[i][j];
                }
            }
        }
    return status;
}

// One CTA per region (J, first structure row, first column) of the level's supernodes.
__global__ void __launch_bounds__(CHOL_BLOCK) k_chol_update(SnView v, const int4* __restrict__ regions, unsigned* error)
{
    __shared__ double As[CHOL_KCHUNK][CHOL_TILE];
    __shared__ double Bs[CHOL_KCHUNK][CHOL_TILE];
    const int4 rg = regions[blockIdx.x];
    const int J = rg.x;
    const int c0 = v.sn_begin[J], w = v.sn_begin[J + 1] - c0;
    const int64_t r0 = v.rows_rp[J];
    const int nr = static_cast<int>(v.rows_rp[J + 1] - r0);
    const int* R = v.rows + r0;
    const int rlo = rg.y, rhi = min(rg.y + CHOL_REGION_ROWS, nr);
    const int clo = rg.z, chi = min(rg.z + CHOL_TILE, w);
    int status = 0;
    for (int u = v.upd_rp[J]; u < v.upd_rp[J + 1]; ++u) {
        const int K = v.upd_k[u];
        const int wK = v.sn_begin[K + 1] - v.sn_begin[K];
        const int64_t q0 = v.rows_rp[K];
        const int nrK = static_cast<int>(v.rows_rp[K + 1] - q0);
        const int* RK = v.rows + q0;
        // K's rows whose place in J is in [rlo, rhi), K's columns of J in [clo, chi)
        const int alo = sn_lower_bound(RK, wK, nrK, R[rlo]);
        const int ahi = sn_lower_bound(RK, alo, nrK, R[rhi - 1] + 1);
        const int blo = sn_lower_bound(RK, wK, nrK, c0 + clo);
        const int bhi = sn_lower_bound(RK, blo, nrK, c0 + chi);
        if (alo < ahi && blo < bhi) status |= chol_update_part(v, J, K, alo, ahi, blo, bhi, As, Bs);
        __syncthreads();
    }
    if (status != 0) atomicOr(error, static_cast<unsigned>(status));
}

// Blocked panel factorization (right-looking, blocks of CHOL_KCHUNK columns): the columns of
// a block are factored one by one as in sn_factor_panel, but their updates reach only the
// block's own columns; the rest of the panel then takes the block's rank-16 update at once as
// a 64 x 64-tiled product (tiles above the diagonal skipped), so the trailing part is read and
// written once per block instead of once per column. Returns 0, or 2 for a non-positive pivot
// (every thread returns it together).
__device__ int chol_panel_blocked(const SnView& v, int J, double (*As)[CHOL_TILE], double (*Bs)[CHOL_TILE])
{
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int c0 = v.sn_begin[J], w = v.sn_begin[J + 1] - c0;
    const int64_t r0 = v.rows_rp[J];
    const int nr = static_cast<int>(v.rows_rp[J + 1] - r0);
    double* P = v.panels + v.panel_off[J];
    for (int cb = 0; cb < w; cb += CHOL_KCHUNK) {
        const int ce = min(cb + CHOL_KCHUNK, w);
        for (int c = cb; c < ce; ++c) {
            double* Pc = P + static_cast<int64_t>(c) * nr;
            if (tid == 0) {
                const double d = Pc[c];
                Pc[c] = d > 0.0 ? sqrt(d) : -1.0;
            }
            __syncthreads();
            const double d = Pc[c];
            if (!(d > 0.0)) return 2;
            const double inv = 1.0 / d;
            for (int r = c + 1 + tid; r < nr; r += CHOL_BLOCK) Pc[r] *= inv;
            __syncthreads();
            for (int r = c + 1 + tid; r < nr; r += CHOL_BLOCK) {
                const double lrc = Pc[r];
                const int cmax = min(r, ce - 1);
                for (int cc = c + 1; cc <= cmax; ++cc) P[static_cast<int64_t>(cc) * nr + r] -= lrc * Pc[cc];
            }
            __syncthreads();
        }
        // trailing update: columns cc >= ce, rows r >= cc, minus sum over the block's columns
        for (int ta = ce; ta < nr; ta += CHOL_TILE)
            for (int tb = ce; tb < w && tb < ta + CHOL_TILE; tb += CHOL_TILE) {
                for (int e = tid; e < CHOL_KCHUNK * CHOL_TILE; e += CHOL_BLOCK) {
                    const int k = e / CHOL_TILE, q = e - k * CHOL_TILE;
                    const bool in = cb + k < ce;
                    const int64_t base = static_cast<int64_t>(cb + k) * nr;
                    As[k][q] = (in && ta + q < nr) ? P[base + ta + q] : 0.0;
                    Bs[k][q] = (in && tb + q < w) ? P[base + tb + q] : 0.0;
                }
                __syncthreads();
                double acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 4
                for (int k = 0; k < CHOL_KCHUNK; ++k) {
                    double x[4], y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) x[i] = As[k][ty + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; ++j) y[j] = Bs[k][tx + 16 * j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] += x[i] * y[j];
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = ta + ty + 16 * i;
                    if (r >= nr) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int cc = tb + tx + 16 * j;
                        if (cc < w && r >= cc) P[static_cast<int64_t>(cc) * nr + r] -= acc[i][j];
                    }
                }
                __syncthreads();
            }
    }
    return 0;
}

__global__ void __launch_bounds__(CHOL_BLOCK) k_chol_panel(SnView v, const int* __restrict__ sns, unsigned* error)
{
    __shared__ double As[CHOL_KCHUNK][CHOL_TILE];
    __shared__ double Bs[CHOL_KCHUNK][CHOL_TILE];
    const int st = chol_panel_blocked(v, sns[blockIdx.x], As, Bs);
    if (st != 0 && threadIdx.x == 0) atomicOr(error, static_cast<unsigned>(st));
}

// The factor of A (ordering perm) with the numeric phase on the device; "" or the reason it
// failed (the caller then factors on the host).
static std::string cholesky_factor_device(const CsrMatrix& A, const std::vector<int>& perm, CholeskyFactor& F,
                                          cudaStream_t s)
{
    SupernodalSymbolic S;
    std::string err = supernodal_symbolic(A, perm, kSupernodalWidth, S);
    if (!err.empty()) return err;
    // update regions of every level: (J, first row, first column), below the diagonal
    const int L = static_cast<int>(S.level_ptr.size()) - 1;
    std::vector<int4> regions;
    std::vector<int> region_ptr(static_cast<size_t>(L) + 1, 0);
    for (int l = 0; l < L; ++l) {
        for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
            const int J = S.level_sn[q];
            if (S.upd_rp[J + 1] == S.upd_rp[J]) continue;
            const int w = S.sn_begin[J + 1] - S.sn_begin[J];
            const int nr = static_cast<int>(S.rows_rp[J + 1] - S.rows_rp[J]);
            for (int rlo = 0; rlo < nr; rlo += CHOL_REGION_ROWS)
                for (int clo = 0; clo < w; clo += CHOL_TILE)
                    if (std::min(rlo + CHOL_REGION_ROWS, nr) > clo) regions.push_back(make_int4(J, rlo, clo, 0));
        }
        region_ptr[l + 1] = static_cast<int>(regions.size());
    }
    DevBuf<int> sn_begin, rows, upd_rp, upd_k, sn_of, Ci, level_sn;
    DevBuf<int64_t> rows_rp, panel_off, Cp;
    DevBuf<double> Cx, panels;
    DevBuf<int4> d_regions;
    DevBuf<unsigned> error;
    cudaError_t e = cudaSuccess;
    auto up = [&](auto& dst, const auto& src) {
        if (e != cudaSuccess) return;
        if ((e = dst.alloc(src.size())) != cudaSuccess) return;
        if (!src.empty()) e = cudaMemcpyAsync(dst.ptr, src.data(), dst.bytes(), cudaMemcpyHostToDevice, s);
    };
    up(sn_begin, S.sn_begin); up(rows, S.rows); up(upd_rp, S.upd_rp); up(upd_k, S.upd_k); up(sn_of, S.sn_of);
    up(Ci, S.Ci); up(level_sn, S.level_sn); up(rows_rp, S.rows_rp); up(panel_off, S.panel_off); up(Cp, S.Cp);
    up(Cx, S.Cx); up(d_regions, regions);
    const size_t np = static_cast<size_t>(S.panel_off[S.nsn]);
    if (e == cudaSuccess) e = panels.alloc(np);
    if (e == cudaSuccess) e = cudaMemsetAsync(panels.ptr, 0, panels.bytes(), s);
    if (e == cudaSuccess) e = error.alloc(1);
    if (e == cudaSuccess) e = cudaMemsetAsync(error.ptr, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return std::string("device Cholesky: ") + cudaGetErrorString(e);
    SnView v{sn_begin.ptr, rows_rp.ptr, rows.ptr, panel_off.ptr, upd_rp.ptr, upd_k.ptr, panels.ptr};
    k_chol_scatter<<<(S.n + 255) / 256, 256, 0, s>>>(S.n, Cp.ptr, Ci.ptr, Cx.ptr, sn_of.ptr, v, error.ptr);
    for (int l = 0; l < L; ++l) {
        const int nreg = region_ptr[l + 1] - region_ptr[l];
        if (nreg > 0) k_chol_update<<<nreg, CHOL_BLOCK, 0, s>>>(v, d_regions.ptr + region_ptr[l], error.ptr);
        const int count = S.level_ptr[l + 1] - S.level_ptr[l];
        if (count > 0) k_chol_panel<<<count, CHOL_BLOCK, 0, s>>>(v, level_sn.ptr + S.level_ptr[l], error.ptr);
    }
    std::vector<double> hp(np);
    unsigned herr = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(hp.data(), panels.ptr, panels.bytes(), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&herr, error.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return std::string("device Cholesky: ") + cudaGetErrorString(e);
    if (herr & 2u) return "H1 metric is not positive definite";
    if (herr) return "device Cholesky: an entry outside the supernodal structure";
    supernodal_to_factor(S, hp, F);
    return std::string();
}

// H1 factor for the current geometry (the reference caches H1Metric/H1Solver on the mesh
// and clears them with the cache on SemiStaticUpdate, src/SimplicialMesh.hpp:368).
static rpb_status ensure_h1(rpb_mesh* m)
{
    Solver& s = *m->solver;
    if (s.h1_version == m->geometry_version) return RPB_OK;
    std::vector<double> V(3 * static_cast<size_t>(m->nV));
    std::vector<int> S(static_cast<size_t>(m->size) * m->N);
    RPB_CUDA(cudaMemcpyAsync(V.data(), m->V.ptr, m->V.bytes(), cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaMemcpyAsync(S.data(), m->S.ptr, m->S.bytes(), cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    const auto t0 = std::chrono::steady_clock::now();
    const CsrMatrix H = assemble_h1(m->dom, V.data(), m->nV, S.data(), m->N, 1.0, 1.0);
    if (s.nd_perm.empty()) s.nd_perm = nested_dissection_ordering(m->tree, S.data(), m->nV);
    CholeskyFactor F;
    // numeric factorization on the device; on host threads if that fails
    s.factor_on_device = cholesky_factor_device(H, s.nd_perm, F, m->stream).empty();
    if (!s.factor_on_device) {
        cudaGetLastError();
        const std::string err = cholesky_factor(H, s.nd_perm, F);
        if (!err.empty()) { set_error(err); return RPB_EINVAL; }
    }
    s.factor_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s.factor_nnz = F.nnz();
    SupernodalSchedule SS;
    const std::string serr = supernodal_schedule(F, kMaxSupernodeWidth, SS);
    if (!serr.empty()) { set_error(serr); return RPB_EINVAL; }
    s.sn_levels_fwd = SS.fwd_levels();
    cudaStream_t st = m->stream;
    auto up = [st](auto& dst, const auto& src) -> cudaError_t {
        cudaError_t e = dst.alloc(src.size());
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(dst.ptr, src.data(), dst.bytes(), cudaMemcpyHostToDevice, st);
    };
    const int n = m->nV;
    std::vector<int> sn_of(n);
    for (int sn = 0; sn < SS.nsn; ++sn)
        for (int c = SS.sn_begin[sn]; c < SS.sn_begin[sn + 1]; ++c) sn_of[c] = sn;
    auto pow2ceil = [](int64_t v) {
        int p = 1;
        while (p < v) p <<= 1;
        return p;
    };
    for (int d = 0; d < 2; ++d) {
        const bool lower = d == 0;
        const std::vector<int64_t>& rp = lower ? F.lower_rp : F.upper_rp;
        const std::vector<int>& ci = lower ? F.lower_ci : F.upper_ci;
        const std::vector<double>& val = lower ? F.lower_val : F.upper_val;
        // each row's entries outside its own supernode
        std::vector<int64_t> xrp(static_cast<size_t>(n) + 1, 0);
        std::vector<int> xci;
        std::vector<double> xval;
        {
            // counted, then filled, by host threads over row ranges
            const int nt = static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
            auto outside = [&](int r, int j) {
                return lower ? (j < SS.sn_begin[sn_of[r]]) : (j >= SS.sn_begin[sn_of[r] + 1]);
            };
            auto pool = [&](auto&& body) {
                std::vector<std::thread> th;
                for (int t = 0; t < nt; ++t)
                    th.emplace_back([&, t] { body(static_cast<int>(static_cast<int64_t>(n) * t / nt),
                                                  static_cast<int>(static_cast<int64_t>(n) * (t + 1) / nt)); });
                for (auto& x : th) x.join();
            };
            pool([&](int r0, int r1) {
                for (int r = r0; r < r1; ++r) {
                    int64_t c = 0;
                    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) c += outside(r, ci[k]) ? 1 : 0;
                    xrp[r + 1] = c;
                }
            });
            for (int r = 0; r < n; ++r) xrp[r + 1] += xrp[r];
            xci.resize(static_cast<size_t>(xrp[n]));
            xval.resize(static_cast<size_t>(xrp[n]));
            pool([&](int r0, int r1) {
                for (int r = r0; r < r1; ++r) {
                    int64_t o = xrp[r];
                    for (int64_t k = rp[r]; k < rp[r + 1]; ++k)
                        if (outside(r, ci[k])) {
                            xci[o] = ci[k];
                            xval[o++] = val[k];
                        }
                }
            });
        }
        // level plans
        const std::vector<int>& lptr = lower ? SS.fwd_level_ptr : SS.bwd_level_ptr;
        const std::vector<int>& lsn = lower ? SS.fwd_level_sn : SS.bwd_level_sn;
        Solver::Direction& D = s.dir[d];
        D.levels.clear();
        std::vector<int> sn_list, row_list;
        for (size_t l = 0; l + 1 < lptr.size(); ++l) {
            bool warp = true;
            int maxw = 0;
            int64_t maxext = 0;
            for (int q = lptr[l]; q < lptr[l + 1]; ++q) {
                const int sn = lsn[q], c0 = SS.sn_begin[sn], w = SS.sn_begin[sn + 1] - c0;
                maxw = std::max(maxw, w);
                const int g = w <= 32 ? 32 / pow2ceil(w) : 1;
                for (int r = c0; r < c0 + w; ++r) {
                    const int64_t len = xrp[r + 1] - xrp[r];
                    maxext = std::max(maxext, len);
                    if (w > 32 || (len + g - 1) / g > kWarpExtIters) warp = false;
                }
            }
            Solver::Level L;
            L.warp = warp;
            if (warp) {
                L.first = static_cast<int>(sn_list.size());
                for (int q = lptr[l]; q < lptr[l + 1]; ++q) sn_list.push_back(lsn[q]);
                L.count = static_cast<int>(sn_list.size()) - L.first;
            } else {
                L.first = static_cast<int>(row_list.size());
                for (int q = lptr[l]; q < lptr[l + 1]; ++q)
                    for (int c = SS.sn_begin[lsn[q]]; c < SS.sn_begin[lsn[q] + 1]; ++c) row_list.push_back(c);
                L.count = static_cast<int>(row_list.size()) - L.first;
                L.g_ext = std::min(SN_BLOCK, std::max(4, pow2ceil((maxext + 3) / 4)));
                L.g_dense = std::min(SN_BLOCK, std::max(4, pow2ceil((maxw + 3) / 4)));
            }
            D.levels.push_back(L);
        }
        RPB_CUDA(up(D.ext_rp, xrp));
        RPB_CUDA(up(D.ext_ci, xci));
        RPB_CUDA(up(D.ext_val, xval));
        RPB_CUDA(up(D.sn_list, sn_list));
        RPB_CUDA(up(D.row_list, row_list));
        RPB_CUDA(up(D.dinv, lower ? SS.dinv : SS.dinvT));
        // the copies read pageable host vectors that go out of scope
        RPB_CUDA(cudaStreamSynchronize(st));
    }
    RPB_CUDA(up(s.perm, F.perm));
    RPB_CUDA(up(s.sn_begin, SS.sn_begin));
    RPB_CUDA(up(s.dinv_off, SS.dinv_off));
    RPB_CUDA(up(s.sn_of, sn_of));
    RPB_CUDA(s.tri.alloc(3 * static_cast<size_t>(n)));
    RPB_CUDA(s.tmp.alloc(3 * static_cast<size_t>(n)));
    RPB_CUDA(s.tbuf.alloc(3 * static_cast<size_t>(n)));
    RPB_CUDA(cudaStreamSynchronize(st));
    s.h1_version = m->geometry_version;
    return RPB_OK;
}

// out = H1^{-1} b (b, out: n x 3 contiguous, device): forward levels on L, backward
// levels on L^T, one or two launches per level
static rpb_status h1_solve(rpb_mesh* m, const double* b, double* out)
{
    Solver& s = *m->solver;
    cudaStream_t st = m->stream;
    for (int d = 0; d < 2; ++d) {
        const bool lower = d == 0;
        const Solver::Direction& D = s.dir[d];
        SnTri A;
        A.sn_begin = s.sn_begin.ptr; A.sn_of = s.sn_of.ptr; A.dinv_off = s.dinv_off.ptr;
        A.ext_rp = D.ext_rp.ptr; A.ext_ci = D.ext_ci.ptr; A.ext_val = D.ext_val.ptr; A.dinv = D.dinv.ptr;
        A.t = s.tbuf.ptr;
        if (lower) {
            A.b = b; A.perm_in = s.perm.ptr; A.y = s.tri.ptr; A.out = nullptr; A.perm_out = nullptr;
        } else {
            A.b = s.tri.ptr; A.perm_in = nullptr; A.y = s.tmp.ptr; A.out = out; A.perm_out = s.perm.ptr;
        }
        for (const Solver::Level& L : D.levels) {
            if (L.warp) {
                const int grid = (L.count + SN_BLOCK / 32 - 1) / (SN_BLOCK / 32);
                const int* list = D.sn_list.ptr + L.first;
                RPB_CUDA(launch_pdl(lower ? k_sn_warp<true> : k_sn_warp<false>, grid, SN_BLOCK, 0, st, A, list, L.count));
            } else {
                const int* rows = D.row_list.ptr + L.first;
                const int ge = static_cast<int>((static_cast<int64_t>(L.count) * L.g_ext + SN_BLOCK - 1) / SN_BLOCK);
                const int gd = static_cast<int>((static_cast<int64_t>(L.count) * L.g_dense + SN_BLOCK - 1) / SN_BLOCK);
                RPB_CUDA(launch_pdl(lower ? k_sn_split_ext<true> : k_sn_split_ext<false>, ge, SN_BLOCK, 0, st, A, rows,
                                    L.count, L.g_ext));
                RPB_CUDA(launch_pdl(lower ? k_sn_split_dense<true> : k_sn_split_dense<false>, gd, SN_BLOCK, 0, st, A,
                                    rows, L.count, L.g_dense));
            }
        }
        RPB_CUDA(cudaGetLastError());
    }
    return RPB_OK;
}

// Y = H1^{-1} L_{2-s} H1^{-1} X   (X, Y: n x 3 contiguous device; Y may alias X)
rpb_status reference_precondition(rpb_mesh* m, double q, double p, const double* X, double* Y)
{
    rpb_status st;
    if ((st = ensure_solver(m)) != RPB_OK) return st;
    if ((st = ensure_h1(m)) != RPB_OK) return st;
    Solver& s = *m->solver;
    const double s_tp = (p - m->dom) / q;
    double* Z = s.vec.ptr + Solver::V_PRE * 3 * static_cast<size_t>(m->nV);
    if ((st = h1_solve(m, X, Z)) != RPB_OK) return st;
    if ((st = plap_multiply_dev(m, 2.0 - s_tp, 1.0, Z, 3, 0.0, Z, 3)) != RPB_OK) return st;
    return h1_solve(m, Z, Y);
}

static rpb_status read_scalars(rpb_mesh* m)
{
    Solver& s = *m->solver;
    RPB_CUDA(cudaMemcpyAsync(s.host_scal, s.scal.ptr, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    return RPB_OK;
}

static rpb_status dot3(rpb_mesh* m, const double* a, const double* b, const double* c, double* out0, double* out1)
{
    Solver& s = *m->solver;
    DotArgs A;
    A.n = m->nV; A.a = a; A.b = b; A.c = c;
    A.partials = s.partials.ptr; A.done = s.done.ptr; A.out0 = out0; A.out1 = out1;
    const int blocks = std::min(1024, (m->nV + 255) / 256);
    k_dot3<<<blocks, 256, 0, m->stream>>>(A);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status apply_preconditioner(rpb_mesh* m, int kind, double q, double p, const double* R, double* Z);  // below

// Solves A Z = B (device, n x 3) by (flexible) PCG. Returns iterations and true residuals.
static rpb_status cg_solve(rpb_mesh* m, double q, double p, const double* B, int max_iter, double tol, int precond,
                           int* iters_out, double* relres_out)
{
    rpb_status st;
    if ((st = ensure_solver(m)) != RPB_OK) return st;
    Solver& s = *m->solver;
    const int n = m->nV;
    const size_t n3 = 3 * static_cast<size_t>(n);
    double* x = s.vec.ptr + Solver::V_X * n3;
    double* r = s.vec.ptr + Solver::V_R * n3;
    double* z = s.vec.ptr + Solver::V_Z * n3;
    double* pv = s.vec.ptr + Solver::V_P * n3;
    double* Ap = s.vec.ptr + Solver::V_AP * n3;
    double* rold = s.vec.ptr + Solver::V_ROLD * n3;
    double* S = s.scal.ptr;
    cudaStream_t stream = m->stream;
    const int eb = (n + 255) / 256;
    const bool flexible = (precond == RPB_PRECOND_LEARNED || precond == RPB_PRECOND_HYBRID);
    // iterations without a 10% drop of the best residual that count as a stall
    constexpr int kStallWindow = 500;
    // iterations per captured graph between host checks of the residuals
    constexpr int kGraphIters = 8;
    int kind = precond;

    // ||B|| per column
    RPB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n3, stream));
    if ((st = dot3(m, B, B, nullptr, S + S_RR, nullptr)) != RPB_OK) return st;
    if ((st = read_scalars(m)) != RPB_OK) return st;
    double bnorm[3], bb[3];
    for (int c = 0; c < 3; ++c) {
        bb[c] = s.host_scal[S_RR + c];
        bnorm[c] = std::sqrt(bb[c]);
    }
    RPB_CUDA(cudaMemcpyAsync(S + S_BB, bb, sizeof(bb), cudaMemcpyHostToDevice, stream));
    double active[3];
    for (int c = 0; c < 3; ++c) active[c] = bnorm[c] > 0 ? 1.0 : 0.0;
    int it = 0;
    double rel[3] = {0, 0, 0};
    int restarts = 0;
    s.last_fallback_iteration = -1;
    double best[3] = {1e300, 1e300, 1e300};
    int since_best = 0;
    bool stalled_flag = false;
    const double tol2 = tol * tol;
    // One CG iteration from a search direction p: A p, step, residual, convergence flags,
    // then the next preconditioned direction. Only launches and device-to-device copies,
    // so K of them are captured into one CUDA graph and replayed between host checks.
    auto iteration = [&](int k) -> rpb_status {
        rpb_status e;
        if ((e = metric_multiply_dev(m, q, p, 1.0, pv, 3, 0.0, Ap, 3, 7)) != RPB_OK) return e;
        if ((e = dot3(m, pv, Ap, nullptr, S + S_PAP, nullptr)) != RPB_OK) return e;
        k_cg_update_rr<<<std::min(1024, eb), 256, 0, stream>>>(n, S, x, r, pv, Ap, flexible ? rold : nullptr,
                                                               s.partials.ptr, s.done.ptr);
        const bool plain = k == RPB_PRECOND_NONE && !flexible;
        k_cg_check<<<1, 1, 0, stream>>>(S, tol2, plain);
        if (!plain) {
            if ((e = apply_preconditioner(m, k, q, p, r, z)) != RPB_OK) return e;
            if ((e = dot3(m, z, r, flexible ? rold : nullptr, S + S_RZ, S + S_ZROLD)) != RPB_OK) return e;
        }
        k_cg_direction<<<eb, 256, 0, stream>>>(n, S, flexible, plain ? r : z, pv);
        RPB_CUDA(cudaGetLastError());
        return RPB_OK;
    };
    cudaGraphExec_t graph = nullptr;
    int graph_kind = -1;
    auto drop_graph = [&]() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    };
    while (true) {
        // r = B - A x (true residual), z = M r, p = z
        if ((st = metric_multiply_dev(m, q, p, -1.0, x, 3, 0.0, r, 3, 7)) != RPB_OK) { drop_graph(); return st; }
        k_axpby3<<<eb, 256, 0, stream>>>(n, 1.0, B, 1.0, r, 3);
        RPB_CUDA(cudaGetLastError());
        if ((st = dot3(m, r, r, nullptr, S + S_RR, nullptr)) != RPB_OK) { drop_graph(); return st; }
        if ((st = read_scalars(m)) != RPB_OK) { drop_graph(); return st; }
        bool done = true;
        for (int c = 0; c < 3; ++c) {
            rel[c] = bnorm[c] > 0 ? std::sqrt(s.host_scal[S_RR + c]) / bnorm[c] : 0.0;
            active[c] = rel[c] > tol ? 1.0 : 0.0;
            if (active[c] != 0.0) done = false;
        }
        if (done || it >= max_iter) break;
        if (stalled_flag && (kind == RPB_PRECOND_LEARNED || kind == RPB_PRECOND_HYBRID)) {
            kind = RPB_PRECOND_REFERENCE;  // fallback on stall
            s.last_fallback_iteration = it;
        }
        if (kind == RPB_PRECOND_HYBRID && restarts == 0) {
            // the weight of the learned operator: an eighth of the ratio of the two parts'
            // energies on the first residual, (r, P_ref r) / (r, M r) / 8 over the three columns
            // (linked tori of 96 x 128 / 192 x 256 vertices: 825 / 849 iterations against 870 /
            // 1,280 with a half and 813 / 887 with a quarter / a sixteenth of the ratio)
            double* zr = s.vec.ptr + Solver::V_HYB * n3;
            if ((st = reference_precondition(m, q, p, r, z)) != RPB_OK) { drop_graph(); return st; }
            if ((st = learned_precondition(m, q, p, r, zr)) != RPB_OK) { drop_graph(); return st; }
            if ((st = dot3(m, r, z, nullptr, S + S_RZ, nullptr)) != RPB_OK) { drop_graph(); return st; }
            if ((st = dot3(m, r, zr, nullptr, S + S_PAP, nullptr)) != RPB_OK) { drop_graph(); return st; }
            if ((st = read_scalars(m)) != RPB_OK) { drop_graph(); return st; }
            double er = 0.0, el = 0.0;
            for (int c = 0; c < 3; ++c) {
                er += s.host_scal[S_RZ + c];
                el += s.host_scal[S_PAP + c];
            }
            const double w = (el > 0.0 && er > 0.0) ? 0.125 * er / el : 0.0;
            RPB_CUDA(cudaMemcpyAsync(S + S_HYB_W, &w, sizeof(double), cudaMemcpyHostToDevice, stream));
            RPB_CUDA(cudaStreamSynchronize(stream));
        }
        stalled_flag = false;
        ++restarts;
        double it_conv[4] = {-1.0, -1.0, -1.0, static_cast<double>(it)};
        RPB_CUDA(cudaMemcpyAsync(S + S_ACTIVE, active, sizeof(active), cudaMemcpyHostToDevice, stream));
        RPB_CUDA(cudaMemcpyAsync(S + S_CONV_IT, it_conv, sizeof(it_conv), cudaMemcpyHostToDevice, stream));
        if ((st = apply_preconditioner(m, kind, q, p, r, z)) != RPB_OK) { drop_graph(); return st; }
        RPB_CUDA(cudaMemcpyAsync(pv, z, sizeof(double) * n3, cudaMemcpyDeviceToDevice, stream));
        if ((st = dot3(m, r, z, nullptr, S + S_RZ, nullptr)) != RPB_OK) { drop_graph(); return st; }
        // batches of kGraphIters iterations as one graph; the remainder launched directly
        // (and everything when the mesh works on the legacy default stream, which cannot
        // be captured)
        const bool use_graph = stream != nullptr;
        if (use_graph && graph_kind != kind) {
            drop_graph();
            cudaGraph_t g = nullptr;
            RPB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            rpb_status cst = RPB_OK;
            for (int k = 0; k < kGraphIters && cst == RPB_OK; ++k) cst = iteration(kind);
            const cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (cst != RPB_OK) { if (g) cudaGraphDestroy(g); return cst; }
            RPB_CUDA(ce);
            const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            RPB_CUDA(ie);
            graph_kind = kind;
        }
        while (it < max_iter) {
            int batch = std::min(kGraphIters, max_iter - it);
            if (use_graph && batch == kGraphIters) {
                RPB_CUDA(cudaGraphLaunch(graph, stream));
            } else {
                for (int k = 0; k < batch; ++k)
                    if ((st = iteration(kind)) != RPB_OK) { drop_graph(); return st; }
            }
            if ((st = read_scalars(m)) != RPB_OK) { drop_graph(); return st; }
            const int done_it = static_cast<int>(s.host_scal[S_IT]);
            bool conv = true, stalled = false;
            int last_conv = 0;
            for (int c = 0; c < 3; ++c) {
                if (active[c] == 0.0) continue;
                const double ci = s.host_scal[S_CONV_IT + c];
                if (ci < 0.0) conv = false;
                else last_conv = std::max(last_conv, static_cast<int>(ci));
                const double rc = bnorm[c] > 0 ? std::sqrt(s.host_scal[S_RR + c]) / bnorm[c] : 0.0;
                if (ci < 0.0 && rc < 0.9 * best[c]) { best[c] = rc; since_best = 0; }
            }
            it = conv ? last_conv : done_it;
            // stall detection only guards the flexible (learned) iteration, which then falls
            // back to the reference preconditioner; fixed-preconditioner CG is never restarted
            since_best += batch;
            if (flexible && (kind == RPB_PRECOND_LEARNED || kind == RPB_PRECOND_HYBRID) && !conv &&
                since_best > kStallWindow)
                stalled = true;
            if (conv || stalled) {
                stalled_flag = stalled;
                since_best = 0;
                break;
            }
        }
        if (restarts > 20) break;
    }
    drop_graph();
    s.last_iterations = it;
    s.last_restarts = restarts;
    if (iters_out) *iters_out = it;
    if (relres_out)
        for (int c = 0; c < 3; ++c) relres_out[c] = rel[c];
    bool ok = true;
    for (int c = 0; c < 3; ++c) ok = ok && !(rel[c] > tol);
    if (!ok) {
        set_error("Solve did not reach the tolerance within max_iter iterations");
        return RPB_ENOTCONV;
    }
    return RPB_OK;
}

rpb_status apply_preconditioner(rpb_mesh* m, int kind, double q, double p, const double* R, double* Z)
{
    if (kind == RPB_PRECOND_NONE) {
        RPB_CUDA(cudaMemcpyAsync(Z, R, sizeof(double) * 3 * static_cast<size_t>(m->nV), cudaMemcpyDeviceToDevice,
                                 m->stream));
        return RPB_OK;
    }
    if (kind == RPB_PRECOND_LEARNED) return learned_precondition(m, q, p, R, Z);
    if (kind == RPB_PRECOND_HYBRID) {
        // Z = P_ref R + w M(R), w fixed at the solve's start (S_HYB_W)
        Solver& s = *m->solver;
        const int n = m->nV;
        double* T = s.vec.ptr + Solver::V_HYB * 3 * static_cast<size_t>(n);
        rpb_status st;
        if ((st = reference_precondition(m, q, p, R, Z)) != RPB_OK) return st;
        if ((st = learned_precondition(m, q, p, R, T)) != RPB_OK) return st;
        k_add_weighted3<<<std::min(1184, (3 * n + 255) / 256), 256, 0, m->stream>>>(n, s.scal.ptr + S_HYB_W, T, Z);
        RPB_CUDA(cudaGetLastError());
        return RPB_OK;
    }
    return reference_precondition(m, q, p, R, Z);
}

}  // namespace rpb

using namespace rpb;

extern "C" {

rpb_status rpb_tpm0_precondition(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX, double beta,
                                 double* Y, int ldY, int nrhs)
{
    if (!m || !X || !Y) { set_error("null argument"); return RPB_EINVAL; }
    if (nrhs != 3) {
        set_error("MultiplyPreconditioner: nrhs = " + std::to_string(nrhs) + " != 3 = AMB_DIM.");
        return RPB_EINVAL;
    }
    if (ldX < 3 || ldY < 3) { set_error("leading dimensions must be >= 3"); return RPB_EINVAL; }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    if ((st = ensure_solver(m)) != RPB_OK) return st;
    cudaStream_t s = m->stream;
    const int n = m->nV;
    RPB_CUDA(copy_rows3(m->X.ptr, 3, X, ldX, n, cudaMemcpyHostToDevice, s));
    if (beta != 0.0)
        RPB_CUDA(copy_rows3(m->Yb.ptr, 3, Y, ldY, n, cudaMemcpyHostToDevice, s));
    double* Z = m->solver->vec.ptr + Solver::V_Z * 3 * static_cast<size_t>(n);
    if ((st = reference_precondition(m, q, p, m->X.ptr, Z)) != RPB_OK) return st;
    k_axpby3<<<(n + 255) / 256, 256, 0, s>>>(n, alpha, Z, beta, m->Yb.ptr, 3);
    RPB_CUDA(cudaGetLastError());
    RPB_CUDA(copy_rows3(Y, ldY, m->Yb.ptr, 3, n, cudaMemcpyDeviceToHost, s));
    RPB_CUDA(cudaStreamSynchronize(s));
    return RPB_OK;
}

rpb_status rpb_tpm0_solve(rpb_mesh* m, double q, double p, double alpha, const double* B, int ldB, double beta,
                          double* X, int ldX, int nrhs, int max_iter, double tol, int precond, int* iterations,
                          double* rel_residual)
{
    if (!m || !B || !X) { set_error("null argument"); return RPB_EINVAL; }
    if (nrhs != 3) {
        set_error("Solve: nrhs = " + std::to_string(nrhs) + " != 3 = AMB_DIM.");
        return RPB_EINVAL;
    }
    if (ldB < 3 || ldX < 3) { set_error("leading dimensions must be >= 3"); return RPB_EINVAL; }
    if (precond < RPB_PRECOND_NONE || precond > RPB_PRECOND_HYBRID) { set_error("unknown preconditioner kind"); return RPB_EINVAL; }
    if (!(tol > 0) || max_iter < 0) { set_error("tolerance must be positive and max_iter >= 0"); return RPB_EINVAL; }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    if ((st = ensure_solver(m)) != RPB_OK) return st;
    cudaStream_t s = m->stream;
    const int n = m->nV;
    double* Bd = m->solver->vec.ptr + Solver::V_B * 3 * static_cast<size_t>(n);
    RPB_CUDA(copy_rows3(Bd, 3, B, ldB, n, cudaMemcpyHostToDevice, s));
    int it = 0;
    double rr[3] = {0, 0, 0};
    rpb_status cs = cg_solve(m, q, p, Bd, max_iter, tol, precond, &it, rr);
    if (cs != RPB_OK && cs != RPB_ENOTCONV) return cs;
    if (iterations) *iterations = it;
    if (rel_residual)
        for (int c = 0; c < 3; ++c) rel_residual[c] = rr[c];
    if (beta != 0.0)
        RPB_CUDA(copy_rows3(m->Yb.ptr, 3, X, ldX, n, cudaMemcpyHostToDevice, s));
    const double* xs = m->solver->vec.ptr + Solver::V_X * 3 * static_cast<size_t>(n);
    k_axpby3<<<(n + 255) / 256, 256, 0, s>>>(n, alpha, xs, beta, m->Yb.ptr, 3);
    RPB_CUDA(cudaGetLastError());
    RPB_CUDA(copy_rows3(X, ldX, m->Yb.ptr, 3, n, cudaMemcpyDeviceToHost, s));
    RPB_CUDA(cudaStreamSynchronize(s));
    return cs;
}

rpb_status rpb_tpm0_solve_info(const rpb_mesh* m, rpb_solve_info* info)
{
    if (!m || !info) { set_error("null argument"); return RPB_EINVAL; }
    info->iterations = m->solver ? m->solver->last_iterations : 0;
    info->restarts = m->solver ? m->solver->last_restarts : 0;
    info->fallback_iteration = m->solver ? m->solver->last_fallback_iteration : -1;
    info->factor_seconds = m->solver ? m->solver->factor_seconds : 0.0;
    info->factor_nnz = m->solver ? m->solver->factor_nnz : 0;
    info->supernode_levels = m->solver ? m->solver->sn_levels_fwd : 0;
    info->factor_on_device = (m->solver && m->solver->factor_on_device) ? 1 : 0;
    return RPB_OK;
}

}  // extern "C"
