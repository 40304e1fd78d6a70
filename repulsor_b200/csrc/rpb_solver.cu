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
#include <vector>

#include "host/sparse_cholesky.hpp"
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
// Level-scheduled supernodal triangular solves with 3 right-hand sides. One launch per
// level of the supernode schedule (host/sparse_cholesky.cpp), one CTA per supernode:
//   phase 1 (warp per row):  t_r = b_r - sum over the row's entries outside the supernode
//                            (all written by earlier levels, i.e. earlier launches),
//   phase 2 (warp per row):  y = D^{-1} t with the inverse of the dense diagonal block.
// Forward: rows of L, external columns < c0, D^{-1} packed lower. Backward: rows of L^T,
// external columns >= c1, D^{-T} packed upper. No inter-CTA waits of any kind.
// ------------------------------------------------------------------------------------------
struct SnArgs {
    const int* level_sn;      // supernodes of this level
    const int* sn_begin;
    const int64_t* rp;
    const int* ci;
    const double* val;
    const int64_t* dinv_off;
    const double* dinv;
    const double* b;          // right-hand side, n x 3
    const int* perm_in;       // if set, row i reads b[perm_in[i]]
    double* y;                // solution in factor order, n x 3
    double* out;              // if set, out[perm_out[i]] = y_i
    const int* perm_out;
};

constexpr int SN_BLOCK = 256;
// widest supernode (3 x 8 bytes of shared memory per row: 24 KB at 1024)
constexpr int kMaxSupernodeWidth = 1024;
// levels with fewer supernodes than this are spread over their rows (two launches)
constexpr int kSplitBelow = 64;

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_solve(SnArgs A)
{
    extern __shared__ double t[];   // w x 3
    const int s = A.level_sn[blockIdx.x];
    const int c0 = A.sn_begin[s], c1 = A.sn_begin[s + 1], w = c1 - c0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < w; r += nw) {
        const int row = c0 + r;
        double s0 = 0, s1 = 0, s2 = 0;
        for (int64_t k = A.rp[row] + lane; k < A.rp[row + 1]; k += 32) {
            const int j = A.ci[k];
            if (LOWER ? (j < c0) : (j >= c1)) {
                const double v = A.val[k];
                s0 += v * A.y[3 * static_cast<int64_t>(j) + 0];
                s1 += v * A.y[3 * static_cast<int64_t>(j) + 1];
                s2 += v * A.y[3 * static_cast<int64_t>(j) + 2];
            }
        }
        s0 = warp_sum_f64(s0);
        s1 = warp_sum_f64(s1);
        s2 = warp_sum_f64(s2);
        if (lane == 0) {
            const int src = A.perm_in ? A.perm_in[row] : row;
            t[3 * r + 0] = A.b[3 * static_cast<int64_t>(src) + 0] - s0;
            t[3 * r + 1] = A.b[3 * static_cast<int64_t>(src) + 1] - s1;
            t[3 * r + 2] = A.b[3 * static_cast<int64_t>(src) + 2] - s2;
        }
    }
    __syncthreads();
    const double* D = A.dinv + A.dinv_off[s];
    for (int r = warp; r < w; r += nw) {
        // LOWER: row r of D^{-1} holds columns 0..r; UPPER: row r of D^{-T} holds columns r..w-1
        const int64_t o = LOWER ? static_cast<int64_t>(r) * (r + 1) / 2
                                : static_cast<int64_t>(r) * w - static_cast<int64_t>(r) * (r - 1) / 2;
        const int cb = LOWER ? 0 : r, len = LOWER ? r + 1 : w - r;
        double s0 = 0, s1 = 0, s2 = 0;
        for (int c = lane; c < len; c += 32) {
            const double d = D[o + c];
            const int tc = 3 * (cb + c);
            s0 += d * t[tc + 0];
            s1 += d * t[tc + 1];
            s2 += d * t[tc + 2];
        }
        s0 = warp_sum_f64(s0);
        s1 = warp_sum_f64(s1);
        s2 = warp_sum_f64(s2);
        if (lane == 0) {
            const int row = c0 + r;
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
    }
}

// Levels with few, wide supernodes run as two launches over all their rows instead
// (one warp per row, many CTAs): the external part into t (global), then y = D^{-1} t.
struct SnSplitArgs {
    const int* rows;          // rows of the level (factor order)
    int nrows;
    const int* sn_of;         // column -> supernode
    const int* sn_begin;
    const int64_t* rp;
    const int* ci;
    const double* val;
    const int64_t* dinv_off;
    const double* dinv;
    const double* b;
    const int* perm_in;
    double* t;                // n x 3 scratch
    double* y;
    double* out;
    const int* perm_out;
};

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_external(SnSplitArgs A)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= A.nrows) return;
    const int row = A.rows[w];
    const int s = A.sn_of[row];
    const int c0 = A.sn_begin[s], c1 = A.sn_begin[s + 1];
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t k = A.rp[row] + lane; k < A.rp[row + 1]; k += 32) {
        const int j = A.ci[k];
        if (LOWER ? (j < c0) : (j >= c1)) {
            const double v = A.val[k];
            s0 += v * A.y[3 * static_cast<int64_t>(j) + 0];
            s1 += v * A.y[3 * static_cast<int64_t>(j) + 1];
            s2 += v * A.y[3 * static_cast<int64_t>(j) + 2];
        }
    }
    s0 = warp_sum_f64(s0);
    s1 = warp_sum_f64(s1);
    s2 = warp_sum_f64(s2);
    if (lane == 0) {
        const int src = A.perm_in ? A.perm_in[row] : row;
        A.t[3 * static_cast<int64_t>(row) + 0] = A.b[3 * static_cast<int64_t>(src) + 0] - s0;
        A.t[3 * static_cast<int64_t>(row) + 1] = A.b[3 * static_cast<int64_t>(src) + 1] - s1;
        A.t[3 * static_cast<int64_t>(row) + 2] = A.b[3 * static_cast<int64_t>(src) + 2] - s2;
    }
}

template <bool LOWER>
__global__ void __launch_bounds__(SN_BLOCK) k_sn_dense(SnSplitArgs A)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= A.nrows) return;
    const int row = A.rows[w];
    const int s = A.sn_of[row];
    const int c0 = A.sn_begin[s], wd = A.sn_begin[s + 1] - c0, r = row - c0;
    const double* D = A.dinv + A.dinv_off[s];
    const int64_t o = LOWER ? static_cast<int64_t>(r) * (r + 1) / 2
                            : static_cast<int64_t>(r) * wd - static_cast<int64_t>(r) * (r - 1) / 2;
    const int cb = LOWER ? 0 : r, len = LOWER ? r + 1 : wd - r;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int c = lane; c < len; c += 32) {
        const double d = D[o + c];
        const int64_t tc = 3 * static_cast<int64_t>(c0 + cb + c);
        s0 += d * A.t[tc + 0];
        s1 += d * A.t[tc + 1];
        s2 += d * A.t[tc + 2];
    }
    s0 = warp_sum_f64(s0);
    s1 = warp_sum_f64(s1);
    s2 = warp_sum_f64(s2);
    if (lane == 0) {
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
}

// ------------------------------------------------------------------------------------------
// CG vector kernels (FP64). Scalars live on the device; per column c:
//   S_RZ rz, S_RZOLD previous rz, S_PAP (p,Ap), S_RR (r,r), S_ZR_OLD (z, r_old)
// ------------------------------------------------------------------------------------------
enum { S_RZ = 0, S_RZOLD = 3, S_PAP = 6, S_RR = 9, S_ZROLD = 12, S_ACTIVE = 15, S_BB = 18, S_CONV_IT = 21, S_IT = 24,
       S_COUNT = 25 };

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
__global__ void k_cg_check(double* S, double tol2)
{
    S[S_IT] += 1.0;
    for (int c = 0; c < 3; ++c) {
        if (S[S_ACTIVE + c] != 0.0 && S[S_RR + c] <= tol2 * S[S_BB + c]) {
            S[S_ACTIVE + c] = 0.0;
            S[S_CONV_IT + c] = S[S_IT];
        }
        S[S_RZOLD + c] = S[S_RZ + c];
    }
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
    const std::string err = cholesky_factor(H, s.nd_perm, F);
    if (!err.empty()) { set_error(err); return RPB_EINVAL; }
    s.factor_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s.factor_nnz = F.nnz();
    SupernodalSchedule SS;
    const std::string serr = supernodal_schedule(F, kMaxSupernodeWidth, SS);
    if (!serr.empty()) { set_error(serr); return RPB_EINVAL; }
    s.sn_levels_fwd = SS.fwd_levels();
    s.sn_levels_bwd = SS.bwd_levels();
    s.fwd_level_ptr = SS.fwd_level_ptr;
    s.bwd_level_ptr = SS.bwd_level_ptr;
    s.fwd_level_width = SS.fwd_level_width;
    s.bwd_level_width = SS.bwd_level_width;
    cudaStream_t st = m->stream;
    auto up = [st](auto& dst, const auto& src) -> cudaError_t {
        cudaError_t e = dst.alloc(src.size());
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(dst.ptr, src.data(), dst.bytes(), cudaMemcpyHostToDevice, st);
    };
    RPB_CUDA(up(s.lo_rp, F.lower_rp));
    RPB_CUDA(up(s.lo_ci, F.lower_ci));
    RPB_CUDA(up(s.lo_val, F.lower_val));
    RPB_CUDA(up(s.up_rp, F.upper_rp));
    RPB_CUDA(up(s.up_ci, F.upper_ci));
    RPB_CUDA(up(s.up_val, F.upper_val));
    RPB_CUDA(up(s.perm, F.perm));
    RPB_CUDA(up(s.sn_begin, SS.sn_begin));
    RPB_CUDA(up(s.fwd_level_sn, SS.fwd_level_sn));
    RPB_CUDA(up(s.bwd_level_sn, SS.bwd_level_sn));
    RPB_CUDA(up(s.dinv_off, SS.dinv_off));
    RPB_CUDA(up(s.dinv, SS.dinv));
    RPB_CUDA(up(s.dinvT, SS.dinvT));
    // levels with fewer supernodes than kSplitBelow run split over their rows
    std::vector<int> sn_of(m->nV);
    for (int sn = 0; sn < SS.nsn; ++sn)
        for (int c = SS.sn_begin[sn]; c < SS.sn_begin[sn + 1]; ++c) sn_of[c] = sn;
    auto split_rows = [&](const std::vector<int>& lptr, const std::vector<int>& lsn, std::vector<int>& rptr,
                          std::vector<int>& rows) {
        const int L = static_cast<int>(lptr.size()) - 1;
        rptr.assign(static_cast<size_t>(L) + 1, 0);
        rows.clear();
        for (int l = 0; l < L; ++l) {
            if (lptr[l + 1] - lptr[l] < kSplitBelow)
                for (int q = lptr[l]; q < lptr[l + 1]; ++q)
                    for (int c = SS.sn_begin[lsn[q]]; c < SS.sn_begin[lsn[q] + 1]; ++c) rows.push_back(c);
            rptr[l + 1] = static_cast<int>(rows.size());
        }
    };
    std::vector<int> frows, brows;
    split_rows(SS.fwd_level_ptr, SS.fwd_level_sn, s.fwd_split_ptr, frows);
    split_rows(SS.bwd_level_ptr, SS.bwd_level_sn, s.bwd_split_ptr, brows);
    RPB_CUDA(up(s.sn_of, sn_of));
    RPB_CUDA(up(s.fwd_split_rows, frows));
    RPB_CUDA(up(s.bwd_split_rows, brows));
    RPB_CUDA(s.tri.alloc(3 * static_cast<size_t>(m->nV)));
    RPB_CUDA(s.tmp.alloc(3 * static_cast<size_t>(m->nV)));
    RPB_CUDA(s.tbuf.alloc(3 * static_cast<size_t>(m->nV)));
    RPB_CUDA(cudaStreamSynchronize(st));
    s.h1_version = m->geometry_version;
    return RPB_OK;
}

// out = H1^{-1} b (b, out: n x 3 contiguous, device): forward levels on L, backward
// levels on L^T, one launch per level
static rpb_status h1_solve(rpb_mesh* m, const double* b, double* out)
{
    Solver& s = *m->solver;
    SnArgs A;
    A.sn_begin = s.sn_begin.ptr; A.dinv_off = s.dinv_off.ptr;
    A.rp = s.lo_rp.ptr; A.ci = s.lo_ci.ptr; A.val = s.lo_val.ptr; A.dinv = s.dinv.ptr;
    A.b = b; A.perm_in = s.perm.ptr; A.y = s.tri.ptr; A.out = nullptr; A.perm_out = nullptr;
    SnSplitArgs P;
    P.sn_of = s.sn_of.ptr; P.sn_begin = s.sn_begin.ptr; P.dinv_off = s.dinv_off.ptr; P.t = s.tbuf.ptr;
    auto level = [&](const SnArgs& a, const int* level_sn, int nsn, int width, const int* rows, int nrows, bool lower) {
        if (nrows > 0) {
            P.rows = rows; P.nrows = nrows;
            P.rp = a.rp; P.ci = a.ci; P.val = a.val; P.dinv = a.dinv;
            P.b = a.b; P.perm_in = a.perm_in; P.y = a.y; P.out = a.out; P.perm_out = a.perm_out;
            const int grid = (nrows + SN_BLOCK / 32 - 1) / (SN_BLOCK / 32);
            if (lower) {
                k_sn_external<true><<<grid, SN_BLOCK, 0, m->stream>>>(P);
                k_sn_dense<true><<<grid, SN_BLOCK, 0, m->stream>>>(P);
            } else {
                k_sn_external<false><<<grid, SN_BLOCK, 0, m->stream>>>(P);
                k_sn_dense<false><<<grid, SN_BLOCK, 0, m->stream>>>(P);
            }
            return;
        }
        SnArgs a2 = a;
        a2.level_sn = level_sn;
        const size_t smem = 3 * sizeof(double) * static_cast<size_t>(width);
        if (lower) k_sn_solve<true><<<nsn, SN_BLOCK, smem, m->stream>>>(a2);
        else k_sn_solve<false><<<nsn, SN_BLOCK, smem, m->stream>>>(a2);
    };
    for (int l = 0; l < s.sn_levels_fwd; ++l)
        level(A, s.fwd_level_sn.ptr + s.fwd_level_ptr[l], s.fwd_level_ptr[l + 1] - s.fwd_level_ptr[l],
              s.fwd_level_width[l], s.fwd_split_rows.ptr + s.fwd_split_ptr[l],
              s.fwd_split_ptr[l + 1] - s.fwd_split_ptr[l], true);
    RPB_CUDA(cudaGetLastError());
    SnArgs U = A;
    U.rp = s.up_rp.ptr; U.ci = s.up_ci.ptr; U.val = s.up_val.ptr; U.dinv = s.dinvT.ptr;
    U.b = s.tri.ptr; U.perm_in = nullptr; U.y = s.tmp.ptr; U.out = out; U.perm_out = s.perm.ptr;
    for (int l = 0; l < s.sn_levels_bwd; ++l)
        level(U, s.bwd_level_sn.ptr + s.bwd_level_ptr[l], s.bwd_level_ptr[l + 1] - s.bwd_level_ptr[l],
              s.bwd_level_width[l], s.bwd_split_rows.ptr + s.bwd_split_ptr[l],
              s.bwd_split_ptr[l + 1] - s.bwd_split_ptr[l], false);
    RPB_CUDA(cudaGetLastError());
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
    const bool flexible = (precond == RPB_PRECOND_LEARNED);
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
        k_cg_check<<<1, 1, 0, stream>>>(S, tol2);
        if ((e = apply_preconditioner(m, k, q, p, r, z)) != RPB_OK) return e;
        if ((e = dot3(m, z, r, flexible ? rold : nullptr, S + S_RZ, S + S_ZROLD)) != RPB_OK) return e;
        k_cg_direction<<<eb, 256, 0, stream>>>(n, S, flexible, z, pv);
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
        if (stalled_flag && kind == RPB_PRECOND_LEARNED) {
            kind = RPB_PRECOND_REFERENCE;  // fallback on stall
            s.last_fallback_iteration = it;
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
            if (flexible && kind == RPB_PRECOND_LEARNED && !conv && since_best > kStallWindow) stalled = true;
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
    if (precond < RPB_PRECOND_NONE || precond > RPB_PRECOND_LEARNED) { set_error("unknown preconditioner kind"); return RPB_EINVAL; }
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
    return RPB_OK;
}

}  // extern "C"
