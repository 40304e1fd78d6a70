// TangentPointMetric0 and PseudoLaplacian on the B200:
//   metric values      TP0 kernels with metric_flag (TP0_Kernel_FF.hpp:295-315,
//                      TP0_Kernel_NF.hpp:313-334), PseudoLaplacian_Kernel_{NF,FF}, full pattern,
//                      one warp per row, row diagonals in the same pass
//   Pre                ClusterTree::Pre (src/ClusterTree.hpp:770-857) with the frozen
//                      mixed-order operator mi_pre (src/ClusterTree.hpp:410-639) and the
//                      PercolateUp as one bottom-up pass
//   block SpMM         KernelMatrixCSR::Dot with TP0_Kernel_MultiplyMetric_Tiny
//                      (TP0_Kernel_MultiplyMetric_Tiny.hpp:89-138) + DiagonalKernelMatrix
//   Post               ClusterTree::Post (src/ClusterTree.hpp:860-943): percolate-down,
//                      clusters-to-primitives and the transposed operator mi_post
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels_energy.cuh"
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

// ------------------------------------------------------------------------------------------
// metric values
// ------------------------------------------------------------------------------------------
struct ValuesArgs {
    int dom, rows;
    const int64_t* rp; const int* ci;
    const void* data;        // PrimDatum* (near rows) or ClusterDatum* (far rows)
    float2* vals;
    double2* diag;
    float s_exp;             // TP0: s_exp of the metric; pseudo-Laplacian: -n/2 - s
};

// One warp per row: a0 = 1/2 (v^T P v + v^T Q v)/r^4 a1, a1 = -2 r^{2 s_exp}
// (TP0_Kernel_FF.hpp:295-315) or the pseudo-Laplacian value -r^{2 s_exp}; the row
// diagonal -sum_j (b/a) (a0, a1) is accumulated in the same pass.
template <bool FAR, bool PL>
__global__ void __launch_bounds__(256) k_metric_values(ValuesArgs A)
{
    using Datum = typename std::conditional<FAR, ClusterDatum, PrimDatum>::type;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= A.rows) return;
    const Datum* base = static_cast<const Datum*>(A.data);
    const Datum X = load_datum(base, i);
    const double inv_a = 1.0 / X.a;
    double d0 = 0.0, d1 = 0.0;
    for (int64_t k = A.rp[i] + lane; k < A.rp[i + 1]; k += 32) {
        const int j = __ldg(A.ci + k);
        const Datum Y = load_datum(base, j);
        float a0, a1;
        if (PL) {
            const float v0 = static_cast<float>(Y.c[0] - X.c[0]);
            const float v1 = static_cast<float>(Y.c[1] - X.c[1]);
            const float v2 = static_cast<float>(Y.c[2] - X.c[2]);
            const float r2 = v0 * v0 + v1 * v1 + v2 * v2;
            a0 = -exp2f(A.s_exp * __log2f(r2));
            a1 = a0;
        } else {
            Proj<float> g;
            if constexpr (FAR) project_clusters(X, Y, g);
            else project_prims(A.dom, X, Y, g);
            const float s = __frcp_rn(g.r2);
            a1 = -2.0f * exp2f(A.s_exp * __log2f(g.r2));
            a0 = 0.5f * (g.cphi + g.cpsi) * s * s * a1;
        }
        A.vals[k] = make_float2(a0, a1);
        // diagonal from the stored (rounded) values with the FP64 weight ratio, so that
        // y_i = sum_j a_ij (x_j - (a_j/a_i) x_i) holds exactly for the operator applied
        const double ba = Y.a * inv_a;
        d0 -= ba * static_cast<double>(a0);
        d1 -= ba * static_cast<double>(a1);
    }
    const double D0 = warp_sum_f64(d0);
    const double D1 = warp_sum_f64(d1);
    if (lane == 0) A.diag[i] = make_double2(D0, D1);
}

static void launch_values(rpb_mesh* m, bool pl, float s_exp, float2* nf, double2* nfd, float2* ff, double2* ffd)
{
    ValuesArgs A;
    A.dom = m->dom;
    A.s_exp = s_exp;
    if (m->near.nnz > 0) {
        A.rows = m->N; A.rp = m->near.rp.ptr; A.ci = m->near.ci.ptr; A.data = m->P_pair.ptr; A.vals = nf; A.diag = nfd;
        if (pl) k_metric_values<false, true><<<(m->N + 7) / 8, 256, 0, m->stream>>>(A);
        else k_metric_values<false, false><<<(m->N + 7) / 8, 256, 0, m->stream>>>(A);
    } else {
        cudaMemsetAsync(nfd, 0, sizeof(double2) * m->N, m->stream);
    }
    if (m->far.nnz > 0) {
        A.rows = m->NC; A.rp = m->far.rp.ptr; A.ci = m->far.ci.ptr; A.data = m->C_pair.ptr; A.vals = ff; A.diag = ffd;
        if (pl) k_metric_values<true, true><<<(m->NC + 7) / 8, 256, 0, m->stream>>>(A);
        else k_metric_values<true, false><<<(m->NC + 7) / 8, 256, 0, m->stream>>>(A);
    } else {
        cudaMemsetAsync(ffd, 0, sizeof(double2) * m->NC, m->stream);
    }
}

// ------------------------------------------------------------------------------------------
// Pre: X (vertices, ldX) -> P_in (primitives, BD = 4*3 or 3) -> C_in (clusters, upsweep)
// ------------------------------------------------------------------------------------------
template <int BD>
struct PreArgs {
    int N, NC, size;
    const int* pre_cols;      // N x size
    const double* pre_vals;   // N x 4 x size
    const double* X;
    int ldX;
    const int* C_begin;
    const int* C_end;
    double* Pin;              // N x BD
    double* Cin;              // NC x BD
    double* local;            // N x BD in-block exclusive prefix
    double* blocks;           // (nblocks + 1) x BD
    unsigned* scan_done;      // last-block counter: the last k_pre block scans `blocks`
};

// Pre operator per primitive (mi_pre / lo_pre rows, src/ClusterTree.hpp:410-639) and the
// in-block prefix sums that give PrimitivesToClusters + PercolateUp as range sums; the
// last block scans the block sums.
template <int BD>
__global__ void __launch_bounds__(SCAN_BLOCK) k_pre(PreArgs<BD> A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int ROWS = BD / 3;  // 4 (mixed order) or 1 (low order)
    double x[BD];
#pragma unroll
    for (int k = 0; k < BD; ++k) x[k] = 0.0;
    if (i < A.N) {
        for (int l = 0; l < A.size; ++l) {
            const int v = A.pre_cols[A.size * i + l];
            const double* xv = A.X + static_cast<int64_t>(A.ldX) * v;
            const double X0 = xv[0], X1 = xv[1], X2 = xv[2];
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const double w = A.pre_vals[(4 * static_cast<int64_t>(i) + r) * A.size + l];
                x[3 * r + 0] += w * X0;
                x[3 * r + 1] += w * X1;
                x[3 * r + 2] += w * X2;
            }
        }
#pragma unroll
        for (int k = 0; k < BD; ++k) A.Pin[BD * static_cast<int64_t>(i) + k] = x[k];
    }
    double tot[BD];
    block_exclusive_scan<BD>(x, tot);
    if (i < A.N) {
#pragma unroll
        for (int k = 0; k < BD; ++k) A.local[BD * static_cast<int64_t>(i) + k] = x[k];
    }
    if (threadIdx.x < BD) A.blocks[BD * static_cast<int64_t>(blockIdx.x) + threadIdx.x] = tot[threadIdx.x];
    last_block_scans_rows<BD>(A.blocks, gridDim.x, A.scan_done);
}

template <int BD>
__global__ void k_cluster_sums(PreArgs<BD> A)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= A.NC) return;
    const int b = A.C_begin[C], e = A.C_end[C];
    const int nb = (A.N + SCAN_BLOCK - 1) / SCAN_BLOCK;
#pragma unroll
    for (int k = 0; k < BD; ++k) {
        const double sb = A.blocks[BD * static_cast<int64_t>(b / SCAN_BLOCK) + k] + A.local[BD * static_cast<int64_t>(b) + k];
        const double se = (e < A.N) ? A.blocks[BD * static_cast<int64_t>(e / SCAN_BLOCK) + k] +
                                          A.local[BD * static_cast<int64_t>(e) + k]
                                    : A.blocks[BD * static_cast<int64_t>(nb) + k];
        A.Cin[BD * static_cast<int64_t>(C) + k] = se - sb;
    }
}

// ------------------------------------------------------------------------------------------
// Block SpMM: y_i = sum_k diag(a0, a1, a1, a1) (x) x_{col(k)} + diag_i (x) x_i, nrhs = 3
// ------------------------------------------------------------------------------------------
template <int BD>
struct SpmmArgs {
    int rows0, rows1;         // near rows [0, rows0), far rows [rows0, rows0 + rows1)
    const int64_t* rp0; const int* ci0; const float2* v0; const double2* d0; const double* x0; double* y0;
    const int64_t* rp1; const int* ci1; const float2* v1; const double2* d1; const double* x1; double* y1;
    bool accumulate;          // y += (very-near add-in) instead of y =
};

// SPMM_LANES lanes per row, striding over the row's blocks (rows hold ~30-60 blocks at
// theta = 0.5). Input rows are gathered in FP64 (the operator's result cancels strongly for
// smooth fields: with the diagonal built from the same stored values, FP64 keeps that
// cancellation exact to ~1e-15). The lanes of a row combine their partial sums by a
// reduce-scatter (BD = 12: 6 + 3 shuffles, each lane ends with 3 of the 12 outputs) or an
// xor butterfly (BD = 3), in a fixed order.
constexpr int SPMM_LANES = 4;

// reduce-scatter / butterfly of the SPMM_LANES partial sums of a row, diagonal term, store
template <int BD>
__device__ __forceinline__ void spmm_finish(const double (&acc)[BD], int sub, bool active, double2 dg,
                                            const double* xi, double* y, bool accumulate)
{
    if constexpr (BD == 12) {
        const bool b1 = sub & 2, b0 = sub & 1;
        double h[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const double send = b1 ? acc[q] : acc[q + 6];
            const double keep = b1 ? acc[q + 6] : acc[q];
            h[q] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
        double f[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double send = b0 ? h[q] : h[q + 3];
            const double keep = b0 ? h[q + 3] : h[q];
            f[q] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
        }
        if (active) {
            const int base = 6 * (b1 ? 1 : 0) + 3 * (b0 ? 1 : 0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int c = base + q;
                const double val = f[q] + (c < 3 ? dg.x : dg.y) * xi[c];
                y[c] = accumulate ? y[c] + val : val;
            }
        }
    } else {
        double a[BD];
#pragma unroll
        for (int c = 0; c < BD; ++c) a[c] = acc[c];
#pragma unroll
        for (int off = 1; off < SPMM_LANES; off <<= 1)
#pragma unroll
            for (int c = 0; c < BD; ++c) a[c] += __shfl_xor_sync(0xffffffffu, a[c], off);
        if (active && sub < BD) {
            double val = a[0];
#pragma unroll
            for (int c = 1; c < BD; ++c) val = (sub == c) ? a[c] : val;
            val += dg.x * xi[sub];
            y[sub] = accumulate ? y[sub] + val : val;
        }
    }
}

// BD = 12: six lanes per row (five rows per warp, two lanes idle); lane s owns outputs
// 2s, 2s+1 and reads the 16-byte piece s of every column row, so one load instruction
// covers five whole 96-byte input rows. Each lane walks all of the row's blocks, four at a
// time with the loads issued first; no cross-lane combination.
constexpr int SPMM6_ROWS_PER_WARP = 5;
__global__ void __launch_bounds__(256) k_block_spmm12_rows6(SpmmArgs<12> A)
{
    const int lane = threadIdx.x & 31, grp = lane / 6, sub = lane - 6 * grp;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * SPMM6_ROWS_PER_WARP + grp;
    if (grp >= SPMM6_ROWS_PER_WARP || row >= A.rows0 + A.rows1) return;
    const bool first = row < A.rows0;
    const int i = first ? row : row - A.rows0;
    const double2* x = reinterpret_cast<const double2*>(first ? A.x0 : A.x1) + sub;
    const int64_t* rp = first ? A.rp0 : A.rp1;
    const int* ci = first ? A.ci0 : A.ci1;
    const float2* vals = first ? A.v0 : A.v1;
    const bool lo_x = 2 * sub < 3, hi_x = 2 * sub + 1 < 3;
    double acc0 = 0.0, acc1 = 0.0;
    const int64_t k1 = rp[i + 1];
    int64_t k = rp[i];
    for (; k + 4 <= k1; k += 4) {
        int j[4];
        float2 a[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            j[q] = __ldg(ci + k + q);
            a[q] = __ldg(vals + k + q);
        }
        double2 t[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = __ldg(x + 6 * static_cast<int64_t>(j[q]));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            acc0 += static_cast<double>(lo_x ? a[q].x : a[q].y) * t[q].x;
            acc1 += static_cast<double>(hi_x ? a[q].x : a[q].y) * t[q].y;
        }
    }
    for (; k < k1; ++k) {
        const int j = __ldg(ci + k);
        const float2 a = __ldg(vals + k);
        const double2 t = __ldg(x + 6 * static_cast<int64_t>(j));
        acc0 += static_cast<double>(lo_x ? a.x : a.y) * t.x;
        acc1 += static_cast<double>(hi_x ? a.x : a.y) * t.y;
    }
    const double2 dg = (first ? A.d0 : A.d1)[i];
    const double2 xi = x[6 * static_cast<int64_t>(i)];
    double* y = (first ? A.y0 : A.y1) + 12 * static_cast<int64_t>(i) + 2 * sub;
    const double v0 = acc0 + (lo_x ? dg.x : dg.y) * xi.x, v1 = acc1 + (hi_x ? dg.x : dg.y) * xi.y;
    if (A.accumulate) {
        y[0] += v0; y[1] += v1;
    } else {
        y[0] = v0; y[1] = v1;
    }
}

template <int BD>
__global__ void __launch_bounds__(256) k_block_spmm(SpmmArgs<BD> A)
{
    static_assert(BD == 12 || BD == 3, "block width 12 (metric) or 3 (pseudo-Laplacian)");
    const int sub = threadIdx.x & (SPMM_LANES - 1);
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / SPMM_LANES;
    const bool active = row < A.rows0 + A.rows1;
    const bool first = row < A.rows0;
    const int i = first ? row : row - A.rows0;
    const double* x = first ? A.x0 : A.x1;
    double acc[BD];
#pragma unroll
    for (int c = 0; c < BD; ++c) acc[c] = 0.0;
    if (active) {
        const int64_t* rp = first ? A.rp0 : A.rp1;
        const int* ci = first ? A.ci0 : A.ci1;
        const float2* vals = first ? A.v0 : A.v1;
        for (int64_t k = rp[i] + sub; k < rp[i + 1]; k += SPMM_LANES) {
            const int j = __ldg(ci + k);
            const float2 a = __ldg(vals + k);
            const double ax = a.x, ay = a.y;
            if constexpr (BD == 12) {
                const double2* xp = reinterpret_cast<const double2*>(x + BD * static_cast<int64_t>(j));
#pragma unroll
                for (int q = 0; q < BD / 2; ++q) {
                    const double2 t = __ldg(xp + q);
                    acc[2 * q] += (2 * q < 3 ? ax : ay) * t.x;
                    acc[2 * q + 1] += (2 * q + 1 < 3 ? ax : ay) * t.y;
                }
            } else {
#pragma unroll
                for (int c = 0; c < BD; ++c) acc[c] += ax * __ldg(x + BD * static_cast<int64_t>(j) + c);
            }
        }
    }
    const double2 dg = active ? (first ? A.d0 : A.d1)[i] : make_double2(0.0, 0.0);
    double* y = (first ? A.y0 : A.y1) + BD * static_cast<int64_t>(i);
    spmm_finish<BD>(acc, sub, active, dg, x + BD * static_cast<int64_t>(i), y, A.accumulate);
}

// ------------------------------------------------------------------------------------------
// Post: Z_i = P_out_i + sum_{ancestors C} C_out_C ; Y_v = alpha sum mi_post Z + beta Y_v
// ------------------------------------------------------------------------------------------
template <int BD>
struct PostArgs {
    int N, nV, size;
    const int* leaf_of;
    const int* C_parent;
    const int* C_up4;
    const double* Pout;
    const double* Cout;
    double* Z;
    const int* vp_rp;
    const int* vp_slot;       // i * size + l
    const double* pre_vals;
    double alpha, beta;
    double* Y;
    int ldY;
};

// POST_LANES consecutive lanes per primitive (vertex): lane p adds the ancestors at
// distances p, p + 4, ... from the leaf (the vertex's slots p, p + 4, ...); an xor
// butterfly combines the lanes' partial sums (every lane ends with the same totals) and the
// lanes write disjoint components.
constexpr int POST_LANES = 4;

template <int BD>
__global__ void k_post_primitives(PostArgs<BD> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / POST_LANES, lane = t % POST_LANES;
    const bool active = i < A.N;
    double z[BD];
#pragma unroll
    for (int c = 0; c < BD; ++c) z[c] = (active && lane == 0) ? A.Pout[BD * static_cast<int64_t>(i) + c] : 0.0;
    if (active) {
        int C = A.leaf_of[i];
        for (int k = 0; k < lane && C >= 0; ++k) C = __ldg(A.C_parent + C);
        for (; C >= 0; C = __ldg(A.C_up4 + C)) {
#pragma unroll
            for (int c = 0; c < BD; ++c) z[c] += A.Cout[BD * static_cast<int64_t>(C) + c];
        }
    }
#pragma unroll
    for (int off = 1; off < POST_LANES; off <<= 1)
#pragma unroll
        for (int c = 0; c < BD; ++c) z[c] += __shfl_xor_sync(0xffffffffu, z[c], off);
    if (!active) return;
#pragma unroll
    for (int c = 0; c < BD; ++c)
        if (c % POST_LANES == lane) A.Z[BD * static_cast<int64_t>(i) + c] = z[c];
}

template <int BD>
__global__ void k_post_vertices(PostArgs<BD> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = t / POST_LANES, lane = t % POST_LANES;
    const bool active = v < A.nV;
    constexpr int ROWS = BD / 3;
    double acc[3] = {0, 0, 0};
    const int k1 = active ? A.vp_rp[v + 1] : 0;
    for (int k = (active ? A.vp_rp[v] : 0) + lane; k < k1; k += POST_LANES) {
        const int slot = A.vp_slot[k];
        const int i = slot / A.size, l = slot - i * A.size;
        const double* z = A.Z + BD * static_cast<int64_t>(i);
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const double w = A.pre_vals[(4 * static_cast<int64_t>(i) + r) * A.size + l];
            acc[0] += w * z[3 * r + 0];
            acc[1] += w * z[3 * r + 1];
            acc[2] += w * z[3 * r + 2];
        }
    }
#pragma unroll
    for (int off = 1; off < POST_LANES; off <<= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
    if (!active || lane >= 3) return;
    const double a = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : acc[2]);
    double* y = A.Y + static_cast<int64_t>(A.ldY) * v + lane;
    *y = A.alpha * a + (A.beta == 0.0 ? 0.0 : A.beta * *y);
}

// ==========================================================================================
// host side
// ==========================================================================================

// Frozen Pre/Post operator (construction-time geometry, as the reference's
// pre_post_initialized flag keeps it): rows 0: a/(n+1) (averaging), rows 1..3: a * D_f.
rpb_status metric_init(rpb_mesh* m, const double* Vh, const int* Sh)
{
    const int N = m->N, size = m->size;
    std::vector<int> cols(static_cast<size_t>(N) * size);
    std::vector<double> vals(static_cast<size_t>(N) * 4 * size, 0.0);
    const double nth = 1.0 / size;
    for (int i = 0; i < N; ++i) {
        const int j = m->tree.perm[i];
        int s[3];
        for (int l = 0; l < size; ++l) s[l] = Sh[static_cast<int64_t>(size) * j + l];
        int ss[3] = {s[0], s[1], s[2]};
        std::sort(ss, ss + size);
        // a = charge * vol from the sorted simplex (SimplexDataKernel::ReadSimplex)
        double df[3][2];
        for (int l = 0; l < size - 1; ++l)
            for (int k = 0; k < 3; ++k) df[k][l] = Vh[3 * static_cast<int64_t>(ss[l + 1]) + k] - Vh[3 * static_cast<int64_t>(ss[0]) + k];
        const int n = size - 1;
        double g[2][2] = {{0, 0}, {0, 0}};
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                for (int k = 0; k < 3; ++k) g[a][b] += df[k][a] * df[k][b];
        double ginv[2][2];
        double vol;
        if (n == 1) {
            vol = std::sqrt(g[0][0]);
            ginv[0][0] = 1.0 / g[0][0];
        } else {
            const double det = g[0][0] * g[1][1] - g[0][1] * g[1][0];
            vol = 0.5 * std::sqrt(det);
            ginv[0][0] = g[1][1] / det; ginv[1][1] = g[0][0] / det; ginv[0][1] = ginv[1][0] = -g[0][1] / det;
        }
        // charges are read back from the device-side copy only for the energy; the
        // operator uses a = mean vertex charge * vol like ReadSimplex
        const double a = vol;  // charges applied below
        double dag[2][3];
        for (int l = 0; l < n; ++l)
            for (int k = 0; k < 3; ++k) {
                double acc = 0;
                for (int b = 0; b < n; ++b) acc += ginv[l][b] * df[k][b];
                dag[l][k] = acc;
            }
        for (int l = 0; l < size; ++l) cols[static_cast<size_t>(size) * i + l] = ss[l];
        for (int l = 0; l < size; ++l) vals[(4 * static_cast<size_t>(i) + 0) * size + l] = a * nth;
        for (int k = 0; k < 3; ++k) {
            double d0 = 0;
            for (int l = 0; l < n; ++l) {
                d0 -= dag[l][k];
                vals[(4 * static_cast<size_t>(i) + 1 + k) * size + l + 1] = a * dag[l][k];
            }
            vals[(4 * static_cast<size_t>(i) + 1 + k) * size + 0] = a * d0;
        }
    }
    // charges (mean of vertex charges) scale a
    {
        std::vector<double> ch(m->nV);
        if (cudaMemcpy(ch.data(), m->charge_v.ptr, sizeof(double) * m->nV, cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error("charge readback failed");
            return RPB_ECUDA;
        }
        for (int i = 0; i < N; ++i) {
            double c = 0;
            for (int l = 0; l < size; ++l) c += ch[cols[static_cast<size_t>(size) * i + l]];
            c /= size;
            for (int k = 0; k < 4 * size; ++k) vals[4 * static_cast<size_t>(i) * size + k] *= c;
        }
    }
    std::vector<int> rp(m->nV + 1, 0), slot(static_cast<size_t>(N) * size);
    for (size_t k = 0; k < cols.size(); ++k) rp[cols[k] + 1]++;
    for (int v = 0; v < m->nV; ++v) rp[v + 1] += rp[v];
    std::vector<int> pos(rp.begin(), rp.end() - 1);
    for (size_t k = 0; k < cols.size(); ++k) slot[pos[cols[k]]++] = static_cast<int>(k);
    cudaStream_t s = m->stream;
    RPB_CUDA(m->pre_cols.alloc(cols.size()));
    RPB_CUDA(m->pre_vals.alloc(vals.size()));
    RPB_CUDA(m->vp_rp.alloc(rp.size()));
    RPB_CUDA(m->vp_slot.alloc(slot.size()));
    RPB_CUDA(cudaMemcpyAsync(m->pre_cols.ptr, cols.data(), m->pre_cols.bytes(), cudaMemcpyHostToDevice, s));
    RPB_CUDA(cudaMemcpyAsync(m->pre_vals.ptr, vals.data(), m->pre_vals.bytes(), cudaMemcpyHostToDevice, s));
    RPB_CUDA(cudaMemcpyAsync(m->vp_rp.ptr, rp.data(), m->vp_rp.bytes(), cudaMemcpyHostToDevice, s));
    RPB_CUDA(cudaMemcpyAsync(m->vp_slot.ptr, slot.data(), m->vp_slot.bytes(), cudaMemcpyHostToDevice, s));
    RPB_CUDA(m->buf_Pin64.alloc(12 * static_cast<size_t>(N)));
    RPB_CUDA(m->buf_scan_local.alloc(12 * static_cast<size_t>(N)));
    RPB_CUDA(m->buf_scan_blocks.alloc(12 * static_cast<size_t>((N + SCAN_BLOCK - 1) / SCAN_BLOCK + 1)));
    RPB_CUDA(m->buf_Cin64.alloc(12 * static_cast<size_t>(m->NC)));
    RPB_CUDA(m->buf_Pout.alloc(12 * static_cast<size_t>(N)));
    RPB_CUDA(m->buf_Cout.alloc(12 * static_cast<size_t>(m->NC)));
    RPB_CUDA(m->buf_Z.alloc(12 * static_cast<size_t>(N)));
    RPB_CUDA(m->X.alloc(3 * static_cast<size_t>(m->nV)));
    RPB_CUDA(m->Yb.alloc(3 * static_cast<size_t>(m->nV)));
    return RPB_OK;
}

static rpb_status ensure_metric_values(rpb_mesh* m, double q, double p)
{
    MetricCache& mc = m->metric;
    if (mc.valid && mc.q == q && mc.p == p) return RPB_OK;
    if (!mc.nf.ptr && m->near.nnz) RPB_CUDA(mc.nf.alloc(m->near.nnz));
    if (!mc.ff.ptr && m->far.nnz) RPB_CUDA(mc.ff.alloc(m->far.nnz));
    if (!mc.nf_diag.ptr) RPB_CUDA(mc.nf_diag.alloc(m->N));
    if (!mc.ff_diag.ptr) RPB_CUDA(mc.ff_diag.alloc(m->NC));
    if (m->verynear.nnz) {
        if (!mc.vf.ptr) RPB_CUDA(mc.vf.alloc(m->verynear.nnz));
        if (!mc.vf_diag.ptr) RPB_CUDA(mc.vf_diag.alloc(m->N));
    }
    const TPExp ex = make_exp(m->dom, q, p);
    launch_values(m, false, static_cast<float>(ex.s_exp_metric), mc.nf.ptr, mc.nf_diag.ptr, mc.ff.ptr, mc.ff_diag.ptr);
    RPB_CUDA(cudaGetLastError());
    if (m->verynear.nnz) {
        RPB_CUDA(cudaMemsetAsync(mc.vf_diag.ptr, 0, mc.vf_diag.bytes(), m->stream));
        rpb_status st = launch_vf_metric(m, ex, mc.vf.ptr, mc.vf_diag.ptr);
        if (st != RPB_OK) return st;
        // once per geometry: pairs in contact make the metric values NaN; report them
        if ((st = vf_take_status(m->vf, m->stream)) != RPB_OK) return st;
    }
    mc.valid = true;
    mc.q = q;
    mc.p = p;
    return RPB_OK;
}

static rpb_status ensure_plap_values(rpb_mesh* m, double s_pl)
{
    PseudoLapCache& pc = m->plap;
    if (pc.valid && pc.s == s_pl) return RPB_OK;
    // stored with the TP0 layout (float2 values / double2 diagonals) for the shared SpMM
    static_assert(sizeof(float2) == 2 * sizeof(float), "layout");
    if (!pc.nf.ptr && m->near.nnz) RPB_CUDA(pc.nf.alloc(2 * m->near.nnz));
    if (!pc.ff.ptr && m->far.nnz) RPB_CUDA(pc.ff.alloc(2 * m->far.nnz));
    if (!pc.nf_diag.ptr) RPB_CUDA(pc.nf_diag.alloc(2 * static_cast<size_t>(m->N)));
    if (!pc.ff_diag.ptr) RPB_CUDA(pc.ff_diag.alloc(2 * static_cast<size_t>(m->NC)));
    if (m->verynear.nnz) {
        if (!pc.vf.ptr) RPB_CUDA(pc.vf.alloc(2 * m->verynear.nnz));
        if (!pc.vf_diag.ptr) RPB_CUDA(pc.vf_diag.alloc(2 * static_cast<size_t>(m->N)));
    }
    launch_values(m, true, static_cast<float>(-m->dom / 2.0 - s_pl), reinterpret_cast<float2*>(pc.nf.ptr),
                  reinterpret_cast<double2*>(pc.nf_diag.ptr), reinterpret_cast<float2*>(pc.ff.ptr),
                  reinterpret_cast<double2*>(pc.ff_diag.ptr));
    RPB_CUDA(cudaGetLastError());
    if (m->verynear.nnz) {
        RPB_CUDA(cudaMemsetAsync(pc.vf_diag.ptr, 0, pc.vf_diag.bytes(), m->stream));
        TPExp ex = make_exp(m->dom, 6.0, 12.0);
        ex.s_exp_metric = -m->dom / 2.0 - s_pl;
        ex.qh = -2;  // marks the pseudo-Laplacian kernel in the very-near quadrature
        rpb_status st = launch_vf_metric(m, ex, reinterpret_cast<float2*>(pc.vf.ptr),
                                         reinterpret_cast<double2*>(pc.vf_diag.ptr));
        if (st != RPB_OK) return st;
        if ((st = vf_take_status(m->vf, m->stream)) != RPB_OK) return st;
    }
    pc.valid = true;
    pc.s = s_pl;
    return RPB_OK;
}

template <int BD>
static rpb_status apply_operator(rpb_mesh* m, const float2* nf, const double2* nfd, const float2* ff,
                                 const double2* ffd, const float2* vf, const double2* vfd, double alpha,
                                 const double* X, int ldX, double beta, double* Y, int ldY, int flags)
{
    cudaStream_t s = m->stream;
    PreArgs<BD> pa;
    pa.N = m->N; pa.NC = m->NC; pa.size = m->size;
    pa.pre_cols = m->pre_cols.ptr; pa.pre_vals = m->pre_vals.ptr;
    pa.X = X; pa.ldX = ldX;
    pa.C_begin = m->C_begin.ptr; pa.C_end = m->C_end.ptr;
    pa.Pin = m->buf_Pin64.ptr; pa.Cin = m->buf_Cin64.ptr;
    pa.local = m->buf_scan_local.ptr; pa.blocks = m->buf_scan_blocks.ptr;
    pa.scan_done = m->done.ptr + 3;
    const int nb = (m->N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_pre<BD><<<nb, SCAN_BLOCK, 0, s>>>(pa);
    k_cluster_sums<BD><<<(m->NC + 255) / 256, 256, 0, s>>>(pa);
    RPB_CUDA(cudaGetLastError());

    const bool NF = (flags & 2) && m->near.nnz > 0;
    const bool FF = (flags & 4) && m->far.nnz > 0;
    const bool VF = (flags & 1) && m->verynear.nnz > 0;
    if (!NF) RPB_CUDA(cudaMemsetAsync(m->buf_Pout.ptr, 0, sizeof(double) * BD * static_cast<size_t>(m->N), s));
    if (!FF) RPB_CUDA(cudaMemsetAsync(m->buf_Cout.ptr, 0, sizeof(double) * BD * static_cast<size_t>(m->NC), s));
    if (NF || FF) {
        SpmmArgs<BD> sa;
        std::memset(&sa, 0, sizeof(sa));
        sa.rows0 = NF ? m->N : 0;
        sa.rp0 = m->near.rp.ptr; sa.ci0 = m->near.ci.ptr; sa.v0 = nf; sa.d0 = nfd;
        sa.x0 = m->buf_Pin64.ptr; sa.y0 = m->buf_Pout.ptr;
        sa.rows1 = FF ? m->NC : 0;
        sa.rp1 = m->far.rp.ptr; sa.ci1 = m->far.ci.ptr; sa.v1 = ff; sa.d1 = ffd;
        sa.x1 = m->buf_Cin64.ptr; sa.y1 = m->buf_Cout.ptr;
        sa.accumulate = false;
        if constexpr (BD == 12) {
            const int warps = (sa.rows0 + sa.rows1 + SPMM6_ROWS_PER_WARP - 1) / SPMM6_ROWS_PER_WARP;
            k_block_spmm12_rows6<<<(warps + 7) / 8, 256, 0, s>>>(sa);
        } else
            k_block_spmm<BD><<<((sa.rows0 + sa.rows1) * SPMM_LANES + 255) / 256, 256, 0, s>>>(sa);
        RPB_CUDA(cudaGetLastError());
    }
    if (VF) {
        SpmmArgs<BD> sa;
        std::memset(&sa, 0, sizeof(sa));
        sa.rows0 = m->N;
        sa.rp0 = m->verynear.rp.ptr; sa.ci0 = m->verynear.ci.ptr; sa.v0 = vf; sa.d0 = vfd;
        sa.x0 = m->buf_Pin64.ptr; sa.y0 = m->buf_Pout.ptr;
        sa.accumulate = true;
        k_block_spmm<BD><<<(sa.rows0 * SPMM_LANES + 255) / 256, 256, 0, s>>>(sa);
        RPB_CUDA(cudaGetLastError());
    }
    PostArgs<BD> po;
    po.N = m->N; po.nV = m->nV; po.size = m->size;
    po.leaf_of = m->leaf_of.ptr; po.C_parent = m->C_parent.ptr; po.C_up4 = m->C_up4.ptr;
    po.Pout = m->buf_Pout.ptr; po.Cout = m->buf_Cout.ptr; po.Z = m->buf_Z.ptr;
    po.vp_rp = m->vp_rp.ptr; po.vp_slot = m->vp_slot.ptr; po.pre_vals = m->pre_vals.ptr;
    po.alpha = alpha; po.beta = beta; po.Y = Y; po.ldY = ldY;
    k_post_primitives<BD><<<static_cast<int>((static_cast<int64_t>(m->N) * POST_LANES + 255) / 256), 256, 0, s>>>(po);
    RPB_CUDA(cudaGetLastError());
    k_post_vertices<BD><<<static_cast<int>((static_cast<int64_t>(m->nV) * POST_LANES + 255) / 256), 256, 0, s>>>(po);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status metric_multiply_dev(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX, double beta,
                               double* Y, int ldY, int flags)
{
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    if (!m->geometry_valid && (st = launch_geometry(m)) != RPB_OK) return st;
    if ((st = ensure_metric_values(m, q, p)) != RPB_OK) return st;
    const MetricCache& mc = m->metric;
    return apply_operator<12>(m, mc.nf.ptr, mc.nf_diag.ptr, mc.ff.ptr, mc.ff_diag.ptr, mc.vf.ptr, mc.vf_diag.ptr,
                              alpha, X, ldX, beta, Y, ldY, flags);
}

rpb_status plap_multiply_dev(rpb_mesh* m, double s_pl, double alpha, const double* X, int ldX, double beta, double* Y,
                             int ldY)
{
    rpb_status st;
    if (!m->geometry_valid && (st = launch_geometry(m)) != RPB_OK) return st;
    if ((st = ensure_plap_values(m, s_pl)) != RPB_OK) return st;
    const PseudoLapCache& pc = m->plap;
    return apply_operator<3>(m, reinterpret_cast<const float2*>(pc.nf.ptr), reinterpret_cast<const double2*>(pc.nf_diag.ptr),
                             reinterpret_cast<const float2*>(pc.ff.ptr), reinterpret_cast<const double2*>(pc.ff_diag.ptr),
                             reinterpret_cast<const float2*>(pc.vf.ptr), reinterpret_cast<const double2*>(pc.vf_diag.ptr),
                             alpha, X, ldX, beta, Y, ldY, 7);
}

}  // namespace rpb

using namespace rpb;

extern "C" {

rpb_status rpb_tpm0_multiply_device(rpb_mesh* m, double q, double p, double alpha, const double* X_dev, int ldX,
                                    double beta, double* Y_dev, int ldY, int nrhs, int flags)
{
    if (!m || !X_dev || !Y_dev) { set_error("null argument"); return RPB_EINVAL; }
    if (nrhs != 3) {
        set_error("MultiplyMetric: nrhs = " + std::to_string(nrhs) + " != 3 = AMB_DIM. Only nrhs = AMB_DIM is accepted.");
        return RPB_EINVAL;
    }
    if (ldX < 3 || ldY < 3) { set_error("leading dimensions must be >= 3"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    return metric_multiply_dev(m, q, p, alpha, X_dev, ldX, beta, Y_dev, ldY, flags);
}

rpb_status rpb_tpm0_multiply(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX, double beta,
                             double* Y, int ldY, int nrhs, int flags)
{
    if (!m || !X || !Y) { set_error("null argument"); return RPB_EINVAL; }
    if (nrhs != 3) {
        set_error("MultiplyMetric: nrhs = " + std::to_string(nrhs) + " != 3 = AMB_DIM. Only nrhs = AMB_DIM is accepted.");
        return RPB_EINVAL;
    }
    if (ldX < 3 || ldY < 3) { set_error("leading dimensions must be >= 3"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = m->stream;
    RPB_CUDA(copy_rows3(m->X.ptr, 3, X, ldX, m->nV, cudaMemcpyHostToDevice, s));
    if (beta != 0.0)
        RPB_CUDA(copy_rows3(m->Yb.ptr, 3, Y, ldY, m->nV, cudaMemcpyHostToDevice, s));
    rpb_status st = metric_multiply_dev(m, q, p, alpha, m->X.ptr, 3, beta, m->Yb.ptr, 3, flags);
    if (st != RPB_OK) return st;
    RPB_CUDA(copy_rows3(Y, ldY, m->Yb.ptr, 3, m->nV, cudaMemcpyDeviceToHost, s));
    RPB_CUDA(cudaStreamSynchronize(s));
    return RPB_OK;
}

}  // extern "C"
