// Learned per-cluster preconditioner for the metric Solve (flexible CG).
//
// For a residual r (vertices x 3) the preconditioner returns z = M(r):
//   1. cluster residual moments R_C = sum_{i in C} a_i mean(r over simplex i): row 0 of
//      the Pre operator (src/ClusterTree.hpp:770-857) followed by the upward sums over
//      the tree, done as range sums over prefix sums (clusters are contiguous ranges),
//   2. 16 features per cluster: R_C / (A_C s) (3, s = RMS of r), centre relative to the
//      root / root diameter (3), averaged unit normal sum(a n)/A (3), log(A_C/A_root)/10,
//      log(d_C/d_root)/10, depth / max depth, and the 4 child-residual norms
//      |R_L|/(A_L s), |R_R|/(A_R s), |R_LL + R_LR|/(A_L s), |R_RL + R_RR|/(A_R s)
//      (zero where the children do not exist),
//   3. an MLP 16 -> 64 -> 64 -> 3 with GELU, BF16 weights and FP32 accumulation gives
//      o_C; the per-component gains g_C = exp(clamp(o_C, +-3)) scale the multilevel
//      coefficient c_C = g_C * R_C * w_C, w_C = (A_C / A_root)^kLevelExponent / A_C,
//   4. every primitive gets Z_i = sum over the clusters containing i of c_C
//      (PercolateDown + ClustersToPrimitives, src/ClusterTree.hpp:706-768) and every
//      vertex z_v = sum_{i at v} a_i/(n+1) Z_i (the transpose of step 1), minus the
//      column means (translations are the kernel of the metric).
// With all gains 1 this is the fixed symmetric positive definite multilevel operator
// W^T E diag(w_C) E^T W; the gains make it nonlinear but homogeneous of degree one in r,
// and z . r > 0 always, so flexible CG cannot break down on it.
//
// Training (rpb_mlp_train_step) on (residual r, correction e) pairs with A e = r: the loss
// 1 - (z.r)^2 / ((z.Az)(e.r)) is the share of ||e||_A^2 that the best step along z = M(r)
// leaves; one metric product Az per pair. Its adjoint runs steps 4 -> 1 backwards
// (primitive moments and range sums again), then the MLP backward pass; weight gradients
// are split-K reductions over the clusters; Adam on FP32 master weights that are rounded
// to the BF16 copy the kernels read.
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "kernels_energy.cuh"
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

constexpr int NF = 16, NH = 64, NO = 3;
constexpr int OFF_W1 = 0;                     // NH x NF
constexpr int OFF_B1 = OFF_W1 + NH * NF;      // NH
constexpr int OFF_W2 = OFF_B1 + NH;           // NH x NH
constexpr int OFF_B2 = OFF_W2 + NH * NH;      // NH
constexpr int OFF_W3 = OFF_B2 + NH;           // NO x NH
constexpr int OFF_B3 = OFF_W3 + NO * NH;      // NO
constexpr int NPARAM = OFF_B3 + NO;           // 5443

// GELU x Phi(x), Phi from the complementary error function of Abramowitz & Stegun 7.1.26
// (absolute error <= 1.5e-7): Phi(-|x|) = 0.5 t P(t) exp(-x^2 / 2), t = 1 / (1 + p |x| / sqrt 2).
// Two MUFU operations (reciprocal, exponential); the activations are rounded to BF16 next.
__device__ __forceinline__ float gelu(float x)
{
    const float z = fabsf(x) * 0.70710678118654752f;
    const float t = __fdividef(1.0f, fmaf(0.3275911f, z, 1.0f));
    const float poly =
        t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
    const float h = 0.5f * poly * __expf(-z * z);
    return x * (x < 0.0f ? h : 1.0f - h);
}
__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// ------------------------------------------------------------------------------------------
// MLP forward / backward, one thread per cluster; weights staged in shared memory as FP32
// from their BF16 copies.
// ------------------------------------------------------------------------------------------
__device__ void stage_weights(const __nv_bfloat16* w, float* sw)
{
    for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) sw[k] = __bfloat162float(w[k]);
    __syncthreads();
}

struct MlpArgs {
    int n;
    const __nv_bfloat16* w;   // NPARAM BF16 weights
    const float* F;           // n x NF
    float* O;                 // n x NO
    float* pre1;              // n x NH (training only)
    float* pre2;              // n x NH (training only)
};

// ------------------------------------------------------------------------------------------
// Forward pass on the tensor cores: a block of 4 warps takes 128 clusters, each warp two
// 16-row tiles; mma.sync m16n8k16 with BF16 operands and FP32 accumulation. Activations
// enter each layer as BF16 (features, GELU outputs), pre-activations and outputs stay FP32.
// Weights are staged to shared memory as BF16 with padded row strides, so that the
// fragment loads of a warp hit 32 distinct banks.
// ------------------------------------------------------------------------------------------
constexpr int MLP_TILE = 128;
constexpr int SF_LD = 24, SH_LD = 72, W1_LD = 24, W2_LD = 72, W3_LD = 72;

struct MlpSmem {
    __nv_bfloat16 W1[NH * W1_LD];
    __nv_bfloat16 W2[NH * W2_LD];
    __nv_bfloat16 W3[8 * W3_LD];          // rows 3..7 zero
    float b1[NH], b2[NH], b3[8];
    __nv_bfloat16 F[MLP_TILE * SF_LD];
    __nv_bfloat16 H[MLP_TILE * SH_LD];
    float O[MLP_TILE * 4];
};

__device__ void stage_mlp_weights(const __nv_bfloat16* w, MlpSmem& sm)
{
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    for (int k = threadIdx.x; k < NH * NF; k += blockDim.x) sm.W1[(k / NF) * W1_LD + k % NF] = w[OFF_W1 + k];
    for (int k = threadIdx.x; k < NH * NH; k += blockDim.x) sm.W2[(k / NH) * W2_LD + k % NH] = w[OFF_W2 + k];
    for (int k = threadIdx.x; k < 8 * NH; k += blockDim.x)
        sm.W3[(k / NH) * W3_LD + k % NH] = (k < NO * NH) ? w[OFF_W3 + k] : zero;
    for (int k = threadIdx.x; k < NH; k += blockDim.x) {
        sm.b1[k] = __bfloat162float(w[OFF_B1 + k]);
        sm.b2[k] = __bfloat162float(w[OFF_B2 + k]);
    }
    if (threadIdx.x < 8) sm.b3[threadIdx.x] = threadIdx.x < NO ? __bfloat162float(w[OFF_B3 + threadIdx.x]) : 0.0f;
}

__device__ __forceinline__ uint32_t ld_bf16x2(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_16816(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One warp: rows 32 w .. 32 w + 31 of the tile (features in sm.F) -> outputs in sm.O;
// pre1/pre2 (training, may be null) receive the FP32 pre-activations of the valid rows
// (global row = row0 + tile row, valid below n).
__device__ void mlp_tile(MlpSmem& sm, int row0, int n, float* pre1, float* pre2)
{
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[2][8][4];
    // layer 1: [32 x 16] x [16 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r = 32 * w + 16 * mt + g;
        uint32_t a[4] = {ld_bf16x2(sm.F + r * SF_LD + 2 * t), ld_bf16x2(sm.F + (r + 8) * SF_LD + 2 * t),
                         ld_bf16x2(sm.F + r * SF_LD + 2 * t + 8), ld_bf16x2(sm.F + (r + 8) * SF_LD + 2 * t + 8)};
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int col = 8 * nt + g;
            const uint32_t bb[2] = {ld_bf16x2(sm.W1 + col * W1_LD + 2 * t), ld_bf16x2(sm.W1 + col * W1_LD + 2 * t + 8)};
            acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
            mma_16816(acc[mt][nt], a, bb);
        }
    }
    auto epilogue = [&](const float* bias, float* pre) {
        __syncwarp();
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int r = 32 * w + 16 * mt + g, col = 8 * nt + 2 * t;
                const float v00 = acc[mt][nt][0] + bias[col], v01 = acc[mt][nt][1] + bias[col + 1];
                const float v10 = acc[mt][nt][2] + bias[col], v11 = acc[mt][nt][3] + bias[col + 1];
                if (pre) {
                    if (row0 + r < n) *reinterpret_cast<float2*>(pre + NH * static_cast<int64_t>(row0 + r) + col) = make_float2(v00, v01);
                    if (row0 + r + 8 < n) *reinterpret_cast<float2*>(pre + NH * static_cast<int64_t>(row0 + r + 8) + col) = make_float2(v10, v11);
                }
                *reinterpret_cast<uint32_t*>(sm.H + r * SH_LD + col) = pack_bf16x2(gelu(v00), gelu(v01));
                *reinterpret_cast<uint32_t*>(sm.H + (r + 8) * SH_LD + col) = pack_bf16x2(gelu(v10), gelu(v11));
            }
        __syncwarp();
    };
    epilogue(sm.b1, pre1);
    // layer 2: [32 x 64] x [64 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = 32 * w + 16 * mt + g, k0 = 16 * ks + 2 * t;
            uint32_t a[4] = {ld_bf16x2(sm.H + r * SH_LD + k0), ld_bf16x2(sm.H + (r + 8) * SH_LD + k0),
                             ld_bf16x2(sm.H + r * SH_LD + k0 + 8), ld_bf16x2(sm.H + (r + 8) * SH_LD + k0 + 8)};
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int col = 8 * nt + g;
                const uint32_t bb[2] = {ld_bf16x2(sm.W2 + col * W2_LD + k0), ld_bf16x2(sm.W2 + col * W2_LD + k0 + 8)};
                mma_16816(acc[mt][nt], a, bb);
            }
        }
    epilogue(sm.b2, pre2);
    // layer 3: [32 x 64] x [64 x 8] (3 outputs)
    float o[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = 32 * w + 16 * mt + g, k0 = 16 * ks + 2 * t;
            uint32_t a[4] = {ld_bf16x2(sm.H + r * SH_LD + k0), ld_bf16x2(sm.H + (r + 8) * SH_LD + k0),
                             ld_bf16x2(sm.H + r * SH_LD + k0 + 8), ld_bf16x2(sm.H + (r + 8) * SH_LD + k0 + 8)};
            const uint32_t bb[2] = {ld_bf16x2(sm.W3 + g * W3_LD + k0), ld_bf16x2(sm.W3 + g * W3_LD + k0 + 8)};
            mma_16816(o[mt], a, bb);
        }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r = 32 * w + 16 * mt + g, col = 2 * t;
        if (col < NO) {
            sm.O[r * 4 + col] = o[mt][0] + sm.b3[col];
            sm.O[(r + 8) * 4 + col] = o[mt][2] + sm.b3[col];
        }
        if (col + 1 < NO) {
            sm.O[r * 4 + col + 1] = o[mt][1] + sm.b3[col + 1];
            sm.O[(r + 8) * 4 + col + 1] = o[mt][3] + sm.b3[col + 1];
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(MLP_TILE) k_mlp_forward(MlpArgs A)
{
    __shared__ MlpSmem sm;
    stage_mlp_weights(A.w, sm);
    const int row0 = blockIdx.x * MLP_TILE;
    const int c = row0 + threadIdx.x;
    for (int k = 0; k < NF; ++k)
        sm.F[threadIdx.x * SF_LD + k] = __float2bfloat16_rn(c < A.n ? A.F[NF * static_cast<int64_t>(c) + k] : 0.0f);
    __syncthreads();
    mlp_tile(sm, row0, A.n, A.pre1, A.pre2);
    __syncthreads();
    if (c < A.n)
        for (int q = 0; q < NO; ++q) A.O[NO * static_cast<int64_t>(c) + q] = sm.O[threadIdx.x * 4 + q];
}

struct MlpBackArgs {
    int n;
    const __nv_bfloat16* w;
    const float* dO;          // n x NO
    const float* pre1;
    const float* pre2;
    float* d2;                // n x NH: dL/dpre2
    float* d1;                // n x NH: dL/dpre1
};

__global__ void __launch_bounds__(128) k_mlp_backward(MlpBackArgs A)
{
    extern __shared__ float sw[];
    stage_weights(A.w, sw);
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.n) return;
    const float do0 = A.dO[NO * static_cast<int64_t>(c)], do1 = A.dO[NO * static_cast<int64_t>(c) + 1],
                do2 = A.dO[NO * static_cast<int64_t>(c) + 2];
    float g2[NH];
#pragma unroll 4
    for (int j = 0; j < NH; ++j) {
        const float dh2 = sw[OFF_W3 + j] * do0 + sw[OFF_W3 + NH + j] * do1 + sw[OFF_W3 + 2 * NH + j] * do2;
        g2[j] = dh2 * gelu_grad(A.pre2[NH * static_cast<int64_t>(c) + j]);
        A.d2[NH * static_cast<int64_t>(c) + j] = g2[j];
    }
    for (int k = 0; k < NH; ++k) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < NH; ++j) s = fmaf(sw[OFF_W2 + NH * j + k], g2[j], s);
        A.d1[NH * static_cast<int64_t>(c) + k] = s * gelu_grad(A.pre1[NH * static_cast<int64_t>(c) + k]);
    }
}

// Split-K weight gradient: partial[b][p][q] = sum_{n in chunk b} G[n][p] * act(X[n][q]),
// with act = identity (X = features) or GELU (X = pre-activations); column p = P means the
// bias gradient (sum of G). P <= 64, Q <= 64.
constexpr int WG_CHUNK = 1024;

// The forward pass feeds each layer BF16 activations, so X (or GELU(X)) is rounded to BF16
// here as well.
__global__ void __launch_bounds__(256) k_weight_grad(int n, const float* G, int P, const float* X, int Q, bool gelu_x,
                                                     float* partial)
{
    __shared__ float sg[32][65];
    __shared__ float sx[32][65];
    const int n0 = blockIdx.x * WG_CHUNK, n1 = min(n, n0 + WG_CHUNK);
    constexpr int OUT_PER_THREAD = (65 * 64 + 255) / 256;
    float acc[OUT_PER_THREAD];
#pragma unroll
    for (int t = 0; t < OUT_PER_THREAD; ++t) acc[t] = 0.0f;
    const int total = P * (Q + 1);
    for (int base = n0; base < n1; base += 32) {
        // columns 0..Q-1: activations, column Q: 1 (the bias), beyond: 0
        for (int e = threadIdx.x; e < 32 * 65; e += blockDim.x) {
            const int r = e / 65, col = e % 65, row = base + r;
            const bool valid = row < n1;
            if (col < 64) sg[r][col] = (valid && col < P) ? G[static_cast<int64_t>(P) * row + col] : 0.0f;
            float x = 0.0f;
            if (valid && col < Q) {
                x = X[static_cast<int64_t>(Q) * row + col];
                if (gelu_x) x = gelu(x);
                x = __bfloat162float(__float2bfloat16_rn(x));
            } else if (valid && col == Q) {
                x = 1.0f;
            }
            sx[r][col] = x;
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < OUT_PER_THREAD; ++t) {
            const int o = threadIdx.x + 256 * t;
            if (o < total) {
                const int p = o / (Q + 1), q = o % (Q + 1);
                float s = acc[t];
#pragma unroll 8
                for (int r = 0; r < 32; ++r) s = fmaf(sg[r][p], sx[r][q], s);
                acc[t] = s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int t = 0; t < OUT_PER_THREAD; ++t) {
        const int o = threadIdx.x + 256 * t;
        if (o < total) partial[static_cast<int64_t>(blockIdx.x) * total + o] = acc[t];
    }
}

// grad[p][q] (weights) and grad_b[p] (bias) = sum over blocks of the partials (fixed order)
__global__ void k_reduce_grad(int nblocks, int P, int Q, const float* partial, float* gW, float* gb)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = P * (Q + 1);
    if (o >= total) return;
    float s = 0.0f;
    for (int b = 0; b < nblocks; ++b) s += partial[static_cast<int64_t>(b) * total + o];
    const int p = o / (Q + 1), q = o % (Q + 1);
    if (q < Q) gW[Q * p + q] = s;
    else gb[p] = s;
}

__global__ void k_adam(int n, float* theta, __nv_bfloat16* w16, const float* g, float* m, float* v, float lr,
                       float b1, float b2, float eps, float bc1, float bc2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float t = theta[k] - lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
    theta[k] = t;
    w16[k] = __float2bfloat16_rn(t);
}

// ------------------------------------------------------------------------------------------
// The preconditioner application in five launches:
//   k_prim_scan     primitive moments a_i mean(r) -> in-block prefix sums; sum of |r|^2
//   k_scan_totals   prefix sums of the block totals; the global sum of |r|^2
//   k_cluster_mlp   per cluster: R_C (and its children's) as prefix-sum differences,
//                   16 features, the MLP, gains, c_C = g_C R_C w_C; sum_C A_C c_C
//   k_prim_expand   Z_i = sum_{C containing i} c_C
//   k_vertex_expand z_v = sum_{i at v} w_i Z_i - mean(z)
// ------------------------------------------------------------------------------------------
constexpr int GAIN_BLOCK = 128;
// Gains g_C = exp(clamp(o_C)) keep z . r > 0 for every residual (flexible CG never meets
// r . z <= 0) and bound the nonlinearity of the preconditioner to [e^-3, e^3] times the
// fixed multilevel operator.
constexpr float GAIN_CLAMP = 3.0f;

struct PrimScanArgs {
    int N, nV, size;
    const int* pre_cols;
    const double* pre_vals;
    const double* R;          // n_v x 3
    double* local;            // N x 3 in-block exclusive prefix sums
    double* blocks;           // (nb + 1) x 3 block totals -> exclusive prefix (row nb: total)
    double* sq_part;          // nb partial sums of |r|^2
};

__global__ void __launch_bounds__(SCAN_BLOCK) k_prim_scan(PrimScanArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[3] = {0, 0, 0}, tot[3];
    if (i < A.N)
        for (int l = 0; l < A.size; ++l) {
            const int u = A.pre_cols[A.size * i + l];
            const double w = A.pre_vals[(4 * static_cast<int64_t>(i)) * A.size + l];
            v[0] += w * A.R[3 * static_cast<int64_t>(u)];
            v[1] += w * A.R[3 * static_cast<int64_t>(u) + 1];
            v[2] += w * A.R[3 * static_cast<int64_t>(u) + 2];
        }
    block_exclusive_scan<3>(v, tot);
    if (i < A.N)
        for (int k = 0; k < 3; ++k) A.local[3 * static_cast<int64_t>(i) + k] = v[k];
    if (threadIdx.x < 3) A.blocks[3 * static_cast<int64_t>(blockIdx.x) + threadIdx.x] = tot[threadIdx.x];
    // |r|^2 over the vertices, grid-strided
    double sq = 0;
    for (int u = i; u < A.nV; u += gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const double x = A.R[3 * static_cast<int64_t>(u) + k];
            sq += x * x;
        }
    __shared__ double sh[SCAN_BLOCK / 32];
    sq = warp_sum_f64(sq);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < SCAN_BLOCK / 32; ++w) t += sh[w];
        A.sq_part[blockIdx.x] = t;
    }
}

// one block: exclusive prefix of the nb block totals (row nb: the total) and the scale
// s = sqrt(sum |r|^2 / (3 n_v))
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_totals(int nb, int nV, double* blocks, const double* sq_part,
                                                            double* scale)
{
    double sq = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) sq += sq_part[b];
    __shared__ double sh[SCAN_BLOCK / 32];
    sq = warp_sum_f64(sq);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < SCAN_BLOCK / 32; ++w) t += sh[w];
        *scale = sqrt(t / (3.0 * nV));
    }
    __syncthreads();
    __shared__ double carry[3];
    if (threadIdx.x < 3) carry[threadIdx.x] = 0.0;
    __syncthreads();
    for (int base = 0; base < nb; base += SCAN_BLOCK) {
        const int i = base + threadIdx.x;
        double v[3], tot[3];
        for (int k = 0; k < 3; ++k) v[k] = (i < nb) ? blocks[3 * static_cast<int64_t>(i) + k] : 0.0;
        block_exclusive_scan<3>(v, tot);
        if (i < nb)
            for (int k = 0; k < 3; ++k) blocks[3 * static_cast<int64_t>(i) + k] = carry[k] + v[k];
        __syncthreads();
        if (threadIdx.x < 3) carry[threadIdx.x] += tot[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x < 3) blocks[3 * static_cast<int64_t>(nb) + threadIdx.x] = carry[threadIdx.x];
}

struct ClusterMlpArgs {
    int N, NC, nV, max_depth;
    const __nv_bfloat16* w;
    const ClusterDatum* C_pair;
    const double* C_an;       // NC x 3: sum of a n over the cluster
    const int* C_begin;
    const int* C_end;
    const int* C_left;
    const int* C_right;
    const int* C_depth;
    const float* C_diam;
    const double* local;      // prefix sums of the primitive moments (k_prim_scan / k_scan_totals)
    const double* blocks;
    const double* scale;
    double* c;                // NC x 3: coefficients
    const float* Fs;          // NC x NFS: the geometric features 3..11 (k_static_features)
    double* csum_part;        // units x 3: partial sums of A_C c_C per 32-cluster unit
    unsigned* done;           // [0] last-block counter, [1] unit counter (zero between launches)
    double* zmean;            // 3: sum_C A_C c_C / n_v = mean of z before its removal
    // training only (may be null)
    float* F;                 // NC x NF
    float* O;                 // NC x NO
    float* pre1;              // NC x NH
    float* pre2;              // NC x NH
    double* Rc;               // NC x 3
    const double* C_w;        // NC: level weights (A_C / A_root)^kLevelExponent / A_C
};

__device__ __forceinline__ void prefix_at(const double* local, const double* blocks, int N, int k, double* out)
{
    const int nb = (N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    if (k < N) {
        for (int q = 0; q < 3; ++q) out[q] = blocks[3 * static_cast<int64_t>(k / SCAN_BLOCK) + q] + local[3 * static_cast<int64_t>(k) + q];
    } else {
        for (int q = 0; q < 3; ++q) out[q] = blocks[3 * static_cast<int64_t>(nb) + q];
    }
}

__device__ __forceinline__ void cluster_moment(const ClusterMlpArgs& A, int C, double* R)
{
    double sb[3], se[3];
    prefix_at(A.local, A.blocks, A.N, A.C_begin[C], sb);
    prefix_at(A.local, A.blocks, A.N, A.C_end[C], se);
    for (int q = 0; q < 3; ++q) R[q] = se[q] - sb[q];
}

// Level exponent of the multilevel coefficients c_C = g_C R_C w_C, w_C = (A_C / A_root)^k / A_C.
// k = 0 weights every level of the tree alike; chosen by FCG iteration counts of the
// untrained operator (all gains 1) on spherical-harmonic icospheres, plain CG residual
// 1e-6, q = 6, p = 12: level 5 / 6 / 7 take 735 / 2,037 / 3,945 iterations at k = 0
// (level 7 stalls into the fallback), 655 / 1,474 / 3,440 at k = 0.5; on level 6, 0.4 and
// 0.6 are within 15 % of 0.5, 0.8 is worse than 0, 1 needs 5,756 and k >= 1.33 stalls.
constexpr double kLevelExponent = 0.5;

// Geometric features of the clusters (3..11 of the 16), once per geometry: centre
// relative to the root over the root diameter, averaged normal, log area ratio, log
// diameter ratio, depth; and the level weights w_C.
constexpr int NFS = 9;
__global__ void k_static_features(int NC, int max_depth, const ClusterDatum* C_pair, const double* C_an,
                                  const float* C_diam, const int* C_depth, float* Fs, double* C_w)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= NC) return;
    const ClusterDatum cd = load_datum(C_pair, C);
    const ClusterDatum root = load_datum(C_pair, 0);
    const double dr = fmax(static_cast<double>(C_diam[0]), 1e-300);
    float* f = Fs + NFS * static_cast<int64_t>(C);
    for (int k = 0; k < 3; ++k) f[k] = static_cast<float>((cd.c[k] - root.c[k]) / dr);
    for (int k = 0; k < 3; ++k) f[3 + k] = static_cast<float>(C_an[3 * static_cast<int64_t>(C) + k] / cd.a);
    f[6] = static_cast<float>(log(cd.a / root.a) / 10.0);
    f[7] = static_cast<float>(log(fmax(static_cast<double>(C_diam[C]), 1e-300) / dr) / 10.0);
    f[8] = static_cast<float>(C_depth[C]) / static_cast<float>(max(max_depth, 1));
    C_w[C] = pow(cd.a / root.a, kLevelExponent) / cd.a;
}

// Persistent: every block stages the weights once, then each of its warps takes units of
// 32 clusters from a global counter (lane = cluster) until none are left: features, the
// MLP on the warp's own 32 rows of the shared tile, gains and coefficients. Per-unit
// partial sums of A_C c_C are added by the last block in unit order (deterministic
// whatever warp took which unit); it also resets both counters.
__global__ void __launch_bounds__(GAIN_BLOCK, 4) k_cluster_mlp(ClusterMlpArgs A)
{
    static_assert(GAIN_BLOCK == MLP_TILE, "one MLP tile per block");
    __shared__ MlpSmem sm;
    __shared__ bool last;
    stage_mlp_weights(A.w, sm);
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int units = (A.NC + 31) / 32;
    const double s = fmax(*A.scale, 1e-300);
    for (;;) {
        int u = 0;
        if (lane == 0) u = static_cast<int>(atomicAdd(A.done + 1, 1u));
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= units) break;
        const int C = 32 * u + lane;
        double cs[3] = {0, 0, 0};
        float f[NF];
        for (int k = 0; k < NF; ++k) f[k] = 0.0f;
        double R[3] = {0, 0, 0};
        double ca = 1.0;
        if (C < A.NC) {
            ca = __ldg(&A.C_pair[C].a);
            cluster_moment(A, C, R);
            for (int k = 0; k < 3; ++k) f[k] = static_cast<float>(R[k] / (ca * s));
            const float* fs = A.Fs + NFS * static_cast<int64_t>(C);
            for (int k = 0; k < NFS; ++k) f[3 + k] = __ldg(fs + k);
            const int L = A.C_left[C], Rr = A.C_right[C];
            if (L >= 0) {
                const double aL = __ldg(&A.C_pair[L].a), aR = __ldg(&A.C_pair[Rr].a);
                double q[3];
                cluster_moment(A, L, q);
                f[12] = static_cast<float>(sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) / (aL * s));
                cluster_moment(A, Rr, q);
                f[13] = static_cast<float>(sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) / (aR * s));
                // children of L together span L: R_LL + R_LR = R_L (as in the reference tree, a
                // cluster is the union of its children); the grandchildren feature uses them
                if (A.C_left[L] >= 0) {
                    double a[3], b[3];
                    cluster_moment(A, A.C_left[L], a);
                    cluster_moment(A, A.C_right[L], b);
                    f[14] = static_cast<float>(sqrt((a[0] + b[0]) * (a[0] + b[0]) + (a[1] + b[1]) * (a[1] + b[1]) +
                                                    (a[2] + b[2]) * (a[2] + b[2])) / (aL * s));
                }
                if (A.C_left[Rr] >= 0) {
                    double a[3], b[3];
                    cluster_moment(A, A.C_left[Rr], a);
                    cluster_moment(A, A.C_right[Rr], b);
                    f[15] = static_cast<float>(sqrt((a[0] + b[0]) * (a[0] + b[0]) + (a[1] + b[1]) * (a[1] + b[1]) +
                                                    (a[2] + b[2]) * (a[2] + b[2])) / (aR * s));
                }
            }
        }
        const int row = 32 * w + lane;
        for (int k = 0; k < NF; ++k) sm.F[row * SF_LD + k] = __float2bfloat16_rn(f[k]);
        __syncwarp();
        mlp_tile(sm, 32 * u - 32 * w, A.NC, A.pre1, A.pre2);
        if (C < A.NC) {
            float o[NO];
            for (int q = 0; q < NO; ++q) o[q] = sm.O[row * 4 + q];
            const double inv_a = __ldg(A.C_w + C);
            for (int q = 0; q < 3; ++q) {
                const float oc = fminf(fmaxf(o[q], -GAIN_CLAMP), GAIN_CLAMP);
                const double cq = exp(static_cast<double>(oc)) * R[q] * inv_a;
                A.c[3 * static_cast<int64_t>(C) + q] = cq;
                cs[q] = ca * cq;
            }
            if (A.F)
                for (int k = 0; k < NF; ++k) A.F[NF * static_cast<int64_t>(C) + k] = f[k];
            if (A.O)
                for (int q = 0; q < NO; ++q) A.O[NO * static_cast<int64_t>(C) + q] = o[q];
            if (A.Rc)
                for (int q = 0; q < 3; ++q) A.Rc[3 * static_cast<int64_t>(C) + q] = R[q];
        }
        for (int q = 0; q < 3; ++q) {
            const double v = warp_sum_f64(cs[q]);
            if (lane == 0) A.csum_part[3 * static_cast<int64_t>(u) + q] = v;
        }
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(A.done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        // thread t adds units t, t + GAIN_BLOCK, ... ; then a fixed tree over the threads
        double t3[3] = {0, 0, 0};
        for (int v = threadIdx.x; v < units; v += GAIN_BLOCK)
            for (int q = 0; q < 3; ++q) t3[q] += __ldcg(A.csum_part + 3 * static_cast<int64_t>(v) + q);
        __shared__ double sh[GAIN_BLOCK / 32][3];
        for (int q = 0; q < 3; ++q) {
            const double v = warp_sum_f64(t3[q]);
            if (lane == 0) sh[w][q] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double t = 0;
            for (int k = 0; k < GAIN_BLOCK / 32; ++k) t += sh[k][threadIdx.x];
            A.zmean[threadIdx.x] = t / A.nV;
        }
        if (threadIdx.x == 0) {
            A.done[0] = 0u;
            A.done[1] = 0u;
        }
    }
}

// Z_i = sum over the clusters containing primitive i of c_C (PercolateDown +
// ClustersToPrimitives as an ancestor walk). EXPAND_LANES consecutive lanes per primitive
// (vertex): lane p takes the ancestors at distances p, p + 4, ... (the vertex's slots
// p, p + 4, ...), an xor butterfly combines the partial sums, lane k < 3 writes component k.
constexpr int EXPAND_LANES = 4;

__global__ void k_prim_expand(int N, const int* leaf_of, const int* C_parent, const int* C_up4, const double* c,
                              double* Z)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / EXPAND_LANES, lane = t % EXPAND_LANES;
    const bool active = i < N;
    double z[3] = {0, 0, 0};
    if (active) {
        int C = leaf_of[i];
        for (int k = 0; k < lane && C >= 0; ++k) C = __ldg(C_parent + C);
        for (; C >= 0; C = __ldg(C_up4 + C))
            for (int m = 0; m < 3; ++m) z[m] += c[3 * static_cast<int64_t>(C) + m];
    }
#pragma unroll
    for (int off = 1; off < EXPAND_LANES; off <<= 1)
#pragma unroll
        for (int m = 0; m < 3; ++m) z[m] += __shfl_xor_sync(0xffffffffu, z[m], off);
    if (!active || lane >= 3) return;
    Z[3 * static_cast<int64_t>(i) + lane] = lane == 0 ? z[0] : (lane == 1 ? z[1] : z[2]);
}

// z_v = sum over the primitives i at v of w_i Z_i, minus the mean of z (translations are
// the kernel of the metric)
__global__ void k_vertex_expand(int nV, int size, const int* vp_rp, const int* vp_slot, const double* pre_vals,
                                const double* Z, const double* zmean, double* z)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = t / EXPAND_LANES, lane = t % EXPAND_LANES;
    const bool active = v < nV;
    double a[3] = {0, 0, 0};
    const int k1 = active ? vp_rp[v + 1] : 0;
    for (int k = (active ? vp_rp[v] : 0) + lane; k < k1; k += EXPAND_LANES) {
        const int slot = vp_slot[k];
        const int i = slot / size, l = slot - i * size;
        const double w = pre_vals[(4 * static_cast<int64_t>(i)) * size + l];
        for (int m = 0; m < 3; ++m) a[m] += w * Z[3 * static_cast<int64_t>(i) + m];
    }
#pragma unroll
    for (int off = 1; off < EXPAND_LANES; off <<= 1)
#pragma unroll
        for (int m = 0; m < 3; ++m) a[m] += __shfl_xor_sync(0xffffffffu, a[m], off);
    if (!active || lane >= 3) return;
    z[3 * static_cast<int64_t>(v) + lane] = (lane == 0 ? a[0] : (lane == 1 ? a[1] : a[2])) - zmean[lane];
}

// per-primitive a*n (3) for the averaged-normal feature
__global__ void k_prim_an(int N, const PrimDatum* P, double* an)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const PrimDatum d = load_datum(P, i);
    for (int k = 0; k < 3; ++k) an[3 * static_cast<int64_t>(i) + k] = d.a * d.n[k];
}

// translation projection helpers: v -= mean (per column); mean from a device sum
__global__ void k_sub_mean(int n, double* v, const double* sums)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) v[3 * static_cast<int64_t>(i) + c] -= sums[c] / n;
}

// Energy-norm loss of one preconditioner application: with e the exact correction (A e = r),
// loss = 1 - (z.r)^2 / ((z.Az)(e.r)) = 1 - cos^2_A(z, e), the share of ||e||_A^2 that the
// best step along z leaves. Gradient wrt z: -2 (z.r)/((z.Az)(e.r)) r + 2 (z.r)^2/((z.Az)^2 (e.r)) Az.
// dots: [0..2] z.r, [3..5] z.Az, [6..8] e.r per column.
__global__ void k_loss_grad(int n, const double* r, const double* Az, const double* dots, double* g, double* loss_acc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double zr = dots[0] + dots[1] + dots[2];
    const double zAz = fmax(dots[3] + dots[4] + dots[5], 1e-300);
    const double er = fmax(dots[6] + dots[7] + dots[8], 1e-300);
    const double c1 = -2.0 * zr / (zAz * er), c2 = 2.0 * zr * zr / (zAz * zAz * er);
    if (i < n)
        for (int c = 0; c < 3; ++c)
            g[3 * static_cast<int64_t>(i) + c] = c1 * r[3 * static_cast<int64_t>(i) + c] + c2 * Az[3 * static_cast<int64_t>(i) + c];
    if (i == 0) *loss_acc += 1.0 - zr * zr / (zAz * er);
}

// dL/do_C = sum_q gc_Cq R_Cq w_C * g_Cq (zero where the clamp is active), plus the
// gradient 2 reg o_C / (3 N_C) of the gain penalty reg * mean(o^2)
__global__ void k_cluster_out_grad(int NC, const double* gc, const float* O, const double* Rc, const ClusterDatum* C_pair,
                                   float reg, const double* C_w, float* dO)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= NC) return;
    const double inv_a = C_w[C];
    for (int q = 0; q < 3; ++q) {
        const int64_t k = 3 * static_cast<int64_t>(C) + q;
        const float o = O[k];
        const bool inside = o > -GAIN_CLAMP && o < GAIN_CLAMP;
        dO[k] = (inside ? static_cast<float>(gc[k] * Rc[k] * inv_a * exp(static_cast<double>(o))) : 0.0f) +
                2.0f * reg * o / (3.0f * NC);
    }
}

// Coefficients of the preconditioner with the gains of an earlier application (O, the
// network's outputs for that residual) on the cluster moments Yc of another vector:
// c_C = exp(clamp(o_C)) Yc_C w_C. With them the application is the linear operator
// the earlier residual's gains define, which the unrolled-solve training needs for its
// adjoint pass.
__global__ void k_frozen_coef(int NC, const float* O, const double* Yc, const double* C_w, double* c)
{
    const int C = blockIdx.x * blockDim.x + threadIdx.x;
    if (C >= NC) return;
    for (int q = 0; q < 3; ++q) {
        const int64_t k = 3 * static_cast<int64_t>(C) + q;
        const float o = fminf(fmaxf(O[k], -GAIN_CLAMP), GAIN_CLAMP);
        c[k] = exp(static_cast<double>(o)) * Yc[k] * C_w[C];
    }
}

// out[c] = sum_i a[3i+c] * b[3i+c] (b == nullptr: column sums); one block, fixed order
__global__ void __launch_bounds__(512) k_dot3_single(int n, const double* a, const double* b, double* out)
{
    __shared__ double sh[16][3];
    double acc[3] = {0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int c = 0; c < 3; ++c) acc[c] += a[3 * static_cast<int64_t>(i) + c] * (b ? b[3 * static_cast<int64_t>(i) + c] : 1.0);
    for (int c = 0; c < 3; ++c) acc[c] = warp_sum_f64(acc[c]);
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 3; ++c) sh[threadIdx.x >> 5][c] = acc[c];
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) t += sh[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
}

// per-primitive residual moment a_i * mean(r over the simplex) (row 0 of the Pre operator)
__global__ void k_prim_moments(int N, int size, const int* pre_cols, const double* pre_vals, const double* R, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double a0 = 0, a1 = 0, a2 = 0;
    for (int l = 0; l < size; ++l) {
        const int v = pre_cols[size * i + l];
        const double w = pre_vals[(4 * static_cast<int64_t>(i)) * size + l];
        a0 += w * R[3 * static_cast<int64_t>(v)];
        a1 += w * R[3 * static_cast<int64_t>(v) + 1];
        a2 += w * R[3 * static_cast<int64_t>(v) + 2];
    }
    out[3 * static_cast<int64_t>(i)] = a0;
    out[3 * static_cast<int64_t>(i) + 1] = a1;
    out[3 * static_cast<int64_t>(i) + 2] = a2;
}

}  // namespace rpb

// ==========================================================================================
// host side
// ==========================================================================================
struct rpb_mlp {
    int device = 0;
    rpb::DevBuf<float> theta, grad, m, v, partial;
    rpb::DevBuf<__nv_bfloat16> w16;
    int64_t step = 0;
};

namespace rpb {

struct LearnedState {
    rpb_mlp* mlp = nullptr;
    int64_t geometry_version = -1;
    int max_depth = 0;
    DevBuf<double> C_an, tmp3, Rc, c, scale, sums, loss, gc, dots, g, r, z, e, Az;
    DevBuf<double> local, blocks, sq_part, csum_part, zmean, C_w;
    DevBuf<unsigned> done;
    DevBuf<float> F, O, dO, pre1, pre2, d1, d2, C_diam;
    DevBuf<int> C_depth;
    DevBuf<float> Fs;         // NC x NFS geometric features
    int mlp_grid = 0;         // resident blocks of k_cluster_mlp on the device
};

static rpb_status range_sums3(rpb_mesh* m, const double* prim3, double* out3)
{
    const int nb = (m->N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_block_scan_rows<3><<<nb, SCAN_BLOCK, 0, m->stream>>>(m->N, prim3, m->buf_scan_local.ptr, m->buf_scan_blocks.ptr);
    k_scan_rows<3><<<1, SCAN_BLOCK, 0, m->stream>>>(m->buf_scan_blocks.ptr, nb);
    k_range_sums<3><<<(m->NC + 255) / 256, 256, 0, m->stream>>>(m->N, m->NC, m->C_begin.ptr, m->C_end.ptr,
                                                                m->buf_scan_local.ptr, m->buf_scan_blocks.ptr, out3);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

static rpb_status ensure_learned(rpb_mesh* m)
{
    if (!m->learned) m->learned = new LearnedState();
    LearnedState& L = *m->learned;
    const size_t NC = m->NC, N = m->N, nV = m->nV;
    if (!L.F.ptr) {
        RPB_CUDA(L.C_an.alloc(3 * NC));
        RPB_CUDA(L.C_w.alloc(NC));
        RPB_CUDA(L.tmp3.alloc(3 * N));
        RPB_CUDA(L.Rc.alloc(3 * NC));
        RPB_CUDA(L.c.alloc(3 * NC));
        const size_t nb = (N + SCAN_BLOCK - 1) / SCAN_BLOCK;
        RPB_CUDA(L.local.alloc(3 * N));
        RPB_CUDA(L.blocks.alloc(3 * (nb + 1)));
        RPB_CUDA(L.sq_part.alloc(nb));
        RPB_CUDA(L.csum_part.alloc(3 * ((NC + 31) / 32)));
        RPB_CUDA(L.zmean.alloc(3));
        RPB_CUDA(L.done.alloc(2));
        RPB_CUDA(L.Fs.alloc(NFS * NC));
        int per_sm = 0, sms = 0;
        RPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cluster_mlp, GAIN_BLOCK, 0));
        RPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device));
        L.mlp_grid = std::max(1, per_sm * sms);
        RPB_CUDA(cudaMemsetAsync(L.done.ptr, 0, L.done.bytes(), m->stream));
        RPB_CUDA(L.scale.alloc(1));
        RPB_CUDA(L.sums.alloc(4));
        RPB_CUDA(L.loss.alloc(1));
        RPB_CUDA(L.gc.alloc(3 * NC));
        RPB_CUDA(L.dots.alloc(9));
        RPB_CUDA(L.g.alloc(3 * nV));
        RPB_CUDA(L.r.alloc(3 * nV));
        RPB_CUDA(L.z.alloc(3 * nV));
        RPB_CUDA(L.e.alloc(3 * nV));
        RPB_CUDA(L.Az.alloc(3 * nV));
        RPB_CUDA(L.F.alloc(NF * NC));
        RPB_CUDA(L.O.alloc(NO * NC));
        RPB_CUDA(L.dO.alloc(NO * NC));
        RPB_CUDA(L.C_diam.alloc(NC));
        RPB_CUDA(L.C_depth.alloc(NC));
        std::vector<float> diam(NC);
        for (size_t C = 0; C < NC; ++C) diam[C] = static_cast<float>(2.0 * std::sqrt(m->tree.C_box[7 * C]));
        RPB_CUDA(cudaMemcpyAsync(L.C_diam.ptr, diam.data(), L.C_diam.bytes(), cudaMemcpyHostToDevice, m->stream));
        RPB_CUDA(cudaMemcpyAsync(L.C_depth.ptr, m->tree.C_depth.data(), L.C_depth.bytes(), cudaMemcpyHostToDevice,
                                 m->stream));
        L.max_depth = m->tree.depth;
        RPB_CUDA(cudaStreamSynchronize(m->stream));
    }
    if (L.geometry_version != m->geometry_version) {
        k_prim_an<<<(m->N + 255) / 256, 256, 0, m->stream>>>(m->N, m->P_pair.ptr, L.tmp3.ptr);
        rpb_status st = range_sums3(m, L.tmp3.ptr, L.C_an.ptr);
        if (st != RPB_OK) return st;
        k_static_features<<<(m->NC + 255) / 256, 256, 0, m->stream>>>(m->NC, L.max_depth, m->C_pair.ptr, L.C_an.ptr,
                                                                      L.C_diam.ptr, L.C_depth.ptr, L.Fs.ptr, L.C_w.ptr);
        RPB_CUDA(cudaGetLastError());
        L.geometry_version = m->geometry_version;
    }
    return RPB_OK;
}

void learned_free(rpb_mesh* m)
{
    delete m->learned;
    m->learned = nullptr;
}

static rpb_status ensure_training_buffers(rpb_mesh* m)
{
    LearnedState& L = *m->learned;
    if (!L.pre1.ptr) {
        const size_t NC = m->NC;
        RPB_CUDA(L.pre1.alloc(NH * NC));
        RPB_CUDA(L.pre2.alloc(NH * NC));
        RPB_CUDA(L.d1.alloc(NH * NC));
        RPB_CUDA(L.d2.alloc(NH * NC));
    }
    return RPB_OK;
}

static rpb_status dot3_dev(rpb_mesh* m, const double* a, const double* b, double* out)
{
    k_dot3_single<<<1, 512, 0, m->stream>>>(m->nV, a, b, out);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

// R_C = sum over the cluster's primitives of a_i mean(r) (Pre row 0, then range sums)
static rpb_status cluster_moments(rpb_mesh* m, const double* R, double* Rc)
{
    k_prim_moments<<<(m->N + 255) / 256, 256, 0, m->stream>>>(m->N, m->size, m->pre_cols.ptr, m->pre_vals.ptr, R,
                                                              m->learned->tmp3.ptr);
    RPB_CUDA(cudaGetLastError());
    return range_sums3(m, m->learned->tmp3.ptr, Rc);
}

// z = M_learned(R) (device, n_v x 3) in five launches; with `training` the features,
// activations, outputs and cluster moments are kept for the backward pass.
static rpb_status learned_forward(rpb_mesh* m, rpb_mlp* mlp, const double* R, double* z, bool training)
{
    LearnedState& L = *m->learned;
    cudaStream_t s = m->stream;
    const int nb = (m->N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    PrimScanArgs ps;
    ps.N = m->N; ps.nV = m->nV; ps.size = m->size;
    ps.pre_cols = m->pre_cols.ptr; ps.pre_vals = m->pre_vals.ptr; ps.R = R;
    ps.local = L.local.ptr; ps.blocks = L.blocks.ptr; ps.sq_part = L.sq_part.ptr;
    k_prim_scan<<<nb, SCAN_BLOCK, 0, s>>>(ps);
    k_scan_totals<<<1, SCAN_BLOCK, 0, s>>>(nb, m->nV, L.blocks.ptr, L.sq_part.ptr, L.scale.ptr);
    ClusterMlpArgs ca;
    ca.N = m->N; ca.NC = m->NC; ca.nV = m->nV; ca.max_depth = L.max_depth;
    ca.w = mlp->w16.ptr; ca.C_pair = m->C_pair.ptr; ca.C_an = L.C_an.ptr;
    ca.C_begin = m->C_begin.ptr; ca.C_end = m->C_end.ptr; ca.C_left = m->C_left.ptr; ca.C_right = m->C_right.ptr;
    ca.C_depth = L.C_depth.ptr; ca.C_diam = L.C_diam.ptr;
    ca.local = L.local.ptr; ca.blocks = L.blocks.ptr; ca.scale = L.scale.ptr;
    ca.c = L.c.ptr; ca.csum_part = L.csum_part.ptr; ca.done = L.done.ptr; ca.zmean = L.zmean.ptr;
    ca.Fs = L.Fs.ptr;
    ca.C_w = L.C_w.ptr;
    ca.F = training ? L.F.ptr : nullptr;
    ca.O = training ? L.O.ptr : nullptr;
    ca.pre1 = training ? L.pre1.ptr : nullptr;
    ca.pre2 = training ? L.pre2.ptr : nullptr;
    ca.Rc = training ? L.Rc.ptr : nullptr;
    k_cluster_mlp<<<std::min(L.mlp_grid, (m->NC + GAIN_BLOCK - 1) / GAIN_BLOCK), GAIN_BLOCK, 0, s>>>(ca);
    k_prim_expand<<<(m->N * EXPAND_LANES + 255) / 256, 256, 0, s>>>(m->N, m->leaf_of.ptr, m->C_parent.ptr, m->C_up4.ptr, L.c.ptr,
                                                      L.tmp3.ptr);
    k_vertex_expand<<<(m->nV * EXPAND_LANES + 255) / 256, 256, 0, s>>>(m->nV, m->size, m->vp_rp.ptr, m->vp_slot.ptr, m->pre_vals.ptr,
                                                        L.tmp3.ptr, L.zmean.ptr, z);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status learned_precondition(rpb_mesh* m, double, double, const double* R, double* Z)
{
    if (!m->learned || !m->learned->mlp) {
        set_error("no learned preconditioner is attached to this mesh (rpb_mesh_set_learned)");
        return RPB_EINVAL;
    }
    rpb_status st = ensure_learned(m);
    if (st != RPB_OK) return st;
    return learned_forward(m, m->learned->mlp, R, Z, false);
}

static rpb_status weight_grads(rpb_mlp* mlp, int n, const float* G, int P, const float* X, int Q, bool gelu_x,
                               float* gW, float* gb, cudaStream_t s)
{
    const int nblocks = (n + WG_CHUNK - 1) / WG_CHUNK;
    const size_t need = static_cast<size_t>(nblocks) * P * (Q + 1);
    if (mlp->partial.n < need) RPB_CUDA(mlp->partial.alloc(need));
    k_weight_grad<<<nblocks, 256, 0, s>>>(n, G, P, X, Q, gelu_x, mlp->partial.ptr);
    k_reduce_grad<<<(P * (Q + 1) + 255) / 256, 256, 0, s>>>(nblocks, P, Q, mlp->partial.ptr, gW, gb);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

// gradient of the MLP parameters for given cluster output gradients dO (all clusters)
static rpb_status mlp_backward(rpb_mlp* mlp, int n, const float* F, const float* pre1, const float* pre2,
                               const float* dO, float* d1, float* d2, float* grad, cudaStream_t s)
{
    MlpBackArgs ba;
    ba.n = n; ba.w = mlp->w16.ptr; ba.dO = dO; ba.pre1 = pre1; ba.pre2 = pre2; ba.d2 = d2; ba.d1 = d1;
    k_mlp_backward<<<(n + 127) / 128, 128, NPARAM * sizeof(float), s>>>(ba);
    RPB_CUDA(cudaGetLastError());
    rpb_status st;
    if ((st = weight_grads(mlp, n, dO, NO, pre2, NH, true, grad + OFF_W3, grad + OFF_B3, s)) != RPB_OK) return st;
    if ((st = weight_grads(mlp, n, d2, NH, pre1, NH, true, grad + OFF_W2, grad + OFF_B2, s)) != RPB_OK) return st;
    if ((st = weight_grads(mlp, n, d1, NH, F, NF, false, grad + OFF_W1, grad + OFF_B1, s)) != RPB_OK) return st;
    return RPB_OK;
}

__global__ void k_accumulate(int n, float* dst, const float* src)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] += src[k];
}

}  // namespace rpb

using namespace rpb;

extern "C" {

int rpb_mlp_param_count(void) { return NPARAM; }

rpb_status rpb_mlp_create(int device, uint64_t seed, rpb_mlp** out)
{
    if (!out) { set_error("null argument"); return RPB_EINVAL; }
    *out = nullptr;
    RPB_CUDA(cudaSetDevice(device));
    auto* mlp = new rpb_mlp();
    mlp->device = device;
    // Xavier-uniform weights, zero biases, a small output layer: all gains start near 1
    std::vector<float> th(NPARAM, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_out, int fan_in, float gain) {
        const float a = gain * std::sqrt(6.0f / (fan_in + fan_out));
        std::uniform_real_distribution<float> U(-a, a);
        for (int k = 0; k < fan_out * fan_in; ++k) th[off + k] = U(rng);
    };
    fill(OFF_W1, NH, NF, 1.0f);
    fill(OFF_W2, NH, NH, 1.0f);
    fill(OFF_W3, NO, NH, 0.01f);
    if (mlp->theta.alloc(NPARAM) || mlp->grad.alloc(NPARAM) || mlp->m.alloc(NPARAM) || mlp->v.alloc(NPARAM) ||
        mlp->w16.alloc(NPARAM)) {
        delete mlp;
        set_error("device allocation failed");
        return RPB_ENOMEM;
    }
    rpb_status st = rpb_mlp_set_params(mlp, th.data());
    if (st != RPB_OK) { delete mlp; return st; }
    *out = mlp;
    return RPB_OK;
}

rpb_status rpb_mlp_destroy(rpb_mlp* mlp)
{
    delete mlp;
    return RPB_OK;
}

rpb_status rpb_mlp_get_params(const rpb_mlp* mlp, float* params)
{
    if (!mlp || !params) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(mlp->device));
    RPB_CUDA(cudaMemcpy(params, mlp->theta.ptr, mlp->theta.bytes(), cudaMemcpyDeviceToHost));
    return RPB_OK;
}

rpb_status rpb_mlp_set_params(rpb_mlp* mlp, const float* params)
{
    if (!mlp || !params) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(mlp->device));
    std::vector<__nv_bfloat16> w(NPARAM);
    for (int k = 0; k < NPARAM; ++k) w[k] = __float2bfloat16_rn(params[k]);
    RPB_CUDA(cudaMemcpy(mlp->theta.ptr, params, mlp->theta.bytes(), cudaMemcpyHostToDevice));
    RPB_CUDA(cudaMemcpy(mlp->w16.ptr, w.data(), mlp->w16.bytes(), cudaMemcpyHostToDevice));
    RPB_CUDA(cudaMemset(mlp->m.ptr, 0, mlp->m.bytes()));
    RPB_CUDA(cudaMemset(mlp->v.ptr, 0, mlp->v.bytes()));
    mlp->step = 0;
    return RPB_OK;
}

rpb_status rpb_mlp_eval(rpb_mlp* mlp, const float* F, int64_t n, const float* dO, float* O, float* grad)
{
    if (!mlp || !F || !O || n <= 0) { set_error("null or empty argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(mlp->device));
    DevBuf<float> dF, dOut, p1, p2, g1, g2, ddO, gr;
    RPB_CUDA(dF.alloc(NF * n));
    RPB_CUDA(dOut.alloc(NO * n));
    RPB_CUDA(p1.alloc(NH * n));
    RPB_CUDA(p2.alloc(NH * n));
    RPB_CUDA(cudaMemcpy(dF.ptr, F, dF.bytes(), cudaMemcpyHostToDevice));
    MlpArgs ma;
    ma.n = static_cast<int>(n); ma.w = mlp->w16.ptr; ma.F = dF.ptr; ma.O = dOut.ptr; ma.pre1 = p1.ptr; ma.pre2 = p2.ptr;
    k_mlp_forward<<<static_cast<unsigned>((n + MLP_TILE - 1) / MLP_TILE), MLP_TILE>>>(ma);
    RPB_CUDA(cudaGetLastError());
    RPB_CUDA(cudaMemcpy(O, dOut.ptr, dOut.bytes(), cudaMemcpyDeviceToHost));
    if (dO && grad) {
        RPB_CUDA(g1.alloc(NH * n));
        RPB_CUDA(g2.alloc(NH * n));
        RPB_CUDA(ddO.alloc(NO * n));
        RPB_CUDA(gr.alloc(NPARAM));
        RPB_CUDA(cudaMemcpy(ddO.ptr, dO, ddO.bytes(), cudaMemcpyHostToDevice));
        rpb_status st = mlp_backward(mlp, static_cast<int>(n), dF.ptr, p1.ptr, p2.ptr, ddO.ptr, g1.ptr, g2.ptr, gr.ptr, 0);
        if (st != RPB_OK) return st;
        RPB_CUDA(cudaMemcpy(grad, gr.ptr, gr.bytes(), cudaMemcpyDeviceToHost));
    }
    return RPB_OK;
}

rpb_status rpb_mesh_set_learned(rpb_mesh* m, rpb_mlp* mlp)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    if (mlp && mlp->device != m->device) { set_error("network and mesh live on different devices"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    rpb_status st = ensure_learned(m);
    if (st != RPB_OK) return st;
    m->learned->mlp = mlp;
    return RPB_OK;
}

rpb_status rpb_tpm0_learned_apply(rpb_mesh* m, const double* R, double* Z)
{
    if (!m || !R || !Z) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    rpb_status st = ensure_learned(m);
    if (st != RPB_OK) return st;
    if (!m->learned->mlp) { set_error("no learned preconditioner attached"); return RPB_EINVAL; }
    LearnedState& L = *m->learned;
    RPB_CUDA(cudaMemcpyAsync(L.r.ptr, R, 3 * sizeof(double) * m->nV, cudaMemcpyHostToDevice, m->stream));
    if ((st = learned_forward(m, L.mlp, L.r.ptr, L.z.ptr, false)) != RPB_OK) return st;
    RPB_CUDA(cudaMemcpyAsync(Z, L.z.ptr, 3 * sizeof(double) * m->nV, cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    return RPB_OK;
}

rpb_status rpb_tpm0_learned_apply_pair(rpb_mesh* m, const double* R, const double* Y, double* Z, double* ZY)
{
    if (!m || !R || !Z || (!Y) != (!ZY)) { set_error("null argument"); return RPB_EINVAL; }
    if (!m->learned || !m->learned->mlp) {
        set_error("no learned preconditioner is attached to this mesh (rpb_mesh_set_learned)");
        return RPB_EINVAL;
    }
    RPB_CUDA(cudaSetDevice(m->device));
    rpb_status st;
    if ((st = ensure_learned(m)) != RPB_OK) return st;
    if ((st = ensure_training_buffers(m)) != RPB_OK) return st;
    LearnedState& L = *m->learned;
    cudaStream_t s = m->stream;
    const size_t n3 = 3 * static_cast<size_t>(m->nV);
    RPB_CUDA(cudaMemcpyAsync(L.r.ptr, R, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if ((st = learned_forward(m, L.mlp, L.r.ptr, L.z.ptr, true)) != RPB_OK) return st;
    RPB_CUDA(cudaMemcpyAsync(Z, L.z.ptr, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (Y) {
        const int eb = (m->nV + 255) / 256;
        RPB_CUDA(cudaMemcpyAsync(L.e.ptr, Y, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
        if ((st = cluster_moments(m, L.e.ptr, L.gc.ptr)) != RPB_OK) return st;
        k_frozen_coef<<<(m->NC + 255) / 256, 256, 0, s>>>(m->NC, L.O.ptr, L.gc.ptr, L.C_w.ptr, L.c.ptr);
        k_prim_expand<<<(m->N * EXPAND_LANES + 255) / 256, 256, 0, s>>>(m->N, m->leaf_of.ptr, m->C_parent.ptr, m->C_up4.ptr, L.c.ptr,
                                                          L.tmp3.ptr);
        RPB_CUDA(cudaMemsetAsync(L.dots.ptr, 0, 3 * sizeof(double), s));
        k_vertex_expand<<<(m->nV * EXPAND_LANES + 255) / 256, 256, 0, s>>>(m->nV, m->size, m->vp_rp.ptr, m->vp_slot.ptr,
                                                                          m->pre_vals.ptr, L.tmp3.ptr,
                                          L.dots.ptr, L.g.ptr);
        if ((st = dot3_dev(m, L.g.ptr, nullptr, L.sums.ptr)) != RPB_OK) return st;
        k_sub_mean<<<eb, 256, 0, s>>>(m->nV, L.g.ptr, L.sums.ptr);
        RPB_CUDA(cudaGetLastError());
        RPB_CUDA(cudaMemcpyAsync(ZY, L.g.ptr, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    RPB_CUDA(cudaStreamSynchronize(s));
    return RPB_OK;
}

rpb_status rpb_mlp_train_step_sens(rpb_mlp* mlp, rpb_mesh* m, const double* R, const double* G, int npairs, double lr,
                                   double reg, double* objective, float* grad)
{
    if (!mlp || !m || !R || !G || npairs <= 0) { set_error("null or empty argument"); return RPB_EINVAL; }
    if (mlp->device != m->device) { set_error("network and mesh live on different devices"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    rpb_status st;
    if ((st = ensure_learned(m)) != RPB_OK) return st;
    if ((st = ensure_training_buffers(m)) != RPB_OK) return st;
    LearnedState& L = *m->learned;
    cudaStream_t s = m->stream;
    const int nV = m->nV;
    const int eb = (nV + 255) / 256;
    const size_t n3 = 3 * static_cast<size_t>(nV);
    DevBuf<float> gsum;
    DevBuf<double> obj;
    RPB_CUDA(gsum.alloc(NPARAM));
    RPB_CUDA(obj.alloc(3 * static_cast<size_t>(npairs)));
    RPB_CUDA(cudaMemsetAsync(gsum.ptr, 0, gsum.bytes(), s));
    for (int k = 0; k < npairs; ++k) {
        RPB_CUDA(cudaMemcpyAsync(L.r.ptr, R + k * n3, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
        RPB_CUDA(cudaMemcpyAsync(L.g.ptr, G + k * n3, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
        if ((st = learned_forward(m, mlp, L.r.ptr, L.z.ptr, true)) != RPB_OK) return st;
        if ((st = dot3_dev(m, L.g.ptr, L.z.ptr, obj.ptr + 3 * k)) != RPB_OK) return st;
        // back through the mean removal, the vertex sum and the cluster expansion
        if ((st = dot3_dev(m, L.g.ptr, nullptr, L.sums.ptr)) != RPB_OK) return st;
        k_sub_mean<<<eb, 256, 0, s>>>(nV, L.g.ptr, L.sums.ptr);
        if ((st = cluster_moments(m, L.g.ptr, L.gc.ptr)) != RPB_OK) return st;
        k_cluster_out_grad<<<(m->NC + 255) / 256, 256, 0, s>>>(m->NC, L.gc.ptr, L.O.ptr, L.Rc.ptr, m->C_pair.ptr,
                                                               static_cast<float>(reg), L.C_w.ptr, L.dO.ptr);
        RPB_CUDA(cudaGetLastError());
        if ((st = mlp_backward(mlp, m->NC, L.F.ptr, L.pre1.ptr, L.pre2.ptr, L.dO.ptr, L.d1.ptr, L.d2.ptr, mlp->grad.ptr,
                               s)) != RPB_OK)
            return st;
        k_accumulate<<<(NPARAM + 255) / 256, 256, 0, s>>>(NPARAM, gsum.ptr, mlp->grad.ptr);
    }
    std::vector<float> gh;
    if (grad) {
        gh.resize(NPARAM);
        RPB_CUDA(cudaMemcpyAsync(gh.data(), gsum.ptr, gsum.bytes(), cudaMemcpyDeviceToHost, s));
    }
    std::vector<double> oh(3 * static_cast<size_t>(npairs));
    RPB_CUDA(cudaMemcpyAsync(oh.data(), obj.ptr, obj.bytes(), cudaMemcpyDeviceToHost, s));
    mlp->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - std::pow(b1, static_cast<float>(mlp->step));
    const float bc2 = 1.0f - std::pow(b2, static_cast<float>(mlp->step));
    if (lr > 0.0)
        k_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(NPARAM, mlp->theta.ptr, mlp->w16.ptr, gsum.ptr, mlp->m.ptr, mlp->v.ptr,
                                                    static_cast<float>(lr), b1, b2, 1e-8f, bc1, bc2);
    RPB_CUDA(cudaGetLastError());
    RPB_CUDA(cudaStreamSynchronize(s));
    if (lr <= 0.0) mlp->step -= 1;
    if (objective) {
        double o = 0;
        for (double v : oh) o += v;
        *objective = o;
    }
    if (grad)
        for (int k = 0; k < NPARAM; ++k) grad[k] = gh[k];
    return RPB_OK;
}

rpb_status rpb_mlp_train_step(rpb_mlp* mlp, rpb_mesh* m, double q, double p, const double* R, const double* E,
                              int npairs, double lr, double reg, double* loss, float* grad)
{
    if (!mlp || !m || !R || !E || npairs <= 0) { set_error("null or empty argument"); return RPB_EINVAL; }
    if (mlp->device != m->device) { set_error("network and mesh live on different devices"); return RPB_EINVAL; }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    if ((st = ensure_learned(m)) != RPB_OK) return st;
    if ((st = ensure_training_buffers(m)) != RPB_OK) return st;
    LearnedState& L = *m->learned;
    cudaStream_t s = m->stream;
    const int nV = m->nV;
    const int eb = (nV + 255) / 256;
    const size_t n3 = 3 * static_cast<size_t>(nV);
    DevBuf<float> gsum;
    RPB_CUDA(gsum.alloc(NPARAM));
    RPB_CUDA(cudaMemsetAsync(gsum.ptr, 0, gsum.bytes(), s));
    RPB_CUDA(cudaMemsetAsync(L.loss.ptr, 0, sizeof(double), s));
    for (int k = 0; k < npairs; ++k) {
        RPB_CUDA(cudaMemcpyAsync(L.r.ptr, R + k * n3, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
        RPB_CUDA(cudaMemcpyAsync(L.e.ptr, E + k * n3, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
        if ((st = learned_forward(m, mlp, L.r.ptr, L.z.ptr, true)) != RPB_OK) return st;
        if ((st = metric_multiply_dev(m, q, p, 1.0, L.z.ptr, 3, 0.0, L.Az.ptr, 3, 7)) != RPB_OK) return st;
        if ((st = dot3_dev(m, L.z.ptr, L.r.ptr, L.dots.ptr)) != RPB_OK) return st;
        if ((st = dot3_dev(m, L.z.ptr, L.Az.ptr, L.dots.ptr + 3)) != RPB_OK) return st;
        if ((st = dot3_dev(m, L.e.ptr, L.r.ptr, L.dots.ptr + 6)) != RPB_OK) return st;
        k_loss_grad<<<eb, 256, 0, s>>>(nV, L.r.ptr, L.Az.ptr, L.dots.ptr, L.g.ptr, L.loss.ptr);
        // back through the mean removal, the vertex sum and the cluster expansion (the
        // transposes: primitive moments and range sums)
        if ((st = dot3_dev(m, L.g.ptr, nullptr, L.sums.ptr)) != RPB_OK) return st;
        k_sub_mean<<<eb, 256, 0, s>>>(nV, L.g.ptr, L.sums.ptr);
        if ((st = cluster_moments(m, L.g.ptr, L.gc.ptr)) != RPB_OK) return st;
        k_cluster_out_grad<<<(m->NC + 255) / 256, 256, 0, s>>>(m->NC, L.gc.ptr, L.O.ptr, L.Rc.ptr, m->C_pair.ptr,
                                                               static_cast<float>(reg), L.C_w.ptr, L.dO.ptr);
        RPB_CUDA(cudaGetLastError());
        if ((st = mlp_backward(mlp, m->NC, L.F.ptr, L.pre1.ptr, L.pre2.ptr, L.dO.ptr, L.d1.ptr, L.d2.ptr, mlp->grad.ptr,
                               s)) != RPB_OK)
            return st;
        k_accumulate<<<(NPARAM + 255) / 256, 256, 0, s>>>(NPARAM, gsum.ptr, mlp->grad.ptr);
    }
    std::vector<float> gh;
    if (grad) {
        gh.resize(NPARAM);
        RPB_CUDA(cudaMemcpyAsync(gh.data(), gsum.ptr, gsum.bytes(), cudaMemcpyDeviceToHost, s));
    }
    // Adam on the mean gradient (the bias corrections carry the 1/npairs)
    mlp->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - std::pow(b1, static_cast<float>(mlp->step));
    const float bc2 = 1.0f - std::pow(b2, static_cast<float>(mlp->step));
    const float np = static_cast<float>(npairs);
    if (lr > 0.0)
        k_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(NPARAM, mlp->theta.ptr, mlp->w16.ptr, gsum.ptr, mlp->m.ptr, mlp->v.ptr,
                                                    static_cast<float>(lr), b1, b2, 1e-8f, bc1 * np, bc2 * np * np);
    RPB_CUDA(cudaGetLastError());
    double l = 0;
    RPB_CUDA(cudaMemcpyAsync(&l, L.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    RPB_CUDA(cudaStreamSynchronize(s));
    if (lr <= 0.0) mlp->step -= 1;
    if (loss) *loss = l / npairs;
    if (grad)
        for (int k = 0; k < NPARAM; ++k) grad[k] = gh[k] / np;
    return RPB_OK;
}

}  // extern "C"
