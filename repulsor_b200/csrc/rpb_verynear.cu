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
// No atomics: the pair thread of entry (i, j), j > i, of the full symmetric pattern
// writes its results into the slots of both entries (i, j) and (j, i) -- the row
// derivative DX into the first, DY into the second, the energy into the first -- and a
// row pass (k_vf_rows) adds each row's slots in pattern order; the energy is summed
// per block and the block partials by the last block in block order, so every result
// is reproducible bit for bit. Obstacle pairs (CROSS: rows are the mesh's primitives,
// columns the obstacle's, TangentPointObstacleEnergy.hpp:62-96) fill only their own
// slot, with the symmetry factor 1/2 of a non-symmetric block cluster tree
// (FMM_Kernel.hpp:43), and form the mesh side's derivative only.
//
// Pairs are classified on the construction-time coordinates (as the reference's block
// cluster tree, whose clustering data SemiStaticUpdate leaves unchanged) but evaluated on
// the current ones. A pair whose primitives touch or intersect at evaluation time has an
// infinite energy and would refine to the level limit along the contact (the number of
// sub-pairs grows like 2^level); such a pair, and any pair needing more than
// VF_MAX_SUBPAIRS sub-pair visits, is not evaluated: its results are set to NaN and a
// status bit is raised, which the host reads when it synchronizes (vf_take_status).
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

constexpr int VF_SLOT = 17;   // per pattern entry: 16 derivative components + the energy
constexpr long long VF_MAX_SUBPAIRS = 1LL << 22;   // sub-pair visits per pair before giving up
constexpr unsigned VF_STATUS_CONTACT = 1u;         // primitives touch or intersect
constexpr unsigned VF_STATUS_WORK = 2u;            // the sub-pair cap was reached

struct VFArgs {
    int dom, N;
    const int64_t* rp;
    const int* ci;
    const double* V;       // row side
    const int* S;
    const int* perm;
    const double* charge_v;
    const double* V_col;   // column side (the mesh itself, or the obstacle for CROSS)
    const int* S_col;
    const int* perm_col;
    const double* charge_col;
    bool cross;
    double theta2;
    int max_level;
    TPExp ex;
    double* part;          // nnz x VF_SLOT entry slots (energy mode: derivative + energy;
                           // metric mode: the two diagonal contributions in [0], [1])
    bool diff;
    float2* vals;          // metric mode: full-pattern values (both triangles written)
    unsigned* status;      // VF_STATUS_* bits raised by pairs that could not be evaluated
};

struct Prim {
    double h[3][3];
    double a;
    double P[6];
};

__device__ void load_prim(int dom, const double* V, const int* S, const int* perm, const double* charge_v, int i,
                          Prim& pr)
{
    const int size = dom + 1;
    SimplexGeom g;
    simplex_geometry(dom, V, S + static_cast<int64_t>(size) * perm[i], charge_v, g);
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) pr.h[c][k] = (c < size) ? g.h[c][k] : 0.0;
    pr.a = g.charge * g.vol;
    projector_packed(dom, g.t, pr.P);
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

// Slot of the transposed entry (j, i) of a symmetric pattern.
__device__ int64_t transposed_slot(const VFArgs& A, int i, int j)
{
    int64_t lo = A.rp[j], hi = A.rp[j + 1];
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (A.ci[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
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
    if (!A.cross && j <= i) return;  // each unordered pair once, by the thread of (i, j), j > i
    Prim X, Y;
    load_prim(A.dom, A.V, A.S, A.perm, A.charge_v, i, X);
    load_prim(A.dom, A.V_col, A.S_col, A.perm_col, A.charge_col, j, Y);
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
    const bool want_dy = A.diff && !A.cross;
    // primitives that touch or intersect now: infinite energy, not evaluated
    const double d2_pair = (A.dom == 2) ? tri_tri_d2(&X.h[0][0], &Y.h[0][0]) : seg_seg_d2(X.h[0], X.h[1], Y.h[0], Y.h[1]);
    unsigned fail = (d2_pair > 0.0) ? 0u : VF_STATUS_CONTACT;
    if (fail) sp = 0;
    long long visits = 0;
    while (sp > 0) {
        if (++visits > VF_MAX_SUBPAIRS) {
            fail = VF_STATUS_WORK;
            break;
        }
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
            if (want_dy) tp0_core<double, 3, 6, true>(A.ex, gy, bp, ap, accY);
        } else {
            e = tp0_core<double, -1, -1, true>(A.ex, gx, ap, bp, accX);
            if (want_dy) tp0_core<double, -1, -1, true>(A.ex, gy, bp, ap, accY);
        }
        e_sum += e;
        if (A.diff) {
            // reference layout: DX[0] = ws (d0 - dx . x), hull slot v = ws lambda_v dx, P part ws dP
            DX[0] += ws * (accX.d0 - (accX.dx[0] * cs[0] + accX.dx[1] * cs[1] + accX.dx[2] * cs[2]));
            for (int c = 0; c < size; ++c)
                for (int kk = 0; kk < 3; ++kk) DX[1 + 3 * c + kk] += ws * ls[c] * accX.dx[kk];
            for (int m = 0; m < 6; ++m) DX[1 + 3 * size + m] += ws * accX.dP[m];
            if (want_dy) {
                DY[0] += wt * (accY.d0 - (accY.dx[0] * ct[0] + accY.dx[1] * ct[1] + accY.dx[2] * ct[2]));
                for (int c = 0; c < size; ++c)
                    for (int kk = 0; kk < 3; ++kk) DY[1 + 3 * c + kk] += wt * lt[c] * accY.dx[kk];
                for (int m = 0; m < 6; ++m) DY[1 + 3 * size + m] += wt * accY.dP[m];
            }
        }
    }
    if (fail) {
        atomicOr(A.status, fail);
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        e_sum = a0_sum = a1_sum = nan;
        for (int m = 0; m < 16; ++m) DX[m] = DY[m] = nan;
    }
    double* slot = A.part + VF_SLOT * k;
    if (METRIC) {
        // the values as stored (FP32), the row diagonals from the stored values so that
        // y_i = sum_j a_ij (x_j - (a_j / a_i) x_i) holds for the applied operator
        const float2 val = make_float2(static_cast<float>(a0_sum), static_cast<float>(a1_sum));
        const int64_t kt = transposed_slot(A, i, j);
        A.vals[k] = val;
        A.vals[kt] = val;
        const double bo = Y.a / X.a, ao = X.a / Y.a;
        slot[0] = -bo * static_cast<double>(val.x);
        slot[1] = -bo * static_cast<double>(val.y);
        double* tslot = A.part + VF_SLOT * kt;
        tslot[0] = -ao * static_cast<double>(val.x);
        tslot[1] = -ao * static_cast<double>(val.y);
        return;
    }
    const double sf = A.cross ? 0.5 : 1.0;
    for (int m = 0; m < 16; ++m) slot[m] = A.diff ? sf * DX[m] : 0.0;
    slot[16] = sf * e_sum;
    if (!A.cross) {
        double* tslot = A.part + VF_SLOT * transposed_slot(A, i, j);
        for (int m = 0; m < 16; ++m) tslot[m] = A.diff ? DY[m] : 0.0;
        tslot[16] = 0.0;
    }
}

struct VFRowArgs {
    int N;
    const int64_t* rp;
    const double* part;
    bool metric, diff;
    double* D_vf;          // energy mode: N x 16 row derivatives (if diff)
    double2* diag;         // metric mode: N row diagonals
    double* block_energy;  // energy mode: one partial per block
    unsigned* done;        // zero between launches
    double* energy_out;
};

// Row pass: each row adds its slots in pattern order; the energy partials of the blocks
// are added by the last block to finish, in block order.
__global__ void k_vf_rows(VFRowArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e_row = 0.0;
    if (i < A.N) {
        const int64_t k0 = A.rp[i], k1 = A.rp[i + 1];
        if (A.metric) {
            double d0 = 0.0, d1 = 0.0;
            for (int64_t k = k0; k < k1; ++k) {
                d0 += A.part[VF_SLOT * k];
                d1 += A.part[VF_SLOT * k + 1];
            }
            A.diag[i] = make_double2(d0, d1);
        } else {
            double D[16];
            for (int m = 0; m < 16; ++m) D[m] = 0.0;
            for (int64_t k = k0; k < k1; ++k) {
                const double* slot = A.part + VF_SLOT * k;
                if (A.diff)
                    for (int m = 0; m < 16; ++m) D[m] += slot[m];
                e_row += slot[16];
            }
            if (A.diff)
                for (int m = 0; m < 16; ++m) A.D_vf[16 * static_cast<int64_t>(i) + m] = D[m];
        }
    }
    if (A.metric) return;
    __shared__ double sh[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    e_row = warp_sum_f64(e_row);
    if (lane == 0) sh[wib] = e_row;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += sh[w];
        A.block_energy[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(A.done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(A.block_energy + b);
        *A.energy_out = s;
        *A.done = 0u;
    }
}

constexpr int VF_ROW_BLOCK = 256;

static VFArgs make_args(rpb_mesh* m, const TPExp& ex)
{
    VFArgs A;
    std::memset(&A, 0, sizeof(A));
    A.dom = m->dom;
    A.N = m->N;
    A.rp = m->verynear.rp.ptr;
    A.ci = m->verynear.ci.ptr;
    A.V = A.V_col = m->V.ptr;
    A.S = A.S_col = m->S.ptr;
    A.perm = A.perm_col = m->perm.ptr;
    A.charge_v = A.charge_col = m->charge_v.ptr;
    A.theta2 = m->settings.theta_near * m->settings.theta_near;
    A.max_level = m->settings.max_refinement;
    A.ex = ex;
    A.status = m->vf.done.ptr + 1;
    return A;
}

int vf_row_blocks(int N) { return (N + VF_ROW_BLOCK - 1) / VF_ROW_BLOCK; }

rpb_status vf_alloc(VFBuffers& b, int64_t nnz, int N)
{
    if (b.part.alloc(VF_SLOT * static_cast<size_t>(nnz)) || b.block_energy.alloc(vf_row_blocks(N)) ||
        b.done.alloc(2) || b.D.alloc(16 * static_cast<size_t>(N))) {
        set_error("device allocation failed (very-near buffers)");
        return RPB_ENOMEM;
    }
    if (cudaMemset(b.done.ptr, 0, 2 * sizeof(unsigned)) != cudaSuccess) {
        set_error("memset failed");
        return RPB_ECUDA;
    }
    return RPB_OK;
}

rpb_status vf_take_status(VFBuffers& b, cudaStream_t s)
{
    if (!b.done.ptr) return RPB_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return RPB_OK;
    unsigned st = 0;
    if (cudaMemcpyAsync(&st, b.done.ptr + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("reading the very-near status failed");
        return RPB_ECUDA;
    }
    if (st == 0) return RPB_OK;
    if (cudaMemsetAsync(b.done.ptr + 1, 0, sizeof(unsigned), s) != cudaSuccess) {
        set_error("memset failed");
        return RPB_ECUDA;
    }
    if (st & VF_STATUS_CONTACT)
        set_error("very-near primitives touch or intersect at the current coordinates: the tangent-point energy is "
                  "infinite there (results are NaN); the pair lists were classified on the construction-time "
                  "coordinates");
    else
        set_error("a very-near pair needed more than 2^22 sub-pair visits of the adaptive quadrature (primitives "
                  "nearly in contact along a line); results are NaN");
    return RPB_EINVAL;
}

static rpb_status launch_vf_pass(const VFArgs& A, int64_t nnz, VFBuffers& b, double* energy_out, bool diff,
                                 cudaStream_t s)
{
    k_verynear<false><<<static_cast<unsigned>((nnz + 63) / 64), 64, 0, s>>>(A);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near kernel launch failed"); return RPB_ECUDA; }
    VFRowArgs R;
    std::memset(&R, 0, sizeof(R));
    R.N = A.N;
    R.rp = A.rp;
    R.part = b.part.ptr;
    R.metric = false;
    R.diff = diff;
    R.D_vf = b.D.ptr;
    R.block_energy = b.block_energy.ptr;
    R.done = b.done.ptr;
    R.energy_out = energy_out;
    k_vf_rows<<<vf_row_blocks(A.N), VF_ROW_BLOCK, 0, s>>>(R);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near row kernel launch failed"); return RPB_ECUDA; }
    return RPB_OK;
}

rpb_status launch_vf(rpb_mesh* m, const TPExp& ex, bool diff)
{
    if (m->verynear.nnz == 0) return RPB_OK;
    VFArgs A = make_args(m, ex);
    A.part = m->vf.part.ptr;
    A.diff = diff;
    return launch_vf_pass(A, m->verynear.nnz, m->vf, m->energy.ptr + 2, diff, m->stream);
}

rpb_status launch_vf_cross(rpb_mesh* m, const rpb_mesh* obstacle, const int64_t* rp, const int* ci, int64_t nnz,
                           VFBuffers& b, const TPExp& ex, bool diff, double* energy_out)
{
    VFArgs A = make_args(m, ex);
    A.rp = rp;
    A.ci = ci;
    A.cross = true;
    A.V_col = obstacle->V.ptr;
    A.S_col = obstacle->S.ptr;
    A.perm_col = obstacle->perm.ptr;
    A.charge_col = obstacle->charge_v.ptr;
    A.part = b.part.ptr;
    A.status = b.done.ptr + 1;
    A.diff = diff;
    return launch_vf_pass(A, nnz, b, energy_out, diff, m->stream);
}

rpb_status launch_vf_metric(rpb_mesh* m, const TPExp& ex, float2* vals, double2* diag)
{
    if (m->verynear.nnz == 0) return RPB_OK;
    VFArgs A = make_args(m, ex);
    A.vals = vals;
    A.part = m->vf.part.ptr;
    if (ex.qh == -2) A.max_level = m->settings.max_refinement < 20 ? m->settings.max_refinement : 20;
    const int64_t n = m->verynear.nnz;
    k_verynear<true><<<static_cast<unsigned>((n + 63) / 64), 64, 0, m->stream>>>(A);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near metric kernel launch failed"); return RPB_ECUDA; }
    VFRowArgs R;
    std::memset(&R, 0, sizeof(R));
    R.N = m->N;
    R.rp = A.rp;
    R.part = A.part;
    R.metric = true;
    R.diag = diag;
    k_vf_rows<<<vf_row_blocks(m->N), VF_ROW_BLOCK, 0, m->stream>>>(R);
    if (cudaGetLastError() != cudaSuccess) { set_error("very-near row kernel launch failed"); return RPB_ECUDA; }
    return RPB_OK;
}

}  // namespace rpb
