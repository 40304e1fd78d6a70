// Energy densities of TangentPointEnergy0 (EnergyBase::SimplexDensities / VertexDensities,
// src/Energies/EnergyBase.hpp:129-150; the density branch of TP0_Kernel_FF/NF,
// src/Energies/TangentPointEnergy0/TP0_Kernel_FF.hpp:214-218; CollectPrimitiveDensities
// and CollectVertexDensities, src/ClusterTree/ClusterTreeBase.hpp:601-729).
//
// For a pair (x, y) the reference adds b |Pv|^q / |v|^p to x's density and a |Qv|^q / |v|^p
// to y's. On the full symmetric patterns a row collects its own side over all its
// partners: rho_row = sum_j b_j u^{q/2} s^{p/2-q/2} with u = v^T P v / |v|^2, s = 1/|v|^2
// (FP64 projection, FP32 kernel, FP64 row sums as in the energy kernels). Far-field
// cluster densities are pushed down to the primitives (sum over the ancestors), so
// sum_i a_i rho_i is the energy. Vertex densities average the simplex densities with the
// weights a_i/(n+1) of the Post operator, divided by the dual volumes.
#include <string>

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

namespace {

template <typename R, int QH, int PH>
__device__ __forceinline__ void density_core(const TPExp& ex, const Proj<R>& g, R a, R b, R& rho, R& energy)
{
    const R s = dev_rcp(g.r2);
    const R u = g.cphi * s, w = g.cpsi * s;
    R uq, wq, se;
    if constexpr (QH > 0 && PH >= QH) {
        uq = ipow_pos(fabs(u), QH - 1) * u;
        wq = ipow_pos(fabs(w), QH - 1) * w;
        se = ipow_pos(s, PH - QH);
    } else {
        const R qh = static_cast<R>(ex.q * 0.5), ph = static_cast<R>(ex.p * 0.5);
        uq = (fabs(u) > R(0)) ? dev_pow(fabs(u), qh) : R(0);
        wq = (fabs(w) > R(0)) ? dev_pow(fabs(w), qh) : R(0);
        se = dev_pow(s, ph - qh);
    }
    rho = b * uq * se;
    energy = a * (uq + wq) * se * b;
}

// One thread per row; rows in tree order. D: rows x 1 densities; energies counted once per
// unordered pair, reduced per block and by the last block.
template <bool FAR, int QH, int PH>
__global__ void __launch_bounds__(256) k_tp0_density(PairArgs A)
{
    using Datum = typename std::conditional<FAR, ClusterDatum, PrimDatum>::type;
    const Datum* base = static_cast<const Datum*>(A.data);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e_row = 0.0;
    if (i < A.rows) {
        const Datum X = load_datum(base, i);
        double rho = 0.0;
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int j = __ldg(A.ci + k);
            const Datum Y = load_datum(base, j);
            bool close = false;
            Proj<float> g;
            if constexpr (FAR) project_clusters(X, Y, g);
            else {
                project_prims(A.dom, X, Y, g);
                const float dd = A.close_factor * (X.diam + Y.diam);
                close = g.r2 < dd * dd;
            }
            if (close) {
                Proj<double> gd;
                if constexpr (!FAR) project_prims(A.dom, X, Y, gd);
                double r, e;
                density_core<double, QH, PH>(A.ex, gd, X.a, Y.a, r, e);
                rho += r;
                if (j > i) e_row += e;
            } else {
                float r, e;
                density_core<float, QH, PH>(A.ex, g, static_cast<float>(X.a), static_cast<float>(Y.a), r, e);
                rho += r;
                if (j > i) e_row += e;
            }
        }
        A.D[i] = rho;
    }
    __shared__ double sh[8];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    e_row = warp_sum_f64(e_row);
    if (lane == 0) sh[wib] = e_row;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) s += sh[w];
        A.block_energy[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(A.done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double s = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(A.block_energy + b);
        s = warp_sum_f64(s);
        __syncthreads();
        if (lane == 0) sh[wib] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (blockDim.x >> 5); ++w) t += sh[w];
            *A.energy_out = t;
            *A.done = 0u;
        }
    }
}

// rho_i = near density + far densities of the clusters containing i (tree order), and the
// simplex output in original order (if out_simplex)
__global__ void k_density_prims(int N, const int* perm, const int* leaf_of, const int* C_parent, const double* dn,
                                const double* df, double* rho, double* out_simplex)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double r = dn[i];
    for (int C = leaf_of[i]; C >= 0; C = C_parent[C]) r += df[C];
    rho[i] = r;
    if (out_simplex) out_simplex[perm[i]] = r;
}

__global__ void k_density_vertices(int nV, int size, const int* vp_rp, const int* vp_slot, const double* pre_vals,
                                   const double* rho, double* out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nV) return;
    double num = 0, den = 0;
    for (int k = vp_rp[v]; k < vp_rp[v + 1]; ++k) {
        const int slot = vp_slot[k];
        const int i = slot / size, l = slot - i * size;
        const double w = pre_vals[(4 * static_cast<int64_t>(i)) * size + l];
        num += w * rho[i];
        den += w;
    }
    out[v] = den > 0 ? num / den : 0.0;
}

template <int QH, int PH>
void launch_density(rpb_mesh* m, const PairArgs& An, const PairArgs& Af)
{
    if (An.rows > 0) k_tp0_density<false, QH, PH><<<(An.rows + 255) / 256, 256, 0, m->stream>>>(An);
    if (Af.rows > 0) k_tp0_density<true, QH, PH><<<(Af.rows + 255) / 256, 256, 0, m->stream>>>(Af);
}

// densities per primitive (tree order) into `rho`; energy into energy_host
rpb_status densities(rpb_mesh* m, double q, double p, double* rho, double* simplex_out, double* energy_host)
{
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    if (m->verynear.nnz > 0) {
        set_error("energy densities are not built for meshes with very-near primitive pairs");
        return RPB_EINVAL;
    }
    if (!m->geometry_valid && (st = launch_geometry(m)) != RPB_OK) return st;
    const TPExp ex = make_exp(m->dom, q, p);
    const int nb_near = (m->N + 255) / 256, nb_far = (m->NC + 255) / 256;
    DevBuf<double> dn, df, partial, e2;
    DevBuf<unsigned> done;
    RPB_CUDA(dn.alloc(m->N));
    RPB_CUDA(df.alloc(m->NC));
    RPB_CUDA(partial.alloc(nb_near + nb_far));
    RPB_CUDA(e2.alloc(2));
    RPB_CUDA(done.alloc(2));
    RPB_CUDA(cudaMemsetAsync(done.ptr, 0, done.bytes(), m->stream));
    RPB_CUDA(cudaMemsetAsync(e2.ptr, 0, e2.bytes(), m->stream));
    RPB_CUDA(cudaMemsetAsync(dn.ptr, 0, dn.bytes(), m->stream));
    RPB_CUDA(cudaMemsetAsync(df.ptr, 0, df.bytes(), m->stream));
    PairArgs An, Af;
    An.col_data = Af.col_data = nullptr;
    An.order = Af.order = nullptr;
    An.dom = Af.dom = m->dom;
    An.ex = Af.ex = ex;
    An.close_factor = Af.close_factor = 0.1f;
    An.rows = m->near.nnz > 0 ? m->N : 0;
    An.rp = m->near.rp.ptr; An.ci = m->near.ci.ptr; An.data = m->P_pair.ptr; An.D = dn.ptr;
    An.block_energy = partial.ptr; An.done = done.ptr; An.energy_out = e2.ptr;
    Af.rows = m->far.nnz > 0 ? m->NC : 0;
    Af.rp = m->far.rp.ptr; Af.ci = m->far.ci.ptr; Af.data = m->C_pair.ptr; Af.D = df.ptr;
    Af.block_energy = partial.ptr + nb_near; Af.done = done.ptr + 1; Af.energy_out = e2.ptr + 1;
    if (ex.qh == 3 && ex.ph == 6) launch_density<3, 6>(m, An, Af);
    else launch_density<-1, -1>(m, An, Af);
    k_density_prims<<<(m->N + 255) / 256, 256, 0, m->stream>>>(m->N, m->perm.ptr, m->leaf_of.ptr, m->C_parent.ptr,
                                                               dn.ptr, df.ptr, rho, simplex_out);
    RPB_CUDA(cudaGetLastError());
    double e[2] = {0, 0};
    RPB_CUDA(cudaMemcpyAsync(e, e2.ptr, sizeof(e), cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    if (energy_host) *energy_host = e[0] + e[1];
    return RPB_OK;
}

}  // namespace
}  // namespace rpb

using namespace rpb;

extern "C" {

rpb_status rpb_tpe0_simplex_densities(rpb_mesh* m, double q, double p, double* density, double* energy)
{
    if (!m || !density) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    DevBuf<double> rho, out;
    RPB_CUDA(rho.alloc(m->N));
    RPB_CUDA(out.alloc(m->N));
    const rpb_status st = densities(m, q, p, rho.ptr, out.ptr, energy);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaMemcpy(density, out.ptr, out.bytes(), cudaMemcpyDeviceToHost));
    return RPB_OK;
}

rpb_status rpb_tpe0_vertex_densities(rpb_mesh* m, double q, double p, double* density, double* energy)
{
    if (!m || !density) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    DevBuf<double> rho, out;
    RPB_CUDA(rho.alloc(m->N));
    RPB_CUDA(out.alloc(m->nV));
    rpb_status st = densities(m, q, p, rho.ptr, nullptr, energy);
    if (st != RPB_OK) return st;
    k_density_vertices<<<(m->nV + 255) / 256, 256, 0, m->stream>>>(m->nV, m->size, m->vp_rp.ptr, m->vp_slot.ptr,
                                                                   m->pre_vals.ptr, rho.ptr, out.ptr);
    RPB_CUDA(cudaGetLastError());
    RPB_CUDA(cudaMemcpyAsync(density, out.ptr, out.bytes(), cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    return RPB_OK;
}

}  // extern "C"
