// TangentPointObstacleEnergy on the B200 (src/Energies/TangentPointObstacleEnergy.hpp:62-96,
// obstacle handling src/SimplicialMesh.hpp:697-756).
//
// A mesh loads an obstacle mesh (rpb_mesh_load_obstacle, SimplicialMesh::LoadObstacle,
// which takes ownership as the reference's unique_ptr argument does). The non-symmetric
// block cluster tree of (mesh tree, obstacle tree) is built once on the host
// (host/tree_builder.cpp build_cross_lists) from the frozen coordinates both trees were
// built from, and uploaded. An evaluation runs the TP0 pair kernel in CROSS mode: rows are
// the mesh's primitives (near) or clusters (far), columns the obstacle's, every pair
// counts with the symmetry factor 1/2, and only the mesh side's moment derivatives are
// formed; they then go through the same collection, chain rule and vertex gather as the
// self energy. Very-near (mesh, obstacle) pairs run the subdivision quadrature in CROSS
// mode (rpb_verynear.cu). The obstacle's own geometry is evaluated once at load (it does
// not move).
#include <algorithm>
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

struct ObstacleState {
    rpb_mesh* mesh = nullptr;      // the obstacle (owned)
    Csr near, far, verynear;
    DevBuf<int> near_order, far_order;
    VFBuffers vf;
    int64_t verynear_nnz = 0, inter_nnz = 0;
    CrossLists lists;              // host copy (patterns for inspection)
    DevBuf<double> D_near, D_far, block_energy, energy;
    DevBuf<unsigned> done;
    int near_blocks = 0, far_blocks = 0;
};

rpb_mesh* obstacle_mesh(const rpb_mesh* m) { return m->obstacle ? m->obstacle->mesh : nullptr; }

void obstacle_free(rpb_mesh* m)
{
    if (!m->obstacle) return;
    rpb_mesh_destroy(m->obstacle->mesh);
    delete m->obstacle;
    m->obstacle = nullptr;
}

namespace {

// Y = beta * Y (beta = 0: Y = 0), n x 3 with leading dimension ldY
__global__ void k_scale_rows(int n, double beta, double* Y, int ldY)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    for (int k = 0; k < 3; ++k) {
        double& y = Y[static_cast<int64_t>(ldY) * v + k];
        y = (beta == 0.0) ? 0.0 : beta * y;
    }
}

template <typename T>
cudaError_t upload_vec(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s)
{
    cudaError_t e = d.alloc(h.size());
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(d.ptr, h.data(), d.bytes(), cudaMemcpyHostToDevice, s);
}

// rows of each 256-row chunk by decreasing length (as for the self-energy lists)
std::vector<int> chunk_order(const CrossPattern& P)
{
    std::vector<int> o(P.rows);
    for (int i = 0; i < P.rows; ++i) o[i] = i;
    for (int c0 = 0; c0 < P.rows; c0 += PAIR_BLOCK) {
        const int c1 = std::min(P.rows, c0 + PAIR_BLOCK);
        std::stable_sort(o.begin() + c0, o.begin() + c1,
                         [&](int a, int b) { return (P.rp[a + 1] - P.rp[a]) > (P.rp[b + 1] - P.rp[b]); });
    }
    return o;
}

template <int QH, int PH>
void launch_cross(rpb_mesh* m, const PairArgs& An, const PairArgs& Af, bool diff)
{
    ObstacleState& O = *m->obstacle;
    if (An.rows > 0) {
        auto k = diff ? k_tp0_pairs<false, QH, PH, true, NEAR_LANES, true> : k_tp0_pairs<false, QH, PH, false, NEAR_LANES, true>;
        k<<<O.near_blocks, PAIR_BLOCK, 0, m->stream>>>(An);
    }
    if (Af.rows > 0) {
        auto k = diff ? k_tp0_pairs<true, QH, PH, true, FAR_LANES, true> : k_tp0_pairs<true, QH, PH, false, FAR_LANES, true>;
        k<<<O.far_blocks, PAIR_BLOCK, 0, m->stream>>>(Af);
    }
}

rpb_status evaluate_obstacle(rpb_mesh* m, double q, double p, bool diff, double alpha, double beta, double* Y_dev,
                             int ldY, double* energy_host)
{
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    if (!m->obstacle) {
        // the reference returns 0 without an obstacle (TangentPointObstacleEnergy::value)
        if (diff) {
            k_scale_rows<<<(m->nV + 255) / 256, 256, 0, m->stream>>>(m->nV, beta, Y_dev, ldY);
            RPB_CUDA(cudaGetLastError());
        }
        if (energy_host) {
            RPB_CUDA(cudaStreamSynchronize(m->stream));
            *energy_host = 0.0;
        }
        return RPB_OK;
    }
    ObstacleState& O = *m->obstacle;
    if (!m->geometry_valid && (st = launch_geometry(m)) != RPB_OK) return st;
    const TPExp ex = make_exp(m->dom, q, p);
    PairArgs An, Af;
    An.dom = Af.dom = m->dom;
    An.ex = Af.ex = ex;
    An.close_factor = Af.close_factor = 0.1f;
    An.rows = O.near.nnz > 0 ? m->N : 0;
    An.rp = O.near.rp.ptr; An.ci = O.near.ci.ptr; An.order = O.near_order.ptr;
    An.data = m->P_pair.ptr; An.col_data = O.mesh->P_pair.ptr; An.D = O.D_near.ptr;
    An.block_energy = O.block_energy.ptr; An.done = O.done.ptr; An.energy_out = O.energy.ptr;

    Af.rows = O.far.nnz > 0 ? m->NC : 0;
    Af.rp = O.far.rp.ptr; Af.ci = O.far.ci.ptr; Af.order = O.far_order.ptr;
    Af.data = m->C_pair.ptr; Af.col_data = O.mesh->C_pair.ptr; Af.D = O.D_far.ptr;
    Af.block_energy = O.block_energy.ptr + O.near_blocks; Af.done = O.done.ptr + 1; Af.energy_out = O.energy.ptr + 1;

    if (An.rows == 0) {
        RPB_CUDA(cudaMemsetAsync(O.energy.ptr, 0, sizeof(double), m->stream));
        if (diff) RPB_CUDA(cudaMemsetAsync(O.D_near.ptr, 0, O.D_near.bytes(), m->stream));
    }
    if (Af.rows == 0) {
        RPB_CUDA(cudaMemsetAsync(O.energy.ptr + 1, 0, sizeof(double), m->stream));
        if (diff) RPB_CUDA(cudaMemsetAsync(O.D_far.ptr, 0, O.D_far.bytes(), m->stream));
    }
    if (ex.qh == 3 && ex.ph == 6) launch_cross<3, 6>(m, An, Af, diff);
    else launch_cross<-1, -1>(m, An, Af, diff);
    RPB_CUDA(cudaGetLastError());
    const bool with_vf = O.verynear.nnz > 0;
    if (with_vf &&
        (st = launch_vf_cross(m, O.mesh, O.verynear.rp.ptr, O.verynear.ci.ptr, O.verynear.nnz, O.vf, ex, diff,
                              O.energy.ptr + 2)) != RPB_OK)
        return st;
    if (diff && (st = launch_collect_gather(m, alpha, beta, Y_dev, ldY, with_vf ? O.vf.D.ptr : nullptr, O.D_near.ptr,
                                            O.D_far.ptr)) != RPB_OK)
        return st;
    if (energy_host) {
        double e[3] = {0, 0, 0};
        RPB_CUDA(cudaMemcpyAsync(e, O.energy.ptr, sizeof(e), cudaMemcpyDeviceToHost, m->stream));
        RPB_CUDA(cudaStreamSynchronize(m->stream));
        *energy_host = (e[2] + e[0]) + e[1];   // (very near + near) + far
        if (with_vf && (st = vf_take_status(O.vf, m->stream)) != RPB_OK) return st;
    }
    return RPB_OK;
}

}  // namespace
}  // namespace rpb

using namespace rpb;

extern "C" {

rpb_status rpb_mesh_load_obstacle(rpb_mesh* m, rpb_mesh* obstacle)
{
    if (!m || !obstacle) { set_error("null argument"); return RPB_EINVAL; }
    if (m == obstacle) { set_error("a mesh cannot be its own obstacle"); return RPB_EINVAL; }
    if (obstacle->device != m->device) { set_error("mesh and obstacle live on different devices"); return RPB_EINVAL; }
    if (obstacle->dom != m->dom) {
        set_error("the obstacle's domain dimension differs from the mesh's");
        return RPB_EINVAL;
    }
    if (obstacle->obstacle) { set_error("the obstacle has an obstacle of its own"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    auto* O = new ObstacleState();
    auto fail = [&](rpb_status st) { O->mesh = nullptr; delete O; return st; };
    const std::string err = build_cross_lists(m->tree, m->V_frozen.data(), m->S_host.data(), obstacle->tree,
                                              obstacle->V_frozen.data(), obstacle->S_host.data(), m->settings,
                                              O->lists);
    if (!err.empty()) { set_error(err); return fail(RPB_EINVAL); }
    cudaStream_t s = m->stream;
    const CrossLists& L = O->lists;
    O->near.rows = L.near.rows; O->near.nnz = L.near.nnz();
    O->far.rows = L.far.rows; O->far.nnz = L.far.nnz();
    O->verynear.rows = L.verynear.rows; O->verynear.nnz = L.verynear.nnz();
    O->verynear_nnz = L.verynear.nnz();
    O->inter_nnz = L.inter.nnz();
    const std::vector<int> no = chunk_order(L.near), fo = chunk_order(L.far);
    O->near_blocks = pair_blocks(m->N, NEAR_LANES);
    O->far_blocks = pair_blocks(m->NC, FAR_LANES);
    if (upload_vec(O->near.rp, L.near.rp, s) || upload_vec(O->near.ci, L.near.ci, s) ||
        upload_vec(O->far.rp, L.far.rp, s) || upload_vec(O->far.ci, L.far.ci, s) ||
        upload_vec(O->near_order, no, s) || upload_vec(O->far_order, fo, s) ||
        upload_vec(O->verynear.rp, L.verynear.rp, s) || upload_vec(O->verynear.ci, L.verynear.ci, s)) {
        set_error("obstacle list upload failed");
        return fail(RPB_ENOMEM);
    }
    if (O->D_near.alloc(10 * static_cast<size_t>(m->N)) || O->D_far.alloc(10 * static_cast<size_t>(m->NC)) ||
        O->block_energy.alloc(O->near_blocks + O->far_blocks) || O->energy.alloc(3) || O->done.alloc(4)) {
        set_error("device allocation failed");
        return fail(RPB_ENOMEM);
    }
    if (O->verynear.nnz > 0) {
        const rpb_status vst = vf_alloc(O->vf, O->verynear.nnz, m->N);
        if (vst != RPB_OK) return fail(vst);
    }
    if (cudaMemsetAsync(O->done.ptr, 0, O->done.bytes(), s) != cudaSuccess ||
        cudaMemsetAsync(O->energy.ptr, 0, O->energy.bytes(), s) != cudaSuccess) {
        set_error("memset failed");
        return fail(RPB_ECUDA);
    }
    // the obstacle's simplex data and cluster moments, once
    if (!obstacle->geometry_valid) {
        const rpb_status st = launch_geometry(obstacle);
        if (st != RPB_OK) return fail(st);
    }
    if (cudaStreamSynchronize(obstacle->stream) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("synchronization failed");
        return fail(RPB_ECUDA);
    }
    obstacle_free(m);
    O->mesh = obstacle;
    m->obstacle = O;
    return RPB_OK;
}

rpb_status rpb_mesh_obstacle_stats(const rpb_mesh* m, int64_t* counts)
{
    if (!m || !counts) { set_error("null argument"); return RPB_EINVAL; }
    if (!m->obstacle) { set_error("no obstacle loaded"); return RPB_EINVAL; }
    const CrossLists& L = m->obstacle->lists;
    counts[0] = L.near.nnz();
    counts[1] = L.far.nnz();
    counts[2] = L.verynear.nnz();
    counts[3] = L.inter.nnz();
    return RPB_OK;
}

rpb_status rpb_mesh_obstacle_pattern(const rpb_mesh* m, int which, int64_t* rowptr, int* colidx)
{
    if (!m || !rowptr || !colidx) { set_error("null argument"); return RPB_EINVAL; }
    if (!m->obstacle) { set_error("no obstacle loaded"); return RPB_EINVAL; }
    const CrossLists& L = m->obstacle->lists;
    const CrossPattern* P = which == 0 ? &L.near : which == 1 ? &L.far : which == 2 ? &L.verynear
                          : which == 3 ? &L.inter : nullptr;
    if (!P) { set_error("pattern must be 0 (near), 1 (far), 2 (very near) or 3 (intersecting)"); return RPB_EINVAL; }
    std::copy(P->rp.begin(), P->rp.end(), rowptr);
    std::copy(P->ci.begin(), P->ci.end(), colidx);
    return RPB_OK;
}

rpb_status rpb_tpoe_value(rpb_mesh* m, double q, double p, double* energy)
{
    if (!m || !energy) { set_error("null argument"); return RPB_EINVAL; }
    return evaluate_obstacle(m, q, p, false, 0.0, 0.0, nullptr, 3, energy);
}

rpb_status rpb_tpoe_differential(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y, int ldY,
                                 double* energy)
{
    if (!m || !Y) { set_error("null argument"); return RPB_EINVAL; }
    if (ldY < 3) { set_error("ldY must be >= AMB_DIM = 3"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    if (beta != 0.0)
        RPB_CUDA(copy_rows3(m->Y.ptr, 3, Y, ldY, m->nV, cudaMemcpyHostToDevice, m->stream));
    double e = 0;
    const rpb_status st = evaluate_obstacle(m, q, p, true, alpha, beta, m->Y.ptr, 3, &e);
    if (st != RPB_OK) return st;
    RPB_CUDA(copy_rows3(Y, ldY, m->Y.ptr, 3, m->nV, cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    if (energy) *energy = e;
    return RPB_OK;
}

rpb_status rpb_tpoe_differential_device(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y_dev,
                                        int ldY, double* energy)
{
    if (!m || !Y_dev) { set_error("null argument"); return RPB_EINVAL; }
    if (ldY < 3) { set_error("ldY must be >= AMB_DIM = 3"); return RPB_EINVAL; }
    return evaluate_obstacle(m, q, p, true, alpha, beta, Y_dev, ldY, energy);
}

}  // extern "C"
