// Energy evaluation that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need the energy: hosts whose
// device memory is owned by a fixed-size arena or pool with no way to hand out more (a
// simulation or renderer that reserves all of its memory at start-up), and real-time or
// inner-loop code that forbids allocation after start-up because an allocation can
// synchronize the device or fail under memory pressure. rpb_tpe0_value_noalloc serves
// them: it runs the same geometry, moment-upsweep and pair kernels as rpb_tpe0_value, but
// its scratch memory (primitive and cluster pair data, prefix sums, block partials) lives
// in one file-scope device array of fixed size instead of buffers owned by an rpb_mesh.
//
// Limits and behaviour:
//  * at most RPB_NOALLOC_MAX_SIMPLICES simplices (40,960) and 2*that-1 clusters; larger
//    meshes are rejected with RPB_EINVAL, and so are meshes with very-near primitive pairs
//    (this entry point evaluates the near and far lists only);
//  * the array (about 12.4 MB) is part of the module: every GPU that loads the library
//    holds it until the process exits;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//    with that device current; make that first call before any stream capture;
//  * all calls share the one array and it keeps the last call's contents, so calls whose
//    work overlaps on the GPU (different streams, or several host threads) race; the
//    counters that must start at zero are cleared at the start of every call;
//  * perm, C_begin and C_end must be the tree of the same mesh as returned by
//    rpb_mesh_tree, and the patterns those of rpb_mesh_pattern: only the sizes are checked;
//  * no cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>
#include <string>

#include "kernels_energy.cuh"
#include "rpb_internal.cuh"

namespace rpb {
namespace {

constexpr int kMaxSimplices = 40960;
constexpr int kMaxClusters = 2 * kMaxSimplices - 1;
constexpr int kMaxBlocksN = (kMaxSimplices + SCAN_BLOCK - 1) / SCAN_BLOCK;
constexpr int kMaxPairBlocksN = pair_blocks(kMaxSimplices, NEAR_LANES);
constexpr int kMaxPairBlocksC = pair_blocks(kMaxClusters, FAR_LANES);

// byte offsets inside the scratch array (each region 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
constexpr size_t kOffPrim = 0;
constexpr size_t kOffClus = align256(kOffPrim + sizeof(PrimDatum) * kMaxSimplices);
constexpr size_t kOffLocal = align256(kOffClus + sizeof(ClusterDatum) * kMaxClusters);
constexpr size_t kOffBlocks = align256(kOffLocal + sizeof(double) * 10 * kMaxSimplices);
constexpr size_t kOffPartials = align256(kOffBlocks + sizeof(double) * 10 * (kMaxBlocksN + 1));
constexpr size_t kOffEnergy = align256(kOffPartials + sizeof(double) * (kMaxPairBlocksN + kMaxPairBlocksC));
constexpr size_t kOffDone = align256(kOffEnergy + sizeof(double) * 2);
constexpr size_t kScratchBytes = align256(kOffDone + sizeof(unsigned) * 4);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
rpb_status scratch_on_current_device(unsigned char** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_error("rpb_tpe0_value_noalloc: no usable current CUDA device");
        return RPB_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("rpb_tpe0_value_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return RPB_ECUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return RPB_OK;
}

template <int QH, int PH>
void launch_energy_pairs(const PairArgs& An, const PairArgs& Af, int nb_near, int nb_far, cudaStream_t s)
{
    if (An.rows > 0) k_tp0_pairs<false, QH, PH, false, NEAR_LANES><<<nb_near, PAIR_BLOCK, 0, s>>>(An);
    if (Af.rows > 0) k_tp0_pairs<true, QH, PH, false, FAR_LANES><<<nb_far, PAIR_BLOCK, 0, s>>>(Af);
}

}  // namespace
}  // namespace rpb

using namespace rpb;

extern "C" rpb_status rpb_tpe0_value_noalloc(int dom_dim, const double* V, int64_t nV, const int* S, int64_t nS,
                                             const int* perm, const int* C_begin, const int* C_end, int64_t nC,
                                             const int64_t* near_rowptr, const int* near_colidx,
                                             const int64_t* far_rowptr, const int* far_colidx, int64_t verynear_nnz,
                                             double q, double p, double* energy, void* stream)
{
    if (dom_dim != 1 && dom_dim != 2) { set_error("rpb_tpe0_value_noalloc: domain dimension must be 1 or 2"); return RPB_EINVAL; }
    if (!V || !S || !perm || !C_begin || !C_end || !near_rowptr || !far_rowptr || !energy || nV <= 0 || nS <= 0) {
        set_error("rpb_tpe0_value_noalloc: null or empty argument");
        return RPB_EINVAL;
    }
    if (verynear_nnz != 0) {
        set_error("rpb_tpe0_value_noalloc: the mesh has very-near primitive pairs (verynear_nnz = " +
                  std::to_string(verynear_nnz) + "), which this entry point does not evaluate; use rpb_tpe0_value");
        return RPB_EINVAL;
    }
    if (nS > kMaxSimplices || nC > kMaxClusters || nC < 1) {
        set_error("rpb_tpe0_value_noalloc: the mesh exceeds the fixed scratch size (at most " +
                  std::to_string(kMaxSimplices) + " simplices and " + std::to_string(kMaxClusters) +
                  " clusters); use rpb_tpe0_value");
        return RPB_EINVAL;
    }
    if (nC > 2 * nS - 1) {
        set_error("rpb_tpe0_value_noalloc: nC = " + std::to_string(nC) + " exceeds 2 nS - 1 = " +
                  std::to_string(2 * nS - 1) + "; pass the tree rpb_mesh_tree returns for this mesh");
        return RPB_EINVAL;
    }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    unsigned char* base = nullptr;
    if ((st = scratch_on_current_device(&base)) != RPB_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int N = static_cast<int>(nS), NC = static_cast<int>(nC);
    auto* P_pair = reinterpret_cast<PrimDatum*>(base + kOffPrim);
    auto* C_pair = reinterpret_cast<ClusterDatum*>(base + kOffClus);
    auto* local = reinterpret_cast<double*>(base + kOffLocal);
    auto* blocks = reinterpret_cast<double*>(base + kOffBlocks);
    auto* partials = reinterpret_cast<double*>(base + kOffPartials);
    auto* e2 = reinterpret_cast<double*>(base + kOffEnergy);
    auto* done = reinterpret_cast<unsigned*>(base + kOffDone);
    if (cudaMemsetAsync(e2, 0, sizeof(double) * 2, s) != cudaSuccess ||
        cudaMemsetAsync(done, 0, sizeof(unsigned) * 4, s) != cudaSuccess) {
        set_error("rpb_tpe0_value_noalloc: clearing the scratch counters failed");
        return RPB_ECUDA;
    }
    GeomArgs g;
    g.dom = dom_dim; g.N = N; g.NC = NC;
    g.V = V; g.S = S; g.charge_v = nullptr; g.perm = perm; g.C_begin = C_begin; g.C_end = C_end;
    g.P_pair = P_pair; g.C_pair = C_pair; g.C_mom = nullptr; g.local = local; g.blocks = blocks;
    const int nb = (N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_geometry_prims<<<nb, SCAN_BLOCK, 0, s>>>(g);
    k_scan_rows<10><<<1, SCAN_BLOCK, 0, s>>>(blocks, nb);
    k_cluster_moments<<<(NC + 255) / 256, 256, 0, s>>>(g);
    const TPExp ex = make_exp(dom_dim, q, p);
    const int nb_near = pair_blocks(N, NEAR_LANES), nb_far = pair_blocks(NC, FAR_LANES);
    PairArgs An, Af;
    An.col_data = Af.col_data = nullptr;
    An.dom = Af.dom = dom_dim;
    An.ex = Af.ex = ex;
    An.close_factor = Af.close_factor = 0.1f;
    An.rows = near_colidx ? N : 0; An.rp = near_rowptr; An.ci = near_colidx; An.order = nullptr; An.data = P_pair;
    An.D = nullptr; An.block_energy = partials; An.done = done; An.energy_out = e2;
    Af.rows = far_colidx ? NC : 0; Af.rp = far_rowptr; Af.ci = far_colidx; Af.order = nullptr; Af.data = C_pair;
    Af.D = nullptr; Af.block_energy = partials + nb_near; Af.done = done + 1; Af.energy_out = e2 + 1;
    if (ex.qh == 3 && ex.ph == 6) launch_energy_pairs<3, 6>(An, Af, nb_near, nb_far, s);
    else launch_energy_pairs<-1, -1>(An, Af, nb_near, nb_far, s);
    k_add_pair<<<1, 1, 0, s>>>(e2, energy);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("rpb_tpe0_value_noalloc: launch failed: ") + cudaGetErrorString(e));
        return RPB_ECUDA;
    }
    return RPB_OK;
}
