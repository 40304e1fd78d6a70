// C ABI of the B200 tangent-point path: mesh lifetime, tree upload, energy and
// differential. Metric and solver entry points live in rpb_metric.cu / rpb_solver.cu.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "../../include/repulsor_b200.h"
#include "host/sparse_cholesky.hpp"
#include "kernels_energy.cuh"
#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

}  // namespace rpb

using namespace rpb;

#define RPB_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);   \
            return e_ == cudaErrorMemoryAllocation ? RPB_ENOMEM : RPB_ECUDA;                  \
        }                                                                                     \
    } while (0)

int64_t rpb_mesh::device_bytes() const
{
    int64_t b = 0;
    b += V.bytes() + charge_v.bytes() + S.bytes() + perm.bytes() + leaf_of.bytes() + C_parent.bytes() +
         C_up4.bytes() + C_left.bytes() + C_right.bytes();
    b += near.rp.bytes() + near.ci.bytes() + far.rp.bytes() + far.ci.bytes() + verynear.rp.bytes() +
         verynear.ci.bytes() + near_order.bytes() + far_order.bytes();
    for (const rpb::TileBufs* t : {&near_tiles, &far_tiles})
        b += t->row0.bytes() + t->cols_rp.bytes() + t->cols.bytes() + t->order.bytes() + t->slot.bytes() +
             t->lane_map.bytes();
    b += P_pair.bytes() + C_pair.bytes() + counter.bytes() + P_near.bytes() + scan_local.bytes() +
         scan_blocks.bytes() + C_begin.bytes() + C_end.bytes();
    b += D_near.bytes() + D_far.bytes() + vf.bytes() + B.bytes() + v_rp.bytes() + v_slot.bytes() + Y.bytes();
    b += block_energy.bytes() + energy.bytes() + done.bytes();
    b += pre_cols.bytes() + pre_vals.bytes() + vp_rp.bytes() + vp_slot.bytes();
    b += buf_Pin64.bytes() + buf_Cin64.bytes() + buf_Pout.bytes() + buf_Cout.bytes() + buf_Z.bytes() + X.bytes() +
         Yb.bytes() + buf_scan_local.bytes() + buf_scan_blocks.bytes();
    b += metric.nf.bytes() + metric.ff.bytes() + metric.vf.bytes() + metric.nf_diag.bytes() +
         metric.ff_diag.bytes() + metric.vf_diag.bytes();
    b += plap.nf.bytes() + plap.ff.bytes() + plap.vf.bytes() + plap.nf_diag.bytes() + plap.ff_diag.bytes() +
         plap.vf_diag.bytes();
    return b;
}

namespace rpb {

// 16 independent FMA chains per thread, fully register resident.
__global__ void k_fma_peak(float* out, int iters, float m)
{
    float r[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) r[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) r[k] = fmaf(r[k], m, 1e-7f);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += r[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
static rpb_status upload(DevBuf<T>& d, const T* h, size_t n, cudaStream_t s)
{
    RPB_CUDA(d.alloc(n));
    if (n) RPB_CUDA(cudaMemcpyAsync(d.ptr, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    return RPB_OK;
}

static rpb_status upload_pattern(Csr& d, const SymPattern& P, cudaStream_t s)
{
    d.rows = P.rows;
    d.nnz = P.nnz();
    rpb_status st = upload(d.rp, P.rp.data(), P.rp.size(), s);
    if (st != RPB_OK) return st;
    return upload(d.ci, P.ci.data(), P.ci.size(), s);
}

TPExp make_exp(int dom, double q, double p)
{
    TPExp e;
    e.q = q;
    e.p = p;
    const double s = (p - dom) / q;
    e.s_exp_metric = -0.5 * (2.0 * (s - 1.0) + dom);
    const double qh = q / 2, ph = p / 2;
    e.qh = (qh == std::floor(qh)) ? static_cast<int>(qh) : -1;
    e.ph = (ph == std::floor(ph)) ? static_cast<int>(ph) : -1;
    return e;
}

rpb_status check_exponents(double q, double p)
{
    if (!(q >= 2.0) || !std::isfinite(q) || !std::isfinite(p) || !(p > 0)) {
        set_error("tangent-point kernels need q >= 2 and p > 0 (the reference rejects q < 0 and 0 < q < 2)");
        return RPB_EINVAL;
    }
    return RPB_OK;
}

// SemiStaticUpdate on the device: simplex data + cluster moments.
rpb_status launch_geometry(rpb_mesh* m)
{
    GeomArgs g;
    g.dom = m->dom;
    g.N = m->N;
    g.NC = m->NC;
    g.V = m->V.ptr;
    g.S = m->S.ptr;
    g.charge_v = m->charge_v.ptr;
    g.perm = m->perm.ptr;
    g.C_begin = m->C_begin.ptr;
    g.C_end = m->C_end.ptr;
    g.P_pair = m->P_pair.ptr;
    g.C_pair = m->C_pair.ptr;
    g.C_mom = nullptr;   // the FP64 moments are not read by any later kernel
    g.local = m->scan_local.ptr;
    g.blocks = m->scan_blocks.ptr;
    const int nb = (m->N + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_geometry_prims<<<nb, SCAN_BLOCK, 0, m->stream>>>(g);
    launch_pdl(k_scan_rows<10>, 1, SCAN_BLOCK, 0, m->stream, m->scan_blocks.ptr, nb);
    launch_pdl(k_cluster_moments, (m->NC + 255) / 256, 256, 0, m->stream, g);
    RPB_CUDA(cudaGetLastError());
    m->geometry_valid = true;
    m->geometry_version++;
    m->metric.valid = false;
    m->plap.valid = false;
    return RPB_OK;
}

// Largest dynamic shared memory a tiled pair kernel may ask for, set once per device for
// every instantiation (the attribute only permits; each launch asks for its tiles' need).
template <int QH, int PH>
static cudaError_t allow_tile_smem_t(int optin)
{
    const int nb = optin, fb = optin;
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, int bytes) {
        // the block's static shared memory counts against the same per-block limit
        cudaFuncAttributes fa;
        cudaError_t r = cudaFuncGetAttributes(&fa, f);
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     bytes - static_cast<int>(fa.sharedSizeBytes));
        if (e == cudaSuccess) e = r;
    };
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled<false, QH, PH, true>), nb);
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled<false, QH, PH, false>), nb);
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled<true, QH, PH, true>), fb);
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled<true, QH, PH, false>), fb);
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled_both<QH, PH, true>), std::max(nb, fb));
    set(reinterpret_cast<const void*>(k_tp0_pairs_tiled_both<QH, PH, false>), std::max(nb, fb));
    return e;
}

static rpb_status allow_tile_smem(int device)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), device) != done.end()) return RPB_OK;
    int optin = 0;
    RPB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    RPB_CUDA((allow_tile_smem_t<3, 6>(optin)));
    RPB_CUDA((allow_tile_smem_t<2, 4>(optin)));
    RPB_CUDA((allow_tile_smem_t<1, 2>(optin)));
    RPB_CUDA((allow_tile_smem_t<-1, -1>(optin)));
    done.push_back(device);
    return RPB_OK;
}

// Tiles [first, first + count) of shard `shard` of `shards` (all tiles for shard < 0).
static void shard_tiles(const TileBufs& t, int shard, int shards, int& first, int& count)
{
    if (shard < 0) { first = 0; count = t.tiles; return; }
    first = static_cast<int>(static_cast<int64_t>(t.tiles) * shard / shards);
    count = static_cast<int>(static_cast<int64_t>(t.tiles) * (shard + 1) / shards) - first;
}

static PairTiles tiles_view(const TileBufs& t, int first)
{
    return PairTiles{t.row0.ptr, t.cols_rp.ptr, t.cols.ptr, t.slot.ptr, t.order.ptr, t.lane_map.ptr, first};
}

// Shared-memory row tiles of a CSR pattern (one kernel block per tile). Tiles are balanced
// by entries and their count is shards x a whole number of waves of resident blocks (no
// partial last wave, whose few blocks would run while the other SMs idle), so that each
// of `shards` GPUs owns whole waves; at most NEAR_TILE_ROWS / FAR_TILE_ROWS rows per tile
// on average. A pattern whose rows exceed the union cap keeps the gather kernel (d.valid
// stays false).
static rpb_status tile_pattern(rpb_mesh* m, int rows, const int64_t* rp, const int* ci, int64_t nnz, int ncols,
                               bool far, const void* kernel, int cap, int shards, TileBufs& d)
{
    cudaStream_t s = m->stream;
    d.valid = false;
    d.tiles = 0;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device) != cudaSuccess) sms = 0;
    auto resident = [&](int max_union, int64_t max_entries) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, PAIR_TILE_THREADS,
                                                          pair_tile_smem(max_union, far, max_entries)) != cudaSuccess)
            return 0;
        return per_sm;
    };
    auto most_entries = [&](const RowTiles& R) {
        int64_t e = 0;
        for (int b = 0; b < R.tiles(); ++b) e = std::max(e, rp[R.row0[b + 1]] - rp[R.row0[b]]);
        return e;
    };
    if (sms <= 0 || nnz == 0) return RPB_OK;
    // resident blocks depend on the tiles' largest union and entry count, the tile size on
    // the resident blocks: start from the union cap and two blocks' share of the entries
    // and re-tile while the count changes
    int per_sm = resident(cap, (nnz + 2 * sms * shards - 1) / (2 * sms * shards));
    RowTiles R;
    int64_t max_entries = 0;
    for (int pass = 0; pass < 3 && per_sm > 0; ++pass) {
        const int64_t slots = static_cast<int64_t>(per_sm) * sms * shards;
        const int64_t tile_rows = far ? FAR_TILE_ROWS : NEAR_TILE_ROWS;
        const int64_t waves = std::max<int64_t>(1, (rows + slots * tile_rows - 1) / (slots * tile_rows));
        const int64_t target = (nnz + waves * slots - 1) / (waves * slots);
        build_row_tiles(rp, ci, rows, ncols, PAIR_TILE_THREADS, target, cap, std::max(1, m->settings.threads), R);
        if (!R.valid) break;
        max_entries = most_entries(R);
        const int now = resident(R.max_union, max_entries);
        if (now == per_sm) break;
        per_sm = now;
    }
    if (per_sm <= 0 || !R.valid || R.tiles() == 0) return RPB_OK;
    // the kernels copy every tile's slots by 16-byte pieces, the last of which may reach up
    // to PAIR_SLOT_PAD - 1 entries past the pattern's end
    R.slot.resize(R.slot.size() + PAIR_SLOT_PAD, 0);
    rpb_status e;
    if ((e = upload(d.row0, R.row0.data(), R.row0.size(), s)) != RPB_OK) return e;
    if ((e = upload(d.cols_rp, R.cols_rp.data(), R.cols_rp.size(), s)) != RPB_OK) return e;
    if ((e = upload(d.cols, R.cols.data(), R.cols.size(), s)) != RPB_OK) return e;
    if ((e = upload(d.order, R.order.data(), R.order.size(), s)) != RPB_OK) return e;
    if ((e = upload(d.slot, R.slot.data(), R.slot.size(), s)) != RPB_OK) return e;
    if ((e = upload(d.lane_map, R.lane_map.data(), R.lane_map.size(), s)) != RPB_OK) return e;
    d.row0_host = R.row0;
    d.tiles = R.tiles();
    d.max_union = R.max_union;
    d.max_entries = max_entries;
    d.valid = true;
    return RPB_OK;
}

// Per-block energy partials for `blocks` blocks of the pair launches (never shrinks).
static rpb_status ensure_block_energy(rpb_mesh* m, int blocks)
{
    if (m->block_energy.n >= static_cast<size_t>(blocks)) return RPB_OK;
    if (m->block_energy.alloc(blocks)) {
        set_error("device allocation failed");
        return RPB_ENOMEM;
    }
    return RPB_OK;
}

// Row tiles of the two patterns for `shards` row shards (1 at mesh creation; more with
// rpb_mesh_set_shards). Sets the launch grids of the pair kernels.
static rpb_status build_pair_tiles(rpb_mesh* m, int shards)
{
    rpb_status st;
    if ((st = allow_tile_smem(m->device)) != RPB_OK) return st;
    m->near_blocks = pair_blocks(m->N, NEAR_LANES);
    m->far_blocks = pair_blocks(m->NC, FAR_LANES);
    const void* kn = reinterpret_cast<const void*>(k_tp0_pairs_tiled<false, 3, 6, true>);
    const void* kf = reinterpret_cast<const void*>(k_tp0_pairs_tiled<true, 3, 6, true>);
    const SymPattern& Pn = m->tree.near;
    const SymPattern& Pf = m->tree.far;
    if ((st = tile_pattern(m, Pn.rows, Pn.rp.data(), Pn.ci.data(), Pn.nnz(), m->N, false, kn, NEAR_TILE_UNION, shards,
                           m->near_tiles)) != RPB_OK)
        return st;
    if ((st = tile_pattern(m, Pf.rows, Pf.rp.data(), Pf.ci.data(), Pf.nnz(), m->NC, true, kf, FAR_TILE_UNION, shards,
                           m->far_tiles)) != RPB_OK)
        return st;
    if (m->near_tiles.valid) m->near_blocks = m->near_tiles.tiles;
    if (m->far_tiles.valid) m->far_blocks = m->far_tiles.tiles;
    m->shards = shards;
    return ensure_block_energy(m, m->near_blocks + m->far_blocks);
}

template <int QH, int PH>
static void launch_pairs_t(rpb_mesh* m, const PairArgs& An, const PairArgs& Af, bool diff, cudaEvent_t between,
                           int shard)
{
    if (An.rows > 0 && Af.rows > 0 && m->near_tiles.valid && m->far_tiles.valid && !between) {
        int nfirst, ncount, ffirst, fcount;
        shard_tiles(m->near_tiles, shard, m->shards, nfirst, ncount);
        shard_tiles(m->far_tiles, shard, m->shards, ffirst, fcount);
        if (ncount > 0 && fcount > 0) {
            const size_t smem = std::max(pair_tile_smem(m->near_tiles.max_union, false, m->near_tiles.max_entries),
                                         pair_tile_smem(m->far_tiles.max_union, true, m->far_tiles.max_entries));
            launch_pdl(diff ? k_tp0_pairs_tiled_both<QH, PH, true> : k_tp0_pairs_tiled_both<QH, PH, false>,
                       ncount + fcount, PAIR_TILE_THREADS, smem, m->stream, An, tiles_view(m->near_tiles, nfirst), Af,
                       tiles_view(m->far_tiles, ffirst), fcount);
            return;
        }
    }
    if (An.rows > 0) {
        const TileBufs& t = m->near_tiles;
        if (t.valid) {
            int first, count;
            shard_tiles(t, shard, m->shards, first, count);
            const size_t smem = pair_tile_smem(t.max_union, false, t.max_entries);
            if (count > 0)
                launch_pdl(diff ? k_tp0_pairs_tiled<false, QH, PH, true> : k_tp0_pairs_tiled<false, QH, PH, false>, count,
                           PAIR_TILE_THREADS, smem, m->stream, An, tiles_view(t, first));
        } else if (diff) k_tp0_pairs<false, QH, PH, true, NEAR_LANES><<<m->near_blocks, PAIR_BLOCK, 0, m->stream>>>(An);
        else k_tp0_pairs<false, QH, PH, false, NEAR_LANES><<<m->near_blocks, PAIR_BLOCK, 0, m->stream>>>(An);
    }
    if (between) cudaEventRecord(between, m->stream);
    if (Af.rows > 0) {
        const TileBufs& t = m->far_tiles;
        if (t.valid) {
            int first, count;
            shard_tiles(t, shard, m->shards, first, count);
            const size_t smem = pair_tile_smem(t.max_union, true, t.max_entries);
            if (count > 0)
                launch_pdl(diff ? k_tp0_pairs_tiled<true, QH, PH, true> : k_tp0_pairs_tiled<true, QH, PH, false>, count,
                           PAIR_TILE_THREADS, smem, m->stream, Af, tiles_view(t, first));
        } else if (diff) k_tp0_pairs<true, QH, PH, true, FAR_LANES><<<m->far_blocks, PAIR_BLOCK, 0, m->stream>>>(Af);
        else k_tp0_pairs<true, QH, PH, false, FAR_LANES><<<m->far_blocks, PAIR_BLOCK, 0, m->stream>>>(Af);
    }
}

// Near- and far-field pair kernels on the mesh stream. shard >= 0: only that row shard's
// tiles (both patterns tiled), derivatives into D_near / D_far (zeroed first), energies into
// energy[0..1]; shard < 0: every row, into the mesh's own buffers.
rpb_status launch_pairs(rpb_mesh* m, const TPExp& ex, bool diff, cudaEvent_t between = nullptr, int shard = -1,
                        double* D_near = nullptr, double* D_far = nullptr)
{
    PairArgs An, Af;
    An.col_data = Af.col_data = nullptr;
    An.dom = Af.dom = m->dom;
    An.ex = Af.ex = ex;
    An.close_factor = Af.close_factor = 0.1f;
    An.rows = m->near.nnz > 0 ? m->N : 0;
    An.rp = m->near.rp.ptr; An.ci = m->near.ci.ptr; An.data = m->P_pair.ptr; An.D = m->D_near.ptr;
    An.order = m->near_order.ptr;
    An.block_energy = m->block_energy.ptr; An.done = m->done.ptr; An.energy_out = m->energy.ptr;

    Af.rows = m->far.nnz > 0 ? m->NC : 0;
    Af.rp = m->far.rp.ptr; Af.ci = m->far.ci.ptr; Af.data = m->C_pair.ptr; Af.D = m->D_far.ptr;
    Af.order = m->far_order.ptr;
    Af.block_energy = m->block_energy.ptr + m->near_blocks; Af.done = m->done.ptr + 1; Af.energy_out = m->energy.ptr + 1;

    if (shard >= 0) {
        An.D = D_near;
        Af.D = D_far;
        RPB_CUDA(cudaMemsetAsync(D_near, 0, sizeof(double) * 10 * static_cast<size_t>(m->N), m->stream));
        RPB_CUDA(cudaMemsetAsync(D_far, 0, sizeof(double) * 10 * static_cast<size_t>(m->NC), m->stream));
        int first, count;
        shard_tiles(m->near_tiles, shard, m->shards, first, count);
        if (count == 0) An.rows = 0;
        shard_tiles(m->far_tiles, shard, m->shards, first, count);
        if (count == 0) Af.rows = 0;
    }
    if (An.rows == 0) {
        RPB_CUDA(cudaMemsetAsync(m->energy.ptr, 0, sizeof(double), m->stream));
        if (diff && shard < 0) RPB_CUDA(cudaMemsetAsync(m->D_near.ptr, 0, m->D_near.bytes(), m->stream));
    }
    if (Af.rows == 0) {
        RPB_CUDA(cudaMemsetAsync(m->energy.ptr + 1, 0, sizeof(double), m->stream));
        if (diff && shard < 0) RPB_CUDA(cudaMemsetAsync(m->D_far.ptr, 0, m->D_far.bytes(), m->stream));
    }
    if (ex.qh == 3 && ex.ph == 6) launch_pairs_t<3, 6>(m, An, Af, diff, between, shard);
    else if (ex.qh == 2 && ex.ph == 4) launch_pairs_t<2, 4>(m, An, Af, diff, between, shard);
    else if (ex.qh == 1 && ex.ph == 2) launch_pairs_t<1, 2>(m, An, Af, diff, between, shard);
    else launch_pairs_t<-1, -1>(m, An, Af, diff, between, shard);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status launch_collect_gather(rpb_mesh* m, double alpha, double beta, double* Y, int ldY, const double* D_vf,
                                 const double* D_near, const double* D_far)
{
    CollectArgs C;
    C.dom = m->dom;
    C.N = m->N;
    C.V = m->V.ptr;
    C.S = m->S.ptr;
    C.charge_v = m->charge_v.ptr;
    C.perm = m->perm.ptr;
    C.leaf_of = m->leaf_of.ptr;
    C.C_parent = m->C_parent.ptr;
    C.C_up4 = m->C_up4.ptr;
    C.C_pair = m->C_pair.ptr;
    C.D_near = D_near ? D_near : m->D_near.ptr;
    C.D_far = D_far ? D_far : m->D_far.ptr;
    C.D_vf = D_vf;
    C.B = m->B.ptr;
    // a plain launch: with programmatic dependent launch the collection's early blocks hold
    // SM resources during the pair kernel's last wave (measured: 9,540 against 9,985 evals/s)
    k_collect_chain<<<(m->N + 255) / 256, 256, 0, m->stream>>>(C);
    RPB_CUDA(cudaGetLastError());
    GatherArgs G;
    G.nV = m->nV;
    G.v_rp = m->v_rp.ptr;
    G.v_slot = m->v_slot.ptr;
    G.B = m->B.ptr;
    G.alpha = alpha;
    G.beta = beta;
    G.Y = Y;
    G.ldY = ldY;
    launch_pdl(k_gather_vertices, static_cast<int>((static_cast<int64_t>(m->nV) * GATHER_LANES + 255) / 256), 256, 0,
               m->stream, G);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

// (very-near + near) + far, the order evaluate() uses on the host
static __global__ void k_sum_energy_parts(const double* e, double* out) { *out = (e[2] + e[0]) + e[1]; }

// Full energy (+ differential into device Y) evaluation on the mesh stream.
rpb_status evaluate(rpb_mesh* m, double q, double p, bool diff, double alpha, double beta, double* Y_dev, int ldY,
                    double* energy_host)
{
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    const TPExp ex = make_exp(m->dom, q, p);
    if (!m->geometry_valid) {
        st = launch_geometry(m);
        if (st != RPB_OK) return st;
    }
    st = launch_pairs(m, ex, diff);
    if (st != RPB_OK) return st;
    const bool with_vf = m->verynear.nnz > 0;
    if (with_vf) {
        st = launch_vf(m, ex, diff);
        if (st != RPB_OK) return st;
    }
    if (diff) {
        st = launch_collect_gather(m, alpha, beta, Y_dev, ldY, with_vf ? m->vf.D.ptr : nullptr, nullptr, nullptr);
        if (st != RPB_OK) return st;
    }
    if (energy_host) {
        double e[3] = {0, 0, 0};
        RPB_CUDA(cudaMemcpyAsync(e, m->energy.ptr, sizeof(double) * 3, cudaMemcpyDeviceToHost, m->stream));
        RPB_CUDA(cudaStreamSynchronize(m->stream));
        *energy_host = (e[2] + e[0]) + e[1];
        if (with_vf && (st = vf_take_status(m->vf, m->stream)) != RPB_OK) return st;
    }
    return RPB_OK;
}

}  // namespace rpb

// ============================================================================================
extern "C" {

rpb_status rpb_default_settings(rpb_settings* s)
{
    if (!s) { set_error("null settings"); return RPB_EINVAL; }
    s->split_threshold = 1;
    s->far_field_separation = 0.5;
    s->near_field_separation = 10.0;
    s->near_field_intersection = 1e10;
    s->max_refinement = 30;
    s->thread_count = 0;
    s->device = 0;
    return RPB_OK;
}

const char* rpb_last_error(void) { return g_last_error.c_str(); }

rpb_status rpb_mesh_create(int dom_dim, int amb_dim, const double* Vh, int64_t nV, const int* Sh, int64_t nS,
                           const double* charges, const rpb_settings* settings, rpb_mesh** out)
{
    if (!out) { set_error("out is null"); return RPB_EINVAL; }
    *out = nullptr;
    if (amb_dim != 3) { set_error("only ambient dimension 3 is supported"); return RPB_EINVAL; }
    if (dom_dim != 1 && dom_dim != 2) { set_error("domain dimension must be 1 or 2"); return RPB_EINVAL; }
    if (!Vh || !Sh || nV <= 0 || nS <= 0) { set_error("empty mesh: (V.Dim(0) <= 0) || (simplices.Dim(0) <= 0)"); return RPB_EINVAL; }
    if (nV > (1ll << 30) || nS > (1ll << 29)) { set_error("mesh too large for 32-bit indices"); return RPB_EINVAL; }
    rpb_settings set;
    rpb_default_settings(&set);
    if (settings) set = *settings;
    if (set.split_threshold != 1) { set_error("only split_threshold = 1 is supported"); return RPB_EINVAL; }
    if (!(set.far_field_separation > 0) || !(set.near_field_separation > 0)) { set_error("separation parameters must be positive"); return RPB_EINVAL; }
    if (set.max_refinement < 0 || set.max_refinement > 60) { set_error("max_refinement must be in [0, 60]"); return RPB_EINVAL; }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= 0) {
        set_error("no CUDA device available: the B200 path has no CPU fallback");
        return RPB_ECUDA;
    }
    if (set.device < 0 || set.device >= dev_count) { set_error("device ordinal out of range"); return RPB_EINVAL; }

    auto* m = new rpb_mesh();
    m->dom = dom_dim;
    m->size = dom_dim + 1;
    m->nV = static_cast<int>(nV);
    m->N = static_cast<int>(nS);
    m->device = set.device;
    m->settings.theta_far = set.far_field_separation;
    m->settings.theta_near = set.near_field_separation;
    m->settings.max_refinement = set.max_refinement;
    m->settings.threads = set.thread_count > 0 ? set.thread_count : std::max(1u, std::thread::hardware_concurrency());
    auto fail = [&](rpb_status st) { delete m; return st; };

    if (cudaSetDevice(m->device) != cudaSuccess) { set_error("cudaSetDevice failed"); return fail(RPB_ECUDA); }
    if (cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking) != cudaSuccess) { set_error("stream creation failed"); return fail(RPB_ECUDA); }
    // the cluster tree's splits and the block cluster tree's traversal on the device (each
    // on the host if the device work fails; both give the same tree and patterns)
    const auto t0 = std::chrono::steady_clock::now();
    {
        std::vector<double> Pser;
        std::string derr;
        m->cluster_tree_on_device =
            build_cluster_tree_device(dom_dim, Vh, m->nV, Sh, m->N, m->tree, Pser, m->own_stream, derr);
        if (!m->cluster_tree_on_device) {
            cudaGetLastError();
            const std::string err = build_cluster_tree(dom_dim, Vh, m->nV, Sh, m->N, m->settings, m->tree, Pser);
            if (!err.empty()) { set_error(err); return fail(RPB_EINVAL); }
        }
        m->block_tree_on_device = build_block_cluster_tree_device(m->tree, Pser, Sh, m->settings, m->own_stream, derr);
        if (!m->block_tree_on_device) {
            cudaGetLastError();
            build_block_cluster_tree(m->tree, Pser, Sh, m->settings);
        }
    }
    m->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    m->NC = m->tree.NC;
    m->V_frozen.assign(Vh, Vh + 3 * static_cast<size_t>(m->nV));
    m->S_host.assign(Sh, Sh + static_cast<size_t>(m->size) * m->N);

    if (cudaMallocHost(reinterpret_cast<void**>(&m->host_energy), 3 * sizeof(double)) != cudaSuccess) {
        set_error("pinned host allocation failed");
        return fail(RPB_ENOMEM);
    }
    m->stream = m->own_stream;
    cudaStream_t s = m->stream;
    const HostTree& T = m->tree;
    std::vector<double> ch(m->nV, 1.0);
    if (charges) std::copy(charges, charges + m->nV, ch.begin());
    rpb_status st;
#define UP(buf, ptr, n) do { st = upload(buf, ptr, n, s); if (st != RPB_OK) return fail(st); } while (0)
    UP(m->V, Vh, 3 * static_cast<size_t>(m->nV));
    UP(m->charge_v, ch.data(), ch.size());
    UP(m->S, Sh, static_cast<size_t>(m->size) * m->N);
    UP(m->perm, T.perm.data(), T.perm.size());
    UP(m->leaf_of, T.leaf_of.data(), T.leaf_of.size());
    UP(m->C_parent, T.C_parent.data(), T.C_parent.size());
    {
        std::vector<int> up4(T.C_parent.size());
        for (size_t C = 0; C < up4.size(); ++C) {
            int a = static_cast<int>(C);
            for (int k = 0; k < 4 && a >= 0; ++k) a = T.C_parent[a];
            up4[C] = a;
        }
        UP(m->C_up4, up4.data(), up4.size());
    }
    UP(m->C_left, T.C_left.data(), T.C_left.size());
    UP(m->C_right, T.C_right.data(), T.C_right.size());
    UP(m->C_begin, T.C_begin.data(), T.C_begin.size());
    UP(m->C_end, T.C_end.data(), T.C_end.size());
    if ((st = upload_pattern(m->near, T.near, s)) != RPB_OK) return fail(st);
    if ((st = upload_pattern(m->far, T.far, s)) != RPB_OK) return fail(st);
    if ((st = upload_pattern(m->verynear, T.verynear, s)) != RPB_OK) return fail(st);
    // vertex -> slot incidence (DerivativeAssembler, src/SimplicialMesh.hpp:625-649)
    {
        std::vector<int> rp(m->nV + 1, 0), slot(static_cast<size_t>(m->size) * m->N);
        for (int64_t k = 0; k < static_cast<int64_t>(m->size) * m->N; ++k) rp[Sh[k] + 1]++;
        for (int v = 0; v < m->nV; ++v) rp[v + 1] += rp[v];
        std::vector<int> pos(rp.begin(), rp.end() - 1);
        for (int64_t k = 0; k < static_cast<int64_t>(m->size) * m->N; ++k) slot[pos[Sh[k]]++] = static_cast<int>(k);
        UP(m->v_rp, rp.data(), rp.size());
        UP(m->v_slot, slot.data(), slot.size());
    }
#undef UP
    if (m->P_pair.alloc(m->N) || m->C_pair.alloc(m->NC) ||
        m->counter.alloc(m->NC) || m->D_near.alloc(10 * static_cast<size_t>(m->N)) ||
        m->scan_local.alloc(10 * static_cast<size_t>(m->N)) ||
        m->scan_blocks.alloc(10 * static_cast<size_t>((m->N + SCAN_BLOCK - 1) / SCAN_BLOCK + 1)) ||
        m->D_far.alloc(10 * static_cast<size_t>(m->NC)) ||
        m->B.alloc(3 * static_cast<size_t>(m->size) * m->N) || m->Y.alloc(3 * static_cast<size_t>(m->nV)) ||
        m->energy.alloc(4) || m->done.alloc(4)) {
        set_error("device allocation failed");
        return fail(RPB_ENOMEM);
    }
    {
        // rows of each 256-row chunk sorted by decreasing length: threads of a warp see
        // similar trip counts while the chunk keeps the tree-order locality of its columns
        auto order_of = [](const SymPattern& P) {
            std::vector<int> o(P.rows);
            for (int i = 0; i < P.rows; ++i) o[i] = i;
            for (int c0 = 0; c0 < P.rows; c0 += PAIR_BLOCK) {
                const int c1 = std::min(P.rows, c0 + PAIR_BLOCK);
                std::stable_sort(o.begin() + c0, o.begin() + c1, [&](int a, int b) {
                    return (P.rp[a + 1] - P.rp[a]) > (P.rp[b + 1] - P.rp[b]);
                });
            }
            return o;
        };
        const std::vector<int> no = order_of(T.near), fo = order_of(T.far);
        if ((st = upload(m->near_order, no.data(), no.size(), s)) != RPB_OK) return fail(st);
        if ((st = upload(m->far_order, fo.data(), fo.size(), s)) != RPB_OK) return fail(st);
        m->near_blocks = pair_blocks(m->N, NEAR_LANES);
        m->far_blocks = pair_blocks(m->NC, FAR_LANES);
        if ((st = build_pair_tiles(m, 1)) != RPB_OK) return fail(st);
    }
    if (cudaMemsetAsync(m->counter.ptr, 0, m->counter.bytes(), s) != cudaSuccess ||
        cudaMemsetAsync(m->done.ptr, 0, m->done.bytes(), s) != cudaSuccess ||
        cudaMemsetAsync(m->energy.ptr, 0, m->energy.bytes(), s) != cudaSuccess) {
        set_error("memset failed");
        return fail(RPB_ECUDA);
    }
    if (m->verynear.nnz > 0) {
        const rpb_status vst = vf_alloc(m->vf, m->verynear.nnz, m->N);
        if (vst != RPB_OK) return fail(vst);
    }
    if ((st = launch_geometry(m)) != RPB_OK) return fail(st);
    if ((st = metric_init(m, Vh, Sh)) != RPB_OK) return fail(st);
    if (cudaStreamSynchronize(s) != cudaSuccess) { set_error("initial upload failed"); return fail(RPB_ECUDA); }
    *out = m;
    return RPB_OK;
}

rpb_status rpb_mesh_destroy(rpb_mesh* m)
{
    if (!m) return RPB_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    solver_free(m);
    learned_free(m);
    obstacle_free(m);
    cudaStream_t s = m->own_stream;
    delete m;  // frees device buffers and the pinned energy slots
    if (s) cudaStreamDestroy(s);
    return RPB_OK;
}

rpb_status rpb_mesh_set_stream(rpb_mesh* m, void* stream)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    m->stream = stream ? static_cast<cudaStream_t>(stream) : m->own_stream;
    return RPB_OK;
}

rpb_status rpb_mesh_get_stream(const rpb_mesh* m, void** stream)
{
    if (!m || !stream) { set_error("null argument"); return RPB_EINVAL; }
    *stream = static_cast<void*>(m->stream);
    return RPB_OK;
}

rpb_status rpb_mesh_stats(const rpb_mesh* m, rpb_stats* o)
{
    if (!m || !o) { set_error("null argument"); return RPB_EINVAL; }
    o->vertex_count = m->nV;
    o->simplex_count = m->N;
    o->cluster_count = m->NC;
    o->tree_depth = m->tree.depth;
    o->near_nnz = m->tree.near.nnz();
    o->far_nnz = m->tree.far.nnz();
    o->verynear_nnz = m->tree.verynear.nnz();
    o->inter_nnz = m->tree.inter.nnz();
    o->tree_build_seconds = m->build_seconds;
    o->device_bytes = m->device_bytes();
    return RPB_OK;
}

rpb_status rpb_mesh_build_info(const rpb_mesh* m, int* cluster_tree_on_device, int* block_tree_on_device)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    if (cluster_tree_on_device) *cluster_tree_on_device = m->cluster_tree_on_device ? 1 : 0;
    if (block_tree_on_device) *block_tree_on_device = m->block_tree_on_device ? 1 : 0;
    return RPB_OK;
}

rpb_status rpb_mesh_tree(const rpb_mesh* m, int* perm, int* C_begin, int* C_end, int* C_left, int* C_right)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    const HostTree& T = m->tree;
    if (perm) std::copy(T.perm.begin(), T.perm.end(), perm);
    if (C_begin) std::copy(T.C_begin.begin(), T.C_begin.end(), C_begin);
    if (C_end) std::copy(T.C_end.begin(), T.C_end.end(), C_end);
    if (C_left) std::copy(T.C_left.begin(), T.C_left.end(), C_left);
    if (C_right) std::copy(T.C_right.begin(), T.C_right.end(), C_right);
    return RPB_OK;
}

rpb_status rpb_mesh_pattern(const rpb_mesh* m, int which, int64_t* rowptr, int* colidx)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    const SymPattern* P = which == 0 ? &m->tree.near : which == 1 ? &m->tree.far : which == 2 ? &m->tree.verynear
                        : which == 3 ? &m->tree.inter : nullptr;
    if (!P) { set_error("pattern id must be 0..3"); return RPB_EINVAL; }
    if (rowptr) std::copy(P->rp.begin(), P->rp.end(), rowptr);
    if (colidx) std::copy(P->ci.begin(), P->ci.end(), colidx);
    return RPB_OK;
}

struct rpb_host_tree {
    HostTree tree;
    TreeSettings settings;
    double seconds = 0;
};

rpb_status rpb_tree_build_host(int dom_dim, const double* V, int64_t nV, const int* S, int64_t nS,
                               const rpb_settings* settings, rpb_host_tree** out)
{
    if (!out) { set_error("out is null"); return RPB_EINVAL; }
    *out = nullptr;
    if (!V || !S || nV <= 0 || nS <= 0) { set_error("empty mesh"); return RPB_EINVAL; }
    if (nV > (1ll << 30) || nS > (1ll << 29)) { set_error("mesh too large for 32-bit indices"); return RPB_EINVAL; }
    rpb_settings set;
    rpb_default_settings(&set);
    if (settings) set = *settings;
    if (set.split_threshold != 1) { set_error("only split_threshold = 1 is supported"); return RPB_EINVAL; }
    TreeSettings ts;
    ts.theta_far = set.far_field_separation;
    ts.theta_near = set.near_field_separation;
    ts.max_refinement = set.max_refinement;
    ts.threads = set.thread_count > 0 ? set.thread_count : std::max(1u, std::thread::hardware_concurrency());
    auto* t = new rpb_host_tree();
    t->settings = ts;
    const auto t0 = std::chrono::steady_clock::now();
    const std::string err = build_tree(dom_dim, V, static_cast<int>(nV), S, static_cast<int>(nS), ts, t->tree);
    if (!err.empty()) { delete t; set_error(err); return RPB_EINVAL; }
    t->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = t;
    return RPB_OK;
}

rpb_status rpb_tree_host_stats(const rpb_host_tree* t, rpb_stats* o)
{
    if (!t || !o) { set_error("null argument"); return RPB_EINVAL; }
    const HostTree& T = t->tree;
    std::memset(o, 0, sizeof(*o));
    o->vertex_count = T.nV;
    o->simplex_count = T.N;
    o->cluster_count = T.NC;
    o->tree_depth = T.depth;
    o->near_nnz = T.near.nnz();
    o->far_nnz = T.far.nnz();
    o->verynear_nnz = T.verynear.nnz();
    o->inter_nnz = T.inter.nnz();
    o->tree_build_seconds = t->seconds;
    return RPB_OK;
}

rpb_status rpb_tree_host_arrays(const rpb_host_tree* t, int* perm, int* C_begin, int* C_end, int* C_left,
                                int* C_right)
{
    if (!t) { set_error("null tree"); return RPB_EINVAL; }
    const HostTree& T = t->tree;
    if (perm) std::copy(T.perm.begin(), T.perm.end(), perm);
    if (C_begin) std::copy(T.C_begin.begin(), T.C_begin.end(), C_begin);
    if (C_end) std::copy(T.C_end.begin(), T.C_end.end(), C_end);
    if (C_left) std::copy(T.C_left.begin(), T.C_left.end(), C_left);
    if (C_right) std::copy(T.C_right.begin(), T.C_right.end(), C_right);
    return RPB_OK;
}

rpb_status rpb_tree_host_pattern(const rpb_host_tree* t, int which, int64_t* rowptr, int* colidx)
{
    if (!t) { set_error("null tree"); return RPB_EINVAL; }
    const SymPattern* P = which == 0 ? &t->tree.near : which == 1 ? &t->tree.far : which == 2 ? &t->tree.verynear
                        : which == 3 ? &t->tree.inter : nullptr;
    if (!P) { set_error("pattern id must be 0..3"); return RPB_EINVAL; }
    if (rowptr) std::copy(P->rp.begin(), P->rp.end(), rowptr);
    if (colidx) std::copy(P->ci.begin(), P->ci.end(), colidx);
    return RPB_OK;
}

rpb_status rpb_tree_host_destroy(rpb_host_tree* t)
{
    delete t;
    return RPB_OK;
}

rpb_status rpb_tree_host_obstacle_pattern(const rpb_host_tree* mesh, const double* V, const int* S,
                                          const rpb_host_tree* obstacle, const double* VO, const int* SO, int which,
                                          int64_t* counts, int64_t* rowptr, int* colidx)
{
    if (!mesh || !obstacle || !V || !S || !VO || !SO || !counts) { set_error("null argument"); return RPB_EINVAL; }
    if (which < 0 || which > 3) { set_error("pattern id must be 0..3"); return RPB_EINVAL; }
    CrossLists L;
    const std::string err = build_cross_lists(mesh->tree, V, S, obstacle->tree, VO, SO, mesh->settings, L);
    if (!err.empty()) { set_error(err); return RPB_EINVAL; }
    counts[0] = L.near.nnz(); counts[1] = L.far.nnz(); counts[2] = L.verynear.nnz(); counts[3] = L.inter.nnz();
    const CrossPattern& P = which == 0 ? L.near : which == 1 ? L.far : which == 2 ? L.verynear : L.inter;
    if (rowptr) std::copy(P.rp.begin(), P.rp.end(), rowptr);
    if (colidx) std::copy(P.ci.begin(), P.ci.end(), colidx);
    return RPB_OK;
}

rpb_status rpb_h1_solve_host(const rpb_host_tree* t, const double* V, const int* S, const double* B, double* X,
                             int nrhs)
{
    if (!t || !V || !S || !B || !X || nrhs <= 0) { set_error("null argument"); return RPB_EINVAL; }
    const HostTree& T = t->tree;
    const CsrMatrix H = assemble_h1(T.dom, V, T.nV, S, T.N, 1.0, 1.0);
    const std::vector<int> perm = nested_dissection_ordering(T, S, T.nV);
    CholeskyFactor F;
    const std::string err = cholesky_factor(H, perm, F);
    if (!err.empty()) { set_error(err); return RPB_EINVAL; }
    const int n = T.nV;
    std::vector<double> y(n);
    for (int c = 0; c < nrhs; ++c) {
        for (int i = 0; i < n; ++i) {  // forward: rows of L, diagonal last
            double s = B[static_cast<int64_t>(nrhs) * F.perm[i] + c];
            const int64_t k1 = F.lower_rp[i + 1] - 1;
            for (int64_t k = F.lower_rp[i]; k < k1; ++k) s -= F.lower_val[k] * y[F.lower_ci[k]];
            y[i] = s / F.lower_val[k1];
        }
        for (int i = n; i-- > 0;) {    // backward: rows of L^T, diagonal first
            double s = y[i];
            const int64_t k0 = F.upper_rp[i];
            for (int64_t k = k0 + 1; k < F.upper_rp[i + 1]; ++k) s -= F.upper_val[k] * y[F.upper_ci[k]];
            y[i] = s / F.upper_val[k0];
        }
        for (int i = 0; i < n; ++i) X[static_cast<int64_t>(nrhs) * F.perm[i] + c] = y[i];
    }
    return RPB_OK;
}

rpb_status rpb_mesh_semistatic_update(rpb_mesh* m, const double* V, int transp)
{
    if (!m || !V) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    if (transp) {
        std::vector<double> t(3 * static_cast<size_t>(m->nV));
        for (int v = 0; v < m->nV; ++v)
            for (int k = 0; k < 3; ++k) t[3 * static_cast<size_t>(v) + k] = V[static_cast<size_t>(k) * m->nV + v];
        RPB_CUDA(cudaMemcpyAsync(m->V.ptr, t.data(), m->V.bytes(), cudaMemcpyHostToDevice, m->stream));
        RPB_CUDA(cudaStreamSynchronize(m->stream));
    } else {
        RPB_CUDA(cudaMemcpyAsync(m->V.ptr, V, m->V.bytes(), cudaMemcpyHostToDevice, m->stream));
    }
    return launch_geometry(m);
}

rpb_status rpb_mesh_semistatic_update_device(rpb_mesh* m, const double* V_dev)
{
    if (!m || !V_dev) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    RPB_CUDA(cudaMemcpyAsync(m->V.ptr, V_dev, m->V.bytes(), cudaMemcpyDeviceToDevice, m->stream));
    return launch_geometry(m);
}

rpb_status rpb_tpe0_value(rpb_mesh* m, double q, double p, double* energy)
{
    if (!m || !energy) { set_error("null argument"); return RPB_EINVAL; }
    return evaluate(m, q, p, false, 0.0, 0.0, nullptr, 3, energy);
}

rpb_status rpb_tpe0_differential_device(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y_dev,
                                        int ldY, double* energy)
{
    if (!m || !Y_dev) { set_error("null argument"); return RPB_EINVAL; }
    if (ldY < 3) { set_error("ldY must be >= AMB_DIM = 3"); return RPB_EINVAL; }
    return evaluate(m, q, p, true, alpha, beta, Y_dev, ldY, energy);
}

rpb_status rpb_mesh_set_shards(rpb_mesh* m, int shards)
{
    if (!m) { set_error("null mesh"); return RPB_EINVAL; }
    if (shards < 1) { set_error("shards must be >= 1"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    rpb_status st = build_pair_tiles(m, shards);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    return RPB_OK;
}

rpb_status rpb_mesh_shard_rows(const rpb_mesh* m, int shard, int64_t* near_rows, int64_t* far_rows)
{
    if (!m || !near_rows || !far_rows) { set_error("null argument"); return RPB_EINVAL; }
    if (shard < 0 || shard >= m->shards) { set_error("shard out of range"); return RPB_EINVAL; }
    const TileBufs* tb[2] = {&m->near_tiles, &m->far_tiles};
    int64_t* out[2] = {near_rows, far_rows};
    const int rows[2] = {m->N, m->NC};
    for (int k = 0; k < 2; ++k) {
        if (!tb[k]->valid) {
            out[k][0] = 0; out[k][1] = shard == 0 ? rows[k] : 0;   // untiled (empty) pattern: shard 0
            continue;
        }
        int first, count;
        shard_tiles(*tb[k], shard, m->shards, first, count);
        out[k][0] = tb[k]->row0_host[first];
        out[k][1] = tb[k]->row0_host[first + count];
    }
    return RPB_OK;
}

rpb_status rpb_mesh_shard_buffer_doubles(const rpb_mesh* m, int64_t* doubles)
{
    if (!m || !doubles) { set_error("null argument"); return RPB_EINVAL; }
    *doubles = 10 * static_cast<int64_t>(m->N) + 10 * static_cast<int64_t>(m->NC) + 1;
    return RPB_OK;
}

rpb_status rpb_tpe0_pairs_shard(rpb_mesh* m, double q, double p, int shard, double* buf)
{
    if (!m || !buf) { set_error("null argument"); return RPB_EINVAL; }
    if (shard < 0 || shard >= m->shards) { set_error("shard out of range"); return RPB_EINVAL; }
    if (m->verynear.nnz > 0) {
        set_error("row-sharded evaluation is not built for meshes with very-near primitive pairs");
        return RPB_EINVAL;
    }
    if ((m->near.nnz > 0 && !m->near_tiles.valid) || (m->far.nnz > 0 && !m->far_tiles.valid)) {
        set_error("row-sharded evaluation needs row tiles (a row exceeds the tile column cap)");
        return RPB_EINVAL;
    }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    if (!m->geometry_valid && (st = launch_geometry(m)) != RPB_OK) return st;
    double* D_near = buf;
    double* D_far = buf + 10 * static_cast<int64_t>(m->N);
    double* e_out = D_far + 10 * static_cast<int64_t>(m->NC);
    if ((st = launch_pairs(m, make_exp(m->dom, q, p), true, nullptr, shard, D_near, D_far)) != RPB_OK) return st;
    k_add_pair<<<1, 1, 0, m->stream>>>(m->energy.ptr, e_out);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status rpb_tpe0_collect_shards(rpb_mesh* m, const double* buf, double alpha, double beta, double* Y_dev, int ldY)
{
    if (!m || !buf || !Y_dev) { set_error("null argument"); return RPB_EINVAL; }
    if (ldY < 3) { set_error("ldY must be >= AMB_DIM = 3"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    const double* D_near = buf;
    const double* D_far = buf + 10 * static_cast<int64_t>(m->N);
    return launch_collect_gather(m, alpha, beta, Y_dev, ldY, nullptr, D_near, D_far);
}

rpb_status rpb_tpe0_energy_device(rpb_mesh* m, double* energy_dev)
{
    if (!m || !energy_dev) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    k_sum_energy_parts<<<1, 1, 0, m->stream>>>(m->energy.ptr, energy_dev);
    RPB_CUDA(cudaGetLastError());
    return RPB_OK;
}

rpb_status rpb_tpe0_differential(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y, int ldY,
                                 double* energy)
{
    if (!m || !Y) { set_error("null argument"); return RPB_EINVAL; }
    if (ldY < 3) { set_error("ldY must be >= AMB_DIM = 3"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(m->device));
    if (beta != 0.0)
        RPB_CUDA(copy_rows3(m->Y.ptr, 3, Y, ldY, m->nV, cudaMemcpyHostToDevice, m->stream));
    // the derivative and the energy parts come back with one synchronization
    rpb_status st = evaluate(m, q, p, true, alpha, beta, m->Y.ptr, 3, nullptr);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaMemcpyAsync(m->host_energy, m->energy.ptr, 3 * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(copy_rows3(Y, ldY, m->Y.ptr, 3, m->nV, cudaMemcpyDeviceToHost, m->stream));
    RPB_CUDA(cudaStreamSynchronize(m->stream));
    if (energy) *energy = (m->host_energy[2] + m->host_energy[0]) + m->host_energy[1];
    if (m->verynear.nnz > 0) return vf_take_status(m->vf, m->stream);
    return RPB_OK;
}

rpb_status rpb_tpe0_stage_times(rpb_mesh* m, double q, double p, int reps, int64_t flush_bytes, double* ms)
{
    if (!m || !ms || reps <= 0) { set_error("bad argument"); return RPB_EINVAL; }
    rpb_status st = check_exponents(q, p);
    if (st != RPB_OK) return st;
    RPB_CUDA(cudaSetDevice(m->device));
    const TPExp ex = make_exp(m->dom, q, p);
    cudaEvent_t ev[5];
    for (auto& e : ev) RPB_CUDA(cudaEventCreate(&e));
    DevBuf<char> flush;
    if (flush_bytes > 0) RPB_CUDA(flush.alloc(static_cast<size_t>(flush_bytes)));
    double acc[5] = {0, 0, 0, 0, 0};
    const bool with_vf = m->verynear.nnz > 0;
    for (int r = 0; r < reps; ++r) {
        if (flush.ptr) RPB_CUDA(cudaMemsetAsync(flush.ptr, r & 0xff, flush.bytes(), m->stream));
        RPB_CUDA(cudaEventRecord(ev[0], m->stream));
        if ((st = launch_geometry(m)) != RPB_OK) return st;
        RPB_CUDA(cudaEventRecord(ev[1], m->stream));
        // near rows | far rows (+ very-near) | collection
        if ((st = launch_pairs(m, ex, true, ev[2])) != RPB_OK) return st;
        if (with_vf && (st = launch_vf(m, ex, true)) != RPB_OK) return st;
        RPB_CUDA(cudaEventRecord(ev[3], m->stream));
        if ((st = launch_collect_gather(m, 1.0, 0.0, m->Y.ptr, 3, with_vf ? m->vf.D.ptr : nullptr, nullptr, nullptr)) !=
            RPB_OK)
            return st;
        RPB_CUDA(cudaEventRecord(ev[4], m->stream));
        RPB_CUDA(cudaEventSynchronize(ev[4]));
        float t;
        cudaEventElapsedTime(&t, ev[0], ev[1]); acc[0] += t;
        cudaEventElapsedTime(&t, ev[1], ev[2]); acc[1] += t;
        cudaEventElapsedTime(&t, ev[2], ev[3]); acc[2] += t;
        cudaEventElapsedTime(&t, ev[3], ev[4]); acc[3] += t;
        cudaEventElapsedTime(&t, ev[0], ev[4]); acc[4] += t;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 5; ++k) ms[k] = acc[k] / reps;
    return RPB_OK;
}

rpb_status rpb_measure_fp32_peak(int device, double* tflops)
{
    if (!tflops) { set_error("null argument"); return RPB_EINVAL; }
    RPB_CUDA(cudaSetDevice(device));
    int sms = 0;
    RPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256, iters = 8192;
    DevBuf<float> out;
    RPB_CUDA(out.alloc(static_cast<size_t>(blocks) * threads));
    cudaEvent_t a, b;
    RPB_CUDA(cudaEventCreate(&a));
    RPB_CUDA(cudaEventCreate(&b));
    k_fma_peak<<<blocks, threads>>>(out.ptr, iters, 1.0001f);
    RPB_CUDA(cudaEventRecord(a));
    k_fma_peak<<<blocks, threads>>>(out.ptr, iters, 1.0001f);
    RPB_CUDA(cudaEventRecord(b));
    RPB_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const double flops = 2.0 * 16.0 * iters * static_cast<double>(blocks) * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return RPB_OK;
}

}  // extern "C"
