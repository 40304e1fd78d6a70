// Per-mesh device state of the B200 tangent-point path.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "host/tree_builder.hpp"
#include "rpb_device.cuh"

namespace rpb {

struct Solver;
struct LearnedState;
struct ObstacleState;
void set_error(const std::string& msg);

template <typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count)
    {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void**>(&ptr), sizeof(T) * count);
    }
    size_t bytes() const { return sizeof(T) * n; }
};

struct Csr {
    DevBuf<int64_t> rp;
    DevBuf<int> ci;
    int rows = 0;
    int64_t nnz = 0;
};

// Metric values on the full symmetric patterns (TP0: two scalars per block, FP32)
// and row diagonals (FP64), cached per (q, p) and geometry state.
struct MetricCache {
    bool valid = false;
    double q = 0, p = 0;
    DevBuf<float2> nf, ff, vf;
    DevBuf<double2> nf_diag, ff_diag, vf_diag;
};

struct PseudoLapCache {
    bool valid = false;
    double s = 0;
    DevBuf<float> nf, ff, vf;
    DevBuf<double> nf_diag, ff_diag, vf_diag;
};

// Very-near quadrature buffers of one list (rpb_verynear.cu): per-entry slots, the row
// derivatives (N x 16, reference layout a, a*hull, a*P) and the energy reduction state.
struct VFBuffers {
    DevBuf<double> part, D, block_energy;
    DevBuf<unsigned> done;
    size_t bytes() const { return part.bytes() + D.bytes() + block_energy.bytes() + done.bytes(); }
};

// Device copy of a pattern's row tiles (RowTiles); valid == false: the gather kernels run.
struct TileBufs {
    DevBuf<int> row0, cols_rp, cols, order, lane_map;
    DevBuf<uint16_t> slot;
    std::vector<int> row0_host;   // tiles + 1: first row of each tile
    int tiles = 0, max_union = 0;
    int64_t max_entries = 0;      // most entries in one tile
    bool valid = false;
};

}  // namespace rpb

struct rpb_mesh {
    int dom = 2, size = 3, nV = 0, N = 0, NC = 0;
    int device = 0;
    double build_seconds = 0;
    bool cluster_tree_on_device = false;  // the splits ran on the device (else on the host)
    bool block_tree_on_device = false;    // the dual traversal ran on the device
    cudaStream_t stream = nullptr;        // stream all work is issued on
    cudaStream_t own_stream = nullptr;    // stream created by the mesh
    double* host_energy = nullptr;        // 3 pinned doubles: energy parts read back with the results
    ~rpb_mesh() { if (host_energy) cudaFreeHost(host_energy); }
    rpb::HostTree tree;
    rpb::TreeSettings settings;

    // mesh
    rpb::DevBuf<double> V, charge_v;
    rpb::DevBuf<int> S;
    // tree
    rpb::DevBuf<int> perm, leaf_of, C_parent, C_left, C_right, C_begin, C_end;
    rpb::DevBuf<int> C_up4;   // fourth ancestor of every cluster (-1 when the root is nearer)
    rpb::Csr near, far, verynear;
    rpb::DevBuf<int> near_order, far_order;             // pair-kernel row order (length-sorted per chunk)
    rpb::TileBufs near_tiles, far_tiles;                // shared-memory row tiles of the two patterns
    // geometry state
    rpb::DevBuf<rpb::PrimDatum> P_pair;
    rpb::DevBuf<rpb::ClusterDatum> C_pair;
    rpb::DevBuf<double> scan_local, scan_blocks;   // prefix sums of the moment upsweep
    rpb::DevBuf<unsigned> counter;
    // near-hull data for very-near quadrature (N x (1 + 3 size + 6), FP64)
    rpb::DevBuf<double> P_near;
    // derivative path
    rpb::DevBuf<double> D_near, D_far, B;
    rpb::VFBuffers vf;                          // very-near quadrature (when the list is not empty)
    rpb::DevBuf<int> v_rp, v_slot;
    rpb::DevBuf<double> Y;
    rpb::DevBuf<double> block_energy, energy;   // energy[0] near, [1] far, [2] very near
    rpb::DevBuf<unsigned> done;                 // last-block counters: [0] near, [1] far pairs,
                                                // [3] the metric Pre kernel's block scan
    int near_blocks = 0, far_blocks = 0;
    int shards = 1;                             // row shards the tiles are grouped for
    int64_t last_step_candidates = 0;           // candidate pairs of the last MaximumSafeStepSize
    // metric: frozen Pre/Post (per primitive in tree order: sorted vertex ids, 4 x size coefficients)
    rpb::DevBuf<int> pre_cols;
    rpb::DevBuf<double> pre_vals;
    rpb::DevBuf<int> vp_rp, vp_slot;        // vertex -> (primitive position * size + corner)
    rpb::DevBuf<double> buf_Pin64, buf_Cin64, buf_Pout, buf_Cout, buf_Z, buf_scan_local, buf_scan_blocks;
    rpb::DevBuf<double> X, Yb;              // staging for host-pointer calls (nV x 3)
    rpb::MetricCache metric;
    rpb::PseudoLapCache plap;
    bool geometry_valid = false;
    int64_t geometry_version = 0;

    // solver state (allocated on first solve)
    rpb::Solver* solver = nullptr;
    // learned preconditioner state (allocated on first use)
    rpb::LearnedState* learned = nullptr;
    // obstacle of TangentPointObstacleEnergy (owned, with its cross block cluster tree)
    rpb::ObstacleState* obstacle = nullptr;
    // frozen coordinates and simplices on the host (the tree was built from them)
    std::vector<double> V_frozen;
    std::vector<int> S_host;

    int64_t device_bytes() const;
};
