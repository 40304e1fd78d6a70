// Host-side construction of Repulsor's ClusterTree and BlockClusterTree for the
// B200 path. The tree and its pair lists are built once per mesh on the host and
// uploaded; SemiStaticUpdate keeps them fixed (src/ClusterTree.hpp:951-993).
//
// Restated behaviour (citations are paths inside HenrikSchumacher/Repulsor):
//  * primitive serialization: src/Primitives/Polytope.hpp:113-160 (frozen coordinates)
//  * AABB from primitives:    src/BoundingVolumes/AABB.hpp:155-237
//  * longest-axis split:      src/BoundingVolumes/AABB_LongestAxisSplit.hpp:134-253
//    (strict x < mid partition with in-place swaps, median fallback via std::nth_element)
//  * depth-first numbering:   src/ClusterTree/Serialize_Thread.hpp:273-314
//  * dual-tree traversal:     src/ClusterTreePairTraversor/Traverse_DepthFirst.hpp:52-258
//  * split kernel / MACs:     src/BlockClusterTree/BlockSplit_Kernel.hpp:164-251, src/GJK.hpp:1162-1183
//  * symmetric CSR patterns:  src/BlockClusterTree.hpp:306-326
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace rpb {

struct TreeSettings {
    double theta_far = 0.5;         // far_field_separation_parameter (src/Settings.hpp:39)
    double theta_near = 10.0;       // AdaptivitySettings::theta (src/Settings.hpp:52)
    int max_refinement = 30;        // AdaptivitySettings::max_refinement (src/Settings.hpp:51)
    int threads = 1;                // host threads for the build
};

// Full symmetric CSR (both triangles), columns sorted, no diagonal entries.
struct SymPattern {
    int rows = 0;
    std::vector<int64_t> rp;        // rows + 1
    std::vector<int> ci;            // nnz
    std::vector<int64_t> diag;      // first position in row i with column > i
    int64_t nnz() const { return rp.empty() ? 0 : rp.back(); }
};

struct HostTree {
    int dom = 2, size = 3;
    int nV = 0, N = 0, NC = 0, depth = 0;
    std::vector<int> perm;          // position -> original simplex (P_ordering)
    std::vector<int> inv_perm;      // original simplex -> position
    std::vector<int> C_begin, C_end, C_left, C_right, C_parent, C_depth;
    std::vector<int> leaf_of;       // position -> leaf cluster
    std::vector<double> C_box;      // NC x 7: r2, centre[3], half-lengths[3]
    SymPattern near, far, verynear, inter;
};

// Builds the cluster tree and the four block-cluster-tree patterns.
// V: nV x 3 (frozen coordinates), S: N x (dom+1) simplices.
// Returns an empty string on success, otherwise an error message.
std::string build_tree(int dom, const double* V, int nV, const int* S, int N, const TreeSettings& set,
                       HostTree& out);

// The two halves of build_tree: the cluster tree (returns the serialized polytopes
// [r2, centre, hull] in tree order, which the block cluster tree reads) and the block
// cluster tree's patterns (host threads; rpb_gputree.cu computes the same on the device).
std::string build_cluster_tree(int dom, const double* V, int nV, const int* S, int N, const TreeSettings& set,
                               HostTree& out, std::vector<double>& P);
void build_block_cluster_tree(HostTree& T, const std::vector<double>& P, const int* S, const TreeSettings& set);

// Rectangular CSR (rows of one tree, columns of another), columns sorted.
struct CrossPattern {
    int rows = 0;
    std::vector<int64_t> rp;
    std::vector<int> ci;
    int64_t nnz() const { return rp.empty() ? 0 : rp.back(); }
};

// Non-symmetric block cluster tree of a mesh tree S against an obstacle tree T
// (BlockClusterTree<..., false>, src/SimplicialMesh.hpp:741-756): every (S, T) block
// pair is visited once, the larger cluster (by squared radius) is split, both when the
// radii are equal. near/verynear/inter rows are S primitives, far rows are S clusters.
struct CrossLists {
    CrossPattern near, far, verynear, inter;
};

std::string build_cross_lists(const HostTree& S, const double* VS, const int* SS, const HostTree& T,
                              const double* VT, const int* ST, const TreeSettings& set, CrossLists& out);

// Row tiles of a CSR pattern for the shared-memory pair kernels: consecutive rows (tree
// order, so spatially close) are grouped until a tile holds target_entries entries, at
// most block_lanes rows and at most max_union distinct columns; a tile's kernel block
// stages the union's column data once and every entry addresses it by its 16-bit slot.
// Inside a tile every row gets a group of lanes (a power of two, at most 32, aligned in
// its warp): all rows start with one lane and the row with the most entries per lane
// doubles its group while the block has lanes left. valid is false when a single row has
// more than max_union entries.
struct RowTiles {
    std::vector<int> row0;          // tiles + 1: first row of each tile
    std::vector<int> cols_rp;       // tiles + 1: offsets into cols
    std::vector<int> cols;          // union columns of each tile, ascending
    std::vector<uint16_t> slot;     // nnz: index of the entry's column in its tile's union
    std::vector<int> order;         // rows; inside each tile by decreasing group size and length
    std::vector<int> lane_map;      // tiles x block_lanes: (row position in the tile's order << 10)
                                    // | ((group size - 1) << 5) | lane in the group; -1 idle
    int block_lanes = 0;
    int max_union = 0;
    bool valid = false;
    int tiles() const { return row0.empty() ? 0 : static_cast<int>(row0.size()) - 1; }
};

void build_row_tiles(const int64_t* rp, const int* ci, int rows, int ncols, int block_lanes, int64_t target_entries,
                     int max_union, int threads, RowTiles& out);

}  // namespace rpb
