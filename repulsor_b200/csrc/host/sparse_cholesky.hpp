// Host-side H1 metric assembly, nested-dissection ordering and sparse Cholesky
// factorization for the reference preconditioner H1^{-1} L_{2-s} H1^{-1}
// (src/Metrics/TangentPointMetric0.hpp:88-126, src/SimplicialMesh/H1Metric.hpp:36-257,
//  src/SimplicialMesh/NestedDissectionOrdering.hpp:3-207).
// The factor is uploaded once per geometry state; the triangular solves run on the GPU.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "tree_builder.hpp"

namespace rpb {

struct CsrMatrix {
    int n = 0;
    std::vector<int64_t> rp;
    std::vector<int> ci;
    std::vector<double> val;
};

// H1 = stiffness_weight * stiffness + mass_weight * mass (P1 elements on the simplices,
// src/SimplicialMesh/H1Metric.hpp:36-169); duplicate entries summed, columns sorted.
CsrMatrix assemble_h1(int dom, const double* V, int nV, const int* S, int N, double stiffness_weight,
                      double mass_weight);

// Vertex permutation by nested dissection along the cluster tree: perm[new] = old.
std::vector<int> nested_dissection_ordering(const HostTree& T, const int* S, int nV);

// widest supernode of the numeric factorization (host/supernodal_chol.hpp)
constexpr int kSupernodalWidth = 256;

// Sparse Cholesky L L^T = P A P^T (supernodal, on host threads: host/supernodal_chol.hpp).
// Returns the factor in both row forms used by the GPU triangular solves:
//   lower: row i of L, columns ascending, diagonal last
//   upper: row i of L^T (= column i of L), columns ascending, diagonal first
struct CholeskyFactor {
    int n = 0;
    std::vector<int> perm;            // perm[new] = old
    std::vector<int64_t> lower_rp, upper_rp;
    std::vector<int> lower_ci, upper_ci;
    std::vector<double> lower_val, upper_val;
    int64_t nnz() const { return lower_rp.empty() ? 0 : lower_rp.back(); }
};

std::string cholesky_factor(const CsrMatrix& A, const std::vector<int>& perm, CholeskyFactor& out);

// Level schedule of the triangular solves by supernodes. Supernodes are contiguous column
// ranges of L: fundamental supernodes (column j+1 is the only child of column j and their
// structures nest), then single-child chains merged into one range, then ranges wider
// than max_width split into consecutive pieces. Within a supernode the dense diagonal
// block D (explicit zeros included) is inverted once on the host, so a supernode is
// solved as t = b - (external part of its rows) followed by y = D^{-1} t. A supernode's
// level is one more than the highest level it reads from: all supernodes of one level
// are independent, and a level is one kernel launch.
struct SupernodalSchedule {
    int n = 0, nsn = 0, max_width = 0;
    std::vector<int> sn_begin;                 // nsn + 1 column offsets
    // forward (L) and backward (L^T) schedules: supernodes grouped by level
    std::vector<int> fwd_level_ptr, fwd_level_sn, fwd_level_width;
    std::vector<int> bwd_level_ptr, bwd_level_sn, bwd_level_width;
    std::vector<int64_t> dinv_off;             // nsn + 1: w (w + 1) / 2 entries per supernode
    std::vector<double> dinv;                  // D^{-1}, packed lower triangle by rows
    std::vector<double> dinvT;                 // D^{-T}, packed upper triangle by rows
    int fwd_levels() const { return static_cast<int>(fwd_level_ptr.size()) - 1; }
    int bwd_levels() const { return static_cast<int>(bwd_level_ptr.size()) - 1; }
};

std::string supernodal_schedule(const CholeskyFactor& F, int max_width, SupernodalSchedule& out);

}  // namespace rpb
