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

// Sparse Cholesky L L^T = P A P^T (up-looking, elimination tree). Returns the factor in
// both row forms used by the GPU triangular solves:
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

}  // namespace rpb
