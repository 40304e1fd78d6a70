// Internal entry points shared between the translation units of librepulsor_b200.
#pragma once

#include <string>

#include "../../include/repulsor_b200.h"
#include "host/tree_builder.hpp"
#include "rpb_device.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

void set_error(const std::string& msg);
TPExp make_exp(int dom, double q, double p);
rpb_status check_exponents(double q, double p);
// the four block-cluster-tree patterns of T on the device (rpb_gputree.cu); false with T
// untouched and err set if the device work failed
bool build_block_cluster_tree_device(HostTree& T, const std::vector<double>& P, const int* S, const TreeSettings& set,
                                     cudaStream_t s, std::string& err);
// the cluster tree of a mesh built on the device (rpb_gputree.cu): the same permutation,
// ranges, links and boxes as build_cluster_tree, and the serialized polytopes in tree order;
// false with err set if the input is invalid or the device work failed
bool build_cluster_tree_device(int dom, const double* V, int nV, const int* S, int N, HostTree& T,
                               std::vector<double>& P, cudaStream_t s, std::string& err);
// the obstacle loaded into m (rpb_mesh_load_obstacle), or null
rpb_mesh* obstacle_mesh(const rpb_mesh* m);

// n rows of 3 doubles between arrays with leading dimensions ld_dst / ld_src (host or
// device): one contiguous copy when both are 3 (a pitched copy of 24-byte rows from
// pageable host memory moves row by row, ~100x slower), a pitched copy otherwise.
inline cudaError_t copy_rows3(void* dst, int ld_dst, const void* src, int ld_src, int64_t n, cudaMemcpyKind kind,
                              cudaStream_t s)
{
    if (ld_dst == 3 && ld_src == 3) return cudaMemcpyAsync(dst, src, sizeof(double) * 3 * n, kind, s);
    return cudaMemcpy2DAsync(dst, sizeof(double) * ld_dst, src, sizeof(double) * ld_src, sizeof(double) * 3, n, kind, s);
}
rpb_status launch_geometry(rpb_mesh* m);
// near/far moment derivatives (mesh buffers when null) and very-near row derivatives (none
// when D_vf is null) -> chain rule -> Y = alpha dE + beta Y
rpb_status launch_collect_gather(rpb_mesh* m, double alpha, double beta, double* Y, int ldY, const double* D_vf,
                                 const double* D_near, const double* D_far);
rpb_status evaluate(rpb_mesh* m, double q, double p, bool diff, double alpha, double beta, double* Y_dev, int ldY,
                    double* energy_host);

// very-near adaptive quadrature (rpb_verynear.cu)
rpb_status vf_alloc(VFBuffers& b, int64_t nnz, int N);
// reads (synchronizing) and clears the status of the last very-near evaluations: RPB_EINVAL
// with the message set if a pair touched or intersected or exceeded the work cap
rpb_status vf_take_status(VFBuffers& b, cudaStream_t s);
rpb_status launch_vf(rpb_mesh* m, const TPExp& ex, bool diff);
rpb_status launch_vf_metric(rpb_mesh* m, const TPExp& ex, float2* vals, double2* diag);
// mesh x obstacle very-near pairs (CSR rp/ci over m's primitives): row derivatives into
// b.D, the energy (symmetry factor 1/2) into *energy_out, on m's stream
rpb_status launch_vf_cross(rpb_mesh* m, const rpb_mesh* obstacle, const int64_t* rp, const int* ci, int64_t nnz,
                           VFBuffers& b, const TPExp& ex, bool diff, double* energy_out);

// metric (rpb_metric.cu)
rpb_status metric_init(rpb_mesh* m, const double* Vh, const int* Sh);
rpb_status metric_multiply_dev(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX, double beta,
                               double* Y, int ldY, int flags);
rpb_status plap_multiply_dev(rpb_mesh* m, double s, double alpha, const double* X, int ldX, double beta, double* Y,
                             int ldY);

// solver (rpb_solver.cu)
void solver_free(rpb_mesh* m);
rpb_status reference_precondition(rpb_mesh* m, double q, double p, const double* X, double* Y);

// learned preconditioner (rpb_learned.cu): Z = MLP correction of the residual R (n x 3, device)
rpb_status learned_precondition(rpb_mesh* m, double q, double p, const double* R, double* Z);
void learned_free(rpb_mesh* m);

// obstacle (rpb_obstacle.cu)
void obstacle_free(rpb_mesh* m);

}  // namespace rpb
