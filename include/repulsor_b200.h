/*
 * repulsor_b200 -- C ABI of the B200 implementation of Repulsor's multipole-
 * accelerated tangent-point path.
 *
 * One `rpb_mesh` replaces a Repulsor `SimplicialMesh` together with its cached
 * ClusterTree / BlockClusterTree and the metric-value cache. All arrays in these
 * signatures are plain host pointers unless the function name ends in `_device`
 * (device pointers on the mesh's CUDA stream). Every function returns an
 * `rpb_status`; `rpb_last_error` gives the message of the last failure.
 *
 * Citations name the reference interface each entry point replaces
 * (paths inside HenrikSchumacher/Repulsor).
 */
#ifndef REPULSOR_B200_H
#define REPULSOR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rpb_status {
    RPB_OK = 0,
    RPB_EINVAL = 1,      /* invalid argument (the reference prints via eprint and does nothing) */
    RPB_ENOTCONV = 2,    /* solver reached max_iter above the tolerance */
    RPB_ESTALL = 3,      /* solver stagnated */
    RPB_ECUDA = 4,       /* CUDA runtime error */
    RPB_ENOMEM = 5,      /* device allocation failed */
    RPB_ETIMEOUT = 6     /* a bounded device-side wait gave up */
} rpb_status;

typedef struct rpb_mesh rpb_mesh;

/* ClusterTreeSettings / BlockClusterTreeSettings / AdaptivitySettings
 * (src/Settings.hpp:5-54, overrides of src/SimplicialMesh.hpp:592-595). */
typedef struct rpb_settings {
    int    split_threshold;          /* only 1 is supported (the reference default) */
    double far_field_separation;     /* theta of the AABB MAC, default 0.5 */
    double near_field_separation;    /* AdaptivitySettings::theta, default 10 */
    double near_field_intersection;  /* AdaptivitySettings::intersection_theta, default 1e10 (unused by the
                                        classification, which the reference also ties to theta) */
    int    max_refinement;           /* very-near subdivision limit, default 30 */
    int    thread_count;             /* host threads for the tree build (0 = hardware concurrency) */
    int    device;                   /* CUDA device ordinal */
} rpb_settings;

typedef struct rpb_stats {
    int64_t vertex_count;
    int64_t simplex_count;
    int64_t cluster_count;
    int64_t tree_depth;
    int64_t near_nnz;                /* full symmetric storage (both triangles) */
    int64_t far_nnz;
    int64_t verynear_nnz;
    int64_t inter_nnz;
    double  tree_build_seconds;
    int64_t device_bytes;            /* device memory held by the mesh */
} rpb_stats;

/* Fills `s` with the reference defaults. */
rpb_status rpb_default_settings(rpb_settings* s);

/* Last error message of this thread ("" if none). */
const char* rpb_last_error(void);

/* --- mesh ------------------------------------------------------------------------------- */

/* SimplicialMesh(V, nV, S, nS[, charges]) (src/SimplicialMesh.hpp:154-220) followed by
 * GetClusterTree()/GetBlockClusterTree() (src/SimplicialMesh.hpp:470-607): builds the
 * cluster tree and the block cluster tree from the frozen coordinates on the device (on
 * host threads if the device work fails; the same tree either way, rpb_mesh_build_info
 * tells which) and keeps them there. V: nV x amb_dim row-major doubles; S: nS x (dom_dim+1)
 * row-major ints;
 * charges: nV doubles or NULL (all ones). Only amb_dim = 3 and dom_dim in {1,2}. */
rpb_status rpb_mesh_create(int dom_dim, int amb_dim, const double* V, int64_t nV, const int* S, int64_t nS,
                           const double* charges, const rpb_settings* settings, rpb_mesh** out);

rpb_status rpb_mesh_destroy(rpb_mesh* m);

rpb_status rpb_mesh_stats(const rpb_mesh* m, rpb_stats* out);

/* Where rpb_mesh_create built the cluster tree (the longest-axis splits,
 * src/ClusterTree/Split_Thread.hpp, src/BoundingVolumes/AABB_LongestAxisSplit.hpp:134-253)
 * and the block cluster tree (the dual traversal, Traverse_DepthFirst.hpp:52-258): 1 on the
 * device, 0 on host threads, the fallback when the device work failed. Both give the same
 * permutation, clusters and pair lists. Either pointer may be NULL. */
rpb_status rpb_mesh_build_info(const rpb_mesh* m, int* cluster_tree_on_device, int* block_tree_on_device);

/* CUDA stream used by all work of this mesh (a cudaStream_t passed as void*).
 * set: the caller keeps ownership of `stream`; NULL restores the mesh's own stream.
 * No reference counterpart: Repulsor runs on host threads only. */
rpb_status rpb_mesh_set_stream(rpb_mesh* m, void* stream);
rpb_status rpb_mesh_get_stream(const rpb_mesh* m, void** stream);

/* SimplicialMesh::SemiStaticUpdate (src/SimplicialMesh.hpp:354-376): new coordinates,
 * same tree and pair lists; recomputes primitive data and the cluster moment upsweep.
 * transp != 0 reads V column-major (3 x nV). The copy of V is queued on the mesh stream:
 * pageable host memory is read before the call returns, page-locked memory (cudaHostAlloc,
 * pinned tensors) only when the stream gets there, so a page-locked V must stay unchanged
 * until the next synchronizing call (Value, Differential with host Y) has returned. */
rpb_status rpb_mesh_semistatic_update(rpb_mesh* m, const double* V, int transp);
rpb_status rpb_mesh_semistatic_update_device(rpb_mesh* m, const double* V_dev);

/* Tree inspection (ClusterTree::PrimitiveOrdering/ClusterBegin/End/Left/Right,
 * src/ClusterTree/ClusterTreeBase.hpp:298-578). Arrays sized simplex_count / cluster_count. */
rpb_status rpb_mesh_tree(const rpb_mesh* m, int* perm, int* C_begin, int* C_end, int* C_left, int* C_right);

/* BlockClusterTree patterns Near()/Far()/VeryNear()/PrimitiveIntersectionMatrix()
 * (src/BlockClusterTree.hpp:161-179). which: 0 near, 1 far, 2 very-near, 3 intersecting.
 * rowptr: rows+1 entries, colidx: nnz entries (full symmetric CSR, sorted). */
rpb_status rpb_mesh_pattern(const rpb_mesh* m, int which, int64_t* rowptr, int* colidx);

/* --- host-only tree construction ---------------------------------------------------------- */

/* ClusterTree + BlockClusterTree construction alone, without a device (the host half of
 * SimplicialMesh::GetClusterTree/GetBlockClusterTree, src/SimplicialMesh.hpp:470-607;
 * ClusterTree ctor src/ClusterTree.hpp:115-180; BlockClusterTree::ComputeBlocks
 * src/BlockClusterTree.hpp:234-330). Used to inspect and cross-check tree parity. */
typedef struct rpb_host_tree rpb_host_tree;
rpb_status rpb_tree_build_host(int dom_dim, const double* V, int64_t nV, const int* S, int64_t nS,
                               const rpb_settings* settings, rpb_host_tree** out);
rpb_status rpb_tree_host_stats(const rpb_host_tree* t, rpb_stats* out);
rpb_status rpb_tree_host_arrays(const rpb_host_tree* t, int* perm, int* C_begin, int* C_end, int* C_left,
                                int* C_right);
rpb_status rpb_tree_host_pattern(const rpb_host_tree* t, int which, int64_t* rowptr, int* colidx);
rpb_status rpb_tree_host_destroy(rpb_host_tree* t);

/* The obstacle lists of rpb_mesh_load_obstacle on the host only: counts[4] = sizes of
 * [near, far, very near, intersecting]; rowptr/colidx (may be NULL) receive list `which`.
 * V, S and VO, SO are the coordinates and simplices the two trees were built from. */
rpb_status rpb_tree_host_obstacle_pattern(const rpb_host_tree* mesh, const double* V, const int* S,
                                          const rpb_host_tree* obstacle, const double* VO, const int* SO, int which,
                                          int64_t* counts, int64_t* rowptr, int* colidx);

/* SimplicialMesh::H1Solver().Solve on the host (src/SimplicialMesh/H1Metric.hpp:208-257):
 * X = H1^{-1} B with H1 = stiffness + mass of the given coordinates, factorized by the
 * same nested-dissection-ordered sparse Cholesky the GPU preconditioner uploads.
 * B, X: nV x nrhs row-major. */
rpb_status rpb_h1_solve_host(const rpb_host_tree* t, const double* V, const int* S, const double* B, double* X,
                             int nrhs);

/* --- TangentPointEnergy0 (src/Energies/TangentPointEnergy0.hpp:35-86) -------------------- */

/* EnergyBase::Value (src/Energies/EnergyBase.hpp:40-56). */
rpb_status rpb_tpe0_value(rpb_mesh* m, double q, double p, double* energy);

/* EnergyBase::Differential(M, alpha, beta, Y, ldY) (src/Energies/EnergyBase.hpp:90-104):
 * Y = alpha * dE + beta * Y, Y: nV x ldY host doubles; returns the energy. */
rpb_status rpb_tpe0_differential(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y, int ldY,
                                 double* energy);

/* Same with Y a device pointer (nV x ldY) on the mesh stream. With `energy` non-NULL the
 * energy is read back (synchronizing the stream); with NULL nothing synchronizes and the
 * call (like rpb_mesh_semistatic_update_device) may be captured into a CUDA graph;
 * rpb_tpe0_energy_device then places the energy in device memory. */
rpb_status rpb_tpe0_differential_device(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y_dev,
                                        int ldY, double* energy);

/* --- TangentPointMetric0 (src/Metrics/TangentPointMetric0.hpp:57-126) ---------------------- */

/* MetricBase::MultiplyMetric (src/Metrics/MetricDimRestricted.hpp:109-139):
 * Y = alpha * A X + beta * Y with nrhs = 3; flags: bit0 VF, bit1 NF, bit2 FF. */
rpb_status rpb_tpm0_multiply(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX, double beta,
                             double* Y, int ldY, int nrhs, int flags);
rpb_status rpb_tpm0_multiply_device(rpb_mesh* m, double q, double p, double alpha, const double* X_dev, int ldX,
                                    double beta, double* Y_dev, int ldY, int nrhs, int flags);

/* MetricBase::MultiplyPreconditioner (src/Metrics/TangentPointMetric0.hpp:88-126):
 * Y = alpha * H1^{-1} L_{2-s} H1^{-1} X + beta * Y. */
rpb_status rpb_tpm0_precondition(rpb_mesh* m, double q, double p, double alpha, const double* X, int ldX,
                                 double beta, double* Y, int ldY, int nrhs);

/* Preconditioner kinds for rpb_tpm0_solve. */
typedef enum rpb_precond {
    RPB_PRECOND_NONE = 0,        /* plain CG */
    RPB_PRECOND_REFERENCE = 1,   /* H1^{-1} L_{2-s} H1^{-1} (the reference's preconditioner) */
    RPB_PRECOND_LEARNED = 2,     /* per-cluster MLP in flexible CG, falls back to REFERENCE on stall */
    RPB_PRECOND_HYBRID = 3       /* flexible CG with z = P_ref r + w M(r): the reference preconditioner
                                    plus the attached network's output, w = (r0, P_ref r0) / (8 (r0, M r0))
                                    on the first residual; falls back to REFERENCE on stall */
} rpb_precond;

/* MetricBase::Solve (src/Metrics/MetricDimRestricted.hpp:232-289):
 * X = alpha * A^{-1} B + beta * X by (flexible) preconditioned CG with FP64 inner
 * products; stops when the true relative residual of every column is <= tol.
 * iterations / rel_residual (3 entries) may be NULL. */
rpb_status rpb_tpm0_solve(rpb_mesh* m, double q, double p, double alpha, const double* B, int ldB, double beta,
                          double* X, int ldX, int nrhs, int max_iter, double tol, int precond, int* iterations,
                          double* rel_residual);

/* Statistics of the last rpb_tpm0_solve on this mesh (the reference's Solver_IterationCount
 * plus what the B200 solver adds). */
typedef struct rpb_solve_info {
    int     iterations;          /* CG iterations (all columns advance together) */
    int     restarts;            /* recurrences restarted from the true residual */
    int     fallback_iteration;  /* iteration at which LEARNED switched to REFERENCE, or -1 */
    int     supernode_levels;    /* launches per triangular solve of the H1 factor (0: none built) */
    double  factor_seconds;      /* H1 assembly + ordering + Cholesky time of the current factor */
    int64_t factor_nnz;          /* nonzeros of the H1 Cholesky factor */
    int     factor_on_device;    /* 1: the numeric factorization ran on the device, 0: on host threads */
} rpb_solve_info;

rpb_status rpb_tpm0_solve_info(const rpb_mesh* m, rpb_solve_info* info);

/* The energy of the last evaluation on this mesh (Value / Differential), written to the
 * device double `energy_dev` asynchronously on the mesh stream (graph-capturable). */
rpb_status rpb_tpe0_energy_device(rpb_mesh* m, double* energy_dev);

/* --- collision-free step size ---------------------------------------------------------------- */

/* SimplicialMesh::MaximumSafeStepSize(vecs, max_time, TOL) (src/SimplicialMesh.hpp:441-468,
 * src/CollisionTree.hpp:175-215, src/CollisionFinder.hpp:94-200): the largest t <= max_time
 * such that the mesh moved by t * velocities (n_v x 3 host doubles) keeps every pair of
 * primitives without a common vertex apart, up to the relative bisection tolerance `tol`
 * (the reference's default is 0.0625). As in the reference the test uses the coordinates
 * the cluster tree was built from. A loaded obstacle (at rest) is included. */
rpb_status rpb_mesh_maximum_safe_step_size(rpb_mesh* m, const double* velocities, double max_time, double tol,
                                           double* t);

/* --- row sharding of one evaluation over several GPUs ------------------------------------- */
/* The reference splits the rows of the Near() and Far() lists over host threads by nonzero
 * count and adds the per-thread derivative slices (src/FMM/FMM_Traversor.hpp:56-147,
 * src/ClusterTree.hpp:1115-1208). Here each of `shards` processes (one per GPU, the same
 * mesh at the same coordinates on every one) evaluates a contiguous range of row tiles,
 * the partial buffers are summed across processes (one all-reduce, e.g. NCCL), and every
 * process applies the chain rule to the sum.
 *
 * rpb_mesh_set_shards regroups the row tiles so that every shard owns whole waves of
 * resident blocks (synchronizes the mesh stream; call before any capture). */
rpb_status rpb_mesh_set_shards(rpb_mesh* m, int shards);
/* Rows [near_rows[0], near_rows[1]) of Near() and [far_rows[0], far_rows[1]) of Far() (tree
 * order) that shard `shard` evaluates. */
rpb_status rpb_mesh_shard_rows(const rpb_mesh* m, int shard, int64_t near_rows[2], int64_t far_rows[2]);
/* Number of doubles of a shard buffer: 10 N (near moment derivatives) + 10 N_C (far) + 1
 * (energy part). */
rpb_status rpb_mesh_shard_buffer_doubles(const rpb_mesh* m, int64_t* doubles);
/* Pair kernels of shard `shard` on the mesh stream into the device buffer `buf`: the
 * moment derivatives of the shard's rows (zero elsewhere; near rows centred at the
 * primitive, far rows with d0 - dx . c_C in their first entry) and its energy part.
 * Meshes with very-near pairs are rejected. */
rpb_status rpb_tpe0_pairs_shard(rpb_mesh* m, double q, double p, int shard, double* buf);
/* Collection, chain rule and vertex gather from the sum of all shards' buffers:
 * Y_dev = alpha dE + beta Y_dev (n_v x ldY, device); the energy is buf[10 N + 10 N_C]. */
rpb_status rpb_tpe0_collect_shards(rpb_mesh* m, const double* buf, double alpha, double beta, double* Y_dev,
                                   int ldY);

/* EnergyBase::SimplexDensities / VertexDensities (src/Energies/EnergyBase.hpp:129-150):
 * energy densities per simplex (original order, n_s values) or per vertex (n_v values; the
 * simplex densities averaged with the weights a_i/(n+1) and divided by the dual volume);
 * sum_i a_i rho_i is the energy, which `energy` (may be NULL) receives. Not built for
 * meshes with very-near primitive pairs. */
rpb_status rpb_tpe0_simplex_densities(rpb_mesh* m, double q, double p, double* density, double* energy);
rpb_status rpb_tpe0_vertex_densities(rpb_mesh* m, double q, double p, double* density, double* energy);

/* --- obstacle energy --------------------------------------------------------------------- */

/* SimplicialMesh::LoadObstacle (src/SimplicialMesh.hpp:697-719): m takes ownership of the
 * obstacle mesh (destroyed with m or when another obstacle is loaded; the caller must not
 * destroy it). Builds the non-symmetric block cluster tree of (m's tree, the obstacle's
 * tree) (GetObstacleBlockClusterTree, src/SimplicialMesh.hpp:741-756) once, from the
 * coordinates both trees were built from. Both meshes must have the same domain
 * dimension and live on the same device. */
rpb_status rpb_mesh_load_obstacle(rpb_mesh* m, rpb_mesh* obstacle);

/* Sizes [near, far, very near, intersecting] of the obstacle lists (rows are m's
 * primitives, or clusters for far; columns the obstacle's). */
rpb_status rpb_mesh_obstacle_stats(const rpb_mesh* m, int64_t* counts);

/* One obstacle list as CSR (rowptr: rows + 1, colidx: nnz); which as for rpb_mesh_pattern. */
rpb_status rpb_mesh_obstacle_pattern(const rpb_mesh* m, int which, int64_t* rowptr, int* colidx);

/* TangentPointObstacleEnergy (src/Energies/TangentPointObstacleEnergy.hpp:62-96): the
 * tangent-point energy of every (mesh, obstacle) pair with the symmetry factor 1/2 of a
 * non-symmetric block cluster tree; 0 without an obstacle. The differential (Y = alpha dE +
 * beta Y) is taken with respect to m's vertices only. */
rpb_status rpb_tpoe_value(rpb_mesh* m, double q, double p, double* energy);
rpb_status rpb_tpoe_differential(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y, int ldY,
                                 double* energy);
/* Same with Y on the device (asynchronous on the mesh stream; energy may be NULL). */
rpb_status rpb_tpoe_differential_device(rpb_mesh* m, double q, double p, double alpha, double beta, double* Y_dev,
                                        int ldY, double* energy);

/* --- learned preconditioner ------------------------------------------------------------ */

/* No counterpart in the reference: a per-cluster MLP (16 -> 64 -> 64 -> 3, GELU, BF16
 * weights, FP32 accumulation) that maps a residual r (n_v x 3) to a correction z. Every
 * cluster C reads 16 features of r and of its geometry (residual moment
 * R_C = sum_{i in C} a_i mean(r), barycentre, averaged normal, area, diameter, tree level,
 * 4 child-residual norms) and emits gains g_C = exp(clamp(o_C, +-3)); z is the multilevel
 * sum over the clusters containing each primitive of g_C R_C / A_C, gathered to the
 * vertices with the weights a_i/(n+1), minus the column means. rpb_tpm0_solve with
 * RPB_PRECOND_LEARNED uses it inside flexible CG and switches to the reference
 * preconditioner (MultiplyPreconditioner) when the residual stalls. */
typedef struct rpb_mlp rpb_mlp;

/* Number of FP32 parameters (W1 64x16, b1 64, W2 64x64, b2 64, W3 3x64, b3 3 = 5443). */
int rpb_mlp_param_count(void);
/* New network on `device`, Xavier-uniform weights from `seed`, zero biases. */
rpb_status rpb_mlp_create(int device, uint64_t seed, rpb_mlp** out);
rpb_status rpb_mlp_destroy(rpb_mlp* mlp);
/* FP32 master parameters (host arrays of rpb_mlp_param_count() floats); set resets Adam. */
rpb_status rpb_mlp_get_params(const rpb_mlp* mlp, float* params);
rpb_status rpb_mlp_set_params(rpb_mlp* mlp, const float* params);
/* Network on n feature rows F (n x 16, host): O (n x 3). With dO (n x 3) and grad
 * (param_count) non-NULL also grad = d(sum dO . O)/d(params) (for gradient checks). */
rpb_status rpb_mlp_eval(rpb_mlp* mlp, const float* F, int64_t n, const float* dO, float* O, float* grad);
/* One Adam step (lr <= 0: none) on npairs (residual R_k, correction E_k) pairs of mesh m
 * (host, n_v x 3 each, consecutive; A E_k = R_k for the metric A of exponents q, p):
 * loss = mean_k 1 - (z_k.R_k)^2 / ((z_k.A z_k)(E_k.R_k)) with z_k = M(R_k), the share of
 * the error energy ||E_k||_A^2 that the best step along z_k leaves, plus reg * mean over
 * clusters and components of o_C^2 (keeps the gains near the multilevel operator's 1).
 * `loss` (without the penalty) and `grad` (param_count floats, with it; either may be
 * NULL) are taken before the step. */
rpb_status rpb_mlp_train_step(rpb_mlp* mlp, rpb_mesh* m, double q, double p, const double* R, const double* E,
                              int npairs, double lr, double reg, double* loss, float* grad);
/* Attach (mlp non-NULL) or detach the network used by RPB_PRECOND_LEARNED on this mesh;
 * the mesh keeps the pointer, the caller keeps ownership. */
rpb_status rpb_mesh_set_learned(rpb_mesh* m, rpb_mlp* mlp);
/* Z = M(R) for one residual (host arrays, n_v x 3, row-major). */
rpb_status rpb_tpm0_learned_apply(rpb_mesh* m, const double* R, double* Z);
/* Z = M(R) and, with Y and ZY non-NULL, ZY = M_R(Y): the preconditioner with the gains the
 * network gave for R applied to another vector Y (the linearization of M at R with the
 * gains held fixed), which the adjoint pass of unrolled-solve training needs. */
rpb_status rpb_tpm0_learned_apply_pair(rpb_mesh* m, const double* R, const double* Y, double* Z, double* ZY);
/* One Adam step (lr <= 0: none) on the objective sum_k G_k . M(R_k) over npairs pairs of
 * residuals R_k and sensitivities G_k = dL/dz_k (host, n_v x 3 each, consecutive), plus
 * reg * mean over clusters and components of o_C^2: the parameter gradient of a loss L that
 * depends on the preconditioner outputs z_k = M(R_k) through G_k, e.g. the residual after
 * an unrolled preconditioned CG. objective (sum_k G_k . z_k) and grad (param_count floats,
 * with the penalty) may be NULL; both are taken before the step. */
rpb_status rpb_mlp_train_step_sens(rpb_mlp* mlp, rpb_mesh* m, const double* R, const double* G, int npairs,
                                   double lr, double reg, double* objective, float* grad);

/* --- energy without device allocation -------------------------------------------------- */

/* No counterpart in the reference (Repulsor has no device path). TangentPointEnergy0
 * Value for callers that cannot allocate device memory when they need the energy: hosts
 * whose device memory belongs to a fixed-size arena or pool, and real-time or inner-loop
 * code that forbids allocation after start-up (an allocation can synchronize the device or
 * fail under memory pressure). All pointers are device pointers the caller owns: V
 * (nV x 3), S (nS x (dom_dim+1)), the tree (perm: nS, C_begin/C_end: nC) and the full
 * symmetric near/far patterns exactly as rpb_mesh_tree/rpb_mesh_pattern return them for
 * this mesh (only sizes are checked); verynear_nnz is rpb_stats.verynear_nnz of the mesh
 * and must be 0 (meshes with very-near pairs give RPB_EINVAL: use rpb_tpe0_value). The
 * energy (1 double) is written asynchronously on `stream`. Unit charges. Scratch lives in
 * one static device array of about 12.4 MB (at most 40,960 simplices and 2 nS - 1
 * clusters; larger meshes give RPB_EINVAL) held by every device that loads the library
 * until the process exits; the first call on a device looks up the array's address and
 * should come before any stream capture; all calls share the array, so calls that overlap
 * on the GPU (other streams, other host threads) race and must be serialised by the
 * caller. Calls no cudaMalloc, cudaFree or allocating library routine. */
rpb_status rpb_tpe0_value_noalloc(int dom_dim, const double* V, int64_t nV, const int* S, int64_t nS,
                                  const int* perm, const int* C_begin, const int* C_end, int64_t nC,
                                  const int64_t* near_rowptr, const int* near_colidx, const int64_t* far_rowptr,
                                  const int* far_colidx, int64_t verynear_nnz, double q, double p, double* energy,
                                  void* stream);

/* --- measurement (no reference counterpart: Repulsor has no device path) ------------------ */

/* Runs `reps` energy+differential evaluations (SemiStaticUpdate geometry + pair kernels +
 * collection) on the mesh stream with CUDA events between the stages and returns the
 * mean milliseconds of each stage: ms[0] geometry/upsweep, ms[1] near-field pairs,
 * ms[2] far-field pairs, ms[3] collection + chain rule + vertex gather, ms[4] total.
 * If flush_bytes > 0 a device buffer of that size is overwritten before every
 * evaluation (outside the timed events) so that no stage starts with a warm L2. */
rpb_status rpb_tpe0_stage_times(rpb_mesh* m, double q, double p, int reps, int64_t flush_bytes, double* ms);

/* Measured FP32 FMA throughput of the device (TFLOP/s), from a register-resident
 * kernel of independent FMA chains timed with CUDA events. */
rpb_status rpb_measure_fp32_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* REPULSOR_B200_H */
