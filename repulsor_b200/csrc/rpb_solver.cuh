// Solver state owned by a mesh (allocated on the first Solve / MultiplyPreconditioner).
#pragma once

#include <vector>

#include "rpb_mesh.cuh"

namespace rpb {

struct LearnedState;

struct Solver {
    ~Solver();
    // CG vectors, each n x 3 FP64
    enum { V_X = 0, V_R, V_Z, V_P, V_AP, V_ROLD, V_B, V_PRE, NVEC };
    DevBuf<double> vec;
    DevBuf<double> scal;          // per-column CG scalars
    DevBuf<double> partials;      // block partials of the dot products
    DevBuf<unsigned> done;
    double* host_scal = nullptr;  // pinned readback of the scalars
    // H1 Cholesky factor (reference preconditioner) and its supernodal level schedule
    int64_t h1_version = -1;
    std::vector<int> nd_perm;
    DevBuf<int64_t> lo_rp, up_rp, dinv_off;
    DevBuf<int> lo_ci, up_ci, perm, sn_begin, fwd_level_sn, bwd_level_sn, sn_of, fwd_split_rows, bwd_split_rows;
    DevBuf<double> lo_val, up_val, dinv, dinvT, tri, tmp, tbuf;
    int sn_levels_fwd = 0, sn_levels_bwd = 0;
    std::vector<int> fwd_level_ptr, bwd_level_ptr, fwd_level_width, bwd_level_width;
    std::vector<int> fwd_split_ptr, bwd_split_ptr;   // per level: rows of split levels (empty range: fused)
    double factor_seconds = 0;
    int64_t factor_nnz = 0;
    // statistics of the last Solve
    int last_iterations = 0, last_restarts = 0, last_fallback_iteration = -1;
};

}  // namespace rpb
