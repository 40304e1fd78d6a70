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
    DevBuf<int> err;              // set when a bounded device wait gives up
    double* host_scal = nullptr;  // pinned readback of the scalars
    // H1 Cholesky factor (reference preconditioner)
    int64_t h1_version = -1;
    std::vector<int> nd_perm;
    DevBuf<int64_t> lo_rp, up_rp;
    DevBuf<int> lo_ci, up_ci, perm, flags;
    DevBuf<double> lo_val, up_val, tri, tmp;
    DevBuf<unsigned> ticket;
    int epoch = 0;
    double factor_seconds = 0;
    int64_t factor_nnz = 0;
};

}  // namespace rpb
