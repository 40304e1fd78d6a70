// Solver state owned by a mesh (allocated on the first Solve / MultiplyPreconditioner).
#pragma once

#include <vector>

#include "rpb_mesh.cuh"

namespace rpb {

struct LearnedState;

struct Solver {
    ~Solver();
    // CG vectors, each n x 3 FP64
    enum { V_X = 0, V_R, V_Z, V_P, V_AP, V_ROLD, V_B, V_PRE, V_HYB, NVEC };
    DevBuf<double> vec;
    DevBuf<double> scal;          // per-column CG scalars
    DevBuf<double> partials;      // block partials of the dot products
    DevBuf<unsigned> done;
    double* host_scal = nullptr;  // pinned readback of the scalars
    // H1 Cholesky factor (reference preconditioner) and its supernodal level schedule
    int64_t h1_version = -1;
    std::vector<int> nd_perm;
    // one launch plan per level: a warp level (sn_list[first .. first + count)) or a split
    // level (row_list[first .. first + count), G lanes per row for the external part and
    // for the diagonal block)
    struct Level {
        bool warp = true;
        int first = 0, count = 0, g_ext = 32, g_dense = 32;
    };
    // per direction (0: forward on L, 1: backward on L^T)
    struct Direction {
        DevBuf<int64_t> ext_rp;
        DevBuf<int> ext_ci, sn_list, row_list;
        DevBuf<double> ext_val, dinv;
        std::vector<Level> levels;
    } dir[2];
    DevBuf<int64_t> dinv_off;
    DevBuf<int> perm, sn_begin, sn_of;
    DevBuf<double> tri, tmp, tbuf;
    int sn_levels_fwd = 0;
    double factor_seconds = 0;
    int64_t factor_nnz = 0;
    bool factor_on_device = false;   // numeric factorization on the device (else host threads)
    // statistics of the last Solve
    int last_iterations = 0, last_restarts = 0, last_fallback_iteration = -1;
};

}  // namespace rpb
