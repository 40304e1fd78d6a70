// Header-only C++20 mirror of Repulsor's tangent-point API over the C ABI of
// librepulsor_b200.so (include/repulsor_b200.h). Link with -lrepulsor_b200.
//
// Mirrored interfaces (HenrikSchumacher/Repulsor):
//   SimplicialMesh<DOM_DIM, AMB_DIM, Real, Int, LInt, SReal, ExtReal>
//       constructors src/SimplicialMesh.hpp:143-222, settings members
//       src/SimplicialMesh/SimplicialMeshBase.hpp:61-63 (src/Settings.hpp:5-54),
//       SemiStaticUpdate src/SimplicialMesh.hpp:354-376
//   TangentPointEnergy0<Mesh_T>   src/Energies/TangentPointEnergy0.hpp:35-45 with the
//       EnergyBase interface src/Energies/EnergyBase.hpp:40-121 (Value and the cached
//       Differential; Differential to a pointer with alpha/beta/ldY and with addto)
//   TangentPointObstacleEnergy<Mesh_T>  src/Energies/TangentPointObstacleEnergy.hpp:48-96,
//       with SimplicialMesh::LoadObstacle (src/SimplicialMesh.hpp:697-719)
//   TangentPointMetric0<Mesh_T>   src/Metrics/TangentPointMetric0.hpp:31-126 with the
//       MetricBase interface src/Metrics/MetricBase.hpp:31-134 (MultiplyMetric,
//       MultiplyPreconditioner, Solve, MetricNorm, PreconditionerNorm,
//       Solver_IterationCount, Solver_RelativeResiduals)
//
// As in the reference, the trees are built on first use, so the settings members may be
// changed after construction; invalid arguments print an error (eprint) and the call does
// nothing. The namespace is Repulsor_B200; `namespace Repulsor = Repulsor_B200;` makes
// existing Repulsor code compile against it unchanged for these classes.
#pragma once

#include <cmath>
#include <cstddef>
#include <iostream>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../repulsor_b200.h"

namespace Repulsor_B200 {

inline void eprint(const std::string& s) { std::cerr << "ERROR: " << s << std::endl; }

struct ClusterTreeSettings {
    int split_threshold = 1;
    int thread_count = 1;
};

struct BlockClusterTreeSettings {
    double far_field_separation_parameter = 0.5;
    double near_field_separation_parameter = 10.;
    double near_field_intersection_parameter = 10000000000.;
    int max_refinement = 30;
};

struct AdaptivitySettings {
    int max_refinement = 30;
    double theta = 10.;
    double intersection_theta = 10000000000.;
};

template <int DOM_DIM_, int AMB_DIM_, typename Real_ = double, typename Int_ = int, typename LInt_ = std::size_t,
          typename SReal_ = double, typename ExtReal_ = double>
class SimplicialMesh {
    static_assert(AMB_DIM_ == 3, "repulsor_b200 is built for ambient dimension 3");
    static_assert(DOM_DIM_ == 1 || DOM_DIM_ == 2, "repulsor_b200 is built for curves and surfaces");

public:
    using Real = Real_;
    using Int = Int_;
    using LInt = LInt_;
    using SReal = SReal_;
    using ExtReal = ExtReal_;
    static constexpr Int DOM_DIM = DOM_DIM_;
    static constexpr Int AMB_DIM = AMB_DIM_;

    mutable ClusterTreeSettings cluster_tree_settings;
    mutable BlockClusterTreeSettings block_cluster_tree_settings;
    mutable AdaptivitySettings adaptivity_settings;

    SimplicialMesh() = default;

    template <typename ExtReal_2, typename ExtInt>
    SimplicialMesh(const ExtReal_2* V, std::size_t vertex_count, const ExtInt* S, std::size_t simplex_count,
                   std::size_t thread_count = 1)
        : SimplicialMesh(V, vertex_count, false, S, simplex_count, false, thread_count)
    {}

    template <typename ExtReal_2, typename ExtInt>
    SimplicialMesh(const ExtReal_2* V, std::size_t vertex_count, bool V_ColMajorQ, const ExtInt* S,
                   std::size_t simplex_count, bool S_ColMajorQ, std::size_t thread_count = 1)
    {
        read(V, vertex_count, V_ColMajorQ, S, simplex_count, S_ColMajorQ);
        cluster_tree_settings.thread_count = static_cast<int>(thread_count);
    }

    template <typename ExtReal_2, typename ExtReal_3, typename ExtInt>
    SimplicialMesh(const ExtReal_2* V, std::size_t vertex_count, bool V_ColMajorQ, const ExtInt* S,
                   std::size_t simplex_count, bool S_ColMajorQ, const ExtReal_3* vertex_charges,
                   std::size_t thread_count = 1)
    {
        read(V, vertex_count, V_ColMajorQ, S, simplex_count, S_ColMajorQ);
        charges_.assign(vertex_charges, vertex_charges + vertex_count);
        cluster_tree_settings.thread_count = static_cast<int>(thread_count);
    }

    SimplicialMesh(const SimplicialMesh&) = delete;
    SimplicialMesh& operator=(const SimplicialMesh&) = delete;
    SimplicialMesh(SimplicialMesh&&) = default;
    SimplicialMesh& operator=(SimplicialMesh&&) = default;

    Int DomDim() const { return DOM_DIM; }
    Int AmbDim() const { return AMB_DIM; }
    Int VertexCount() const { return nV_; }
    Int SimplexCount() const { return nS_; }
    Int ThreadCount() const { return cluster_tree_settings.thread_count; }
    const std::vector<double>& VertexCoordinates() const { return V_; }
    const std::vector<int>& Simplices() const { return S_; }

    // New vertex positions with the same trees (src/SimplicialMesh.hpp:354-376).
    template <typename ExtReal_2>
    void SemiStaticUpdate(const ExtReal_2* V, bool transp = false)
    {
        for (Int v = 0; v < nV_; ++v)
            for (Int k = 0; k < AMB_DIM; ++k)
                V_[AMB_DIM * v + k] = static_cast<double>(transp ? V[nV_ * k + v] : V[AMB_DIM * v + k]);
        clear_cache();
        if (h_) check(rpb_mesh_semistatic_update(h_.get(), V_.data(), 0), "SemiStaticUpdate");
    }

    // The device mesh (built on first use from the current settings).
    rpb_mesh* Handle() const
    {
        if (!h_ && nV_ > 0) {
            rpb_settings s;
            rpb_default_settings(&s);
            s.split_threshold = cluster_tree_settings.split_threshold;
            s.far_field_separation = block_cluster_tree_settings.far_field_separation_parameter;
            s.near_field_separation = adaptivity_settings.theta;
            s.near_field_intersection = adaptivity_settings.intersection_theta;
            s.max_refinement = adaptivity_settings.max_refinement;
            s.thread_count = cluster_tree_settings.thread_count;
            s.device = device_;
            rpb_mesh* m = nullptr;
            if (check(rpb_mesh_create(DOM_DIM, AMB_DIM, V_.data(), nV_, S_.data(), nS_,
                                      charges_.empty() ? nullptr : charges_.data(), &s, &m),
                      "SimplicialMesh"))
                h_.reset(m);
        }
        return h_.get();
    }

    // Device ordinal used when the device mesh is created.
    void SetDevice(int device) { device_ = device; }

    // SimplicialMesh::LoadObstacle (src/SimplicialMesh.hpp:697-719): the mesh takes the
    // obstacle over; it must have the same domain dimension.
    void LoadObstacle(std::unique_ptr<SimplicialMesh> obstacle)
    {
        if (!obstacle || !Handle() || !obstacle->Handle()) return;
        if (check(rpb_mesh_load_obstacle(Handle(), obstacle->h_.get()), "LoadObstacle")) {
            obstacle->h_.release();    // now owned by this mesh's device object
            obstacle_ = std::move(obstacle);
        }
        clear_cache();
    }

    // Result caches of the energies (src/Energies/EnergyBase.hpp:46-51); SemiStaticUpdate clears them.
    struct Cache {
        bool has_value = false;
        double value = 0;
        std::vector<double> differential;
    };
    Cache& GetCache(const std::string& tag) const { return cache_[tag]; }
    void clear_cache() const { cache_.clear(); }

    static bool check(rpb_status st, const std::string& where)
    {
        if (st == RPB_OK) return true;
        eprint(className() + "::" + where + ": " + rpb_last_error());
        return false;
    }

    static std::string className()
    {
        return "SimplicialMesh<" + std::to_string(DOM_DIM) + "," + std::to_string(AMB_DIM) + ">";
    }

private:
    struct Deleter {
        void operator()(rpb_mesh* m) const { rpb_mesh_destroy(m); }
    };

    template <typename ExtReal_2, typename ExtInt>
    void read(const ExtReal_2* V, std::size_t nV, bool V_col, const ExtInt* S, std::size_t nS, bool S_col)
    {
        nV_ = static_cast<Int>(nV);
        nS_ = static_cast<Int>(nS);
        V_.resize(AMB_DIM * nV);
        S_.resize((DOM_DIM + 1) * nS);
        for (std::size_t v = 0; v < nV; ++v)
            for (int k = 0; k < AMB_DIM; ++k)
                V_[AMB_DIM * v + k] = static_cast<double>(V_col ? V[nV * k + v] : V[AMB_DIM * v + k]);
        for (std::size_t i = 0; i < nS; ++i)
            for (int k = 0; k <= DOM_DIM; ++k)
                S_[(DOM_DIM + 1) * i + k] = static_cast<int>(S_col ? S[nS * k + i] : S[(DOM_DIM + 1) * i + k]);
    }

    Int nV_ = 0, nS_ = 0;
    int device_ = 0;
    std::vector<double> V_, charges_;
    std::vector<int> S_;
    mutable std::unique_ptr<rpb_mesh, Deleter> h_;
    mutable std::unordered_map<std::string, Cache> cache_;
    std::unique_ptr<SimplicialMesh> obstacle_;   // host side of a loaded obstacle
};

template <typename Mesh_T>
class TangentPointEnergy0 {
public:
    using Real = typename Mesh_T::Real;
    using Int = typename Mesh_T::Int;
    using ExtReal = typename Mesh_T::ExtReal;

    TangentPointEnergy0(Real q_, Real p_) : q(q_), p(p_) {}
    explicit TangentPointEnergy0(Real p_) : q(p_), p(2 * p_) {}

    // Value of the energy, cached on the mesh.
    ExtReal Value(const Mesh_T& M) const
    {
        auto& c = M.GetCache(ClassName());
        if (!c.has_value) {
            double e = 0;
            if (!M.Handle() || !Mesh_T::check(rpb_tpe0_value(M.Handle(), q, p, &e), ClassName() + "::Value")) return 0;
            c.value = e;
            c.has_value = true;
        }
        return c.value;
    }

    // Differential (n_v x 3, row-major), cached on the mesh together with the value.
    const std::vector<double>& Differential(const Mesh_T& M) const
    {
        auto& c = M.GetCache(ClassName());
        if (c.differential.empty()) {
            std::vector<double> D(static_cast<std::size_t>(M.VertexCount()) * Mesh_T::AMB_DIM, 0.0);
            double e = 0;
            if (M.Handle() &&
                Mesh_T::check(rpb_tpe0_differential(M.Handle(), q, p, 1.0, 0.0, D.data(), Mesh_T::AMB_DIM, &e),
                              ClassName() + "::Differential")) {
                c.differential = std::move(D);
                c.value = e;
                c.has_value = true;
            }
        }
        return c.differential;
    }

    // Y = alpha * dE + beta * Y (leading dimension ldY); returns the energy. No caching.
    ExtReal Differential(const Mesh_T& M, ExtReal alpha, ExtReal beta, ExtReal* Y, Int ldY) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        Mesh_T::check(rpb_tpe0_differential(M.Handle(), q, p, alpha, beta, Y, ldY, &e), ClassName() + "::Differential");
        return e;
    }

    ExtReal Differential(const Mesh_T& M, ExtReal* Y, bool addto = false) const
    {
        return Differential(M, ExtReal(1), ExtReal(addto ? 1 : 0), Y, Mesh_T::AMB_DIM);
    }

    // Energy densities per simplex / per vertex (src/Energies/EnergyBase.hpp:129-150);
    // return the energy.
    ExtReal SimplexDensities(const Mesh_T& M, ExtReal* density) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        Mesh_T::check(rpb_tpe0_simplex_densities(M.Handle(), q, p, density, &e), ClassName() + "::SimplexDensities");
        return e;
    }

    ExtReal VertexDensities(const Mesh_T& M, ExtReal* density) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        Mesh_T::check(rpb_tpe0_vertex_densities(M.Handle(), q, p, density, &e), ClassName() + "::VertexDensities");
        return e;
    }

    std::string ClassName() const
    {
        return "TangentPointEnergy0<" + std::to_string(Mesh_T::DOM_DIM) + "," + std::to_string(Mesh_T::AMB_DIM) + ">(" +
               std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;
};

// TangentPointObstacleEnergy (src/Energies/TangentPointObstacleEnergy.hpp:48-96): the
// tangent-point energy of the mesh against its loaded obstacle; 0 without one.
template <typename Mesh_T>
class TangentPointObstacleEnergy {
public:
    using Real = typename Mesh_T::Real;
    using Int = typename Mesh_T::Int;
    using ExtReal = typename Mesh_T::ExtReal;

    TangentPointObstacleEnergy(Real q_, Real p_) : q(q_), p(p_) {}

    ExtReal Value(const Mesh_T& M) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        Mesh_T::check(rpb_tpoe_value(M.Handle(), q, p, &e), ClassName() + "::Value");
        return e;
    }

    ExtReal Differential(const Mesh_T& M, ExtReal alpha, ExtReal beta, ExtReal* Y, Int ldY) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        Mesh_T::check(rpb_tpoe_differential(M.Handle(), q, p, alpha, beta, Y, ldY, &e), ClassName() + "::Differential");
        return e;
    }

    std::string ClassName() const
    {
        return "TangentPointObstacleEnergy<" + std::to_string(Mesh_T::DOM_DIM) + "," + std::to_string(Mesh_T::AMB_DIM) +
               ">(" + std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;
};

template <typename Mesh_T>
class TangentPointMetric0 {
public:
    using Real = typename Mesh_T::Real;
    using Int = typename Mesh_T::Int;
    using ExtReal = typename Mesh_T::ExtReal;

    TangentPointMetric0(Real q_, Real p_) : q(q_), p(p_) {}
    explicit TangentPointMetric0(Real p_) : q(p_), p(2 * p_) {}

    // Y = alpha * A X + beta * Y (src/Metrics/MetricDimRestricted.hpp:109-139).
    void MultiplyMetric(const Mesh_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta, ExtReal* Y, Int ldY,
                        Int nrhs, bool VF_flag = true, bool NF_flag = true, bool FF_flag = true) const
    {
        if (!nrhs_ok(nrhs, "MultiplyMetric") || !M.Handle()) return;
        const int flags = (VF_flag ? 1 : 0) | (NF_flag ? 2 : 0) | (FF_flag ? 4 : 0);
        Mesh_T::check(rpb_tpm0_multiply(M.Handle(), q, p, alpha, X, ldX, beta, Y, ldY, nrhs, flags),
                      ClassName() + "::MultiplyMetric");
    }

    // Y = alpha * H1^{-1} L_{2-s} H1^{-1} X + beta * Y (src/Metrics/TangentPointMetric0.hpp:88-126).
    void MultiplyPreconditioner(const Mesh_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta, ExtReal* Y,
                                Int ldY, Int nrhs) const
    {
        if (!nrhs_ok(nrhs, "MultiplyPreconditioner") || !M.Handle()) return;
        Mesh_T::check(rpb_tpm0_precondition(M.Handle(), q, p, alpha, X, ldX, beta, Y, ldY, nrhs),
                      ClassName() + "::MultiplyPreconditioner");
    }

    // X = alpha * A^{-1} B + beta * X (src/Metrics/MetricDimRestricted.hpp:232-289).
    void Solve(const Mesh_T& M, ExtReal alpha, const ExtReal* B, Int ldB, ExtReal beta, ExtReal* X, Int ldX, Int nrhs,
               Int max_iter, Real tolerance) const
    {
        if (!nrhs_ok(nrhs, "Solve") || !M.Handle()) return;
        int it = 0;
        double rr[3] = {0, 0, 0};
        const rpb_status st = rpb_tpm0_solve(M.Handle(), q, p, alpha, B, ldB, beta, X, ldX, nrhs, max_iter, tolerance,
                                             precond, &it, rr);
        iter = it;
        rel_residuals.assign(rr, rr + 3);
        if (st != RPB_ENOTCONV) Mesh_T::check(st, ClassName() + "::Solve");
    }

    ExtReal MetricNorm(const Mesh_T& M, const ExtReal* X, Int ldX, Int nrhs) const
    {
        std::vector<double> Xc(static_cast<std::size_t>(M.VertexCount()) * nrhs), Y(Xc.size(), 0.0);
        for (Int v = 0; v < M.VertexCount(); ++v)
            for (Int k = 0; k < nrhs; ++k) Xc[nrhs * v + k] = X[ldX * v + k];
        MultiplyMetric(M, 1, Xc.data(), nrhs, 0, Y.data(), nrhs, nrhs);
        double s = 0;
        for (std::size_t k = 0; k < Y.size(); ++k) s += Xc[k] * Y[k];
        return std::sqrt(s);
    }

    ExtReal PreconditionerNorm(const Mesh_T& M, const ExtReal* X, Int ldX, Int nrhs) const
    {
        std::vector<double> Xc(static_cast<std::size_t>(M.VertexCount()) * nrhs), Y(Xc.size(), 0.0);
        for (Int v = 0; v < M.VertexCount(); ++v)
            for (Int k = 0; k < nrhs; ++k) Xc[nrhs * v + k] = X[ldX * v + k];
        MultiplyPreconditioner(M, 1, Xc.data(), nrhs, 0, Y.data(), nrhs, nrhs);
        double s = 0;
        for (std::size_t k = 0; k < Y.size(); ++k) s += Xc[k] * Y[k];
        return std::sqrt(s);
    }

    Int Solver_IterationCount() const { return iter; }
    std::vector<double> Solver_RelativeResiduals() const { return rel_residuals; }

    // B200 extra: the preconditioner Solve uses (RPB_PRECOND_REFERENCE by default).
    void SetPreconditioner(rpb_precond kind) { precond = kind; }

    std::string ClassName() const
    {
        return "TangentPointMetric0<" + std::to_string(Mesh_T::DOM_DIM) + "," + std::to_string(Mesh_T::AMB_DIM) + ">(" +
               std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;

private:
    bool nrhs_ok(Int nrhs, const char* tag) const
    {
        if (nrhs == Mesh_T::AMB_DIM) return true;
        eprint(ClassName() + "::" + tag + ": nrhs = " + std::to_string(nrhs) + " != " + std::to_string(Mesh_T::AMB_DIM) +
               " = AMB_DIM");
        return false;
    }

    int precond = RPB_PRECOND_REFERENCE;
    mutable Int iter = 0;
    mutable std::vector<double> rel_residuals;
};

}  // namespace Repulsor_B200
