// Header-only C++20 mirror of Repulsor's tangent-point API over the C ABI of
// librepulsor_b200.so (include/repulsor_b200.h). Link with -lrepulsor_b200.
//
// Mirrored interfaces (HenrikSchumacher/Repulsor):
//   SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>
//       src/SimplicialMesh/SimplicialMeshBase.hpp:8-230 (settings members :61-63,
//       SemiStaticUpdate :104, MaximumSafeStepSize :134-139, LoadObstacle/GetObstacle
//       :186-188, WriteToFile :204)
//   SimplicialMesh<DOM_DIM, AMB_DIM, Real, Int, LInt, SReal, ExtReal>
//       constructors src/SimplicialMesh.hpp:143-222, SemiStaticUpdate :354-376,
//       WriteToFile :780-818
//   SimplicialMesh_Factory<MeshBase_T, MinDom, MaxDom, MinAmb, MaxAmb>
//       src/SimplicialMesh/SimplicialMesh_Factory.hpp:8-246 (Make, Make_FromFile)
//   EnergyBase<MeshBase_T>        src/Energies/EnergyBase.hpp:8-163 (cached Value and
//       Differential, Differential to a pointer with alpha/beta/ldY and with addto,
//       SimplexDensities, VertexDensities)
//   MetricBase<MeshBase_T>        src/Metrics/MetricBase.hpp:8-134 (MultiplyMetric,
//       MultiplyPreconditioner, Solve, MetricNorm, PreconditionerNorm,
//       Solver_IterationCount, Solver_RelativeResiduals)
//   TangentPointEnergy0<Mesh_T>   src/Energies/TangentPointEnergy0.hpp:35-45
//   TangentPointMetric0<Mesh_T>   src/Metrics/TangentPointMetric0.hpp:31-126
//   TangentPointObstacleEnergy<Mesh_T>  src/Energies/TangentPointObstacleEnergy.hpp:48-96
//   TangentPointEnergy0_Factory / TangentPointMetric0_Factory
//       src/Energies/TangentPointEnergy/TP_Factory.hpp:8-89 (Make(dom, amb, q, p))
//   TangentPointObstacleEnergy_Factory
//       src/Energies/TangentPointEnergy/TPO_Factory.hpp:8-95 (Make(dom_S, dom_T, amb, q, p))
//   Tensor1 / Tensor2  minimal stand-ins for the Tensors library's containers that the
//       reference uses as TangentVector_T / CotangentVector_T (contiguous, row-major)
//
// As in the reference, the trees are built on first use, so the settings members may be
// changed after construction; invalid arguments print an error (eprint) and the call does
// nothing. The namespace is Repulsor_B200; `namespace Repulsor = Repulsor_B200;` lets code
// written against these reference classes compile against it.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../repulsor_b200.h"

namespace Repulsor_B200 {

inline void eprint(const std::string& s) { std::cerr << "ERROR: " << s << std::endl; }

// ---------------------------------------------------------------------------------------
// Containers
// ---------------------------------------------------------------------------------------

template <typename T, typename I>
class Tensor1 {
public:
    Tensor1() = default;
    explicit Tensor1(I n) : a_(static_cast<std::size_t>(n), T(0)) {}
    Tensor1(I n, T init) : a_(static_cast<std::size_t>(n), init) {}
    template <typename S>
    Tensor1(const S* src, I n) : a_(src, src + n) {}

    T* data() { return a_.data(); }
    const T* data() const { return a_.data(); }
    I Size() const { return static_cast<I>(a_.size()); }
    I Dim(I) const { return Size(); }
    T& operator[](I i) { return a_[static_cast<std::size_t>(i)]; }
    const T& operator[](I i) const { return a_[static_cast<std::size_t>(i)]; }
    T& operator()(I i) { return (*this)[i]; }
    const T& operator()(I i) const { return (*this)[i]; }
    T Max() const { return a_.empty() ? T(0) : *std::max_element(a_.begin(), a_.end()); }

private:
    std::vector<T> a_;
};

template <typename T, typename I>
std::ostream& operator<<(std::ostream& s, const Tensor1<T, I>& t)
{
    s << "{ ";
    for (I i = 0; i < t.Size(); ++i) s << (i ? ", " : "") << t[i];
    return s << " }";
}

template <typename T, typename I>
class Tensor2 {
public:
    Tensor2() = default;
    Tensor2(I m, I n) : d0_(m), d1_(n), a_(static_cast<std::size_t>(m) * static_cast<std::size_t>(n), T(0)) {}
    Tensor2(I m, I n, T init) : d0_(m), d1_(n), a_(static_cast<std::size_t>(m) * static_cast<std::size_t>(n), init) {}

    T* data() { return a_.data(); }
    const T* data() const { return a_.data(); }
    T* data(I i) { return a_.data() + static_cast<std::size_t>(i) * d1_; }
    const T* data(I i) const { return a_.data() + static_cast<std::size_t>(i) * d1_; }
    I Dim(I k) const { return k == 0 ? d0_ : (k == 1 ? d1_ : I(0)); }
    I Size() const { return static_cast<I>(a_.size()); }
    T& operator()(I i, I j) { return a_[static_cast<std::size_t>(i) * d1_ + j]; }
    const T& operator()(I i, I j) const { return a_[static_cast<std::size_t>(i) * d1_ + j]; }

    void Fill(T x) { std::fill(a_.begin(), a_.end(), x); }
    void SetZero() { Fill(T(0)); }

    // Uniformly distributed entries in [0, 1) from a fixed-seed generator (reproducible,
    // and independent of the host's entropy source).
    void Random(std::uint64_t seed = 0x5eedULL)
    {
        std::mt19937_64 g{seed};
        std::uniform_real_distribution<double> u(0.0, 1.0);
        for (T& x : a_) x = static_cast<T>(u(g));
    }

    // Reads d0 rows of d1 entries with leading dimension ld; writes them likewise.
    template <typename S>
    void Read(const S* src, I ld)
    {
        for (I i = 0; i < d0_; ++i)
            for (I j = 0; j < d1_; ++j) (*this)(i, j) = static_cast<T>(src[static_cast<std::size_t>(i) * ld + j]);
    }
    template <typename S>
    void Write(S* dst, I ld) const
    {
        for (I i = 0; i < d0_; ++i)
            for (I j = 0; j < d1_; ++j) dst[static_cast<std::size_t>(i) * ld + j] = static_cast<S>((*this)(i, j));
    }

    Tensor2& operator*=(T s)
    {
        for (T& x : a_) x *= s;
        return *this;
    }
    template <typename S>
    Tensor2& operator+=(const Tensor2<S, I>& b)
    {
        if (b.Dim(0) != d0_ || b.Dim(1) != d1_) {
            eprint("Tensor2::operator+=: dimensions do not match");
            return *this;
        }
        for (std::size_t k = 0; k < a_.size(); ++k) a_[k] += static_cast<T>(b.data()[k]);
        return *this;
    }
    template <typename S>
    Tensor2& operator-=(const Tensor2<S, I>& b)
    {
        if (b.Dim(0) != d0_ || b.Dim(1) != d1_) {
            eprint("Tensor2::operator-=: dimensions do not match");
            return *this;
        }
        for (std::size_t k = 0; k < a_.size(); ++k) a_[k] -= static_cast<T>(b.data()[k]);
        return *this;
    }

private:
    I d0_ = 0, d1_ = 0;
    std::vector<T> a_;
};

// ---------------------------------------------------------------------------------------
// Settings (src/Settings.hpp:5-54)
// ---------------------------------------------------------------------------------------

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

// ---------------------------------------------------------------------------------------
// Meshes
// ---------------------------------------------------------------------------------------

template <typename Real_, typename Int_, typename LInt_, typename SReal_ = Real_, typename ExtReal_ = Real_>
class SimplicialMeshBase {
    static_assert(std::is_integral_v<Int_> && std::is_integral_v<LInt_>, "Int and LInt must be integral types");
    static_assert(std::is_same_v<Real_, double> && std::is_same_v<ExtReal_, double>,
                  "repulsor_b200 takes and returns double at its host boundary");

public:
    using Real = Real_;
    using Int = Int_;
    using LInt = LInt_;
    using SReal = SReal_;
    using ExtReal = ExtReal_;
    using TangentVector_T = Tensor2<ExtReal, Int>;
    using CotangentVector_T = Tensor2<ExtReal, Int>;

    mutable ClusterTreeSettings cluster_tree_settings;
    mutable BlockClusterTreeSettings block_cluster_tree_settings;
    mutable AdaptivitySettings adaptivity_settings;

    SimplicialMeshBase() = default;
    virtual ~SimplicialMeshBase() = default;
    SimplicialMeshBase(const SimplicialMeshBase&) = delete;
    SimplicialMeshBase& operator=(const SimplicialMeshBase&) = delete;

    virtual Int DomDim() const = 0;
    virtual Int AmbDim() const = 0;
    Int VertexCount() const { return V_.Dim(0); }
    Int SimplexCount() const { return S_.Dim(0); }
    Int ThreadCount() const { return cluster_tree_settings.thread_count; }
    const Tensor2<Real, Int>& VertexCoordinates() const { return V_; }
    const Tensor2<Int, Int>& Simplices() const { return S_; }

    // New vertex positions with the same trees (src/SimplicialMesh.hpp:354-376).
    void SemiStaticUpdate(const ExtReal* V, bool transp = false) const
    {
        const Int nV = VertexCount(), m = AmbDim();
        for (Int v = 0; v < nV; ++v)
            for (Int k = 0; k < m; ++k) V_(v, k) = transp ? V[static_cast<std::size_t>(nV) * k + v] : V[m * v + k];
        ClearCache();
        if (h_) check(rpb_mesh_semistatic_update(h_.get(), V_.data(), 0), "SemiStaticUpdate");
    }

    // Largest collision-free step along vecs (src/SimplicialMesh.hpp:441-468).
    ExtReal MaximumSafeStepSize(const ExtReal* vecs, ExtReal max_time, ExtReal TOL = ExtReal(0.0625),
                                bool transp = false)
    {
        if (!Handle()) return 0;
        const Int nV = VertexCount(), m = AmbDim();
        std::vector<double> U(static_cast<std::size_t>(nV) * m);
        for (Int v = 0; v < nV; ++v)
            for (Int k = 0; k < m; ++k)
                U[static_cast<std::size_t>(m) * v + k] = transp ? vecs[static_cast<std::size_t>(nV) * k + v] : vecs[m * v + k];
        double t = 0;
        if (!check(rpb_mesh_maximum_safe_step_size(Handle(), U.data(), max_time, TOL, &t), "MaximumSafeStepSize"))
            return 0;
        return t;
    }

    // SimplicialMesh::LoadObstacle (src/SimplicialMesh.hpp:697-719): the mesh takes the
    // obstacle over; it must have the same domain dimension.
    void LoadObstacle(std::unique_ptr<SimplicialMeshBase> obstacle)
    {
        if (!obstacle || !Handle() || !obstacle->Handle()) return;
        if (check(rpb_mesh_load_obstacle(Handle(), obstacle->h_.get()), "LoadObstacle")) {
            obstacle->h_.release();    // now owned by this mesh's device object
            obstacle_ = std::move(obstacle);
        }
        ClearCache();
    }

    const SimplicialMeshBase& GetObstacle() const
    {
        if (!obstacle_) eprint(ClassName() + "::GetObstacle: no obstacle loaded; returning the mesh itself.");
        return obstacle_ ? *obstacle_ : *this;
    }

    bool ObstacleLoadedQ() const { return static_cast<bool>(obstacle_); }

    // SimplicialMesh::WriteToFile (src/SimplicialMesh.hpp:780-818): the text format that
    // SimplicialMesh_Factory::Make_FromFile reads.
    void WriteToFile(const std::filesystem::path& file) const
    {
        std::ofstream s(file);
        if (!s.good()) {
            eprint(ClassName() + "::WriteToFile: file " + file.string() + " could not be opened.");
            return;
        }
        const Int nV = VertexCount(), nS = SimplexCount(), m = AmbDim(), sz = DomDim() + 1;
        s << "domain_dimension\t" << DomDim() << "\n";
        s << "ambient_dimension\t" << m << "\n";
        s << "vertex_count\t" << nV << "\n";
        s << "simplex_count\t" << nS << "\n";
        s << std::scientific << std::uppercase << std::setprecision(std::numeric_limits<Real>::digits10 + 1);
        for (Int v = 0; v < nV; ++v) {
            for (Int k = 0; k < m; ++k) s << V_(v, k) << "\t";
            s << "\n";
        }
        for (Int i = 0; i < nS; ++i) {
            for (Int k = 0; k < sz; ++k) s << S_(i, k) << "\t";
            s << "\n";
        }
    }

    // The device mesh (built on first use from the current settings).
    rpb_mesh* Handle() const
    {
        if (!h_ && VertexCount() > 0) {
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
            if (check(rpb_mesh_create(DomDim(), AmbDim(), V_.data(), VertexCount(), S32_.data(), SimplexCount(),
                                      charges_.empty() ? nullptr : charges_.data(), &s, &m),
                      "SimplicialMesh"))
                h_.reset(m);
        }
        return h_.get();
    }

    // Device ordinal used when the device mesh is created.
    void SetDevice(int device) { device_ = device; }

    // Result caches of the energies (CachedObject, src/Energies/EnergyBase.hpp:46-83);
    // SemiStaticUpdate and LoadObstacle clear them.
    struct Cache {
        bool has_value = false;
        ExtReal value = 0;
        bool has_differential = false;
        CotangentVector_T differential;
    };
    Cache& GetCache(const std::string& tag) const { return cache_[tag]; }
    bool InCacheQ(const std::string& tag) const { return cache_.count(tag) > 0; }
    void ClearCache() const { cache_.clear(); }

    bool check(rpb_status st, const std::string& where) const
    {
        if (st == RPB_OK) return true;
        eprint(ClassName() + "::" + where + ": " + rpb_last_error());
        return false;
    }

    virtual std::string ClassName() const { return "SimplicialMeshBase"; }

protected:
    template <typename ExtReal_2, typename ExtInt>
    void read(Int dom, Int amb, const ExtReal_2* V, Int nV, bool V_col, const ExtInt* S, Int nS, bool S_col)
    {
        V_ = Tensor2<Real, Int>(nV, amb);
        S_ = Tensor2<Int, Int>(nS, dom + 1);
        S32_.resize(static_cast<std::size_t>(nS) * (dom + 1));
        for (Int v = 0; v < nV; ++v)
            for (Int k = 0; k < amb; ++k)
                V_(v, k) = static_cast<Real>(V_col ? V[static_cast<std::size_t>(nV) * k + v] : V[amb * v + k]);
        for (Int i = 0; i < nS; ++i)
            for (Int k = 0; k <= dom; ++k) {
                S_(i, k) = static_cast<Int>(S_col ? S[static_cast<std::size_t>(nS) * k + i] : S[(dom + 1) * i + k]);
                S32_[static_cast<std::size_t>(dom + 1) * i + k] = static_cast<int>(S_(i, k));
            }
    }

    struct Deleter {
        void operator()(rpb_mesh* m) const { rpb_mesh_destroy(m); }
    };

    int device_ = 0;
    mutable Tensor2<Real, Int> V_;
    Tensor2<Int, Int> S_;
    std::vector<int> S32_;
    std::vector<double> charges_;
    mutable std::unique_ptr<rpb_mesh, Deleter> h_;
    mutable std::unordered_map<std::string, Cache> cache_;
    std::unique_ptr<SimplicialMeshBase> obstacle_;   // host side of a loaded obstacle
};

template <int DOM_DIM_, int AMB_DIM_, typename Real_ = double, typename Int_ = int, typename LInt_ = std::size_t,
          typename SReal_ = Real_, typename ExtReal_ = Real_>
class SimplicialMesh : public SimplicialMeshBase<Real_, Int_, LInt_, SReal_, ExtReal_> {
    static_assert(AMB_DIM_ == 3, "repulsor_b200 is built for ambient dimension 3");
    static_assert(DOM_DIM_ == 1 || DOM_DIM_ == 2, "repulsor_b200 is built for curves and surfaces");
    using Base = SimplicialMeshBase<Real_, Int_, LInt_, SReal_, ExtReal_>;

public:
    using Real = Real_;
    using Int = Int_;
    using LInt = LInt_;
    using SReal = SReal_;
    using ExtReal = ExtReal_;
    using MeshBase_T = Base;
    static constexpr Int DOM_DIM = DOM_DIM_;
    static constexpr Int AMB_DIM = AMB_DIM_;

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
        this->read(DOM_DIM, AMB_DIM, V, static_cast<Int>(vertex_count), V_ColMajorQ, S, static_cast<Int>(simplex_count),
                   S_ColMajorQ);
        this->cluster_tree_settings.thread_count = static_cast<int>(std::max<std::size_t>(1, thread_count));
    }

    template <typename ExtReal_2, typename ExtReal_3, typename ExtInt>
    SimplicialMesh(const ExtReal_2* V, std::size_t vertex_count, bool V_ColMajorQ, const ExtInt* S,
                   std::size_t simplex_count, bool S_ColMajorQ, const ExtReal_3* vertex_charges,
                   std::size_t thread_count = 1)
        : SimplicialMesh(V, vertex_count, V_ColMajorQ, S, simplex_count, S_ColMajorQ, thread_count)
    {
        this->charges_.assign(vertex_charges, vertex_charges + vertex_count);
    }

    Int DomDim() const override { return DOM_DIM; }
    Int AmbDim() const override { return AMB_DIM; }

    std::string ClassName() const override { return className(); }
    static std::string className()
    {
        return "SimplicialMesh<" + std::to_string(DOM_DIM) + "," + std::to_string(AMB_DIM) + ">";
    }
};

namespace detail {
// Mesh text format of SimplicialMesh_Factory::Make_FromFile / SimplicialMesh::WriteToFile
// (src/SimplicialMesh/SimplicialMesh_Factory.hpp:160-246, src/SimplicialMesh.hpp:780-818):
// four "name value" lines (domain dimension, ambient dimension, vertex count, simplex
// count; the names are not checked), then the coordinates and the simplices row by row.
struct MeshFile {
    long long dom = -1, amb = -1, nV = -1, nS = -1;
    std::vector<double> V;
    std::vector<long long> S;
};

inline bool read_mesh_file(const std::filesystem::path& file, MeshFile& f)
{
    std::ifstream s(file);
    if (!s.good()) return false;
    std::string name;
    s >> name >> f.dom >> name >> f.amb >> name >> f.nV >> name >> f.nS;
    if (!s || f.dom < 0 || f.amb < 1 || f.nV < 0 || f.nS < 0) return false;
    f.V.resize(static_cast<std::size_t>(f.nV * f.amb));
    f.S.resize(static_cast<std::size_t>(f.nS * (f.dom + 1)));
    for (double& x : f.V) s >> x;
    for (long long& i : f.S) s >> i;
    return static_cast<bool>(s);
}
}  // namespace detail

template <class MeshBase_T, int... N>
class SimplicialMesh_Factory;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal, int MinDomDim_,
          int MaxDomDim_, int MinAmbDim_, int MaxAmbDim_>
class SimplicialMesh_Factory<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>, MinDomDim_, MaxDomDim_, MinAmbDim_,
                             MaxAmbDim_> {
    static_assert(MinDomDim_ <= MaxDomDim_, "MinDomDim_ <= MaxDomDim_ required.");
    static_assert(MinAmbDim_ <= MaxAmbDim_, "MinAmbDim_ <= MaxAmbDim_ required.");

public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;

    // Meshes of domain dimension simplex_size - 1 in [MinDom, MaxDom] and ambient
    // dimension in [MinAmb, MaxAmb]; this build has (1, 3) and (2, 3).
    template <typename ExtInt>
    [[nodiscard]] std::unique_ptr<MeshBase_T> Make(const ExtReal* vertex_coords, Int vertex_count, Int amb_dim,
                                                   bool vertex_coords_ColMajorQ, const ExtInt* simplices,
                                                   Int simplex_count, Int simplex_size, bool simplices_ColMajorQ,
                                                   Int thread_count = 1) const
    {
        const Int dom_dim = simplex_size - 1;
        if (dom_dim < MinDomDim_ || dom_dim > MaxDomDim_) {
            eprint(ClassName() + "::Make: dom_dim is out of range.");
            return Error(dom_dim, amb_dim);
        }
        if (amb_dim < MinAmbDim_ || amb_dim > MaxAmbDim_) {
            eprint(ClassName() + "::Make: amb_dim is out of range.");
            return Error(dom_dim, amb_dim);
        }
        if (amb_dim != 3 || (dom_dim != 1 && dom_dim != 2)) return Error(dom_dim, amb_dim);
        if (dom_dim == 1)
            return std::make_unique<SimplicialMesh<1, 3, Real, Int, LInt, SReal, ExtReal>>(
                vertex_coords, vertex_count, vertex_coords_ColMajorQ, simplices, simplex_count, simplices_ColMajorQ,
                thread_count);
        return std::make_unique<SimplicialMesh<2, 3, Real, Int, LInt, SReal, ExtReal>>(
            vertex_coords, vertex_count, vertex_coords_ColMajorQ, simplices, simplex_count, simplices_ColMajorQ,
            thread_count);
    }

    [[nodiscard]] std::unique_ptr<MeshBase_T> Make_FromFile(const std::filesystem::path& file, Int thread_count) const
    {
        detail::MeshFile f;
        if (!detail::read_mesh_file(file, f)) {
            eprint("Make_FromFile: File " + file.string() + " could not be opened or read.");
            return nullptr;
        }
        return Make(f.V.data(), static_cast<Int>(f.nV), static_cast<Int>(f.amb), false, f.S.data(),
                    static_cast<Int>(f.nS), static_cast<Int>(f.dom + 1), false, thread_count);
    }

    std::string ClassName() const
    {
        return "SimplicialMesh_Factory<" + std::to_string(MinDomDim_) + "," + std::to_string(MaxDomDim_) + "," +
               std::to_string(MinAmbDim_) + "," + std::to_string(MaxAmbDim_) + ">";
    }

private:
    std::unique_ptr<MeshBase_T> Error(Int dom_dim, Int amb_dim) const
    {
        eprint(ClassName() + " cannot create SimplicialMesh with domain dimension " + std::to_string(dom_dim) +
               " and ambient dimension " + std::to_string(amb_dim) + ".");
        return nullptr;
    }
};

// ---------------------------------------------------------------------------------------
// Energies
// ---------------------------------------------------------------------------------------

template <typename MeshBase_T>
class EnergyBase;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal>
class EnergyBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>> {
public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;
    using TangentVector_T = typename MeshBase_T::TangentVector_T;
    using CotangentVector_T = typename MeshBase_T::CotangentVector_T;

    virtual ~EnergyBase() = default;

    // Value of the energy, cached on the mesh (src/Energies/EnergyBase.hpp:40-56).
    ExtReal Value(const MeshBase_T& M) const
    {
        auto& c = M.GetCache(ClassName());
        if (!c.has_value) {
            double e = 0;
            if (!M.Handle() || !M.check(value(M, &e), ClassName() + "::Value")) return 0;
            c.value = e;
            c.has_value = true;
        }
        return c.value;
    }

    // Differential (n_v x AMB_DIM), cached on the mesh together with the value
    // (src/Energies/EnergyBase.hpp:62-88).
    const CotangentVector_T& Differential(const MeshBase_T& M) const
    {
        auto& c = M.GetCache(ClassName());
        if (!c.has_differential) {
            CotangentVector_T D(M.VertexCount(), M.AmbDim());
            double e = 0;
            if (M.Handle() && M.check(differential(M, 1.0, 0.0, D.data(), M.AmbDim(), &e), ClassName() + "::Differential")) {
                c.differential = std::move(D);
                c.has_differential = true;
                if (!c.has_value) {
                    c.value = e;
                    c.has_value = true;
                }
            }
        }
        return c.differential;
    }

    // Y = alpha * dE + beta * Y (leading dimension ldY); returns the energy; no caching.
    ExtReal Differential(const MeshBase_T& M, ExtReal alpha, ExtReal beta, ExtReal* Y, Int ldY) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        M.check(differential(M, alpha, beta, Y, ldY, &e), ClassName() + "::Differential");
        return e;
    }

    ExtReal Differential(const MeshBase_T& M, ExtReal* Y, bool addto = false) const
    {
        return Differential(M, ExtReal(1), ExtReal(addto ? 1 : 0), Y, M.AmbDim());
    }

    // Energy densities per simplex / per vertex (src/Energies/EnergyBase.hpp:129-150);
    // return the energy.
    ExtReal SimplexDensities(const MeshBase_T& M, ExtReal* density) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        M.check(densities(M, false, density, &e), ClassName() + "::SimplexDensities");
        return e;
    }

    ExtReal VertexDensities(const MeshBase_T& M, ExtReal* density) const
    {
        double e = 0;
        if (!M.Handle()) return 0;
        M.check(densities(M, true, density, &e), ClassName() + "::VertexDensities");
        return e;
    }

    virtual std::string ClassName() const = 0;

protected:
    virtual rpb_status value(const MeshBase_T& M, double* e) const = 0;
    virtual rpb_status differential(const MeshBase_T& M, double alpha, double beta, double* Y, Int ldY,
                                    double* e) const = 0;
    virtual rpb_status densities(const MeshBase_T& M, bool per_vertex, double* density, double* e) const = 0;
};

template <typename Mesh_T>
class TangentPointEnergy0;

template <int DOM_DIM, int AMB_DIM, typename Real, typename Int, typename LInt, typename SReal, typename ExtReal>
class TangentPointEnergy0<SimplicialMesh<DOM_DIM, AMB_DIM, Real, Int, LInt, SReal, ExtReal>>
    : public EnergyBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>> {
    using Base = EnergyBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>>;
    using MeshBase_T = typename Base::MeshBase_T;

public:
    TangentPointEnergy0(Real q_, Real p_) : q(q_), p(p_) {}
    explicit TangentPointEnergy0(Real p_) : q(p_), p(2 * p_) {}

    std::string ClassName() const override
    {
        return "TangentPointEnergy0<" + std::to_string(DOM_DIM) + "," + std::to_string(AMB_DIM) + ">(" +
               std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;

protected:
    rpb_status value(const MeshBase_T& M, double* e) const override { return rpb_tpe0_value(M.Handle(), q, p, e); }
    rpb_status differential(const MeshBase_T& M, double alpha, double beta, double* Y, Int ldY,
                            double* e) const override
    {
        return rpb_tpe0_differential(M.Handle(), q, p, alpha, beta, Y, static_cast<int>(ldY), e);
    }
    rpb_status densities(const MeshBase_T& M, bool per_vertex, double* density, double* e) const override
    {
        return per_vertex ? rpb_tpe0_vertex_densities(M.Handle(), q, p, density, e)
                          : rpb_tpe0_simplex_densities(M.Handle(), q, p, density, e);
    }
};

// TangentPointObstacleEnergy (src/Energies/TangentPointObstacleEnergy.hpp:48-96): the
// tangent-point energy of the mesh against its loaded obstacle; 0 without one.
template <typename Mesh_T>
class TangentPointObstacleEnergy;

template <int DOM_DIM, int AMB_DIM, typename Real, typename Int, typename LInt, typename SReal, typename ExtReal>
class TangentPointObstacleEnergy<SimplicialMesh<DOM_DIM, AMB_DIM, Real, Int, LInt, SReal, ExtReal>>
    : public EnergyBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>> {
    using Base = EnergyBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>>;
    using MeshBase_T = typename Base::MeshBase_T;

public:
    TangentPointObstacleEnergy(Real q_, Real p_) : q(q_), p(p_) {}

    std::string ClassName() const override
    {
        return "TangentPointObstacleEnergy<" + std::to_string(DOM_DIM) + "," + std::to_string(AMB_DIM) + ">(" +
               std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;

protected:
    rpb_status value(const MeshBase_T& M, double* e) const override { return rpb_tpoe_value(M.Handle(), q, p, e); }
    rpb_status differential(const MeshBase_T& M, double alpha, double beta, double* Y, Int ldY,
                            double* e) const override
    {
        return rpb_tpoe_differential(M.Handle(), q, p, alpha, beta, Y, static_cast<int>(ldY), e);
    }
    rpb_status densities(const MeshBase_T&, bool, double*, double*) const override
    {
        eprint(ClassName() + ": densities of the obstacle energy are not built.");
        return RPB_EINVAL;
    }
};

// ---------------------------------------------------------------------------------------
// Metrics
// ---------------------------------------------------------------------------------------

template <typename MeshBase_T>
class MetricBase;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal>
class MetricBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>> {
public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;
    using TangentVector_T = typename MeshBase_T::TangentVector_T;
    using CotangentVector_T = typename MeshBase_T::CotangentVector_T;
    using SolverVector_T = Tensor1<Real, Int>;

    virtual ~MetricBase() = default;

    // Y = alpha * A X + beta * Y (src/Metrics/MetricDimRestricted.hpp:109-139).
    virtual void MultiplyMetric(const MeshBase_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta,
                                ExtReal* Y, Int ldY, Int nrhs, bool VF_flag = true, bool NF_flag = true,
                                bool FF_flag = true) const = 0;

    void MultiplyMetric(const MeshBase_T& M, ExtReal alpha, const TangentVector_T& X, ExtReal beta,
                        CotangentVector_T& Y, bool VF_flag = true, bool NF_flag = true, bool FF_flag = true) const
    {
        this->MultiplyMetric(M, alpha, X.data(), X.Dim(1), beta, Y.data(), Y.Dim(1), X.Dim(1), VF_flag, NF_flag, FF_flag);
    }

    // Y = alpha * P X + beta * Y.
    virtual void MultiplyPreconditioner(const MeshBase_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta,
                                        ExtReal* Y, Int ldY, Int nrhs) const = 0;

    // X = alpha * A^{-1} B + beta * X.
    virtual void Solve(const MeshBase_T& M, ExtReal alpha, const ExtReal* B, Int ldB, ExtReal beta, ExtReal* X,
                       Int ldX, Int nrhs, Int max_iter, Real tolerance) const = 0;

    ExtReal MetricNorm(const MeshBase_T& M, const ExtReal* X, Int ldX, Int nrhs) const
    {
        return norm(M, X, ldX, nrhs, false);
    }

    ExtReal PreconditionerNorm(const MeshBase_T& M, const ExtReal* X, Int ldX, Int nrhs) const
    {
        return norm(M, X, ldX, nrhs, true);
    }

    Int Solver_IterationCount() const { return iter; }
    SolverVector_T Solver_RelativeResiduals() const { return rel_residuals; }

    virtual std::string ClassName() const = 0;

protected:
    mutable Int iter = 0;
    mutable SolverVector_T rel_residuals;

private:
    ExtReal norm(const MeshBase_T& M, const ExtReal* X, Int ldX, Int nrhs, bool precond) const
    {
        Tensor2<Real, Int> Xc(M.VertexCount(), nrhs), Y(M.VertexCount(), nrhs);
        Xc.Read(X, ldX);
        if (precond)
            MultiplyPreconditioner(M, 1, Xc.data(), nrhs, 0, Y.data(), nrhs, nrhs);
        else
            MultiplyMetric(M, 1, Xc.data(), nrhs, 0, Y.data(), nrhs, nrhs);
        double s = 0;
        for (Int k = 0; k < Y.Size(); ++k) s += Xc.data()[k] * Y.data()[k];
        return std::sqrt(s);
    }
};

template <typename Mesh_T>
class TangentPointMetric0;

template <int DOM_DIM, int AMB_DIM, typename Real, typename Int, typename LInt, typename SReal, typename ExtReal>
class TangentPointMetric0<SimplicialMesh<DOM_DIM, AMB_DIM, Real, Int, LInt, SReal, ExtReal>>
    : public MetricBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>> {
    using Base = MetricBase<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>>;
    using MeshBase_T = typename Base::MeshBase_T;

public:
    TangentPointMetric0(Real q_, Real p_) : q(q_), p(p_) {}
    explicit TangentPointMetric0(Real p_) : q(p_), p(2 * p_) {}

    using Base::MultiplyMetric;

    void MultiplyMetric(const MeshBase_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta, ExtReal* Y,
                        Int ldY, Int nrhs, bool VF_flag = true, bool NF_flag = true,
                        bool FF_flag = true) const override
    {
        if (!nrhs_ok(nrhs, "MultiplyMetric") || !M.Handle()) return;
        const int flags = (VF_flag ? 1 : 0) | (NF_flag ? 2 : 0) | (FF_flag ? 4 : 0);
        M.check(rpb_tpm0_multiply(M.Handle(), q, p, alpha, X, static_cast<int>(ldX), beta, Y, static_cast<int>(ldY),
                                  static_cast<int>(nrhs), flags),
                ClassName() + "::MultiplyMetric");
    }

    // Y = alpha * H1^{-1} L_{2-s} H1^{-1} X + beta * Y (src/Metrics/TangentPointMetric0.hpp:88-126).
    void MultiplyPreconditioner(const MeshBase_T& M, ExtReal alpha, const ExtReal* X, Int ldX, ExtReal beta,
                                ExtReal* Y, Int ldY, Int nrhs) const override
    {
        if (!nrhs_ok(nrhs, "MultiplyPreconditioner") || !M.Handle()) return;
        M.check(rpb_tpm0_precondition(M.Handle(), q, p, alpha, X, static_cast<int>(ldX), beta, Y,
                                      static_cast<int>(ldY), static_cast<int>(nrhs)),
                ClassName() + "::MultiplyPreconditioner");
    }

    // X = alpha * A^{-1} B + beta * X (src/Metrics/MetricDimRestricted.hpp:232-289).
    void Solve(const MeshBase_T& M, ExtReal alpha, const ExtReal* B, Int ldB, ExtReal beta, ExtReal* X, Int ldX,
               Int nrhs, Int max_iter, Real tolerance) const override
    {
        if (!nrhs_ok(nrhs, "Solve") || !M.Handle()) return;
        int it = 0;
        double rr[3] = {0, 0, 0};
        const rpb_status st = rpb_tpm0_solve(M.Handle(), q, p, alpha, B, static_cast<int>(ldB), beta, X,
                                             static_cast<int>(ldX), static_cast<int>(nrhs), static_cast<int>(max_iter),
                                             tolerance, precond, &it, rr);
        this->iter = it;
        this->rel_residuals = typename Base::SolverVector_T(rr, 3);
        if (st != RPB_ENOTCONV) M.check(st, ClassName() + "::Solve");
    }

    // B200 extra: the preconditioner Solve uses (RPB_PRECOND_REFERENCE by default).
    void SetPreconditioner(rpb_precond kind) { precond = kind; }

    std::string ClassName() const override
    {
        return "TangentPointMetric0<" + std::to_string(DOM_DIM) + "," + std::to_string(AMB_DIM) + ">(" +
               std::to_string(q) + "," + std::to_string(p) + ")";
    }

    Real q, p;

private:
    bool nrhs_ok(Int nrhs, const char* tag) const
    {
        if (nrhs == AMB_DIM) return true;
        eprint(ClassName() + "::" + tag + ": nrhs = " + std::to_string(nrhs) + " != " + std::to_string(AMB_DIM) +
               " = AMB_DIM");
        return false;
    }

    int precond = RPB_PRECOND_REFERENCE;
};

// ---------------------------------------------------------------------------------------
// Factories (runtime dispatch on the dimensions)
// ---------------------------------------------------------------------------------------

namespace detail {
template <template <class> class CLASS, typename Root, typename Real, typename Int, typename LInt, typename SReal,
          typename ExtReal>
std::unique_ptr<Root> make_dispatch(const std::string& who, int min_dom, int max_dom, int min_amb, int max_amb,
                                    Int dom_dim, Int amb_dim, Real q, Real p)
{
    if (dom_dim < min_dom || dom_dim > max_dom) {
        eprint(who + "::Make: dom_dim is out of range.");
    } else if (amb_dim < min_amb || amb_dim > max_amb) {
        eprint(who + "::Make: amb_dim is out of range.");
    } else if (amb_dim == 3 && dom_dim == 1) {
        return std::make_unique<CLASS<SimplicialMesh<1, 3, Real, Int, LInt, SReal, ExtReal>>>(q, p);
    } else if (amb_dim == 3 && dom_dim == 2) {
        return std::make_unique<CLASS<SimplicialMesh<2, 3, Real, Int, LInt, SReal, ExtReal>>>(q, p);
    }
    eprint(who + " cannot create an instance with domain dimension " + std::to_string(dom_dim) +
           " and ambient dimension " + std::to_string(amb_dim) + ".");
    return nullptr;
}
}  // namespace detail

template <class MeshBase_T, int... N>
class TangentPointEnergy0_Factory;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal, int MIN_DOM_DIM,
          int MAX_DOM_DIM, int MIN_AMB_DIM, int MAX_AMB_DIM>
class TangentPointEnergy0_Factory<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>, MIN_DOM_DIM, MAX_DOM_DIM,
                                  MIN_AMB_DIM, MAX_AMB_DIM> {
public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;
    [[nodiscard]] std::unique_ptr<EnergyBase<MeshBase_T>> Make(Int dom_dim, Int amb_dim, Real q, Real p) const
    {
        return detail::make_dispatch<TangentPointEnergy0, EnergyBase<MeshBase_T>, Real, Int, LInt, SReal, ExtReal>(
            "TangentPointEnergy0_Factory", MIN_DOM_DIM, MAX_DOM_DIM, MIN_AMB_DIM, MAX_AMB_DIM, dom_dim, amb_dim, q, p);
    }
};

template <class MeshBase_T, int... N>
class TangentPointMetric0_Factory;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal, int MIN_DOM_DIM,
          int MAX_DOM_DIM, int MIN_AMB_DIM, int MAX_AMB_DIM>
class TangentPointMetric0_Factory<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>, MIN_DOM_DIM, MAX_DOM_DIM,
                                  MIN_AMB_DIM, MAX_AMB_DIM> {
public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;
    [[nodiscard]] std::unique_ptr<MetricBase<MeshBase_T>> Make(Int dom_dim, Int amb_dim, Real q, Real p) const
    {
        return detail::make_dispatch<TangentPointMetric0, MetricBase<MeshBase_T>, Real, Int, LInt, SReal, ExtReal>(
            "TangentPointMetric0_Factory", MIN_DOM_DIM, MAX_DOM_DIM, MIN_AMB_DIM, MAX_AMB_DIM, dom_dim, amb_dim, q, p);
    }
};

template <class MeshBase_T, int... N>
class TangentPointObstacleEnergy_Factory;

template <typename Real, typename Int, typename LInt, typename SReal, typename ExtReal, int MIN_DOM_DIM_S,
          int MAX_DOM_DIM_S, int MIN_DOM_DIM_T, int MAX_DOM_DIM_T, int MIN_AMB_DIM, int MAX_AMB_DIM>
class TangentPointObstacleEnergy_Factory<SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>, MIN_DOM_DIM_S,
                                         MAX_DOM_DIM_S, MIN_DOM_DIM_T, MAX_DOM_DIM_T, MIN_AMB_DIM, MAX_AMB_DIM> {
public:
    using MeshBase_T = SimplicialMeshBase<Real, Int, LInt, SReal, ExtReal>;
    // The mesh (S) and the obstacle (T) must have the same domain dimension in this build.
    [[nodiscard]] std::unique_ptr<EnergyBase<MeshBase_T>> Make(Int dom_dim_S, Int dom_dim_T, Int amb_dim, Real q,
                                                               Real p) const
    {
        const std::string who = "TangentPointObstacleEnergy_Factory";
        if (dom_dim_T < MIN_DOM_DIM_T || dom_dim_T > MAX_DOM_DIM_T) {
            eprint(who + "::Make: dom_dim_T is out of range.");
            return nullptr;
        }
        if (dom_dim_S != dom_dim_T) {
            eprint(who + " cannot create an obstacle energy between domain dimensions " + std::to_string(dom_dim_S) +
                   " and " + std::to_string(dom_dim_T) + ".");
            return nullptr;
        }
        return detail::make_dispatch<TangentPointObstacleEnergy, EnergyBase<MeshBase_T>, Real, Int, LInt, SReal,
                                     ExtReal>(who, MIN_DOM_DIM_S, MAX_DOM_DIM_S, MIN_AMB_DIM, MAX_AMB_DIM, dom_dim_S,
                                              amb_dim, q, p);
    }
};

}  // namespace Repulsor_B200
