// Follows Repulsor's own example program (Example/main.cpp of HenrikSchumacher/Repulsor)
// call for call through the header-only mirror: base types SimplicialMeshBase /
// EnergyBase / MetricBase, the four factories, a mesh made from arrays in memory, energy,
// differential (cached, pointer, both at once), metric products with tensors, the
// gradient by Solve, MaximumSafeStepSize, SemiStaticUpdate, the energy of the moved mesh,
// an obstacle loaded from arrays and the obstacle energy and its differential.
//
// Usage: example_main MESH_FILE OBSTACLE_FILE [split_threshold [far_theta [obstacle_first]]]
// The files are in the reference's mesh text format (the example compiles its arrays in
// from Meshes/TwoSpheres.hpp; here they are read into arrays first). Prints one
// "name value" line per quantity for the comparison with the Python mirror.
//
// In the example's order the obstacle is loaded after the mesh has moved along the
// gradient by a step that did not know the obstacle; on TwoSpheres (0.0078 apart) the
// moved sphere then intersects the obstacle, and the obstacle energy of intersecting very
// near pairs is infinite: the library reports this as an error. With "obstacle_first"
// the obstacle is loaded right after the mesh, so that the step size accounts for it.
#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "repulsor_b200/Repulsor.hpp"

namespace Repulsor = Repulsor_B200;

using Int = int;
using LInt = std::size_t;
using Real = double;

namespace {

// progress on stderr, so that a run that stops early shows how far it came
void step(const char* what)
{
    std::fprintf(stderr, "step: %s\n", what);
    std::fflush(stderr);
}

struct Arrays {
    Int dom_dim = 0, amb_dim = 0, vertex_count = 0, simplex_count = 0;
    std::vector<Real> V;
    std::vector<Int> S;
};

bool read_arrays(const char* path, Arrays& a)
{
    Repulsor::detail::MeshFile f;
    if (!Repulsor::detail::read_mesh_file(path, f)) return false;
    a.dom_dim = static_cast<Int>(f.dom);
    a.amb_dim = static_cast<Int>(f.amb);
    a.vertex_count = static_cast<Int>(f.nV);
    a.simplex_count = static_cast<Int>(f.nS);
    a.V = f.V;
    a.S.assign(f.S.begin(), f.S.end());
    return true;
}

double max_abs(const double* x, std::size_t n)
{
    double m = 0;
    for (std::size_t k = 0; k < n; ++k) m = std::fmax(m, std::fabs(x[k]));
    return m;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 3) return 1;
    Arrays mesh, obstacle;
    if (!read_arrays(argv[1], mesh) || !read_arrays(argv[2], obstacle)) return 1;
    const int split_threshold = argc > 3 ? std::stoi(argv[3]) : 2;
    const double far_theta = argc > 4 ? std::stod(argv[4]) : 0.25;
    const bool obstacle_first = argc > 5 && std::string(argv[5]) == "obstacle_first";

    int thread_count = 1;

    using Mesh_T = Repulsor::SimplicialMeshBase<Real, Int, LInt>;
    Repulsor::SimplicialMesh_Factory<Mesh_T, 2, 2, 3, 3> mesh_factory;

    using Energy_T = Repulsor::EnergyBase<Mesh_T>;
    using Metric_T = Repulsor::MetricBase<Mesh_T>;

    Repulsor::TangentPointEnergy0_Factory<Mesh_T, 2, 2, 3, 3> TPE_factory;
    Repulsor::TangentPointMetric0_Factory<Mesh_T, 2, 2, 3, 3> TPM_factory;

    const Int dom_dim = mesh.dom_dim, amb_dim = mesh.amb_dim;

    std::unique_ptr<Mesh_T> M_ptr = mesh_factory.Make(mesh.V.data(), mesh.vertex_count, amb_dim, false, mesh.S.data(),
                                                      mesh.simplex_count, dom_dim + 1, false, thread_count);
    if (!M_ptr) return 2;
    auto& M = *M_ptr;

    M.cluster_tree_settings.split_threshold = split_threshold;
    M.block_cluster_tree_settings.far_field_separation_parameter = far_theta;
    M.adaptivity_settings.theta = 10.0;

    const Real q = 6;
    const Real p = 12;

    if (obstacle_first) {
        step("LoadObstacle");
        M.LoadObstacle(mesh_factory.Make(obstacle.V.data(), obstacle.vertex_count, amb_dim, false, obstacle.S.data(),
                                         obstacle.simplex_count, dom_dim + 1, false, thread_count));
    }

    std::unique_ptr<Energy_T> tpe_ptr = TPE_factory.Make(dom_dim, amb_dim, q, p);
    std::unique_ptr<Metric_T> tpm_ptr = TPM_factory.Make(dom_dim, amb_dim, q, p);
    if (!tpe_ptr || !tpm_ptr) return 3;

    const auto& tpe = *tpe_ptr;
    const auto& tpm = *tpm_ptr;

    step("Value");
    Real en = tpe.Value(M);
    std::printf("energy %.17g\n", en);

    Mesh_T::CotangentVector_T diff;
    step("Differential");
    diff = tpe.Differential(M);
    std::printf("differential_max %.17g\n", max_abs(diff.data(), static_cast<std::size_t>(diff.Size())));

    tpe.Differential(M, diff.data());
    en = tpe.Differential(M, diff.data());
    std::printf("energy_pointer %.17g\n", en);

    Mesh_T::TangentVector_T X(M.VertexCount(), M.AmbDim());
    Mesh_T::CotangentVector_T Y(M.VertexCount(), M.AmbDim());
    step("MultiplyMetric");
    X.Random();
    const Real alpha = 1.0;
    const Real beta = 0.0;
    tpm.MultiplyMetric(M, alpha, X, beta, Y);
    tpm.MultiplyMetric(M, alpha, X, beta, Y);
    tpm.MultiplyMetric(M, alpha, X, beta, Y);
    // <X, A X> >= 0 and A annihilates constants: report the Rayleigh quotient's sign only
    double xay = 0;
    for (Int k = 0; k < X.Size(); ++k) xay += X.data()[k] * Y.data()[k];
    std::printf("metric_xax_nonnegative %d\n", xay >= -1e-12 * std::fabs(xay) ? 1 : 0);

    const Int max_iter = 100;
    const Real relative_tolerance = 0.00001;
    step("Solve");
    Mesh_T::TangentVector_T gradient(M.VertexCount(), M.AmbDim());
    tpm.Solve(M, Real(1), diff.data(), M.AmbDim(), Real(0), gradient.data(), M.AmbDim(), M.AmbDim(), max_iter,
              relative_tolerance);
    std::printf("solve_iterations %d\n", static_cast<int>(tpm.Solver_IterationCount()));
    std::printf("solve_relative_residual_max %.6g\n", tpm.Solver_RelativeResiduals().Max());
    std::printf("gradient_max %.17g\n", max_abs(gradient.data(), static_cast<std::size_t>(gradient.Size())));

    Mesh_T::TangentVector_T downward_gradient = gradient;
    downward_gradient *= -1.;

    step("MaximumSafeStepSize");
    const Real t = M.MaximumSafeStepSize(downward_gradient.data(), 1.);
    std::printf("step_size %.17g\n", t);
    std::fflush(stdout);

    X = downward_gradient;
    X *= t;
    X += M.VertexCoordinates();
    step("SemiStaticUpdate");
    M.SemiStaticUpdate(X.data());

    Real en_new = tpe.Value(M);
    std::printf("energy_new %.17g\n", en_new);
    std::printf("energy_decreased %d\n", en_new < en ? 1 : 0);

    if (!obstacle_first) {
        step("LoadObstacle");
        M.LoadObstacle(mesh_factory.Make(obstacle.V.data(), obstacle.vertex_count, amb_dim, false, obstacle.S.data(),
                                         obstacle.simplex_count, dom_dim + 1, false, thread_count));
    }
    std::printf("obstacle_vertex_count %d\n", static_cast<int>(M.GetObstacle().VertexCount()));
    std::printf("obstacle_simplex_count %d\n", static_cast<int>(M.GetObstacle().SimplexCount()));

    Repulsor::TangentPointObstacleEnergy_Factory<Mesh_T, 2, 2, 2, 2, 3, 3> TPOE_factory;
    std::unique_ptr<Energy_T> tpo_ptr = TPOE_factory.Make(dom_dim, dom_dim, amb_dim, q, p);
    if (!tpo_ptr) return 4;
    const auto& tpo = *tpo_ptr;

    step("obstacle Value");
    en = tpo.Value(M);
    std::printf("obstacle_energy %.17g\n", en);
    step("obstacle Differential");
    diff = tpo.Differential(M);
    std::printf("obstacle_differential_max %.17g\n", max_abs(diff.data(), static_cast<std::size_t>(diff.Size())));
    step("done");
    return 0;
}
