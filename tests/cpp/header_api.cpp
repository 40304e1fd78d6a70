// Drives the header-only C++20 mirror (include/repulsor_b200/Repulsor.hpp) through its
// concrete classes: read a mesh file in the reference's text format (the factory's
// Make_FromFile), evaluate TangentPointEnergy0 Value/Differential/SimplexDensities,
// multiply the metric, solve, load an obstacle and evaluate TangentPointObstacleEnergy.
// Output: energy, |dE|_max, sum(A dE), iterations, the relative residual, the energy
// from the densities call and the obstacle energy, one per line.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include "repulsor_b200/Repulsor.hpp"

namespace Repulsor = Repulsor_B200;

template <int DOM>
int run(const Repulsor::SimplicialMeshBase<double, int, std::size_t>& file_mesh)
{
    using Mesh_T = Repulsor::SimplicialMesh<DOM, 3>;
    const int nV = file_mesh.VertexCount(), nS = file_mesh.SimplexCount();
    const std::vector<double> V(file_mesh.VertexCoordinates().data(), file_mesh.VertexCoordinates().data() + 3 * nV);
    const std::vector<int> S(file_mesh.Simplices().data(), file_mesh.Simplices().data() + (DOM + 1) * nS);
    Mesh_T M(V.data(), nV, S.data(), nS, 4);
    M.block_cluster_tree_settings.far_field_separation_parameter = 0.5;
    M.adaptivity_settings.theta = 10.0;
    Repulsor::TangentPointEnergy0<Mesh_T> tpe(6.0, 12.0);
    Repulsor::TangentPointMetric0<Mesh_T> tpm(6.0, 12.0);
    const double E = tpe.Value(M);
    const auto& Dt = tpe.Differential(M);
    if (Dt.Dim(0) != nV || Dt.Dim(1) != 3) return 2;
    const std::vector<double> D(Dt.data(), Dt.data() + Dt.Size());
    double dmax = 0;
    for (double d : D) dmax = std::fmax(dmax, std::fabs(d));
    std::vector<double> Y(3 * nV, 0.0), X(3 * nV, 0.0);
    tpm.MultiplyMetric(M, 1.0, D.data(), 3, 0.0, Y.data(), 3, 3);
    double ysum = 0;
    for (double y : Y) ysum += y;
    // right-hand side: the differential without its column means (the metric's kernel)
    std::vector<double> B(D);
    for (int k = 0; k < 3; ++k) {
        double m = 0;
        for (int v = 0; v < nV; ++v) m += B[3 * v + k];
        for (int v = 0; v < nV; ++v) B[3 * v + k] -= m / nV;
    }
    tpm.SetPreconditioner(RPB_PRECOND_NONE);
    tpm.Solve(M, 1.0, B.data(), 3, 0.0, X.data(), 3, 3, 20000, 1e-6);
    const auto rr = tpm.Solver_RelativeResiduals();
    const double rmax = rr.Max();
    std::vector<double> rho(nS);
    const double Ed = tpe.SimplexDensities(M, rho.data());
    // an obstacle: the mesh shifted by 3 along z, loaded into the mesh
    std::vector<double> VO(V);
    for (int v = 0; v < nV; ++v) VO[3 * v + 2] += 3.0;
    M.LoadObstacle(std::make_unique<Mesh_T>(VO.data(), nV, S.data(), nS, 4));
    Repulsor::TangentPointObstacleEnergy<Mesh_T> tpo(6.0, 12.0);
    const double Eo = tpo.Value(M);
    std::printf("%.17g\n%.17g\n%.17g\n%d\n%.6g\n%.17g\n%.17g\n", E, dmax, ysum,
                static_cast<int>(tpm.Solver_IterationCount()), rmax, Ed, Eo);
    // errors follow the reference: print and do nothing
    tpm.MultiplyMetric(M, 1.0, D.data(), 3, 0.0, Y.data(), 3, 2);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 1;
    using MeshBase_T = Repulsor::SimplicialMeshBase<double, int, std::size_t>;
    Repulsor::SimplicialMesh_Factory<MeshBase_T, 1, 2, 3, 3> factory;
    std::unique_ptr<MeshBase_T> M = factory.Make_FromFile(argv[1], 4);
    if (!M) return 1;
    return M->DomDim() == 1 ? run<1>(*M) : run<2>(*M);
}
