// The reference's solver program (src/Solver.cpp:17-73) with its EulerSolver replaced by
// EulerSolverGPU: the reference's own config parser, mesh reader, connectivity, metrics, FlowField
// and WriteSolution around the GPU Run().  This is what a maintainer's main() becomes; it is built
// by `make -C oracle adapter` (which compiles the reference's front end from its sources) and run
// by tests/test_gpu_adapter.py, whose output files must equal the reference program's.
//
//   e3d_gpu_main <case.e3d> [exact|fp64] [solver_ms total_ms]
//
// With timings given, summary.txt is written with them instead of the measured ones (so that two
// runs can be compared byte for byte).
#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>

#include "EulerSolverGPU.hpp"
#include "mesh/Mesh.hpp"
#include "mesh/Metrics.hpp"
#include "parallelization/MPIHandler.hpp"
#include "parser/SimConfig.hpp"
#include "solver/FlowField.hpp"
#include "solver/WriteSolution.hpp"

int main(int argc, char *argv[]) {
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    E3D::Parallel::MPIHandler e3d_mpi(argc, argv);
    if (argc < 2) {
        std::cerr << "Usage : e3d_gpu_main <configFile.e3d> [exact|fp64] [solver_ms total_ms]" << std::endl;
        return 2;
    }
    const int precision = argc >= 3 && std::string(argv[2]) == "exact" ? E3D_PREC_FP64_EXACT : E3D_PREC_FP64;
    try {
        E3D::Parser::SimConfig config(argv[1], e3d_mpi.getRankID(), e3d_mpi.getPoolSize());
        E3D::Mesh<E3D::Parser::MeshPartition> mesh(config.getPartitionedMeshFiles()[e3d_mpi.getRankID()],
                                                   e3d_mpi.getRankID());
        mesh.solveConnectivity();
        e3d_mpi.updateRequesterID(mesh.getMPIelements());
        e3d_mpi.sortInterface();
        E3D::Metrics metrics(mesh, e3d_mpi.getRankID(), config);
        E3D::Solver::FlowField flow(config, mesh);
        E3D::Solver::EulerSolverGPU solver(flow, e3d_mpi, mesh, config, metrics, precision);
        const auto t1 = clock::now();
        solver.Run();
        const auto t2 = clock::now();
        E3D::Solver::WriteSolution writeSolution(flow, mesh, config, e3d_mpi);
        const auto t3 = clock::now();
        long solverMs = std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count();
        long totalMs = std::chrono::duration_cast<std::chrono::milliseconds>(t3 - t0).count();
        if (argc >= 5) {
            solverMs = std::atol(argv[3]);
            totalMs = std::atol(argv[4]);
        }
        solver.WriteSummary(solverMs, totalMs);
        std::cout << "iterations " << solver.stats().iterations << " device_ms " << solver.stats().device_ms << "\n";
    } catch (const std::exception &e) {
        std::cerr << "e3d_gpu_main: " << e.what() << std::endl;
        return 1;
    }
    e3d_mpi.finalize();
    return 0;
}
