// EulerSolverGPU: drop-in for the reference's E3D::Solver::EulerSolver (include/solver/EulerSolver.hpp:89-223)
// that runs the solver loop on one B200 through the euler3d_b200 C ABI.
//
// Same constructor arguments and the same Run() / WriteSummary() calls as the reference class, so the
// reference's main (src/Solver.cpp:56-69) only changes the type name.  The constructor reads what
// EulerSolver reads from Mesh, Metrics, SimConfig and FlowField (the ghost-cell lists, face2element,
// element2face, normals, areas, centres, volumes, flow settings); Run() uploads the FlowField, runs
// e3d_solver_run and writes every FlowField array back through its setters, so WriteSolution and the
// reference's output code run unchanged.
//
// Header-only; compile it together with the reference headers and link libeuler3d_b200.so.
#pragma once

#include <array>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "euler3d_b200.h"
#include "mesh/Mesh.hpp"
#include "mesh/Metrics.hpp"
#include "parallelization/MPIHandler.hpp"
#include "parser/SimConfig.hpp"
#include "solver/FlowField.hpp"

namespace E3D::Solver {

class EulerSolverGPU {
public:
    EulerSolverGPU(FlowField &flow, const E3D::Parallel::MPIHandler &mpi, const E3D::Mesh<E3D::Parser::MeshPartition> &mesh,
                   const E3D::Parser::SimConfig &config, const E3D::Metrics &metrics, int precision = E3D_PREC_FP64,
                   bool useConfigScheme = false)
        : _flow(flow), _mpi(mpi), _mesh(mesh), _config(config) {
        if (mpi.getPoolSize() != 1) throw std::runtime_error("EulerSolverGPU runs one whole mesh per GPU (one partition)");
        const int nCells = mesh.GetnElemTot(), nFaces = mesh.GetnFace();
        // element -> face CSR from the public per-element getter
        _c2fPtr.resize(nCells + 1, 0);
        for (int e = 0; e < nCells; e++) {
            int n = 0;
            const int *f = mesh.GetElement2FaceID(e, n);
            _c2fPtr[e + 1] = _c2fPtr[e] + n;
            _c2f.insert(_c2f.end(), f, f + n);
        }
        e3d_mesh_desc d{};
        d.n_cells = nCells;
        d.n_faces = nFaces;
        d.n_faces_int = mesh.GetnFaceInt();
        d.face2cell = mesh.GetFace2ElementID(0);  // the face2element vector is contiguous
        // Vector3<double> is three packed doubles, so the metric vectors are x,y,z arrays
        d.face_unit_normal = &metrics.getFaceNormalsUnit()[0].x;
        d.face_normal = &metrics.getFaceNormals()[0].x;
        d.face_area = metrics.getFaceSurfaces().data();
        d.face_center = &metrics.getFaceCenters()[0].x;
        d.cell_volume = metrics.getCellVolumes().data();
        d.cell2face_ptr = _c2fPtr.data();
        d.cell2face = _c2f.data();
        d.n_wall = (int32_t)mesh.GetWallGhostCellsIDs().size();
        d.wall_ghost = mesh.GetWallGhostCellsIDs().data();
        d.wall_interior = mesh.GetWallAdjacentGhostCellIDs().data();
        d.wall_face = mesh.GetWallAdjacentFaceIDs().data();
        d.n_farfield = (int32_t)mesh.GetFarfieldGhostCellsIDs().size();
        d.farfield_ghost = mesh.GetFarfieldGhostCellsIDs().data();
        d.farfield_interior = mesh.GetFarfieldAdjacentToGhostCellsIDs().data();
        d.farfield_face = mesh.GetFarfieldAdjacentFaceIDs().data();
        d.n_sym = (int32_t)mesh.GetSymmetryGhostCellsIDs().size();
        d.sym_ghost = mesh.GetSymmetryGhostCellsIDs().data();
        d.sym_interior = mesh.GetSymmetryAdjacentGhostCellIDs().data();
        d.sym_face = mesh.GetSymmetryAdjacentFaceIDs().data();

        e3d_flow_params p{};
        p.gamma = config.getGamma();
        p.mach = flow.getM_inf();
        p.aoa_deg = config.getAoA();
        p.cfl = config.getCFL();
        p.sref = config.getSref();
        p.cref = config.getCref();
        E3D::Vector3<double> ref = config.getMeshRefPoint();
        p.ref_point[0] = ref.x;
        p.ref_point[1] = ref.y;
        p.ref_point[2] = ref.z;
        p.cl_axis = config.getMeshOrientationCL().first;
        p.cl_sign = config.getMeshOrientationCL().second;
        p.cd_axis = config.getMeshOrientationCD().first;
        p.cd_sign = config.getMeshOrientationCD().second;
        p.cm_axis = config.getMeshOrientationCM().first;
        p.cm_sign = config.getMeshOrientationCM().second;
        // The reference parses SCHEME= but never reads it: it always runs Roe (Solver::AUSM is declared,
        // include/solver/ConvectiveFluxesSchemes.h:27-30, and never defined or called).  The same by
        // default; useConfigScheme runs AUSM for SCHEME= 1.
        p.scheme = useConfigScheme && config.getSolverScheme() == E3D::Parser::SimConfig::SolverScheme::AUSM
                       ? E3D_SCHEME_AUSM
                       : E3D_SCHEME_ROE;
        p.precision = precision;
        p.ordering = E3D_ORDER_SPATIAL;
        // TIME_INTEGRATION= (EulerSolver's constructor, src/solver/EulerSolver.cpp:49-56); the
        // implicit scheme is a stub there that never updates the state
        switch (config.getTemporalScheme()) {
            case E3D::Parser::SimConfig::TemporalScheme::RK5: p.integrator = E3D_INTEGRATOR_RK5; break;
            case E3D::Parser::SimConfig::TemporalScheme::EXPLICIT_EULER: p.integrator = E3D_INTEGRATOR_EULER; break;
            default: throw std::runtime_error("TIME_INTEGRATION= 1 (implicit Euler) is not supported on the GPU");
        }
        p.residual_smoothing = config.getResidualSmoothing() ? 1 : 0;
        check(e3d_solver_create(&d, &p, &_solver), "e3d_solver_create");
        if ((size_t)e3d_solver_state_size(_solver) != flow.Getrho().size())
            throw std::runtime_error("every boundary face needs a wall, farfield or sym marker");
    }

    ~EulerSolverGPU() { e3d_solver_destroy(_solver); }
    EulerSolverGPU(const EulerSolverGPU &) = delete;
    EulerSolverGPU &operator=(const EulerSolverGPU &) = delete;

    // EulerSolver::Run (src/solver/EulerSolver.cpp:60-167) on the GPU.
    void Run() {
        const size_t n = _flow.Getrho().size();
        std::array<std::vector<double>, 8> st;
        st[0] = _flow.Getrho();
        st[1] = _flow.GetU_Velocity();
        st[2] = _flow.GetV_Velocity();
        st[3] = _flow.GetW_Velocity();
        st[4] = _flow.GetP();
        st[5] = _flow.GetE();
        st[6] = _flow.GetH();
        st[7] = _flow.GetMach();
        const double *in[8];
        for (int k = 0; k < 8; k++) in[k] = st[k].data();
        check(e3d_solver_set_state(_solver, in), "e3d_solver_set_state");
        e3d_run_params rp{};
        rp.max_iter = _config.getMaxNumberIterations();
        rp.sampling = _config.getSamplingPeriod();
        rp.min_residual = _config.getMinResidual();
        rp.min_aerocoeff_error = _config.getMinAeroCoeffError();
        check(e3d_solver_run(_solver, &rp, &_stats), "e3d_solver_run");
        double *out[8];
        for (int k = 0; k < 8; k++) out[k] = st[k].data();
        check(e3d_solver_get_state(_solver, out), "e3d_solver_get_state");
        for (size_t i = 0; i < n; i++) {
            _flow.setRho((int)i, st[0][i]);
            _flow.setU((int)i, st[1][i]);
            _flow.setV((int)i, st[2][i]);
            _flow.setW((int)i, st[3][i]);
            _flow.setP((int)i, st[4][i]);
            _flow.setE((int)i, st[5][i]);
            _flow.setH((int)i, st[6][i]);
            _flow.setM((int)i, st[7][i]);
        }
        std::vector<double> hist(_stats.n_rms);
        int32_t cnt = 0;
        check(e3d_solver_rms_history(_solver, hist.data(), (int32_t)hist.size(), &cnt), "e3d_solver_rms_history");
        _rms = hist;
        // residuals.dat, which the reference writes row by row during Run() (ResidualsFile,
        // include/solver/ResidualsFile.hpp:18-48): the same rows, written once the run is over
        if (_mpi.getRankID() == 0)
            check(e3d_solver_write_residuals(_solver, (_config.GetoutputDir() / "residuals.dat").c_str()),
                  "e3d_solver_write_residuals");
    }

    // EulerSolver::WriteSummary (src/solver/EulerSolver.cpp:169-198): cp_part_N.dat and summary.txt,
    // byte for byte as the reference writes them.  The .sol/.bry files come from the reference's own
    // WriteSolution on the FlowField that Run() filled.
    void WriteSummary(long solverTimer, long totalTimer) {
        const std::string cp = "cp_part_" + std::to_string(_mpi.getRankID()) + ".dat";
        check(e3d_solver_write_cp(_solver, (_config.GetoutputDir() / cp).c_str()), "e3d_solver_write_cp");
        if (_mpi.getRankID() == 0)
            check(e3d_solver_write_summary(_solver, (_config.GetoutputDir() / "summary.txt").c_str(), solverTimer,
                                           totalTimer, _mpi.getPoolSize()),
                  "e3d_solver_write_summary");
    }

    const e3d_run_stats &stats() const { return _stats; }
    const std::vector<double> &rmsHistory() const { return _rms; }

private:
    static void check(e3d_status s, const char *what) {
        if (s != E3D_OK) throw std::runtime_error(std::string(what) + ": " + e3d_last_error());
    }
    FlowField &_flow;
    const E3D::Parallel::MPIHandler &_mpi;
    const E3D::Mesh<E3D::Parser::MeshPartition> &_mesh;
    const E3D::Parser::SimConfig &_config;
    std::vector<int32_t> _c2fPtr, _c2f;
    e3d_solver *_solver = nullptr;
    e3d_run_stats _stats{};
    std::vector<double> _rms;
};

}  // namespace E3D::Solver
