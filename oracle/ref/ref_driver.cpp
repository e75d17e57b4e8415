/*
 * Checker driver around the UNMODIFIED Euler3D reference solver sources.
 *
 * Test infrastructure only (built by oracle/Makefile into oracle/_ref/, never
 * linked into the product).  It mirrors the reference executable's main
 * (src/Solver.cpp:19-73): parse the .e3d config, read the partition file,
 * solve connectivity, compute metrics, initialise the flow field and build
 * EulerSolver; it then drives the reference's own member functions and dumps
 * their results as raw little-endian arrays so that the tests can compare the
 * CUDA path with the reference bit for bit or to a stated tolerance.
 *
 * Modes
 *   mesh    <cfg> <out>            connectivity, metrics and ghost lists
 *   run     <cfg> <out>            EulerSolver::Run() exactly as main() calls it
 *   history <cfg> <out> <iters>    one Run() iteration at a time, recording the
 *                                  density RMS at full precision each iteration
 *   stage   <cfg> <out> [state]    one iteration body step by step (updateBC,
 *                                  computeResidual, updateDeltaTime, RungeKutta)
 *                                  from the freestream or a given state
 *   bench   <cfg> <warm> <iters>   time Run() over <iters> iterations
 *   outputs <cfg> <out> <solver_ms> <total_ms>   Run(), WriteSummary and WriteSolution: the
 *                                  reference's own output files
 *
 * Private members are reached through the access-specifier macro below only
 * to READ the solver's residual / time-step vectors, to reset its iteration
 * counter and to call its private steps in the order Run() calls them.
 */
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <regex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "mesh/Mesh.hpp"
#include "mesh/Metrics.hpp"
#include "parallelization/MPIHandler.hpp"
#include "parser/SimConfig.hpp"
#include "solver/EulerSolver.hpp"
#include "solver/FlowField.hpp"
#include "solver/WriteSolution.hpp"
#undef private
#undef protected

using namespace E3D;

namespace {

std::string g_out;

template<typename T>
void dump(const std::string &name, const T *p, size_t n) {
	std::string path = g_out + "/" + name;
	FILE *f = std::fopen(path.c_str(), "wb");
	if (!f) {
		std::fprintf(stderr, "cannot write %s\n", path.c_str());
		std::exit(2);
	}
	if (n) std::fwrite(p, sizeof(T), n, f);
	std::fclose(f);
}

template<typename T>
void dumpv(const std::string &name, const std::vector<T> &v) { dump(name, v.data(), v.size()); }

void dumpVec3(const std::string &name, const std::vector<Vector3<double>> &v) {
	std::vector<double> flat(3 * v.size());
	for (size_t i = 0; i < v.size(); i++) {
		flat[3 * i] = v[i].x;
		flat[3 * i + 1] = v[i].y;
		flat[3 * i + 2] = v[i].z;
	}
	dumpv(name, flat);
}

void dumpState(Solver::FlowField &ff, const std::string &prefix) {
	dumpv(prefix + "rho.f64", ff.Getrho());
	dumpv(prefix + "u.f64", ff.GetU_Velocity());
	dumpv(prefix + "v.f64", ff.GetV_Velocity());
	dumpv(prefix + "w.f64", ff.GetW_Velocity());
	dumpv(prefix + "p.f64", ff.GetP());
	dumpv(prefix + "E.f64", ff.GetE());
	dumpv(prefix + "H.f64", ff.GetH());
	dumpv(prefix + "M.f64", ff.GetMach());
}

void loadState(Solver::FlowField &ff, const std::string &path) {
	size_t n = ff.Getrho().size();
	std::vector<double> buf(8 * n);
	FILE *f = std::fopen(path.c_str(), "rb");
	if (!f || std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) {
		std::fprintf(stderr, "cannot read %zu doubles from %s\n", buf.size(), path.c_str());
		std::exit(2);
	}
	std::fclose(f);
	for (size_t i = 0; i < n; i++) {
		ff.setRho((int) i, buf[0 * n + i]);
		ff.setU((int) i, buf[1 * n + i]);
		ff.setV((int) i, buf[2 * n + i]);
		ff.setW((int) i, buf[3 * n + i]);
		ff.setP((int) i, buf[4 * n + i]);
		ff.setE((int) i, buf[5 * n + i]);
		ff.setH((int) i, buf[6 * n + i]);
		ff.setM((int) i, buf[7 * n + i]);
	}
}

void dumpResiduals(const std::vector<Solver::ResidualVar> &r, const std::string &name) {
	std::vector<double> flat(5 * r.size());
	for (size_t i = 0; i < r.size(); i++) {
		flat[5 * i + 0] = r[i].m_rhoV_residual;
		flat[5 * i + 1] = r[i].m_rho_uV_residual;
		flat[5 * i + 2] = r[i].m_rho_vV_residual;
		flat[5 * i + 3] = r[i].m_rho_wV_residual;
		flat[5 * i + 4] = r[i].m_rho_HV_residual;
	}
	dumpv(name, flat);
}

void writeText(const std::string &name, const std::string &text) {
	std::ofstream f(g_out + "/" + name);
	f << text;
}

std::string fmt17(double x) {
	char b[64];
	std::snprintf(b, sizeof b, "%.17g", x);
	return b;
}

}// namespace

int main(int argc, char **argv) {
	if (argc < 4) {
		std::fprintf(stderr, "usage: %s mesh|run|history|stage|bench <config.e3d> <outdir|warm> [arg]\n", argv[0]);
		return 2;
	}
	std::string mode = argv[1];
	std::string cfgPath = argv[2];
	if (mode != "bench") {
		g_out = argv[3];
		std::filesystem::create_directories(g_out);
	}

	int fakeArgc = 1;
	char name[] = "e3d_ref_driver";
	char *fakeArgvData[] = {name, nullptr};
	char **fakeArgv = fakeArgvData;
	Parallel::MPIHandler e3d_mpi(fakeArgc, fakeArgv);

	auto t0 = std::chrono::steady_clock::now();
	Parser::SimConfig config(cfgPath, e3d_mpi.getRankID(), e3d_mpi.getPoolSize());
	Mesh<Parser::MeshPartition> localmesh(config.getPartitionedMeshFiles()[e3d_mpi.getRankID()], e3d_mpi.getRankID());
	localmesh.solveConnectivity();
	e3d_mpi.updateRequesterID(localmesh.getMPIelements());
	e3d_mpi.sortInterface();
	Metrics metrics(localmesh, e3d_mpi.getRankID(), config);
	Solver::FlowField flow(config, localmesh);
	auto t1 = std::chrono::steady_clock::now();
	double setupSeconds = std::chrono::duration<double>(t1 - t0).count();

	if (mode == "mesh") {
		int nElem = localmesh.GetnElemTot();
		int nFace = localmesh.GetnFace();
		std::vector<int> f2e(localmesh.face2element->begin(), localmesh.face2element->end());
		dumpv("face2elem.i32", f2e);
		dumpv("elem2face_ptr.i32", *localmesh.element2faceStart);
		dumpv("elem2face.i32", *localmesh.element2face);
		dumpv("elem2elem.i32", *localmesh.element2element);
		dumpv("face2node_ptr.i32", *localmesh.face2nodeStart);
		dumpv("face2node.i32", *localmesh.face2node);
		dumpVec3("face_normal.f64", metrics.getFaceNormals());
		dumpVec3("face_unit_normal.f64", metrics.getFaceNormalsUnit());
		dumpVec3("face_center.f64", metrics.getFaceCenters());
		dumpv("face_area.f64", metrics.getFaceSurfaces());
		dumpv("cell_volume.f64", metrics.getCellVolumes());
		dumpVec3("cell_centroid.f64", metrics.getCellCentroids());
		dumpv("wall_ghost.i32", localmesh.GetWallGhostCellsIDs());
		dumpv("wall_interior.i32", localmesh.GetWallAdjacentGhostCellIDs());
		dumpv("wall_face.i32", localmesh.GetWallAdjacentFaceIDs());
		dumpv("farfield_ghost.i32", localmesh.GetFarfieldGhostCellsIDs());
		dumpv("farfield_interior.i32", localmesh.GetFarfieldAdjacentToGhostCellsIDs());
		dumpv("farfield_face.i32", localmesh.GetFarfieldAdjacentFaceIDs());
		dumpv("sym_ghost.i32", localmesh.GetSymmetryGhostCellsIDs());
		dumpv("sym_interior.i32", localmesh.GetSymmetryAdjacentGhostCellIDs());
		dumpv("sym_face.i32", localmesh.GetSymmetryAdjacentFaceIDs());
		std::ostringstream meta;
		meta << "n_elem " << nElem << "\nn_face " << nFace << "\nn_face_int " << localmesh.GetnFaceInt()
		     << "\nn_total " << flow.getTotalElemsCount() << "\nn_domain " << flow.getTotalDomainCounts()
		     << "\nsetup_s " << setupSeconds << "\n";
		writeText("meta.txt", meta.str());
		return 0;
	}

	Solver::EulerSolver solver(flow, e3d_mpi, localmesh, config, metrics);

	if (mode == "run") {
		auto a = std::chrono::steady_clock::now();
		solver.Run();
		auto b = std::chrono::steady_clock::now();
		dumpState(flow, "");
		std::ostringstream meta;
		meta << "iterations " << solver._nbInteration << "\nrun_s " << std::chrono::duration<double>(b - a).count()
		     << "\nsetup_s " << setupSeconds << "\nCL " << fmt17(solver._CL) << "\nCD " << fmt17(solver._CD)
		     << "\nCM " << fmt17(solver._CM) << "\nforce " << fmt17(solver._forceCoefficients.x) << " "
		     << fmt17(solver._forceCoefficients.y) << " " << fmt17(solver._forceCoefficients.z) << "\nmoment "
		     << fmt17(solver._momentCoefficients.x) << " " << fmt17(solver._momentCoefficients.y) << " "
		     << fmt17(solver._momentCoefficients.z) << "\n";
		writeText("meta.txt", meta.str());
		return 0;
	}

	if (mode == "outputs") {
		// the files a run writes (src/Solver.cpp:58-67): residuals.dat during Run(), then
		// WriteSummary (summary.txt, cp_part_0.dat) with the given timings, then WriteSolution
		// (<partition>.sol, <partition>.bry)
		if (argc < 6) return 2;
		solver.Run();
		solver.WriteSummary(std::atol(argv[4]), std::atol(argv[5]));
		Solver::WriteSolution ws(flow, localmesh, config, e3d_mpi);
		return 0;
	}

	if (mode == "history") {
		if (argc < 5) return 2;
		int iters = std::atoi(argv[4]);
		const_cast<Parser::SimConfig &>(config)._maxIter = 1;
		std::vector<double> rms;
		for (int it = 0; it < iters; it++) {
			solver._nbInteration = 0;
			solver.Run();
			double sum = solver.computeRMS();
			rms.push_back(std::sqrt(sum / flow.getTotalDomainCounts()));
		}
		dumpv("rms.f64", rms);
		dumpState(flow, "");
		return 0;
	}

	if (mode == "stage") {
		if (argc >= 5) loadState(flow, argv[4]);
		// Run()'s prologue (src/solver/EulerSolver.cpp:65-78), then one loop body.
		solver.sortGhostCells();
		solver._residuals.resize(localmesh.GetnElemTot(), Solver::ResidualVar(0.0, 0.0, 0.0, 0.0, 0.0));
		solver._deltaT.resize(localmesh.GetnElemTot(), 0);
		solver.resetResiduals();
		solver.updateBC();
		dumpState(flow, "bc_");
		solver.computeResidual();
		dumpResiduals(solver._residuals, "residual.f64");
		solver.updateDeltaTime();
		dumpv("dt.f64", solver._deltaT);
		solver.RungeKutta();
		dumpResiduals(solver._residuals, "residual_stage5.f64");
		double sum = solver.computeRMS();
		std::vector<double> rms{std::sqrt(sum / flow.getTotalDomainCounts())};
		dumpv("rms.f64", rms);
		dumpState(flow, "rk_");
		return 0;
	}

	if (mode == "bench") {
		int warm = std::atoi(argv[3]);
		int iters = argc >= 5 ? std::atoi(argv[4]) : 1;
		auto &cfg = const_cast<Parser::SimConfig &>(config);
		cfg._minResidual = 0.0;
		cfg._minAeroCoeffError = 0.0;
		double warmSeconds = 0.0;
		if (warm > 0) {
			cfg._maxIter = warm;
			auto a = std::chrono::steady_clock::now();
			solver.Run();
			warmSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
		}
		cfg._maxIter = iters;
		solver._nbInteration = 0;
		auto a = std::chrono::steady_clock::now();
		solver.Run();
		double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
		std::fflush(stdout);
		std::cout << std::flush;
		std::printf("\n{\"cells\": %d, \"iterations\": %d, \"seconds\": %.9g, \"warm_seconds\": %.9g, \"setup_seconds\": %.6g}\n",
		            localmesh.GetnElemTot(), solver._nbInteration, s, warmSeconds, setupSeconds);
		return 0;
	}
	std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
	return 2;
}
