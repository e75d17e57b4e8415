/*
 * Timing driver for the UNMODIFIED Euler3D reference solver on N host cores through its own
 * multi-rank path (test infrastructure: the CPU baseline beside the GPU numbers; built by
 * oracle/Makefile `ref-fast` with the reference's Release flags and the shared-memory MPI of this
 * directory, never linked into the product).
 *
 *   E3D_MPI_RANKS=N e3d_ref_mpi <config.e3d> <warm-up iterations> <timed iterations> [fast]
 *
 * It follows the reference solver program (src/Solver.cpp:19-73): every rank parses its .par
 * partition file, solves the connectivity, sets up the MPI interfaces, computes the metrics,
 * initialises the flow field and builds EulerSolver; then EulerSolver::Run() runs the warm-up
 * iterations and, after a barrier, the timed ones.  Rank 0 prints one line
 *   E3D_REF_MPI {"ranks": N, "cells": ..., "iterations": ..., "seconds": <slowest rank>, ...}
 * With E3D_REF_DUMP=<dir>, every rank also writes its final flow state to <dir>/state_<rank>.f64.
 *
 * With `fast`, the face search of Connectivity::SolveElement2Element and the boundary-list search
 * of Mesh::updateWall/Farfield/SymmetryGhostCell -- O(elements x nodes) and O(boundary faces^2),
 * hours on the 12.6M-cell mesh -- are replaced by the euler3d_b200 library's mesh preparation
 * (e3d_mesh_from_arrays) run on the same parsed elements and markers; its arrays are the
 * reference's own numbering bit for bit (tests/test_mesh_prep.py).  Everything else, and all that
 * is timed, is the reference's code: the parser, Connectivity's node lists, updateMPIGhostCells,
 * MPIHandler, Metrics, FlowField and EulerSolver::Run with its halo exchange and Allreduce.
 */
// every standard header the reference's headers use comes first: the access-specifier macro below
// is for the reference's classes only
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
#undef private
#undef protected

#include "euler3d_b200.h"

using namespace E3D;

namespace {

std::vector<int> int_array(const e3d_mesh *pm, const char *name) {
	const void *data = nullptr;
	int64_t n = 0;
	int32_t is_double = 0;
	if (e3d_mesh_array(pm, name, &data, &n, &is_double) != E3D_OK || is_double) {
		std::fprintf(stderr, "e3d_mesh_array(%s): %s\n", name, e3d_last_error());
		std::exit(2);
	}
	const int32_t *p = static_cast<const int32_t *>(data);
	return std::vector<int>(p, p + n);
}

// Mesh<MeshPartition>::solveConnectivity (include/mesh/Mesh.hpp:36-105) with its two searches done
// by the euler3d_b200 mesh preparation on the same parsed input.
void fast_connectivity(Mesh<Parser::MeshPartition> &m) {
	auto &c = m.connectivityObj;
	c._nNode = m.GetMeshNodeCount();
	c.SolveElement2node(m.GetInteriorElementVector());
	c.ComputeVTKLinkedLists(m.GetInteriorVTKID());
	c.SolveNode2element();

	const auto &nodes = m.GetNodeVector();
	std::vector<double> xyz(3 * nodes.size());
	for (size_t i = 0; i < nodes.size(); i++) {
		xyz[3 * i] = nodes[i].getX();
		xyz[3 * i + 1] = nodes[i].getY();
		xyz[3 * i + 2] = nodes[i].getZ();
	}
	std::vector<int32_t> vtk(m.GetInteriorVTKID().begin(), m.GetInteriorVTKID().end());
	std::vector<int32_t> eptr(c._element2nodeStart.begin(), c._element2nodeStart.end());
	std::vector<int32_t> enodes(c._element2node.begin(), c._element2node.end());
	std::vector<std::string> tags;
	std::vector<int32_t> mptr{0}, fptr{0}, fnodes;
	for (const auto &[tag, elems] : m.GetBoundaryConditionVector()) {
		tags.push_back(tag);
		for (const auto &e : elems) {
			for (int nd : e.getElemNodes()) fnodes.push_back(nd);
			fptr.push_back((int32_t) fnodes.size());
		}
		mptr.push_back((int32_t) (fptr.size() - 1));
	}
	std::vector<const char *> tagp;
	for (const auto &t : tags) tagp.push_back(t.c_str());
	e3d_mesh *pm = nullptr;
	if (e3d_mesh_from_arrays((int32_t) nodes.size(), xyz.data(), (int32_t) vtk.size(), vtk.data(), eptr.data(),
	                         enodes.data(), (int32_t) tags.size(), tagp.data(), mptr.data(), fptr.data(), fnodes.data(),
	                         1.0, 1, &pm) != E3D_OK) {
		std::fprintf(stderr, "e3d_mesh_from_arrays: %s\n", e3d_last_error());
		std::exit(2);
	}
	e3d_mesh_info info{};
	e3d_mesh_info_get(pm, &info);
	c._nFace = info.n_faces;
	c._nFaceInt = info.n_faces_int;
	c._element2faceStart = int_array(pm, "cell2face_ptr");
	c._element2elementStart = c._element2faceStart;
	c._element2face = int_array(pm, "cell2face");
	c._element2element = int_array(pm, "cell2cell");
	c._face2element = int_array(pm, "face2cell");
	c._face2nodeStart = int_array(pm, "face2node_ptr");
	c._face2node = int_array(pm, "face2node");

	// the rest of solveConnectivity, as the reference does it
	m.node2element = std::make_unique<std::vector<int>>(c._node2element);
	m.node2elementStart = std::make_unique<std::vector<int>>(c._node2elementStart);
	m.element2element = std::make_unique<std::vector<int>>(c._element2element);
	m.element2elementStart = std::make_unique<std::vector<int>>(c._element2elementStart);
	m.element2face = std::make_unique<std::vector<int>>(c._element2face);
	m.element2faceStart = std::make_unique<std::vector<int>>(c._element2faceStart);
	m.face2element = std::make_unique<std::vector<int>>(c._face2element);
	m.face2node = std::make_unique<std::vector<int>>(c._face2node);
	m.face2nodeStart = std::make_unique<std::vector<int>>(c._face2nodeStart);
	m.updateMPIGhostCells();
	m.WallGhostCellIDs = int_array(pm, "wall_ghost");
	m.WallAdjacentToGhostCellIDs = int_array(pm, "wall_interior");
	m.WallAdjacentFaceIDs = int_array(pm, "wall_face");
	m.FarfieldGhostCellIDs = int_array(pm, "farfield_ghost");
	m.FarfieldAdjacentToGhostCellIDs = int_array(pm, "farfield_interior");
	m.FarfieldAdjacentFaceIDs = int_array(pm, "farfield_face");
	m.SymmetryGhostCellIDs = int_array(pm, "sym_ghost");
	m.SymmetryAdjacentGhostCellIDs = int_array(pm, "sym_interior");
	m.SymmetryAdjacentFaceIDs = int_array(pm, "sym_face");
	e3d_mesh_destroy(pm);
	// the collectives solveConnectivity ends with (Mesh.hpp:90-92), so every rank keeps the same sequence
	std::array<int, 4> stats{(int) m.FarfieldGhostCellIDs.size(), (int) m.WallGhostCellIDs.size(),
	                         (int) m.SymmetryGhostCellIDs.size(), m.GetMpiElemsCount()};
	std::array<int, 4> sum{0, 0, 0, 0};
	MPI_Reduce(&stats, &sum, 4, MPI_INT, MPI_SUM, 0, MPI_COMM_WORLD);
	MPI_Barrier(MPI_COMM_WORLD);
}

double seconds_since(std::chrono::steady_clock::time_point t) {
	return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

}// namespace

int main(int argc, char **argv) {
	if (argc < 4) {
		std::fprintf(stderr, "usage: E3D_MPI_RANKS=N %s <config.e3d> <warm> <iters> [fast]\n", argv[0]);
		return 2;
	}
	const std::string cfgPath = argv[1];
	const int warm = std::atoi(argv[2]), iters = std::atoi(argv[3]);
	const bool fast = argc >= 5 && std::string(argv[4]) == "fast";

	auto t0 = std::chrono::steady_clock::now();
	Parallel::MPIHandler e3d_mpi(argc, argv);
	const int rank = e3d_mpi.getRankID(), size = e3d_mpi.getPoolSize();
	Parser::SimConfig config(cfgPath, rank, size);
	Mesh<Parser::MeshPartition> localmesh(config.getPartitionedMeshFiles()[rank], rank);
	auto tc = std::chrono::steady_clock::now();
	if (fast) fast_connectivity(localmesh);
	else localmesh.solveConnectivity();
	const double connectivitySeconds = seconds_since(tc);
	MPI_Barrier(MPI_COMM_WORLD);
	e3d_mpi.updateRequesterID(localmesh.getMPIelements());
	e3d_mpi.sortInterface();
	Metrics metrics(localmesh, rank, config);
	MPI_Barrier(MPI_COMM_WORLD);
	Solver::FlowField flow(config, localmesh);
	Solver::EulerSolver solver(flow, e3d_mpi, localmesh, config, metrics);
	const double setupSeconds = seconds_since(t0);

	auto &cfg = const_cast<Parser::SimConfig &>(config);
	cfg._minResidual = 0.0;
	cfg._minAeroCoeffError = 0.0;
	double warmSeconds = 0.0;
	if (warm > 0) {
		cfg._maxIter = warm;
		auto a = std::chrono::steady_clock::now();
		solver.Run();
		warmSeconds = seconds_since(a);
	}
	cfg._maxIter = iters;
	solver._nbInteration = 0;
	MPI_Barrier(MPI_COMM_WORLD);
	auto a = std::chrono::steady_clock::now();
	solver.Run();
	double s = seconds_since(a);
	std::fflush(stdout);

	if (const char *dir = std::getenv("E3D_REF_DUMP")) {
		// each rank's flow state (rho u v w p E H M, cells then ghosts) as raw doubles, for checks
		const std::string path = std::string(dir) + "/state_" + std::to_string(rank) + ".f64";
		FILE *f = std::fopen(path.c_str(), "wb");
		if (!f) return 2;
		const std::vector<const std::vector<double> *> fields{&flow.Getrho(), &flow.GetU_Velocity(), &flow.GetV_Velocity(),
		                                                      &flow.GetW_Velocity(), &flow.GetP(), &flow.GetE(),
		                                                      &flow.GetH(), &flow.GetMach()};
		for (const auto *v : fields) std::fwrite(v->data(), sizeof(double), v->size(), f);
		std::fclose(f);
	}
	std::vector<double> all(size);
	MPI_Gather(&s, 1, MPI_DOUBLE, all.data(), 1, MPI_DOUBLE, 0, MPI_COMM_WORLD);
	int cells = localmesh.GetMeshInteriorElemCount(), total = 0;
	MPI_Allreduce(&cells, &total, 1, MPI_INT, MPI_SUM, MPI_COMM_WORLD);
	if (rank == 0) {
		const double tmax = *std::max_element(all.begin(), all.end());
		const double tmin = *std::min_element(all.begin(), all.end());
		std::printf("\nE3D_REF_MPI {\"ranks\": %d, \"cells\": %d, \"iterations\": %d, \"seconds\": %.9g, "
		            "\"seconds_min_rank\": %.9g, \"warm_iterations\": %d, \"warm_seconds\": %.6g, \"setup_seconds\": %.6g, "
		            "\"connectivity_seconds_rank0\": %.6g, \"fast_connectivity\": %s}\n",
		            size, total, solver._nbInteration, tmax, tmin, warm, warmSeconds, setupSeconds, connectivitySeconds,
		            fast ? "true" : "false");
		std::fflush(stdout);
	}
	e3d_mpi.finalize();
	return 0;
}
