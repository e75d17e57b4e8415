/*
 * euler3d_b200.h -- C ABI of the B200 (sm_100a) Euler3D explicit-solver hot path.
 *
 * The library replaces, for one GPU, the inside of the reference solver's
 * EulerSolver::Run() loop: ghost-cell boundary updates, the face flux residual,
 * the local time step, the 5-stage Runge-Kutta update and the residual / force
 * reductions.  Plain C types only; every pointer here is a HOST pointer unless a
 * name says otherwise.  All functions return an e3d_status; on failure
 * e3d_last_error() holds a message (per calling thread).
 *
 * Numbering: every array is in the reference's own cell and face numbering
 * (cells 0..n_cells-1 interior; the ghost cell of boundary face f is
 * n_cells + f - n_faces_int; faces 0..n_faces_int-1 interior), so results can
 * be written straight back into the reference's FlowField.  The device keeps
 * its own locality-ordered copy internally.
 *
 * Threading: a solver handle belongs to one host thread at a time; work is
 * ordered on the handle's CUDA stream.
 */
#ifndef EULER3D_B200_H
#define EULER3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define E3D_ABI_VERSION 3

typedef enum e3d_status {
	E3D_OK = 0,
	E3D_ERR_INVALID_ARG = 1, /* null pointer, inconsistent sizes, bad enum value */
	E3D_ERR_OOM = 2,         /* host or device allocation failed */
	E3D_ERR_NONFINITE = 3,   /* the solution developed a NaN/Inf or a non-positive density/pressure */
	E3D_ERR_TIMEOUT = 4,     /* a bounded wait on the device ran out */
	E3D_ERR_CUDA = 5,        /* a CUDA call failed, or no usable sm_100 device */
	E3D_ERR_MESH = 6         /* malformed mesh or mesh file */
} e3d_status;

/* Flux scheme (the reference's SCHEME= key, src/parser/SimConfig.cpp:127-129). */
enum { E3D_SCHEME_ROE = 0, E3D_SCHEME_AUSM = 1 };

/* Arithmetic of the hot path.
 *   FP64_EXACT : double precision in the reference's own operation order, no FMA
 *                contraction; bit-for-bit equal to the reference for the state,
 *                residual and time step (reductions differ in summation order only).
 *   FP64       : double precision with restructured arithmetic (fewer divisions and
 *                square roots, FMA); agrees with the reference to round-off.
 *   FP32_FLUX  : fluxes, face states and time step in single precision; conservative
 *                state, Runge-Kutta accumulation and all reductions in double. */
enum { E3D_PREC_FP64_EXACT = 0, E3D_PREC_FP64 = 1, E3D_PREC_FP32_FLUX = 2 };

/* Cell ordering used on the device (results are always returned in reference order):
 * reference order, reverse Cuthill-McKee of the cell graph, or Morton order of the cell centres
 * (spatially compact groups of cells, which the face-tile kernel needs). */
enum { E3D_ORDER_NATIVE = 0, E3D_ORDER_RCM = 1, E3D_ORDER_SPATIAL = 2 };

/* Time integration (the reference's TIME_INTEGRATION= key, src/parser/SimConfig.cpp:130-148, and
 * EulerSolver's constructor, src/solver/EulerSolver.cpp:49-56): RK5 is TIME_INTEGRATION= 2
 * (EulerSolver::RungeKutta, :425-472); EULER is TIME_INTEGRATION= 0, explicit Euler
 * (EulerSolver::EulerExplicit, :419-423: W += R * (-dt / V) on the carried conservative state).
 * TIME_INTEGRATION= 1 (EulerImplicit, :474-480) never updates the state in the reference and has
 * no counterpart here. */
enum { E3D_INTEGRATOR_RK5 = 0, E3D_INTEGRATOR_EULER = 1 };

/* Why e3d_solver_run stopped (the exits of EulerSolver::Run, src/solver/EulerSolver.cpp:100-152). */
enum { E3D_STOP_MAX_ITER = 0, E3D_STOP_RESIDUAL = 1, E3D_STOP_COEFFICIENTS = 2, E3D_STOP_STALL = 3 };

/* ------------------------------------------------------------------------------------------
 * Mesh preparation.  Replaces Mesh<MeshPartition>::solveConnectivity
 * (include/mesh/Mesh.hpp:36-105, src/connectivity/Connectivity.cpp:5-362), the ghost-cell
 * classification (include/mesh/Mesh.hpp:471-707) and the Metrics constructor
 * (src/mesh/Metrics.cpp:9-335).  Same numbering and the same IEEE results as the reference.
 * ------------------------------------------------------------------------------------------ */
typedef struct e3d_mesh e3d_mesh;

/* Read an SU2 mesh or single-domain .par partition file (src/parser/SU2MeshParser.cpp:12-240,
 * src/parser/MeshPartition.cpp:15-112) and prepare it.  cref divides the coordinates
 * (src/mesh/Metrics.cpp:12-19).  n_threads <= 0 uses all host cores. */
e3d_status e3d_mesh_read(const char *path, double cref, int32_t n_threads, e3d_mesh **out);

/* Prepare a mesh held in memory.  Volume elements: VTK type (10 tetra, 12 hexa, 13 wedge,
 * 14 pyramid) and CSR node lists.  Markers: n_markers tags; marker m owns surface faces
 * marker_ptr[m] .. marker_ptr[m+1]-1, face k has nodes face_nodes[face_ptr[k] .. face_ptr[k+1]-1]. */
e3d_status e3d_mesh_from_arrays(int32_t n_nodes, const double *xyz, int32_t n_elems, const int32_t *elem_vtk,
                                const int32_t *elem_ptr, const int32_t *elem_nodes, int32_t n_markers,
                                const char *const *marker_tags, const int32_t *marker_ptr, const int32_t *face_ptr,
                                const int32_t *face_nodes, double cref, int32_t n_threads, e3d_mesh **out);

/* Sizes of a prepared mesh. */
typedef struct e3d_mesh_info {
	int32_t n_cells, n_faces, n_faces_int, n_nodes;
	int32_t n_wall, n_farfield, n_sym;
} e3d_mesh_info;
e3d_status e3d_mesh_info_get(const e3d_mesh *mesh, e3d_mesh_info *info);

/* Read-only view of one prepared array by name: "face2cell", "cell2face_ptr", "cell2face",
 * "cell2cell", "face2node_ptr", "face2node", "face_normal", "face_unit_normal", "face_center",
 * "face_area", "cell_volume", "cell_centroid", "{wall,farfield,sym}_{ghost,interior,face}",
 * "partition_cell_ptr" (empty unless read from partition files).
 * *is_double says whether the data is double (else int32).  Valid until e3d_mesh_destroy. */
e3d_status e3d_mesh_array(const e3d_mesh *mesh, const char *name, const void **data, int64_t *count,
                          int32_t *is_double);
void e3d_mesh_destroy(e3d_mesh *mesh);

/* ------------------------------------------------------------------------------------------
 * Solver.  The descriptor carries what EulerSolver reads from Mesh and Metrics
 * (include/solver/EulerSolver.hpp:91-95, :206-210); all pointers are host arrays in the
 * reference numbering, copied during e3d_solver_create and not retained.
 * ------------------------------------------------------------------------------------------ */
typedef struct e3d_mesh_desc {
	int32_t n_cells;                  /* Mesh::GetnElemTot */
	int32_t n_faces;                  /* Mesh::GetnFace */
	int32_t n_faces_int;              /* Mesh::GetnFaceInt */
	const int32_t *face2cell;         /* [2*n_faces]  Mesh::GetFace2ElementID */
	const double *face_unit_normal;   /* [3*n_faces]  Metrics::getFaceNormalsUnit */
	const double *face_normal;        /* [3*n_faces]  Metrics::getFaceNormals */
	const double *face_area;          /* [n_faces]    Metrics::getFaceSurfaces */
	const double *face_center;        /* [3*n_faces]  Metrics::getFaceCenters */
	const double *cell_volume;        /* [n_cells]    Metrics::getCellVolumes */
	const int32_t *cell2face_ptr;     /* [n_cells+1]  Mesh::GetElement2FaceID */
	const int32_t *cell2face;
	int32_t n_wall;                   /* Mesh::GetWallGhostCellsIDs / AdjacentGhostCellIDs / AdjacentFaceIDs */
	const int32_t *wall_ghost, *wall_interior, *wall_face;
	int32_t n_farfield;               /* Mesh::GetFarfield... */
	const int32_t *farfield_ghost, *farfield_interior, *farfield_face;
	int32_t n_sym;                    /* Mesh::GetSymmetry... */
	const int32_t *sym_ghost, *sym_interior, *sym_face;
} e3d_mesh_desc;

/* The partition files of a multi-partition case (PARTITION_FILES= n, the .par files E3D_PRE writes,
 * src/partition/Partition.cpp, read per rank by MeshPartition, src/parser/MeshPartition.cpp:39-112),
 * merged into one mesh for one GPU: nodes shared by partitions are joined through the
 * inter-partition faces (NINTERNAL_MARKER) both sides list, elements are concatenated partition by
 * partition -- e3d_mesh_array "partition_cell_ptr" gives the first cell of each -- and boundary
 * markers merged by tag.  Fails with E3D_ERR_MESH on inconsistent partitions. */
e3d_status e3d_mesh_read_partitions(const char *const *paths, int32_t n_parts, double cref, int32_t n_threads,
                                    e3d_mesh **out);

/* <partition>.bry, WriteSolution::writeBoundaryFile (src/solver/WriteSolution.cpp:57-76): every wall
 * face's interior cell and node ids, byte for byte as the reference writes it. */
e3d_status e3d_mesh_write_boundary(const e3d_mesh *mesh, const char *path);

/* Fill a descriptor whose pointers refer to a prepared mesh's arrays. */
e3d_status e3d_mesh_describe(const e3d_mesh *mesh, e3d_mesh_desc *desc);

typedef struct e3d_flow_params {
	double gamma;                     /* GAMMA= */
	double mach;                      /* FlowField::getM_inf */
	double aoa_deg;                   /* AOA= */
	double cfl;                       /* CFL= */
	double sref, cref;                /* SREF= CREF= */
	double ref_point[3];              /* MESH_REF_POINT_{X,Y,Z}= */
	int32_t cl_axis, cl_sign;         /* SimConfig::getMeshOrientationCL */
	int32_t cd_axis, cd_sign;         /* SimConfig::getMeshOrientationCD */
	int32_t cm_axis, cm_sign;         /* SimConfig::getMeshOrientationCM */
	int32_t scheme;                   /* E3D_SCHEME_* */
	int32_t precision;                /* E3D_PREC_* */
	int32_t ordering;                 /* E3D_ORDER_* */
	int32_t device;                   /* CUDA device ordinal */
	void *stream;                     /* cudaStream_t to run on, or NULL for a library-owned stream */
	int32_t no_autotune;              /* 1: skip the creation-time timing of the stage-kernel variants
	                                     and use the face-tile kernel (what a batch runs anyway) */
	int32_t integrator;               /* E3D_INTEGRATOR_* (TIME_INTEGRATION=) */
	int32_t residual_smoothing;       /* RESIDUAL_SMOOTHING=: EulerSolver::smoothResiduals
	                                     (src/solver/EulerSolver.cpp:483-518) on every residual that
	                                     updates the state; FP64 and FP64_EXACT only */
} e3d_flow_params;

typedef struct e3d_solver e3d_solver;

/* Replaces the EulerSolver constructor (src/solver/EulerSolver.cpp:21-58) plus the FlowField
 * freestream initialisation (src/solver/FlowField.cpp:68-101): uploads the mesh and sets
 * every cell and ghost to the freestream. */
e3d_status e3d_solver_create(const e3d_mesh_desc *mesh, const e3d_flow_params *params, e3d_solver **out);
void e3d_solver_destroy(e3d_solver *solver);

/* What the handle holds on the device and what its autotuner chose.  At creation the solver times
 * each stage-kernel variant available for its precision on this mesh -- per-cell gather and face
 * tiles at several register budgets (occupancies), the persistent face-tile kernel, and face
 * colouring at two block sizes (faces per block) -- with writes redirected to scratch, and keeps the
 * fastest. */
typedef struct e3d_solver_info {
	int32_t n_cells, n_ghosts, n_faces;
	int32_t stage_variant;            /* variant in use */
	int32_t n_variants;
	float variant_ms[8];              /* measured duration of one stage per variant, n_variants of
	                                     them (-1: not available for this mesh and precision) */
	int32_t tile_smem_bytes;          /* dynamic shared memory of one face-tile block (0: no tiles) */
	int64_t device_bytes;             /* device memory held by the handle */
} e3d_solver_info;
e3d_status e3d_solver_info_get(const e3d_solver *solver, e3d_solver_info *info);

/* Number of entries of each state array: n_cells + (n_faces - n_faces_int). */
int64_t e3d_solver_state_size(const e3d_solver *solver);

/* Flow state in FlowField's layout (include/solver/FlowField.hpp:29-59): the 8 arrays
 * rho, u, v, w, p, E, H, M, each e3d_solver_state_size() long, interior cells then ghosts. */
e3d_status e3d_solver_set_state(e3d_solver *solver, const double *const state[8]);
e3d_status e3d_solver_get_state(e3d_solver *solver, double *const state[8]);
e3d_status e3d_solver_set_freestream(e3d_solver *solver);

typedef struct e3d_run_params {
	int32_t max_iter;                 /* MAX_ITER= */
	int32_t sampling;                 /* SAMPLING= (force coefficients every this many iterations) */
	double min_residual;              /* MIN_RESIDUAL= (absolute density RMS) */
	double min_aerocoeff_error;       /* MIN_AEROCOEFF_ERROR= (0 disables the coefficient exit) */
	int32_t check_every;              /* iterations per CUDA-graph launch between host checks of the
	                                     stop flag (0: 32); iterations past a stop are no-ops */
	int32_t profile_stages;           /* 0: CUDA graphs; 1: launch directly and time every stage
	                                     kernel with CUDA events (stats.stage_ms); 2: CUDA graphs as
	                                     with 0, with an event pair captured around every stage kernel,
	                                     so the stages are timed as they run back to back
	                                     (stats.stage_ms over the iterations that ran) */
	int32_t stage_kernel;             /* 0: the autotuned stage kernel; 1, 2: per-cell gather with two
	                                     register budgets (FP64 modes); 3: face tiles; 4: persistent
	                                     face tiles with a producer warp streaming tiles to consumer
	                                     warps; 5: face tiles at seven blocks per SM (FP64) or eight
	                                     (FP32_FLUX); 6, 7: face colouring, one launch per class of
	                                     faces that share no cell, 128 or 512 faces per block (FP64)
	                                     (kept for later runs) */
	double min_residual_drop;         /* > 0: also stop once the density RMS is below this fraction of
	                                     the run's first RMS (a relative tolerance such as 1e-8); 0 off.
	                                     No counterpart in the reference, whose test is absolute. */
	int32_t stall_window;             /* > 0: also stop (E3D_STOP_STALL) once the density RMS has set no
	                                     new minimum for this many iterations -- the residual has hit
	                                     the floor of the arithmetic (FP32_FLUX); 0 off.  No counterpart
	                                     in the reference. */
	double stall_below;               /* > 0: the stall test starts once the RMS is below this fraction of
	                                     the first RMS (initial transients do not count) */
} e3d_run_params;

typedef struct e3d_run_stats {
	int32_t iterations;               /* EulerSolver::_nbInteration at exit */
	int32_t stop_reason;              /* E3D_STOP_* */
	int32_t n_rms;                    /* iterations whose RMS was computed (history length) */
	double last_rms;                  /* density RMS of the last iteration run */
	double cl, cd, cm;                /* last sampled coefficients (EulerSolver::_CL/_CD/_CM) */
	double force[3], moment[3];       /* last sampled force / moment coefficient vectors */
	double device_ms;                 /* device time of the iterations (CUDA events) */
	int64_t kernel_launches;          /* kernels this call launched */
	double stage_ms;                  /* profile_stages: summed duration of the stage kernels */
	int64_t stage_launches;           /* profile_stages: stage kernels timed */
} e3d_run_stats;

/* Replaces EulerSolver::Run (src/solver/EulerSolver.cpp:60-167): iterate RK5 steps from the
 * current device state until MAX_ITER, the residual test or the coefficient test stops it. */
e3d_status e3d_solver_run(e3d_solver *solver, const e3d_run_params *params, e3d_run_stats *stats);

/* e3d_solver_run for callers that must not allocate device memory once set-up is done: a serving
 * loop that runs inside a fixed, pre-reserved memory budget, or code running where the CUDA
 * allocator may not be called.  e3d_solver_run itself may allocate (its history buffer grows with
 * max_iter and it instantiates CUDA graphs); this call allocates nothing.  It computes the same
 * iterations with the same kernels, launched directly, and keeps its scratch (the per-block RMS
 * partial sums and the RMS history) in one 1.5 MiB file-scope device array that every device loading
 * the library holds until the process exits.  Limits: at most 16,777,216 cells and 65,536
 * iterations per call; larger requests fail with E3D_ERR_INVALID_ARG.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  All calls share the array, so calls that overlap on the GPU race on it.  The
 * density RMS of every iteration run is copied to rms_history (up to history_capacity entries;
 * NULL skips it).  params->stage_kernel must be 0.  After this call the state, the stats, the wall
 * Cp (e3d_solver_wall_cp, e3d_solver_write_cp) and e3d_solver_write_summary / _write_solution are
 * this run's; the handle keeps no RMS history or coefficient samples of it, so
 * e3d_solver_rms_history and e3d_solver_coefficient_history report no entries and
 * e3d_solver_write_residuals fails with E3D_ERR_INVALID_ARG until the next e3d_solver_run.
 * No counterpart in the reference. */
e3d_status e3d_solver_run_noalloc(e3d_solver *solver, const e3d_run_params *params, e3d_run_stats *stats,
                                  double *rms_history, int32_t history_capacity);

/* Fault-path check without a fault: the number of polls the stage kernels make on a tile's data
 * barrier before their bounded wait gives up (default and maximum 4,194,304; a negative value
 * restores the default).  With 0 every wait gives up at once: the kernel lets the copies it issued
 * land, marks the run failed and returns, the run stops after that stage with E3D_ERR_TIMEOUT, and
 * the handle stays usable.  Face-tile stage kernels only (the per-cell gather kernels never wait).
 * Kept for later runs of this solver, also inside a batch.  No counterpart in the reference, which
 * has no device waits. */
e3d_status e3d_solver_set_wait_limit(e3d_solver *solver, int32_t polls);

/* Accuracy check of the FP64 mode's fast reciprocal and reciprocal square root (single-precision
 * seed, one series refinement step): for the n arguments x (host memory) writes, to out (host,
 * 4 n doubles), out[4 i] = the FP64 mode's 1/x, out[4 i + 1] = CUDA's 1.0 / x, out[4 i + 2] = the
 * FP64 mode's 1/sqrt(x) and out[4 i + 3] = CUDA's rsqrt(x), evaluated on `device`.  No counterpart
 * in the reference, whose solver divides and takes square roots in IEEE double precision. */
e3d_status e3d_fast_reciprocals(int32_t device, const double *x, int64_t n, double *out);

/* Density RMS of every iteration of the last e3d_solver_run (the residuals.dat column). */
e3d_status e3d_solver_rms_history(e3d_solver *solver, double *out, int32_t capacity, int32_t *count);

/* One call of EulerSolver::updateBC + computeResidual + updateDeltaTime at the current state
 * (src/solver/EulerSolver.cpp:201-251, :303-359, :362-367): updates the ghost cells and
 * returns the residual R [5*n_cells, cell-major] and time step dt [n_cells].  Either output
 * may be NULL. */
e3d_status e3d_solver_residual(e3d_solver *solver, double *residual, double *dt);

/* AeroCoefficients::Update (src/solver/AeroCoefficients.cpp:38-52) on the current state. */
e3d_status e3d_solver_coefficients(e3d_solver *solver, double force[3], double moment[3]);

/* The coefficient samples of the last run: 7 doubles each -- the iteration, the force and the moment
 * coefficient vectors -- one per SAMPLING-th iteration (the rows EulerSolver::PrintInfo writes to
 * residuals.dat, src/solver/EulerSolver.cpp:253-259).  *count receives the number of samples. */
e3d_status e3d_solver_coefficient_history(e3d_solver *solver, double *samples, int32_t capacity, int32_t *count);
/* Pressure coefficient of every wall face (reference wall order) at the last sample of the last run
 * (AeroCoefficients::_cp; zero before the first sample) or of the last e3d_solver_coefficients. */
e3d_status e3d_solver_wall_cp(e3d_solver *solver, double *cp, int32_t capacity, int32_t *count);

/* The reference's output files of the last run, byte for byte as the reference writes them:
 *   residuals.dat   ResidualsFile (include/solver/ResidualsFile.hpp:18-48): one row per sample, plus
 *                   the row the residual exit prints (src/solver/EulerSolver.cpp:100-108)
 *   cp_part_N.dat   EulerSolver::PrintCp (:283-303): wall Cp of the last sample and face centroids
 *   <partition>.sol WriteSolution::writeSolutionFile (src/solver/WriteSolution.cpp:30-55): the
 *                   interior cells' density, velocity, pressure and energy
 *   summary.txt     EulerSolver::WriteSummary (:169-198), the TOML the reference's toml++ prints,
 *                   with the caller's timings (milliseconds) and core count */
e3d_status e3d_solver_write_residuals(e3d_solver *solver, const char *path);
e3d_status e3d_solver_write_cp(e3d_solver *solver, const char *path);
e3d_status e3d_solver_write_solution(e3d_solver *solver, const char *path);
e3d_status e3d_solver_write_summary(e3d_solver *solver, const char *path, int64_t solver_ms, int64_t total_ms,
                                    int32_t n_cores);

/* ------------------------------------------------------------------------------------------
 * Batches: many solvers advanced together.  No counterpart in the reference, whose solver runs one
 * mesh per process.
 *
 * A batch runs the RK iterations of its members -- solver handles of any mesh sizes and flow
 * conditions, on one device and of one precision -- in shared launches: each Runge-Kutta stage is
 * ONE kernel over the concatenated face tiles of every running member (block -> member, tile),
 * each member's RMS and stop test and its force coefficients one block each of two more kernels,
 * and a step's iterations are one CUDA graph.  Every member keeps its own state, CFL, scheme, stop
 * criteria and iteration counters on the device; a member that meets its stop condition stops
 * updating at once, while the others go on.  Each member computes exactly what e3d_solver_run
 * computes for it alone, with any stage kernel (every stage kernel of a precision gives the same
 * bits): same states, RMS history, counters and coefficients.
 *
 * A solver belongs to the batch from e3d_batch_add until it is retired or removed; meanwhile the
 * other e3d_solver_* calls on it fail with E3D_ERR_INVALID_ARG (e3d_solver_destroy removes it).
 * One host thread drives a batch at a time. */
typedef struct e3d_batch e3d_batch;

/* An empty batch on `device`, running on `stream` (cudaStream_t, or NULL for a batch-owned stream). */
e3d_status e3d_batch_create(int32_t device, void *stream, e3d_batch **out);
/* Removes every member (their state stays on the device, usable again) and frees the batch. */
void e3d_batch_destroy(e3d_batch *batch);

/* Starts a run of `solver` inside the batch, as e3d_solver_run would start it: fresh counters, the
 * solver's current state, params' stop criteria (params->stage_kernel, check_every and
 * profile_stages are ignored).  The solver's mesh must fit the face-tile kernel. */
e3d_status e3d_batch_add(e3d_batch *batch, e3d_solver *solver, const e3d_run_params *params);

/* Runs `iterations` more iterations (rounded up to an even number) of every running member and
 * waits for them.  n_active (may be NULL) receives how many members are still running. */
e3d_status e3d_batch_step(e3d_batch *batch, int32_t iterations, int32_t *n_active);

/* Takes up to `capacity` members whose runs have stopped out of the batch, in the order they were
 * added: solvers[i] and (when not NULL) stats[i] -- the e3d_run_stats their e3d_solver_run would
 * have returned, device_ms and kernel_launches being those of the batch steps they took part in --
 * and status[i]: E3D_OK, E3D_ERR_NONFINITE or E3D_ERR_TIMEOUT as e3d_solver_run would return.
 * *count receives the number taken. */
e3d_status e3d_batch_retire(e3d_batch *batch, e3d_solver **solvers, e3d_run_stats *stats, e3d_status *status,
                            int32_t capacity, int32_t *count);

/* Takes `solver` out of the batch whether or not its run has stopped; stats as e3d_batch_retire. */
e3d_status e3d_batch_remove(e3d_batch *batch, e3d_solver *solver, e3d_run_stats *stats);

/* The stage kernel of a batch's launches:
 *   E3D_BATCH_KERNEL_TILES  one block of 128 threads per (member, tile) entry of the table (default)
 *   E3D_BATCH_KERNEL_WS     one persistent block per SM walking the table: a producer warp copies each
 *                           entry's member arguments and tile data into a ring of shared-memory buffers
 *                           ahead of five consumer groups that evaluate them
 * Both compute the same bits.  No counterpart in the reference. */
enum { E3D_BATCH_KERNEL_TILES = 0, E3D_BATCH_KERNEL_WS = 1 };
e3d_status e3d_batch_set_kernel(e3d_batch *batch, int32_t kernel);

typedef struct e3d_batch_info {
	int32_t n_members;                /* members (running or stopped, not yet retired) */
	int32_t n_running;                /* members whose runs have not stopped */
	int32_t n_tiles;                  /* face tiles in the stage launches of the last step */
	int32_t graph_builds;             /* CUDA graphs instantiated so far */
	int64_t member_device_bytes;      /* e3d_solver_info.device_bytes summed over the members */
	int64_t device_bytes;             /* device memory held by the batch itself */
	double last_step_ms;              /* device time of the last e3d_batch_step */
	int64_t kernel_launches;          /* kernels launched by all steps so far */
} e3d_batch_info;
e3d_status e3d_batch_info_get(const e3d_batch *batch, e3d_batch_info *info);

const char *e3d_status_string(e3d_status status);
const char *e3d_last_error(void);
int32_t e3d_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* EULER3D_B200_H */
