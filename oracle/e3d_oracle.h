/*
 * e3d_oracle: CPU restatement of the Euler3D explicit-solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls this
 * library; the tests, the smoke check and the CPU-baseline leg of the bench use
 * it as the checker the CUDA path is compared with.
 *
 * Parity is pinned: the tests compare this restatement bit for bit with the
 * unmodified reference solver (compiled into oracle/_ref by oracle/Makefile)
 * and with golden arrays that solver produced (tests/golden/).
 *
 * Every function follows the reference's arithmetic in the reference's
 * expression order (so that IEEE double results are identical) and cites the
 * reference file:line it restates.  Arrays are in the reference's own cell and
 * face numbering:
 *   cells 0..n_cells-1 are interior; ghost cell of boundary face f (f >=
 *   n_faces_int) is n_cells + (f - n_faces_int)
 *   (src/connectivity/Connectivity.cpp:212-244).
 */
#ifndef E3D_ORACLE_H
#define E3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	int n_cells;                    /* interior cells (Mesh::GetnElemTot) */
	int n_faces;                    /* Mesh::GetnFace */
	int n_faces_int;                /* Mesh::GetnFaceInt */
	const int *face2cell;           /* [2*n_faces] Mesh::GetFace2ElementID */
	const double *face_unit_normal; /* [3*n_faces] Metrics::getFaceNormalsUnit */
	const double *face_normal;      /* [3*n_faces] Metrics::getFaceNormals */
	const double *face_area;        /* [n_faces]   Metrics::getFaceSurfaces */
	const double *face_center;      /* [3*n_faces] Metrics::getFaceCenters */
	const double *cell_volume;      /* [n_cells]   Metrics::getCellVolumes */
	const int *cell2face_ptr;       /* [n_cells+1] Mesh::GetElement2FaceID */
	const int *cell2face;
	int n_wall;                     /* Mesh::GetWall{GhostCells,AdjacentGhostCell,AdjacentFace}IDs */
	const int *wall_ghost, *wall_interior, *wall_face;
	int n_farfield;                 /* Mesh::GetFarfield... */
	const int *farfield_ghost, *farfield_interior, *farfield_face;
	int n_sym;                      /* Mesh::GetSymmetry... */
	const int *sym_ghost, *sym_interior, *sym_face;
} orc_mesh;

typedef struct {
	double gamma, cfl, mach, aoa_deg;
	double rho_inf, p_inf, u_inf, v_inf, w_inf, E_inf, H_inf, M_inf; /* filled by orc_flow_init */
	double sref, cref, ref_point[3];
	int cl_axis, cl_sign, cd_axis, cd_sign, cm_axis, cm_sign;
	int scheme;                     /* 0 Roe (the reference), 1 AUSM (declared, never defined, in the reference) */
	int integrator;                 /* 0 RK5 (TIME_INTEGRATION= 2), 1 explicit Euler (TIME_INTEGRATION= 0) */
	int smoothing;                  /* RESIDUAL_SMOOTHING= */
} orc_flow;

typedef struct {                    /* each array holds n_cells + (n_faces - n_faces_int) values */
	double *rho, *u, *v, *w, *p, *E, *H, *M;
} orc_state;

typedef struct {
	int max_iter;
	int sampling;
	double min_residual;
	double min_aerocoeff_error;
	double *rms_history;            /* optional [max_iter]: density RMS of every iteration run */
} orc_run_params;

typedef struct {
	int iterations;                 /* EulerSolver::_nbInteration at exit */
	int converged;                  /* 1 RMS below MIN_RESIDUAL, 2 coefficients stagnated, 0 max_iter,
	                                   3 residual smoothing met a NaN (where the reference exits the process) */
	int n_rms;                      /* entries written to rms_history */
	double last_rms;
	double cl, cd, cm;
	double force[3], moment[3];
	long long smooth_sweeps;        /* Jacobi sweeps of residual smoothing, summed over the run */
} orc_run_stats;

/* FlowField::Initialize (src/solver/FlowField.cpp:68-101) */
void orc_flow_init(orc_flow *fl);
void orc_state_freestream(const orc_mesh *m, const orc_flow *fl, orc_state *s);

/* EulerSolver::updateBC (src/solver/EulerSolver.cpp:201-251) */
void orc_update_bc(const orc_mesh *m, const orc_flow *fl, orc_state *s);
/* EulerSolver::computeResidual (src/solver/EulerSolver.cpp:303-359); R is [5*n_cells], zeroed here */
void orc_compute_residual(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double *R);
/* EulerSolver::updateDeltaTime + TimeStepMethod2 (src/solver/TimeIntegration.cpp:8-40) */
void orc_time_step(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double *dt);
/* Solver::Roe (src/solver/ConvectiveFluxesSchemes.cpp:10-165) on face f */
void orc_roe(const orc_mesh *m, const orc_flow *fl, const orc_state *s, int f, double F[5]);
/* AUSM of Liou & Steffen (J. Comput. Phys. 107, 23-39, 1993) on face f.  The reference declares
 * Solver::AUSM (include/solver/ConvectiveFluxesSchemes.h:27-30) but never defines it, so this one is
 * not pinned to the reference; computeResidual uses it in place of Roe when fl->scheme == 1. */
void orc_ausm(const orc_mesh *m, const orc_flow *fl, const orc_state *s, int f, double F[5]);
/* EulerSolver::RungeKutta (src/solver/EulerSolver.cpp:425-472): R holds the residual of the current
 * state on entry (smoothed when fl->smoothing) and the stage-5 residual on return; dt is scratch
 * [n_cells].  Stages 2-5 smooth their residual when fl->smoothing (:456-458).  Returns the Jacobi
 * sweeps of that smoothing, or -1 if it met a NaN. */
long long orc_runge_kutta(const orc_mesh *m, const orc_flow *fl, orc_state *s, double *R, double *dt);
/* EulerSolver::smoothResiduals (src/solver/EulerSolver.cpp:483-518): Jacobi passes
 * R_c = (R0_c + 0.25 sum_{interior neighbours j} R_j) / (1 + 0.25 n_faces(c)), neighbours in
 * element2element (= element2face) order.  As the reference's loop behaves: one pass if its
 * largest change is <= 1e-16, else two.  Returns the number of passes, or -1 if a change of the
 * first pass is NaN (the reference then exits the process). */
long long orc_smooth_residuals(const orc_mesh *m, double *R);
/* EulerSolver::EulerExplicit (src/solver/EulerSolver.cpp:419-423): TimeStepMethod2, ExplicitEuler
 * (src/solver/TimeIntegration.cpp:78-91) and FlowField::Update (src/solver/FlowField.cpp:103-138).
 * W [5*n_cells] is the conservative state FlowField keeps (_rho, _rhou, _rhov, _rhow, _rhoE), updated
 * in place; dt is scratch [n_cells]. */
void orc_euler_explicit(const orc_mesh *m, const orc_flow *fl, orc_state *s, double *W, const double *R, double *dt);
/* EulerSolver::computeRMS (src/solver/EulerSolver.cpp:382-389) followed by the sqrt of :99 */
double orc_rms(const orc_mesh *m, const double *R);
/* AeroCoefficients::Update (src/solver/AeroCoefficients.cpp:38-52) */
void orc_aero_coefficients(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double force[3],
                           double moment[3]);
/* EulerSolver::Run (src/solver/EulerSolver.cpp:60-167); returns 0, or -1 on allocation failure */
int orc_run(const orc_mesh *m, const orc_flow *fl, orc_state *s, const orc_run_params *rp, orc_run_stats *st);

#ifdef __cplusplus
}
#endif
#endif
