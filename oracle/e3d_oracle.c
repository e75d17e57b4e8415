/*
 * e3d_oracle.c -- CPU restatement of the Euler3D explicit-solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see e3d_oracle.h).  Each function restates the
 * reference function cited beside it.  Expressions keep the reference's
 * association order, std::pow(x, 2) is written x * x (the exact value GCC
 * folds it to) and no fused multiply-add is allowed (-ffp-contract=off), so
 * results are the reference's IEEE doubles bit for bit; the tests check that.
 */
#include "e3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_E3D 3.141592653589793238 /* FlowField::E3D_PI, include/solver/FlowField.hpp:93 */

static int n_ghost(const orc_mesh *m) { return m->n_faces - m->n_faces_int; }

/* FlowField::Initialize, src/solver/FlowField.cpp:68-101 (rho_inf = p_inf = 1,
 * include/solver/FlowField.hpp:138-139; w_inf = 0). */
void orc_flow_init(orc_flow *fl) {
	double g = fl->gamma;
	fl->rho_inf = 1.0;
	fl->p_inf = 1.0;
	fl->M_inf = fl->mach;
	fl->u_inf = fl->mach * sqrt(g) * cos(fl->aoa_deg * (PI_E3D / 180));
	fl->v_inf = fl->mach * sqrt(g) * sin(fl->aoa_deg * (PI_E3D / 180));
	fl->w_inf = 0.0;
	fl->E_inf = fl->p_inf / ((g - 1) * fl->rho_inf) +
	            ((fl->u_inf * fl->u_inf + fl->v_inf * fl->v_inf + fl->w_inf * fl->w_inf) / 2.0);
	fl->H_inf = fl->E_inf + (fl->p_inf / fl->rho_inf);
}

void orc_state_freestream(const orc_mesh *m, const orc_flow *fl, orc_state *s) {
	int n = m->n_cells + n_ghost(m);
	for (int i = 0; i < n; i++) {
		s->rho[i] = fl->rho_inf;
		s->u[i] = fl->u_inf;
		s->v[i] = fl->v_inf;
		s->w[i] = fl->w_inf;
		s->p[i] = fl->p_inf;
		s->E[i] = fl->E_inf;
		s->H[i] = fl->H_inf;
		s->M[i] = fl->M_inf;
	}
}

/* ---------------------------------------------------------------- boundary ghosts */

static void set_ghost(orc_state *s, int g, double rho, double u, double v, double w, double M, double p, double E,
                      double H) {
	s->rho[g] = rho;
	s->u[g] = u;
	s->v[g] = v;
	s->w[g] = w;
	s->M[g] = M;
	s->p[g] = p;
	s->E[g] = E;
	s->H[g] = H;
}

/* Shared tail of the subsonic / wall / symmetry ghost states: Mach, E and H of the ghost. */
static void finish_ghost(const orc_flow *fl, orc_state *s, int g, double rho, double u, double v, double w,
                         double p, double c) {
	double q2 = u * u + v * v + w * w;
	double M = sqrt(q2) / c;
	double E = p / ((fl->gamma - 1) * rho) + (q2 / 2.0);
	double H = E + (p / rho);
	set_ghost(s, g, rho, u, v, w, M, p, E, H);
}

/* BC::FarfieldSubsonicInflow, src/solver/PhysicalBC.cpp:43-79 */
static void bc_subsonic_inflow(const orc_flow *fl, orc_state *s, int g, int d, const double *n) {
	double c = sqrt(fl->gamma * (s->p[d] / s->rho[d]));
	double p = 0.5 * (fl->p_inf + s->p[d] -
	                  s->rho[d] * c *
	                          ((n[0] * (fl->u_inf - s->u[d])) + (n[1] * (fl->v_inf - s->v[d])) +
	                           (n[2] * (fl->w_inf - s->w[d]))));
	double rho = fl->rho_inf + (p - fl->p_inf) / (c * c);
	double u = fl->u_inf - n[0] * (fl->p_inf - p) / (s->rho[d] * c);
	double v = fl->v_inf - n[1] * (fl->p_inf - p) / (s->rho[d] * c);
	double w = fl->w_inf - n[2] * (fl->p_inf - p) / (s->rho[d] * c);
	finish_ghost(fl, s, g, rho, u, v, w, p, c);
}

/* BC::FarfieldSubsonicOutflow, src/solver/PhysicalBC.cpp:82-121 */
static void bc_subsonic_outflow(const orc_flow *fl, orc_state *s, int g, int d, const double *n) {
	double c = sqrt(fl->gamma * (s->p[d] / s->rho[d]));
	double p = fl->p_inf;
	double rho = s->rho[d] + (p - s->p[d]) / (c * c);
	double u = s->u[d] + n[0] * (s->p[d] - p) / (s->rho[d] * c);
	double v = s->v[d] + n[1] * (s->p[d] - p) / (s->rho[d] * c);
	double w = s->w[d] + n[2] * (s->p[d] - p) / (s->rho[d] * c);
	finish_ghost(fl, s, g, rho, u, v, w, p, c);
}

/* BC::Wall and BC::Symmetry (identical arithmetic), src/solver/PhysicalBC.cpp:124-162 and :165-231 */
static void bc_mirror(const orc_flow *fl, orc_state *s, int g, int d, const double *n) {
	double c = sqrt(fl->gamma * (s->p[d] / s->rho[d]));
	double V = s->u[d] * n[0] + s->v[d] * n[1] + s->w[d] * n[2];
	double u = s->u[d] - 2 * V * n[0];
	double v = s->v[d] - 2 * V * n[1];
	double w = s->w[d] - 2 * V * n[2];
	finish_ghost(fl, s, g, s->rho[d], u, v, w, s->p[d], c);
}

/* EulerSolver::updateBC, src/solver/EulerSolver.cpp:201-251 (no MPI ghosts on one domain). */
void orc_update_bc(const orc_mesh *m, const orc_flow *fl, orc_state *s) {
	for (int i = 0; i < m->n_farfield; i++) {
		int g = m->farfield_ghost[i], d = m->farfield_interior[i];
		const double *n = m->face_unit_normal + 3 * (size_t) m->farfield_face[i];
		/* the branch is chosen from the ghost's own previous state, :211-226 */
		double V = s->u[g] * n[0] + s->v[g] * n[1] + s->w[g] * n[2];
		double M = s->M[g];
		if (M >= 1.0 && V > 0.0) { /* BC::FarfieldSupersonicOutflow, PhysicalBC.cpp:26-40 */
			set_ghost(s, g, s->rho[d], s->u[d], s->v[d], s->w[d], s->M[d], s->p[d], s->E[d], s->H[d]);
		} else if (M < 1.0 && V > 0.0) {
			bc_subsonic_outflow(fl, s, g, d, n);
		} else if (M >= 1.0 && V <= 0.0) { /* BC::FarfieldSupersonicInflow, PhysicalBC.cpp:11-23 */
			set_ghost(s, g, fl->rho_inf, fl->u_inf, fl->v_inf, fl->w_inf, fl->M_inf, fl->p_inf, fl->E_inf,
			          fl->H_inf);
		} else if (M < 1.0 && V <= 0.0) {
			bc_subsonic_inflow(fl, s, g, d, n);
		}
	}
	for (int i = 0; i < m->n_wall; i++)
		bc_mirror(fl, s, m->wall_ghost[i], m->wall_interior[i], m->face_unit_normal + 3 * (size_t) m->wall_face[i]);
	for (int i = 0; i < m->n_sym; i++)
		bc_mirror(fl, s, m->sym_ghost[i], m->sym_interior[i], m->face_unit_normal + 3 * (size_t) m->sym_face[i]);
}

/* ---------------------------------------------------------------- fluxes */

/* Solver::Roe, src/solver/ConvectiveFluxesSchemes.cpp:10-165.  First-order Roe flux between the
 * face's left and right cells with Harten's entropy fix on the acoustic waves, delta = c_L / 15. */
static void roe_lr(const orc_flow *fl, const orc_state *s, int L, int R, const double *n, double F[5]) {
	const double g = fl->gamma;
	double rl = s->rho[L], rr = s->rho[R];
	double sl = sqrt(rl), sr = sqrt(rr);
	double rt = sqrt(rl * rr);
	double ul = s->u[L], ur = s->u[R], vl = s->v[L], vr = s->v[R], wl = s->w[L], wr = s->w[R];
	double hl = s->H[L], hr = s->H[R], pl = s->p[L], pr = s->p[R];

	/* Roe averages, :48-55 */
	double ut = (ul * sl + ur * sr) / (sl + sr);
	double vt = (vl * sl + vr * sr) / (sl + sr);
	double wt = (wl * sl + wr * sr) / (sl + sr);
	double ht = (hl * sl + hr * sr) / (sl + sr);
	double q2t = ut * ut + vt * vt + wt * wt;
	double ct = sqrt((g - 1.0) * (ht - q2t / 2));

	/* contravariant velocities and jumps, :60-70 */
	double Vt = ut * n[0] + vt * n[1] + wt * n[2];
	double Vl = ul * n[0] + vl * n[1] + wl * n[2];
	double Vr = ur * n[0] + vr * n[1] + wr * n[2];
	double drho = rr - rl, du = ur - ul, dv = vr - vl, dw = wr - wl, dp = pr - pl, dV = Vr - Vl;

	/* central part: mean of the two physical fluxes, :92-104 */
	double fr[5] = {rr * Vr, rr * Vr * ur + pr * n[0], rr * Vr * vr + pr * n[1], rr * Vr * wr + pr * n[2],
	                rr * Vr * hr};
	double fll[5] = {rl * Vl, rl * Vl * ul + pl * n[0], rl * Vl * vl + pl * n[1], rl * Vl * wl + pl * n[2],
	                 rl * Vl * hl};

	/* Harten's entropy fix on |V - c| and |V + c| with delta from the LEFT cell, :107-122 */
	double cl = sqrt(g * pl / rl);
	double delta = (1.0 / 15.0) * cl;
	double lam1 = fabs(Vt - ct);
	if (!(fabs(Vt - ct) > delta)) lam1 = ((Vt - ct) * (Vt - ct) + delta * delta) / (2.0 * delta);
	double lam5 = fabs(Vt + ct);
	if (!(fabs(Vt + ct) > delta)) lam5 = ((Vt + ct) * (Vt + ct) + delta * delta) / (2.0 * delta);

	/* wave 1 (V - c), :125-132 */
	double e1[5] = {1.0, ut - ct * n[0], vt - ct * n[1], wt - ct * n[2], ht - ct * Vt};
	/* waves 2-4 (V, no fix), :134-149 */
	double e2[5] = {1.0, ut, vt, wt, q2t * 0.5};
	double e2b[5] = {0.0, rt * (du - dV * n[0]), rt * (dv - dV * n[1]), rt * (dw - dV * n[2]),
	                 rt * (ut * du + vt * dv + wt * dw - Vt * dV)};
	/* wave 5 (V + c), :151-158 */
	double e5[5] = {1.0, ut + ct * n[0], vt + ct * n[1], wt + ct * n[2], ht + ct * Vt};

	for (int i = 0; i < 5; i++) {
		double d1 = e1[i] * lam1 * (dp - rt * ct * dV) / (2.0 * (ct * ct));
		double d234 = (e2[i] * (drho - dp / (ct * ct)) + e2b[i]) * fabs(Vt);
		double d5 = e5[i] * lam5 * (dp + rt * ct * dV) / (2.0 * (ct * ct));
		F[i] = (fr[i] + fll[i]) * 0.5 - 0.5 * (d1 + d234 + d5);
	}
}

void orc_roe(const orc_mesh *m, const orc_flow *fl, const orc_state *s, int f, double F[5]) {
	roe_lr(fl, s, m->face2cell[2 * f], m->face2cell[2 * f + 1], m->face_unit_normal + 3 * (size_t) f, F);
}

/* AUSM (Liou & Steffen 1993): interface Mach number from the split Mach numbers of both sides,
 * interface pressure from the split pressures, and the convected quantities rho*c*(1,u,v,w,H) taken
 * from the upwind side of the interface Mach number. */
static void ausm_lr(const orc_flow *fl, const orc_state *s, int L, int R, const double *n, double F[5]) {
	const double g = fl->gamma;
	double cl = sqrt(g * s->p[L] / s->rho[L]);
	double cr = sqrt(g * s->p[R] / s->rho[R]);
	double Vl = s->u[L] * n[0] + s->v[L] * n[1] + s->w[L] * n[2];
	double Vr = s->u[R] * n[0] + s->v[R] * n[1] + s->w[R] * n[2];
	double Ml = Vl / cl, Mr = Vr / cr;
	double mp, pp, mm, pm;
	if (fabs(Ml) <= 1.0) {
		mp = 0.25 * (Ml + 1.0) * (Ml + 1.0);
		pp = mp * (2.0 - Ml);
	} else {
		mp = 0.5 * (Ml + fabs(Ml));
		pp = Ml > 0.0 ? 1.0 : 0.0;
	}
	if (fabs(Mr) <= 1.0) {
		mm = -0.25 * (Mr - 1.0) * (Mr - 1.0);
		pm = -mm * (2.0 + Mr);
	} else {
		mm = 0.5 * (Mr - fabs(Mr));
		pm = Mr < 0.0 ? 1.0 : 0.0;
	}
	double mi = mp + mm;
	double pi = pp * s->p[L] + pm * s->p[R];
	double ml = mi > 0.0 ? mi : 0.0, mr = mi < 0.0 ? mi : 0.0;
	double al = ml * (s->rho[L] * cl), ar = mr * (s->rho[R] * cr);
	F[0] = al + ar;
	F[1] = al * s->u[L] + ar * s->u[R] + pi * n[0];
	F[2] = al * s->v[L] + ar * s->v[R] + pi * n[1];
	F[3] = al * s->w[L] + ar * s->w[R] + pi * n[2];
	F[4] = al * s->H[L] + ar * s->H[R];
}

void orc_ausm(const orc_mesh *m, const orc_flow *fl, const orc_state *s, int f, double F[5]) {
	ausm_lr(fl, s, m->face2cell[2 * f], m->face2cell[2 * f + 1], m->face_unit_normal + 3 * (size_t) f, F);
}

static void face_flux(const orc_mesh *m, const orc_flow *fl, const orc_state *s, int f, double F[5]) {
	if (fl->scheme == 1) orc_ausm(m, fl, s, f, F);
	else orc_roe(m, fl, s, f, F);
}

/* Solver::Fc, src/solver/ConvectiveFluxesSchemes.cpp:167-187: physical flux of the ghost state. */
static void ghost_flux(const orc_state *s, int g, const double *n, double V, double F[5]) {
	double rho = s->rho[g];
	F[0] = rho * V;
	F[1] = rho * s->u[g] * V + s->p[g] * n[0];
	F[2] = rho * s->v[g] * V + s->p[g] * n[1];
	F[3] = rho * s->w[g] * V + s->p[g] * n[2];
	F[4] = rho * s->H[g] * V;
}

static int cmp_int(const void *a, const void *b) {
	int x = *(const int *) a, y = *(const int *) b;
	return (x > y) - (x < y);
}

static int *sorted_copy(const int *v, int n) {
	int *c = (int *) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
	if (!c) return NULL;
	if (n) memcpy(c, v, sizeof(int) * (size_t) n);
	qsort(c, (size_t) n, sizeof(int), cmp_int);
	return c;
}

static int contains(const int *sorted, int n, int key) {
	return n > 0 && bsearch(&key, sorted, (size_t) n, sizeof(int), cmp_int) != NULL;
}

/* EulerSolver::computeResidual, src/solver/EulerSolver.cpp:303-359: interior faces scatter
 * +F*S to the left and -F*S to the right cell, then boundary faces add to their interior cell:
 * wall -> pressure only (:331-339), symmetry -> Roe against the mirrored ghost (:343-346),
 * anything else -> physical flux of the ghost (:349-357).  The ghost lists are searched with
 * binary search over sorted copies as the reference does (sortGhostCells, :398-407). */
void orc_compute_residual(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double *R) {
	memset(R, 0, sizeof(double) * 5 * (size_t) m->n_cells);
	double F[5];
	for (int f = 0; f < m->n_faces_int; f++) {
		int L = m->face2cell[2 * f], Rc = m->face2cell[2 * f + 1];
		face_flux(m, fl, s, f, F);
		double S = m->face_area[f];
		for (int k = 0; k < 5; k++) {
			double t = F[k] * S;
			R[5 * (size_t) L + k] += t;
			R[5 * (size_t) Rc + k] -= t;
		}
	}
	int *wall = sorted_copy(m->wall_ghost, m->n_wall);
	int *sym = sorted_copy(m->sym_ghost, m->n_sym);
	for (int f = m->n_faces_int; f < m->n_faces; f++) {
		int L = m->face2cell[2 * f], G = m->face2cell[2 * f + 1];
		double S = m->face_area[f];
		const double *n = m->face_unit_normal + 3 * (size_t) f;
		if (contains(wall, m->n_wall, G)) {
			F[0] = 0;
			F[1] = n[0] * s->p[G];
			F[2] = n[1] * s->p[G];
			F[3] = n[2] * s->p[G];
			F[4] = 0;
		} else if (contains(sym, m->n_sym, G)) {
			face_flux(m, fl, s, f, F);
		} else {
			double V = s->u[G] * n[0] + s->v[G] * n[1] + s->w[G] * n[2];
			ghost_flux(s, G, n, V, F);
		}
		for (int k = 0; k < 5; k++) R[5 * (size_t) L + k] += F[k] * S;
	}
	free(wall);
	free(sym);
}

/* TimeStepMethod2, src/solver/TimeIntegration.cpp:8-40, for every interior cell
 * (EulerSolver::updateDeltaTime, src/solver/EulerSolver.cpp:362-367). */
void orc_time_step(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double *dt) {
	for (int c = 0; c < m->n_cells; c++) {
		double sx = 0, sy = 0, sz = 0;
		for (int k = m->cell2face_ptr[c]; k < m->cell2face_ptr[c + 1]; k++) {
			const double *S = m->face_normal + 3 * (size_t) m->cell2face[k];
			sx += fabs(S[0]);
			sy += fabs(S[1]);
			sz += fabs(S[2]);
		}
		double a = sqrt(fl->gamma * s->p[c] / s->rho[c]);
		double lx = 0.5 * (fabs(s->u[c]) + a) * sx;
		double ly = 0.5 * (fabs(s->v[c]) + a) * sy;
		double lz = 0.5 * (fabs(s->w[c]) + a) * sz;
		dt[c] = fl->cfl * m->cell_volume[c] / (lx + ly + lz);
	}
}

/* Primitive recovery of FlowField::Update / updateWRungeKutta (src/solver/FlowField.cpp:118-127,
 * :150-159) from the conservative state w of cell c. */
static void set_primitives(const orc_flow *fl, orc_state *s, int c, const double w[5]) {
	const double g = fl->gamma;
	double rho = w[0];
	double u = w[1] / rho, v = w[2] / rho, ww = w[3] / rho, E = w[4] / rho;
	double q2 = u * u + v * v + ww * ww;
	double p = (g - 1) * rho * (E - q2 / 2.0);
	s->rho[c] = rho;
	s->u[c] = u;
	s->v[c] = v;
	s->w[c] = ww;
	s->E[c] = E;
	s->p[c] = p;
	s->H[c] = E + (p / rho);
	s->M[c] = sqrt(g * (p / rho)) / sqrt(q2);
}

/* One stage: W = W0 - alpha*dt*R/V followed by FlowField::updateWRungeKutta's primitive recovery,
 * src/solver/EulerSolver.cpp:441-450 / :461-470 and src/solver/FlowField.cpp:140-171. */
static void rk_update(const orc_mesh *m, const orc_flow *fl, orc_state *s, const double *W0, const double *R,
                      const double *dt, double alpha) {
	for (int c = 0; c < m->n_cells; c++) {
		double vol = m->cell_volume[c];
		double w[5];
		for (int k = 0; k < 5; k++) w[k] = W0[5 * (size_t) c + k] - alpha * dt[c] * R[5 * (size_t) c + k] / vol;
		set_primitives(fl, s, c, w);
	}
}

/* EulerSolver::smoothResiduals, src/solver/EulerSolver.cpp:483-518.  The neighbours of cell c are
 * the other cells of its faces in element2face order, which is the reference's element2element
 * order (both are filled per local face, src/connectivity/Connectivity.cpp:184-218); ghost
 * neighbours count in the denominator but not in the sum.
 * The reference's loop runs at most two passes: each pass ends with diff.clear() (:514), so the
 * next pass measures its changes over an empty vector (its std::transform writes into the cleared
 * vector's storage, :505), finds error = 0 and leaves the loop.  One pass if the first pass's
 * largest change is <= 1e-16, otherwise exactly two; only the first pass is checked for NaN. */
static void smooth_pass(const orc_mesh *m, const double *orig, const double *last, double *R) {
	const double epsilon = 0.25;
	for (int c = 0; c < m->n_cells; c++) {
		double sum[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
		const int n_surr = m->cell2face_ptr[c + 1] - m->cell2face_ptr[c];
		for (int k = m->cell2face_ptr[c]; k < m->cell2face_ptr[c + 1]; k++) {
			const int f = m->cell2face[k];
			const int j = m->face2cell[2 * f] == c ? m->face2cell[2 * f + 1] : m->face2cell[2 * f];
			if (j < m->n_cells)
				for (int q = 0; q < 5; q++) sum[q] += last[5 * (size_t) j + q] * epsilon;
		}
		for (int q = 0; q < 5; q++) R[5 * (size_t) c + q] = (orig[5 * (size_t) c + q] + sum[q]) / (1 + n_surr * epsilon);
	}
}

long long orc_smooth_residuals(const orc_mesh *m, double *R) {
	const size_t n5 = 5 * (size_t) m->n_cells;
	double *orig = (double *) calloc(n5 ? n5 : 1, sizeof(double));
	double *last = (double *) calloc(n5 ? n5 : 1, sizeof(double));
	if (!orig || !last) {
		free(orig);
		free(last);
		return -1;
	}
	memcpy(orig, R, sizeof(double) * n5);
	memcpy(last, R, sizeof(double) * n5);
	smooth_pass(m, orig, last, R);
	double error = 0.0;
	for (size_t i = 0; i < n5; i++) {
		double d = fabs(last[i] - R[i]);
		if (isnan(d)) {
			free(orig);
			free(last);
			return -1;
		}
		if (d > error) error = d;
	}
	long long sweeps = 1;
	if (error > 1e-16) {
		memcpy(last, R, sizeof(double) * n5);
		smooth_pass(m, orig, last, R);
		sweeps = 2;
	}
	free(orig);
	free(last);
	return sweeps;
}

/* EulerSolver::EulerExplicit, src/solver/EulerSolver.cpp:419-423 (updateDeltaTime,
 * TimeIntegration :369-374 with ExplicitEuler src/solver/TimeIntegration.cpp:78-91, updateW). */
void orc_euler_explicit(const orc_mesh *m, const orc_flow *fl, orc_state *s, double *W, const double *R, double *dt) {
	orc_time_step(m, fl, s, dt);
	for (int c = 0; c < m->n_cells; c++) {
		double coeff = -dt[c] / m->cell_volume[c];
		double *w = W + 5 * (size_t) c;
		for (int q = 0; q < 5; q++) w[q] += R[5 * (size_t) c + q] * coeff;
		set_primitives(fl, s, c, w);
	}
}

/* EulerSolver::RungeKutta, src/solver/EulerSolver.cpp:425-472 */
long long orc_runge_kutta(const orc_mesh *m, const orc_flow *fl, orc_state *s, double *R, double *dt) {
	static const double alphas[4] = {0.1263, 0.2375, 0.4414, 1.0};
	long long sweeps = 0;
	double *W0 = (double *) malloc(sizeof(double) * 5 * (size_t) (m->n_cells > 0 ? m->n_cells : 1));
	if (!W0) return -1;
	for (int c = 0; c < m->n_cells; c++) { /* W0 from the primitives, :431-438 */
		double rho = s->rho[c];
		W0[5 * (size_t) c + 0] = rho;
		W0[5 * (size_t) c + 1] = s->u[c] * rho;
		W0[5 * (size_t) c + 2] = s->v[c] * rho;
		W0[5 * (size_t) c + 3] = s->w[c] * rho;
		W0[5 * (size_t) c + 4] = s->E[c] * rho;
	}
	orc_time_step(m, fl, s, dt);
	rk_update(m, fl, s, W0, R, dt, 0.0533);
	for (int k = 0; k < 4; k++) {
		orc_update_bc(m, fl, s);
		orc_compute_residual(m, fl, s, R);
		if (fl->smoothing) {
			long long n = orc_smooth_residuals(m, R);
			if (n < 0) {
				free(W0);
				return -1;
			}
			sweeps += n;
		}
		orc_time_step(m, fl, s, dt);
		rk_update(m, fl, s, W0, R, dt, alphas[k]);
	}
	free(W0);
	return sweeps;
}

double orc_rms(const orc_mesh *m, const double *R) {
	double sum = 0.0;
	for (int c = 0; c < m->n_cells; c++) sum += R[5 * (size_t) c] * R[5 * (size_t) c];
	return sqrt(sum / m->n_cells);
}

/* AeroCoefficients ctor + Update, src/solver/AeroCoefficients.cpp:5-52.  The centre-of-pressure
 * division at :48 is a no-op in the reference (Vector3::operator/= returns a copy,
 * include/utils/Vector3.h:107-109), so the lever arm uses the plain sum of coeff*centroid. */
void orc_aero_coefficients(const orc_mesh *m, const orc_flow *fl, const orc_state *s, double force[3],
                           double moment[3]) {
	double u2 = fl->u_inf * fl->u_inf + fl->v_inf * fl->v_inf + fl->w_inf * fl->w_inf;
	double cpf = 1 / (0.5 * fl->rho_inf * u2);
	double F[3] = {0, 0, 0}, CP[3] = {0, 0, 0};
	for (int i = 0; i < m->n_wall; i++) {
		int cell = m->wall_interior[i];
		const double *S = m->face_normal + 3 * (size_t) m->wall_face[i];
		const double *x = m->face_center + 3 * (size_t) m->wall_face[i];
		double cp = cpf * (s->p[cell] - fl->p_inf);
		for (int k = 0; k < 3; k++) {
			double coeff = S[k] * cp * fl->cref / fl->sref;
			F[k] += coeff;
			CP[k] += coeff * x[k];
		}
	}
	double lever[3] = {fl->ref_point[0] - CP[0], fl->ref_point[1] - CP[1], fl->ref_point[2] - CP[2]};
	moment[0] = (F[1] * lever[2] - F[2] * lever[1]) / fl->cref;
	moment[1] = (F[2] * lever[0] - F[0] * lever[2]) / fl->cref;
	moment[2] = (F[0] * lever[1] - F[1] * lever[0]) / fl->cref;
	force[0] = F[0];
	force[1] = F[1];
	force[2] = F[2];
}

/* EulerSolver::Run, src/solver/EulerSolver.cpp:60-167, with ConvergenceCriteria :261-279 and the
 * CL/CD/CM selection of PrintInfo :253-256. */
int orc_run(const orc_mesh *m, const orc_flow *fl, orc_state *s, const orc_run_params *rp, orc_run_stats *st) {
	double *R = (double *) malloc(sizeof(double) * 5 * (size_t) (m->n_cells > 0 ? m->n_cells : 1));
	double *dt = (double *) malloc(sizeof(double) * (size_t) (m->n_cells > 0 ? m->n_cells : 1));
	double *W = NULL;
	if (fl->integrator == 1) W = (double *) malloc(sizeof(double) * 5 * (size_t) (m->n_cells > 0 ? m->n_cells : 1));
	if (!R || !dt || (fl->integrator == 1 && !W)) {
		free(R);
		free(dt);
		free(W);
		return -1;
	}
	memset(st, 0, sizeof *st);
	if (W) /* FlowField's conservative arrays, FlowField::Initialize (src/solver/FlowField.cpp:86-95) */
		for (int c = 0; c < m->n_cells; c++) {
			double rho = s->rho[c];
			W[5 * (size_t) c + 0] = rho;
			W[5 * (size_t) c + 1] = rho * s->u[c];
			W[5 * (size_t) c + 2] = rho * s->v[c];
			W[5 * (size_t) c + 3] = rho * s->w[c];
			W[5 * (size_t) c + 4] = rho * s->E[c];
		}
	int it = 0, counter = 0;
	double cl = 0, cd = 0, cm = 0;
	int sampling = rp->sampling > 0 ? rp->sampling : 1;
	while (it < rp->max_iter) {
		orc_update_bc(m, fl, s);
		orc_compute_residual(m, fl, s, R);
		if (fl->smoothing) {
			long long n = orc_smooth_residuals(m, R);
			if (n < 0) {
				st->converged = 3;
				break;
			}
			st->smooth_sweeps += n;
		}
		if (fl->integrator == 1) {
			orc_euler_explicit(m, fl, s, W, R, dt);
		} else {
			long long n = orc_runge_kutta(m, fl, s, R, dt);
			if (n < 0) {
				st->converged = 3;
				break;
			}
			st->smooth_sweeps += n;
		}
		double rms = orc_rms(m, R);
		if (rp->rms_history) rp->rms_history[st->n_rms] = rms;
		st->n_rms++;
		st->last_rms = rms;
		if (rms < rp->min_residual) {
			st->converged = 1;
			break;
		}
		it += 1;
		if (it % sampling == 0) {
			double old[3] = {cl, cd, cm};
			orc_aero_coefficients(m, fl, s, st->force, st->moment);
			cl = st->force[fl->cl_axis] * fl->cl_sign;
			cd = st->force[fl->cd_axis] * fl->cd_sign;
			cm = st->moment[fl->cm_axis] * fl->cm_sign;
			double tol = rp->min_aerocoeff_error;
			int ok = fabs(old[0] - cl) < tol && fabs(old[1] - cd) < tol && fabs(old[2] - cm) < tol;
			counter = ok ? counter + 1 : 0;
			if (counter >= 2) {
				st->converged = 2;
				break;
			}
		}
	}
	st->iterations = it;
	st->cl = cl;
	st->cd = cd;
	st->cm = cm;
	free(R);
	free(dt);
	free(W);
	return 0;
}
