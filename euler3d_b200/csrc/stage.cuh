// Device code of one Runge-Kutta stage of the Euler3D explicit solver, templated on the
// arithmetic policy.  Included by stage_exact.cu (compiled with -fmad=false: every double
// operation in the reference's order, no contraction) and stage_fast.cu (restructured
// arithmetic with FMA, one reciprocal per face, rsqrt instead of sqrt + divide).
//
// Layout on the device (cells in a locality order chosen on the host):
//   cptr[N+1], cf[M]  CSR of each cell's faces sorted by the reference face id, so a cell adds
//                     its face contributions in exactly the order the reference's face loop
//                     does (src/solver/EulerSolver.cpp:306-358) -> deterministic, no atomics.
//                     cf.x = (index << 3) | tag, cf.y = face geometry slot.
//   fgeo[F]           double4 (unit normal x,y,z ; area)
//   cgeo[N]           double4 (sum|Sx|, sum|Sy|, sum|Sz| over the cell's faces ; volume)
//   q[2][3N]          double2 x3 per cell: (rho,u) (v,w) (p,H), ping-pong between stages
//   w0[5 x stride]    conservative state at the start of the RK step (SoA, stride = N rounded up
//                     to 32 so that every tile's segment is 16-byte aligned for bulk copies)
//   ecell[N]          energy E of the last completed RK step (or of the loaded state)
//   ghost[8G]         ghost cells, 8 doubles each: rho u v w p E H M
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "euler3d_b200.h"

namespace e3d {

enum : int { TAG_LEFT = 0, TAG_RIGHT = 1, TAG_WALL = 2, TAG_SYM = 3, TAG_FAR = 4, TAG_FROZEN = 5 };
constexpr int kTagBits = 3;
// Threads per block of the stage kernels, and cells per face tile.  Of tiles of 64, 128 and 256
// cells, 128 ran the FP64 tile stage fastest on B200 (12.6M tetrahedra: 0.97, 0.85 and 0.93 ms):
// more, smaller blocks per SM interleave their load and compute phases better, until the halo
// share of smaller tiles costs more than that gains.
constexpr int kStageThreads = 128;
constexpr int kTileCells = kStageThreads;   // cells owned by one face tile (one per thread)
constexpr int kTileLocalBits = 10;          // local (owned + halo) cell index in a tile face entry
constexpr unsigned short kNoContrib = 0xFFFF;

struct Freestream {
    double rho, u, v, w, p, E, H, M;
};

// Run control shared by the kernels of e3d_solver_run; lives in device memory.
struct Control {
    int done;          // nonzero: every later kernel returns at once
    int stop_reason;   // E3D_STOP_*
    int it;            // EulerSolver::_nbInteration
    int n_rms;         // iterations whose RMS has been computed
    int counter;       // consecutive stagnated coefficient samples (src/solver/EulerSolver.cpp:142-147)
    int sample_now;    // this iteration samples the force coefficients
    int minit_valid;   // interior Mach of the loaded state still holds (no stage has run since)
    int nonfinite;     // the RMS became NaN/Inf
    int max_iter, sampling, hist_cap;
    int fault;         // a bounded wait in a kernel gave up
    double min_res, min_aero, last_rms, cl, cd, cm;
    double min_drop;   // > 0: also stop once the RMS is below min_drop x the run's first RMS
    double rms0;       // RMS of the run's first iteration
    int n_samples;     // coefficient samples taken (residuals.dat rows)
    int sample_cap;    // capacity of the sample record
    int stall_window;  // > 0: stop once the RMS has set no new minimum for this many iterations
    int since_best;    // iterations since the RMS last set a new minimum
    double best_rms;   // smallest RMS of the run so far
    double stall_below;  // the stall test counts only once RMS < stall_below x the first RMS (0: always)
    double force[3], moment[3];
};

struct StageArgs {
    int n_cells, n_ghosts;
    const int *__restrict__ cptr;
    const int2 *__restrict__ cf;
    const double4 *__restrict__ fgeo;
    const double4 *__restrict__ cgeo;
    const double2 *__restrict__ qin;
    double2 *__restrict__ qout;
    double *__restrict__ w0;
    double *__restrict__ ecell;
    const double *__restrict__ minit;
    double *__restrict__ ghost;
    double *__restrict__ partials;   // per-block sum of R_rho^2 (last stage only)
    Control *ctl;
    Freestream fs;
    double gamma, cfl, alpha;
    int scheme;                      // E3D_SCHEME_ROE or E3D_SCHEME_AUSM (uniform: no divergence)
    int first_stage;                 // stage 1 of an iteration (may read the loaded interior Mach)
    int last_stage;                  // stage 5: write W0/E for the next step and the RMS partials
    int residual_only;               // e3d_solver_residual: write R and dt, leave the state
    double *__restrict__ r_out;      // [5N] reference order (residual_only)
    double *__restrict__ dt_out;     // [N]  reference order (residual_only)
    const int *__restrict__ new2old;
    int w0_stride;                   // row stride of w0
    // face-tile kernel: tile t owns cells [t*kTileCells, ...); its halo cells, face records and
    // the per-cell contribution lists (see tile_kernel)
    const int *__restrict__ tile_halo_ptr;   // halo count of tile t = ptr[t+1] - ptr[t]
    const int *__restrict__ tile_halo;       // halo cells of tile t at [t * halo_stride, ...), then -1
    const int *__restrict__ tile_face_ptr;   // face count of tile t = ptr[t+1] - ptr[t]
    const char *__restrict__ tile_rec;       // FaceRec blocks, one 16-byte aligned block per tile
    const long long *__restrict__ tile_rec_off;  // byte offset of tile t's block
    const unsigned short *__restrict__ tile_contrib;
    int max_contrib;                 // contribution slots per cell (max faces of a cell)
    int smem_cells;                  // max owned + halo cells of a tile
    int smem_faces;                  // max faces of a tile
    int *fault;                      // set when a bounded wait gives up (reported as a timeout)
    int halo_stride;                 // entries per tile in tile_halo (the largest halo)
    int n_tiles;                     // tiles of the mesh
    int pipe_grid;                   // tile_ws_kernel: persistent blocks (one per SM)
    int ws_buffers;                  // tile_ws_kernel: tile buffers in shared memory
    // FP32_FLUX mode: float cell records (rho,u,v,w | p,H,sqrt(rho),rsqrt(gamma p rho)), float
    // face records and float cell geometry; W0 stays double
    const float4 *__restrict__ q32in;
    float4 *__restrict__ q32out;
    const char *__restrict__ tile_rec32;
    const long long *__restrict__ tile_rec32_off;
    const float4 *__restrict__ cgeo32;
    int integrator;                  // E3D_INTEGRATOR_RK5 or E3D_INTEGRATOR_EULER (uniform)
    int split;                       // residual phase of a split stage: write R to r_dev, no update
    double *__restrict__ r_dev;      // [5 x w0_stride] residual of a split stage (device order); the
                                     // update phase reads the smoothed residual from here
    double *__restrict__ rsq;        // FP64_EXACT: R_rho^2 of every cell in reference order (last stage),
                                     // summed sequentially like EulerSolver::computeRMS; else null
    int wait_polls;                  // polls of a tile's data barrier before the wait gives up (kWaitLimit;
                                     // fewer, down to 0, only to exercise the timeout path)
    int ghost_out;                   // write wall / symmetry ghost records although this is not a last
                                     // stage (the residual phase of a split last stage)
};

// One face of a tile: code = l | r << 10 | tag << 20 (local cell indices; r unused for boundary
// faces), ghost slot for boundary faces, unit normal and area.
struct FaceRec {
    int code;
    int ghost;
    double nx, ny, nz, S;
};
static_assert(sizeof(FaceRec) == 40, "FaceRec layout");

// FP32_FLUX mode face record.
struct FaceRec32 {
    int code;
    int ghost;
    float nx, ny, nz, S;
};
static_assert(sizeof(FaceRec32) == 24, "FaceRec32 layout");

struct Prim {
    double rho, u, v, w, p, H;
};

__device__ __forceinline__ Prim load_prim(const double2 *__restrict__ q, int c) {
    double2 a = q[3 * c], b = q[3 * c + 1], d = q[3 * c + 2];
    return Prim{a.x, a.y, b.x, b.y, d.x, d.y};
}

__device__ __forceinline__ void store_prim(double2 *__restrict__ q, int c, const Prim &s) {
    q[3 * c] = make_double2(s.rho, s.u);
    q[3 * c + 1] = make_double2(s.v, s.w);
    q[3 * c + 2] = make_double2(s.p, s.H);
}

// store_prim with streaming stores (st.global.cs): a stage's new states are read back only by the
// next stage, after far more traffic than L2 holds on large meshes.
__device__ __forceinline__ void store_prim_cs(double2 *__restrict__ q, int c, const Prim &s) {
    __stcs(q + 3 * c, make_double2(s.rho, s.u));
    __stcs(q + 3 * c + 1, make_double2(s.v, s.w));
    __stcs(q + 3 * c + 2, make_double2(s.p, s.H));
}

// ------------------------------------------------------------------------------ fast reciprocals
// FP64 path only (never FP64_EXACT): reciprocal and reciprocal square root from the single-
// precision hardware approximations (PTX rcp.approx.ftz.f32 / rsqrt.approx.ftz.f32, relative error
// below 2^-22), refined in one step by the truncated series of the exact correction.  With the seed
// y0 and e = 1 - x y0 (|e| < 2^-22), 1/x = y0 / (1 - e) = y0 (1 + e + e^2 + ...); with
// e = 1 - x y0^2, 1/sqrt(x) = y0 (1 - e)^(-1/2) = y0 (1 + e/2 + 3e^2/8 + ...).  Keeping the terms up
// to e^2 leaves a truncation error of order e^3 < 2^-66, far below double rounding: over 10^7 random
// arguments and seed errors the results were within 1 (reciprocal) and 2 (reciprocal square root)
// units in the last place of the correctly rounded values, where two Newton-Raphson steps (each
// squares the error; Markstein, IBM J. Res. Dev. 34, 1990) gave up to 3, with a longer dependency
// chain and more operations.  The seed is used when the single-precision argument lies in
// [2^-99, 2^99) (its bits, sign included, between 0x0E000000 and 0x71000000: one integer compare
// instead of two double-precision ones), so that seed and result are normal floats; anything else
// (zero, tiny or huge magnitudes, negative arguments of the square root, NaN and Inf) takes the IEEE
// double operation.
__device__ __forceinline__ bool seed_ok(float xf) {
    return __float_as_uint(xf) - 0x0E000000u < 0x63000000u;
}

__device__ __forceinline__ double rcp_nr(double x) {
    const float xf = (float)x;
    if (!seed_ok(fabsf(xf))) return 1.0 / x;
    float yf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(xf));
    const double y = (double)yf;
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);  // y (1 + e + e^2)
}

__device__ __forceinline__ double rsqrt_nr(double x) {
    const float xf = (float)x;
    if (!seed_ok(xf)) return rsqrt(x);
    float yf;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(xf));
    const double y = (double)yf;
    const double e = fma(-(x * y), y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);  // y (1 + e/2 + 3e^2/8)
}

// ------------------------------------------------------------------------------ Roe flux
// Exact: Solver::Roe (src/solver/ConvectiveFluxesSchemes.cpp:10-165) operation by operation.
__device__ __forceinline__ void roe_exact(const Prim &L, const Prim &R, double nx, double ny, double nz,
                                          double g, double F[5]) {
    double sl = sqrt(L.rho), sr = sqrt(R.rho);
    double rt = sqrt(L.rho * R.rho);
    double ut = (L.u * sl + R.u * sr) / (sl + sr);
    double vt = (L.v * sl + R.v * sr) / (sl + sr);
    double wt = (L.w * sl + R.w * sr) / (sl + sr);
    double ht = (L.H * sl + R.H * sr) / (sl + sr);
    double q2t = ut * ut + vt * vt + wt * wt;
    double ct = sqrt((g - 1.0) * (ht - q2t / 2));
    double Vt = ut * nx + vt * ny + wt * nz;
    double Vl = L.u * nx + L.v * ny + L.w * nz;
    double Vr = R.u * nx + R.v * ny + R.w * nz;
    double drho = R.rho - L.rho, du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w, dp = R.p - L.p, dV = Vr - Vl;
    double cl = sqrt(g * L.p / L.rho);
    double delta = (1.0 / 15.0) * cl;
    double lam1 = fabs(Vt - ct);
    if (!(fabs(Vt - ct) > delta)) lam1 = ((Vt - ct) * (Vt - ct) + delta * delta) / (2.0 * delta);
    double lam5 = fabs(Vt + ct);
    if (!(fabs(Vt + ct) > delta)) lam5 = ((Vt + ct) * (Vt + ct) + delta * delta) / (2.0 * delta);
    double c2x2 = 2.0 * (ct * ct);
    double s1 = dp - rt * ct * dV, s5 = dp + rt * ct * dV, s2 = drho - dp / (ct * ct), aV = fabs(Vt);
    double n[3] = {nx, ny, nz};
    double ulr[3][2] = {{L.u, R.u}, {L.v, R.v}, {L.w, R.w}};
    double tl[3] = {ut, vt, wt};
    double dd[3] = {du, dv, dw};
    // mass
    {
        double favg = (R.rho * Vr + L.rho * Vl) * 0.5;
        double d1 = 1.0 * lam1 * s1 / c2x2;
        double d234 = (1.0 * s2 + 0.0) * aV;
        double d5 = 1.0 * lam5 * s5 / c2x2;
        F[0] = favg - 0.5 * (d1 + d234 + d5);
    }
    // momentum
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double fr = R.rho * Vr * ulr[k][1] + R.p * n[k];
        double fl = L.rho * Vl * ulr[k][0] + L.p * n[k];
        double d1 = (tl[k] - ct * n[k]) * lam1 * s1 / c2x2;
        double d234 = (tl[k] * s2 + rt * (dd[k] - dV * n[k])) * aV;
        double d5 = (tl[k] + ct * n[k]) * lam5 * s5 / c2x2;
        F[1 + k] = (fr + fl) * 0.5 - 0.5 * (d1 + d234 + d5);
    }
    // energy
    {
        double fr = R.rho * Vr * R.H, fl = L.rho * Vl * L.H;
        double d1 = (ht - ct * Vt) * lam1 * s1 / c2x2;
        double d234 = (q2t * 0.5 * s2 + rt * (ut * du + vt * dv + wt * dw - Vt * dV)) * aV;
        double d5 = (ht + ct * Vt) * lam5 * s5 / c2x2;
        F[4] = (fr + fl) * 0.5 - 0.5 * (d1 + d234 + d5);
    }
}

// Fast: the same flux rearranged as F = (F_L + F_R - sum_k a_k r_k) / 2 with the wave strengths
// a_k formed once, Roe weights from one reciprocal, c~ and 1/c~^2 from one rsqrt, and the left
// sound speed from rsqrt(gamma p rho).  sl, sr = sqrt(rho) and rcl = rsqrt(gamma p_L rho_L) come
// from the caller (the gather kernel computes them once per cell, the tile kernels once per face).
// The FP64 kernels are compiled without multiply-add contraction and fuse where the source says
// fma(), so the rounding is fixed by the source: every kernel variant, alone or batched, computes
// the same bits whatever its register budget.
__device__ __forceinline__ void roe_fast(const Prim &L, const Prim &R, double sl, double sr, double rcl,
                                         double nx, double ny, double nz, double g, double F[5]) {
    double inv = rcp_nr(sl + sr);
    double wl = sl * inv, wr = sr * inv;
    double ut = fma(L.u, wl, R.u * wr);
    double vt = fma(L.v, wl, R.v * wr);
    double wt = fma(L.w, wl, R.w * wr);
    double ht = fma(L.H, wl, R.H * wr);
    double rt = sl * sr;
    double q2t = fma(ut, ut, fma(vt, vt, wt * wt));
    double c2 = (g - 1.0) * fma(-0.5, q2t, ht);
    double rc = rsqrt_nr(c2);
    double ct = c2 * rc, ic2 = rc * rc;
    double Vt = fma(ut, nx, fma(vt, ny, wt * nz));
    double Vl = fma(L.u, nx, fma(L.v, ny, L.w * nz));
    double Vr = fma(R.u, nx, fma(R.v, ny, R.w * nz));
    double drho = R.rho - L.rho, dp = R.p - L.p, dV = Vr - Vl;
    double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
    // Harten's fix with delta = c_L / 15 (c_L = gamma p_L * rsqrt(gamma p_L rho_L))
    double gpl = g * L.p;
    double delta = (1.0 / 15.0) * (gpl * rcl);
    double lam1 = fabs(Vt - ct), lam5 = fabs(Vt + ct);
    if (!(lam1 > delta) || !(lam5 > delta)) {
        double h = 7.5 * (L.rho * rcl);  // 1 / (2 delta)
        if (!(lam1 > delta)) lam1 = fma(lam1, lam1, delta * delta) * h;
        if (!(lam5 > delta)) lam5 = fma(lam5, lam5, delta * delta) * h;
    }
    double rcdv = rt * ct * dV;
    double a1 = 0.5 * lam1 * (dp - rcdv) * ic2;
    double a5 = 0.5 * lam5 * (dp + rcdv) * ic2;
    double aV = fabs(Vt);
    double a2 = aV * fma(-dp, ic2, drho);
    double a3 = aV * rt;
    double a15 = a1 + a5, d51 = (a5 - a1) * ct, asum = a15 + a2;
    double mL = L.rho * Vl, mR = R.rho * Vr, pp = L.p + R.p;
    F[0] = 0.5 * (mL + mR - asum);
    F[1] = 0.5 * (fma(mL, L.u, fma(mR, R.u, pp * nx)) - fma(asum, ut, fma(d51, nx, a3 * fma(-dV, nx, du))));
    F[2] = 0.5 * (fma(mL, L.v, fma(mR, R.v, pp * ny)) - fma(asum, vt, fma(d51, ny, a3 * fma(-dV, ny, dv))));
    F[3] = 0.5 * (fma(mL, L.w, fma(mR, R.w, pp * nz)) - fma(asum, wt, fma(d51, nz, a3 * fma(-dV, nz, dw))));
    F[4] = 0.5 * (fma(mL, L.H, mR * R.H) -
                  fma(a15, ht, fma(d51, Vt, fma(a2, 0.5 * q2t, a3 * fma(-Vt, dV, fma(ut, du, fma(vt, dv, wt * dw)))))));
}

// ------------------------------------------------------------------------------ AUSM flux
// AUSM of Liou & Steffen (J. Comput. Phys. 107, 23-39, 1993).  Exact: the oracle's operation order
// (oracle/e3d_oracle.c ausm_lr).  Fast: sound speeds from rsqrt(gamma p rho) (rl, rr from the caller).
__device__ __forceinline__ void ausm_split(double M, double &mp, double &pp, double &mm, double &pm, bool left) {
    if (left) {
        if (fabs(M) <= 1.0) {
            mp = 0.25 * (M + 1.0) * (M + 1.0);
            pp = mp * (2.0 - M);
        } else {
            mp = 0.5 * (M + fabs(M));
            pp = M > 0.0 ? 1.0 : 0.0;
        }
    } else {
        if (fabs(M) <= 1.0) {
            mm = -0.25 * (M - 1.0) * (M - 1.0);
            pm = -mm * (2.0 + M);
        } else {
            mm = 0.5 * (M - fabs(M));
            pm = M < 0.0 ? 1.0 : 0.0;
        }
    }
}

__device__ __forceinline__ void ausm_tail(const Prim &L, const Prim &R, double cl, double cr, double Vl, double Vr,
                                          double Ml, double Mr, double nx, double ny, double nz, double F[5]) {
    double mp = 0, pp = 0, mm = 0, pm = 0;
    ausm_split(Ml, mp, pp, mm, pm, true);
    ausm_split(Mr, mp, pp, mm, pm, false);
    (void)Vl;
    (void)Vr;
    double mi = mp + mm;
    double pi = pp * L.p + pm * R.p;
    double ml = mi > 0.0 ? mi : 0.0, mr = mi < 0.0 ? mi : 0.0;
    double al = ml * (L.rho * cl), ar = mr * (R.rho * cr);
    F[0] = al + ar;
    F[1] = al * L.u + ar * R.u + pi * nx;
    F[2] = al * L.v + ar * R.v + pi * ny;
    F[3] = al * L.w + ar * R.w + pi * nz;
    F[4] = al * L.H + ar * R.H;
}

__device__ __forceinline__ void ausm_exact(const Prim &L, const Prim &R, double nx, double ny, double nz, double g,
                                           double F[5]) {
    double cl = sqrt(g * L.p / L.rho);
    double cr = sqrt(g * R.p / R.rho);
    double Vl = L.u * nx + L.v * ny + L.w * nz;
    double Vr = R.u * nx + R.v * ny + R.w * nz;
    ausm_tail(L, R, cl, cr, Vl, Vr, Vl / cl, Vr / cr, nx, ny, nz, F);
}

__device__ __forceinline__ void ausm_fast(const Prim &L, const Prim &R, double rl, double rr, double nx, double ny,
                                          double nz, double g, double F[5]) {
    // c = gamma p / sqrt(gamma p rho); 1/c = rho / sqrt(gamma p rho)
    double cl = g * L.p * rl, cr = g * R.p * rr;
    double Vl = fma(L.u, nx, fma(L.v, ny, L.w * nz));
    double Vr = fma(R.u, nx, fma(R.v, ny, R.w * nz));
    ausm_tail(L, R, cl, cr, Vl, Vr, Vl * (L.rho * rl), Vr * (R.rho * rr), nx, ny, nz, F);
}

// ------------------------------------------------------------------------------ ghost states
// Ghost record: rho u v w p E H M.
__device__ __forceinline__ void ghost_store(double *gp, double rho, double u, double v, double w, double p,
                                            double E, double H, double M) {
    double2 *g2 = reinterpret_cast<double2 *>(gp);
    g2[0] = make_double2(rho, u);
    g2[1] = make_double2(v, w);
    g2[2] = make_double2(p, E);
    g2[3] = make_double2(H, M);
}

// Tail shared by subsonic farfield, wall and symmetry ghosts (src/solver/PhysicalBC.cpp:62-66).
__device__ __forceinline__ void ghost_finish(double *gp, double g, double rho, double u, double v, double w,
                                             double p, double c, Prim &out) {
    double q2 = u * u + v * v + w * w;
    double M = sqrt(q2) / c;
    double E = p / ((g - 1) * rho) + (q2 / 2.0);
    double H = E + (p / rho);
    ghost_store(gp, rho, u, v, w, p, E, H, M);
    out = Prim{rho, u, v, w, p, H};
}

// BC::Wall / BC::Symmetry (src/solver/PhysicalBC.cpp:124-231): mirrored velocity.  The kernels
// never read a wall or symmetry ghost back (it is rebuilt from its interior cell at every stage), so
// its record is written only when `store` says so (the last stage of an iteration, and
// e3d_solver_residual): the state a run leaves is the same, with a fifth of the ghost writes.
// Without the store only what the face flux needs is formed (H for symmetry faces).
__device__ __forceinline__ void ghost_mirror(double *gp, double g, const Prim &d, double nx, double ny, double nz,
                                             Prim &out, bool store, bool need_h) {
    double V = d.u * nx + d.v * ny + d.w * nz;
    double u = d.u - 2 * V * nx;
    double v = d.v - 2 * V * ny;
    double w = d.w - 2 * V * nz;
    if (store) {
        double c = sqrt(g * (d.p / d.rho));
        ghost_finish(gp, g, d.rho, u, v, w, d.p, c, out);
    } else {
        double H = 0.0;
        if (need_h) {  // ghost_finish's E and H, in its operation order
            double q2 = u * u + v * v + w * w;
            double E = d.p / ((g - 1) * d.rho) + (q2 / 2.0);
            H = E + (d.p / d.rho);
        }
        out = Prim{d.rho, u, v, w, d.p, H};
    }
}

// Farfield ghost (EulerSolver::updateBC, src/solver/EulerSolver.cpp:205-227): the branch comes
// from the ghost's previous Mach and normal velocity; d_M / d_E are the interior Mach and energy.
__device__ __forceinline__ void ghost_farfield(double *gp, double g, const Freestream &fs, const Prim &d,
                                               double d_M, double d_E, double nx, double ny, double nz,
                                               Prim &out) {
    double2 gu = reinterpret_cast<const double2 *>(gp)[0];
    double2 gv = reinterpret_cast<const double2 *>(gp)[1];
    double gM = gp[7];
    double V = gu.y * nx + gv.x * ny + gv.y * nz;
    if (gM >= 1.0 && V > 0.0) {  // BC::FarfieldSupersonicOutflow, PhysicalBC.cpp:26-40
        ghost_store(gp, d.rho, d.u, d.v, d.w, d.p, d_E, d.H, d_M);
        out = d;
    } else if (gM < 1.0 && V > 0.0) {  // BC::FarfieldSubsonicOutflow, PhysicalBC.cpp:82-121
        double c = sqrt(g * (d.p / d.rho));
        double p = fs.p;
        double rho = d.rho + (p - d.p) / (c * c);
        double u = d.u + nx * (d.p - p) / (d.rho * c);
        double v = d.v + ny * (d.p - p) / (d.rho * c);
        double w = d.w + nz * (d.p - p) / (d.rho * c);
        ghost_finish(gp, g, rho, u, v, w, p, c, out);
    } else if (gM >= 1.0 && V <= 0.0) {  // BC::FarfieldSupersonicInflow, PhysicalBC.cpp:11-23
        ghost_store(gp, fs.rho, fs.u, fs.v, fs.w, fs.p, fs.E, fs.H, fs.M);
        out = Prim{fs.rho, fs.u, fs.v, fs.w, fs.p, fs.H};
    } else if (gM < 1.0 && V <= 0.0) {  // BC::FarfieldSubsonicInflow, PhysicalBC.cpp:43-79
        double c = sqrt(g * (d.p / d.rho));
        double p = 0.5 * (fs.p + d.p - d.rho * c * ((nx * (fs.u - d.u)) + (ny * (fs.v - d.v)) + (nz * (fs.w - d.w))));
        double rho = fs.rho + (p - fs.p) / (c * c);
        double u = fs.u - nx * (fs.p - p) / (d.rho * c);
        double v = fs.v - ny * (fs.p - p) / (d.rho * c);
        double w = fs.w - nz * (fs.p - p) / (d.rho * c);
        ghost_finish(gp, g, rho, u, v, w, p, c, out);
    } else {  // NaN Mach or velocity: the reference leaves the ghost as it is
        double2 gph = reinterpret_cast<const double2 *>(gp)[2];
        out = Prim{gu.x, gu.y, gv.x, gv.y, gph.x, gp[6]};
    }
}

// Physical flux of a ghost state with V = u_ghost . n (Solver::Fc, ConvectiveFluxesSchemes.cpp:167-187).
__device__ __forceinline__ void ghost_flux(const Prim &s, double nx, double ny, double nz, double F[5]) {
    double V = s.u * nx + s.v * ny + s.w * nz;
    F[0] = s.rho * V;
    F[1] = s.rho * s.u * V + s.p * nx;
    F[2] = s.rho * s.v * V + s.p * ny;
    F[3] = s.rho * s.w * V + s.p * nz;
    F[4] = s.rho * s.H * V;
}

// ------------------------------------------------------------------------------ shared pieces
template <int NT = kStageThreads>
__device__ __forceinline__ void block_sum_store(double v, double *dst) {
    __shared__ double warp_sums[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < NT / 32 ? warp_sums[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) *dst = v;
    }
}

// Boundary face of interior cell c (state me): updates its ghost cell (EulerSolver::updateBC,
// src/solver/EulerSolver.cpp:201-251) and either writes the face flux to F (wall: pressure term,
// :331-339; farfield / unclassified: physical flux of the ghost, :349-357) and returns false, or
// leaves the mirrored ghost in gs and returns true (symmetry: Roe against the ghost, :343-346).
__device__ __forceinline__ bool boundary_face(const StageArgs &a, int tag, double *gp, int c, const Prim &me,
                                              const double4 &fg, double F[5], Prim &gs) {
    const double g = a.gamma;
    const bool store = a.last_stage || a.residual_only || a.ghost_out;
    if (tag == TAG_WALL) {
        ghost_mirror(gp, g, me, fg.x, fg.y, fg.z, gs, store, false);
        F[0] = 0;
        F[1] = fg.x * gs.p;
        F[2] = fg.y * gs.p;
        F[3] = fg.z * gs.p;
        F[4] = 0;
        return false;
    }
    if (tag == TAG_SYM) {
        ghost_mirror(gp, g, me, fg.x, fg.y, fg.z, gs, store, true);
        return true;
    }
    if (tag == TAG_FAR) {
        double q2 = me.u * me.u + me.v * me.v + me.w * me.w;
        // interior Mach as FlowField stores it (c/|u|, FlowField.cpp:157) unless the loaded state's
        // still holds; E is exact at stage 1 (ecell), recomputed from H at later stages
        double dM = (a.first_stage && a.ctl->minit_valid) ? a.minit[c] : sqrt(g * (me.p / me.rho)) / sqrt(q2);
        double dE = a.first_stage ? a.ecell[c] : me.H - me.p / me.rho;
        ghost_farfield(gp, g, a.fs, me, dM, dE, fg.x, fg.y, fg.z, gs);
    } else {  // unclassified boundary: the ghost keeps its (freestream) state
        double2 g0 = reinterpret_cast<const double2 *>(gp)[0];
        double2 g1 = reinterpret_cast<const double2 *>(gp)[1];
        double2 g2 = reinterpret_cast<const double2 *>(gp)[2];
        gs = Prim{g0.x, g0.y, g1.x, g1.y, g2.x, gp[6]};
    }
    ghost_flux(gs, fg.x, fg.y, fg.z, F);
    return false;
}

// Time step, Runge-Kutta update and primitive recovery of cell c from its residual R, the cell's
// W0 and geometry; returns this cell's R_rho^2 on the last stage (for the RMS), else 0.
template <bool EXACT>
__device__ __forceinline__ double finish_cell(const StageArgs &a, int c, const Prim &me, double r_me,
                                              const double R[5], const double W0[5], const double4 cg) {
    const double g = a.gamma;
    // local time step, TimeStepMethod2 (src/solver/TimeIntegration.cpp:8-40)
    double lam, dt;
    if (EXACT) {
        double snd = sqrt(g * me.p / me.rho);
        double lx = 0.5 * (fabs(me.u) + snd) * cg.x;
        double ly = 0.5 * (fabs(me.v) + snd) * cg.y;
        double lz = 0.5 * (fabs(me.w) + snd) * cg.z;
        lam = lx + ly + lz;
        dt = a.cfl * cg.w / lam;
    } else {
        double snd = g * me.p * r_me;
        lam = 0.5 * fma(fabs(me.u) + snd, cg.x, fma(fabs(me.v) + snd, cg.y, (fabs(me.w) + snd) * cg.z));
        dt = a.residual_only ? a.cfl * cg.w / lam : 0.0;  // the update below needs only alpha*cfl/lam
    }
    if (a.residual_only) {
        const int o = a.new2old[c];
#pragma unroll
        for (int k = 0; k < 5; k++) a.r_out[5 * (size_t)o + k] = R[k];
        a.dt_out[o] = dt;
        return 0.0;
    }
    if (a.split) {  // residual smoothing runs between this residual and the update
        const size_t st = (size_t)a.w0_stride;
#pragma unroll
        for (int k = 0; k < 5; k++) a.r_dev[k * st + c] = R[k];
        return 0.0;
    }
    double W[5];
    if (a.integrator == E3D_INTEGRATOR_EULER) {
        // ExplicitEuler (src/solver/TimeIntegration.cpp:78-91) and FlowField::Update
        // (src/solver/FlowField.cpp:103-117): W += R * (-dt / V), W the carried conservative state
        if (EXACT) {
            const double coeff = -dt / cg.w;
#pragma unroll
            for (int k = 0; k < 5; k++) W[k] = W0[k] + R[k] * coeff;
        } else {
            const double coef = a.cfl * rcp_nr(lam);  // dt / V
#pragma unroll
            for (int k = 0; k < 5; k++) W[k] = fma(-coef, R[k], W0[k]);
        }
    } else if (EXACT) {
        // W = W0 - alpha dt R / V and primitive recovery (EulerSolver.cpp:461-470, FlowField.cpp:140-171)
#pragma unroll
        for (int k = 0; k < 5; k++) W[k] = W0[k] - a.alpha * dt * R[k] / cg.w;
    } else {
        double coef = a.alpha * a.cfl * rcp_nr(lam);  // alpha dt / V
#pragma unroll
        for (int k = 0; k < 5; k++) W[k] = fma(-coef, R[k], W0[k]);
    }
    Prim s;
    double E;
    s.rho = W[0];
    if (EXACT) {
        s.u = W[1] / s.rho;
        s.v = W[2] / s.rho;
        s.w = W[3] / s.rho;
        E = W[4] / s.rho;
        double q2 = s.u * s.u + s.v * s.v + s.w * s.w;
        s.p = (g - 1) * s.rho * (E - q2 / 2.0);
        s.H = E + (s.p / s.rho);
    } else {
        double ir = rcp_nr(s.rho);
        s.u = W[1] * ir;
        s.v = W[2] * ir;
        s.w = W[3] * ir;
        E = W[4] * ir;
        s.p = (g - 1.0) * fma(-0.5, fma(W[1], s.u, fma(W[2], s.v, W[3] * s.w)), W[4]);
        s.H = (W[4] + s.p) * ir;
    }
    store_prim_cs(a.qout, c, s);
    if (!a.last_stage) return 0.0;
    const size_t st = (size_t)a.w0_stride;
    if (a.integrator == E3D_INTEGRATOR_EULER) {  // the conservative state itself carries over
#pragma unroll
        for (int k = 0; k < 5; k++) __stcs(a.w0 + k * st + c, W[k]);
        __stcs(a.ecell + c, E);
        if (a.rsq) a.rsq[a.new2old[c]] = R[0] * R[0];
        return R[0] * R[0];
    }
    // the next step's W0 from the primitives (EulerSolver.cpp:431-438)
    __stcs(a.w0 + 0 * st + c, s.rho);
    __stcs(a.w0 + 1 * st + c, s.u * s.rho);
    __stcs(a.w0 + 2 * st + c, s.v * s.rho);
    __stcs(a.w0 + 3 * st + c, s.w * s.rho);
    __stcs(a.w0 + 4 * st + c, E * s.rho);
    __stcs(a.ecell + c, E);
    if (a.rsq) a.rsq[a.new2old[c]] = R[0] * R[0];
    return R[0] * R[0];
}

// ------------------------------------------------------------------------------ gather kernel
// One thread per cell; the cell walks its own faces and evaluates each flux itself (an interior
// face is evaluated by both of its cells).  MINB: resident blocks per SM the register allocation
// must allow (an occupancy variant the autotuner chooses per mesh).
template <bool EXACT, int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) stage_kernel(StageArgs a) {
    if (!a.residual_only && a.ctl->done) return;  // uniform across the grid
    const int c = blockIdx.x * kStageThreads + threadIdx.x;
    const double g = a.gamma;
    double r2 = 0.0;
    if (c < a.n_cells) {
        const Prim me = load_prim(a.qin, c);
        // sqrt(rho) and rsqrt(gamma p rho) of this cell, shared by all its faces (fast path)
        double s_me = 0.0, r_me = 0.0;
        if (!EXACT) {
            s_me = me.rho * rsqrt_nr(me.rho);
            r_me = rsqrt_nr(g * me.p * me.rho);
        }
        double R[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        const int e0 = a.cptr[c], e1 = a.cptr[c + 1];
        for (int e = e0; e < e1; e++) {
            const int2 ent = a.cf[e];
            const int tag = ent.x & ((1 << kTagBits) - 1);
            const int idx = ent.x >> kTagBits;
            const double4 fg = a.fgeo[ent.y];
            double F[5];
            // Operands of the Roe flux in (left, right) order.  Interior faces select them per lane
            // instead of branching, so a warp whose cells sit on either side of their faces runs one
            // flux evaluation, not two.  The right cell subtracts F*S as F*(-S) (same IEEE result).
            Prim fl, fr;
            double sS = fg.w;
            bool roe = true;
            double s_l = s_me, s_r = s_me, r_l = r_me, r_nb = r_me;
            if (tag <= TAG_RIGHT) {
                const Prim nb = load_prim(a.qin, idx);
                const bool left = tag == TAG_LEFT;
                fl = left ? me : nb;
                fr = left ? nb : me;
                sS = left ? fg.w : -fg.w;
                if (!EXACT) {
                    double s_nb = nb.rho * rsqrt_nr(nb.rho);
                    r_nb = rsqrt_nr(g * nb.p * nb.rho);
                    s_l = left ? s_me : s_nb;
                    s_r = left ? s_nb : s_me;
                    r_l = left ? r_me : r_nb;
                }
            } else {
                Prim gs;
                roe = boundary_face(a, tag, a.ghost + 8 * (size_t)idx, c, me, fg, F, gs);
                fl = me;
                fr = gs;  // symmetry ghost: rho and p are the cell's, so s_r = s_me
            }
            if (roe) {
                if (a.scheme == 1) {
                    if (EXACT) ausm_exact(fl, fr, fg.x, fg.y, fg.z, g, F);
                    else ausm_fast(fl, fr, r_l, tag == TAG_LEFT ? r_nb : r_me, fg.x, fg.y, fg.z, g, F);
                } else {
                    if (EXACT) roe_exact(fl, fr, fg.x, fg.y, fg.z, g, F);
                    else roe_fast(fl, fr, s_l, s_r, r_l, fg.x, fg.y, fg.z, g, F);
                }
            }
#pragma unroll
            for (int k = 0; k < 5; k++) R[k] += F[k] * sS;
        }
        double W0[5];
#pragma unroll
        for (int k = 0; k < 5; k++) W0[k] = a.w0[(size_t)k * a.w0_stride + c];
        r2 = finish_cell<EXACT>(a, c, me, r_me, R, W0, a.cgeo[c]);
    }
    if (a.last_stage && !a.residual_only) block_sum_store(r2, a.partials + blockIdx.x);
}

// ------------------------------------------------------------------------------ face colouring
// FP64 mode only.  The faces are split into colour classes in which no two faces share a cell.  One
// launch per class evaluates each face once and adds its F*S to the residuals of its cells in
// global memory (the left cell's plus, the right cell's minus) with no atomics: within a class every
// cell receives at most one contribution.  A last kernel runs the time step and the update from the
// accumulated residuals.  Each cell sums its faces in class order, a fixed order, so the results are
// deterministic; it is not the reference's face order, so FP64_EXACT never takes this path.
struct ColourFace {
    int l;          // interior cell (device index): the face's left cell
    int r;          // right cell (interior face) or ghost index (boundary face)
    int tag;        // TAG_LEFT for an interior face, else the boundary class
    int pad;
    double nx, ny, nz, S;  // unit normal (from l to r) and area
};
static_assert(sizeof(ColourFace) == 48, "ColourFace layout");

// The residual accumulator: one 48-byte record per cell (R0..R4 and a pad), so that the update of
// a scattered cell moves two 32-byte sectors instead of five.
__device__ __forceinline__ void colour_add(double2 *__restrict__ rc, int c, const double F[5], double S, bool plus) {
    double2 *r = rc + 3 * (size_t)c;
    double2 r0 = r[0], r1 = r[1], r2 = r[2];
    if (plus) {
        r0.x += F[0] * S;
        r0.y += F[1] * S;
        r1.x += F[2] * S;
        r1.y += F[3] * S;
        r2.x += F[4] * S;
    } else {
        r0.x -= F[0] * S;
        r0.y -= F[1] * S;
        r1.x -= F[2] * S;
        r1.y -= F[3] * S;
        r2.x -= F[4] * S;
    }
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
}

// One face per thread over class [f, f + n); rc is the residual accumulator (3 double2 per cell).
template <int NT>
__global__ void __launch_bounds__(NT) colour_kernel(StageArgs a, const ColourFace *__restrict__ f, int n,
                                                    double2 *__restrict__ rc) {
    if (!a.residual_only && a.ctl->done) return;  // uniform across the grid
    const int i = blockIdx.x * NT + threadIdx.x;
    if (i >= n) return;
    const ColourFace cf = f[i];
    const double g = a.gamma;
    const double4 fg = make_double4(cf.nx, cf.ny, cf.nz, cf.S);
    const Prim L = load_prim(a.qin, cf.l);
    double F[5];
    if (cf.tag == TAG_LEFT) {
        const Prim R = load_prim(a.qin, cf.r);
        if (a.scheme == 1)
            ausm_fast(L, R, rsqrt_nr(g * L.p * L.rho), rsqrt_nr(g * R.p * R.rho), fg.x, fg.y, fg.z, g, F);
        else
            roe_fast(L, R, L.rho * rsqrt_nr(L.rho), R.rho * rsqrt_nr(R.rho), rsqrt_nr(g * L.p * L.rho), fg.x, fg.y,
                     fg.z, g, F);
        colour_add(rc, cf.l, F, fg.w, true);
        colour_add(rc, cf.r, F, fg.w, false);
        return;
    }
    Prim gs;
    if (boundary_face(a, cf.tag, a.ghost + 8 * (size_t)cf.r, cf.l, L, fg, F, gs)) {
        // symmetry ghost: rho and p are the cell's
        const double rl = rsqrt_nr(g * L.p * L.rho);
        if (a.scheme == 1) ausm_fast(L, gs, rl, rl, fg.x, fg.y, fg.z, g, F);
        else {
            const double sl = L.rho * rsqrt_nr(L.rho);
            roe_fast(L, gs, sl, sl, rl, fg.x, fg.y, fg.z, g, F);
        }
    }
    colour_add(rc, cf.l, F, fg.w, true);
}

// After the last class: time step and update of every cell from its accumulated residual (the
// update, the split residual phase or the residual-only output, as finish_cell does for the other
// stage kernels), RMS partials per block of kStageThreads cells.
template <int = 0>  // instantiated in the FP64 translation unit only
__global__ void __launch_bounds__(kStageThreads) colour_finish_kernel(StageArgs a, const double2 *__restrict__ rc) {
    if (!a.residual_only && a.ctl->done) return;  // uniform across the grid
    const int c = blockIdx.x * kStageThreads + threadIdx.x;
    double r2 = 0.0;
    if (c < a.n_cells) {
        const Prim me = load_prim(a.qin, c);
        const size_t st = (size_t)a.w0_stride;
        const double2 r0 = rc[3 * (size_t)c], r1 = rc[3 * (size_t)c + 1], r2v = rc[3 * (size_t)c + 2];
        const double R[5] = {r0.x, r0.y, r1.x, r1.y, r2v.x};
        double W0[5];
#pragma unroll
        for (int k = 0; k < 5; k++) W0[k] = a.w0[k * st + c];
        r2 = finish_cell<false>(a, c, me, rsqrt_nr(a.gamma * me.p * me.rho), R, W0, a.cgeo[c]);
    }
    if (a.last_stage && !a.residual_only) block_sum_store(r2, a.partials + blockIdx.x);
}

// ------------------------------------------------------------------------------ async copies
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bulk (TMA) copy global -> this CTA's shared memory, completing on bar.  dst, src 16-byte
// aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// L2 policy for data a stage reads once (face records, contribution lists): the lines it brings in
// are the first to be replaced, so that the state rows neighbouring tiles re-read as halo cells stay
// in L2 longer.
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// bulk_g2s under an L2 cache policy.
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}

// Bulk prefetch of a global range into L2 (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n cp.async.wait_group 0;" ::: "memory");
}

constexpr int kWaitLimit = 1 << 22;  // polls of a barrier before the kernel gives up and reports

__device__ __forceinline__ uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

// ------------------------------------------------------------------------------ face tiles
// A tile is kTileCells consecutive cells (a spatially compact group in the Morton cell order).
// Its data, staged in shared memory:
//   st[LC]   48-byte states: owned cells (one bulk copy) then halo cells (outside neighbours,
//            gathered with cp.async)
//   rec[FC]  FaceRec of every face touching the tile (one bulk copy)
//   ct[MC][T]   contribution lists (one bulk copy)
// W0 and the cell geometry (only ever read by the thread that owns the cell) stay in global
// memory: their rows are prefetched into L2 when the tile starts and read, coalesced, into
// registers before the flux phase ends.  Keeping them out of shared memory lets seven blocks share
// an SM.
// Evaluation: every face touching the tile is evaluated once (a face shared with another tile is
// evaluated by both) and its F*S (5 doubles, 40 bytes) written over the face's own 40-byte record,
// which only the thread evaluating the face reads; each cell then sums its faces' F*S in ascending
// reference face id, the order of the reference's face loop, so results are deterministic and, in
// exact mode, the reference's bit for bit.
struct TileBuf {
    double2 *st;
    FaceRec *rec;
    unsigned short *ct;
};

__host__ __device__ __forceinline__ size_t tile_buf_bytes(int LC, int FC, int MC) {
    return (size_t)LC * 48 + ((40u * (size_t)FC + 15) & ~(size_t)15) + (size_t)MC * kTileCells * 2;
}

__device__ __forceinline__ TileBuf tile_buf_at(unsigned char *base, int LC, int FC, int MC) {
    TileBuf b;
    b.st = reinterpret_cast<double2 *>(base);
    b.rec = reinterpret_cast<FaceRec *>(base + (size_t)LC * 48);
    b.ct = reinterpret_cast<unsigned short *>(base + (size_t)LC * 48 + round16(40u * FC));
    return b;
}

// One thread issues the tile's bulk copies onto bar (expecting their byte count); nf and rec_off are
// the tile's face count and record offset.
__device__ __forceinline__ void tile_issue_bulk(const StageArgs &a, int tile, int nf, long long rec_off,
                                                const TileBuf &b, uint64_t *bar) {
    const int T = kTileCells, MC = a.max_contrib;
    const int c0 = tile * T, nloc = min(T, a.n_cells - c0);
    const uint32_t b_state = (uint32_t)nloc * 48u;
    const uint32_t b_rec = round16(40u * (uint32_t)nf);
    const uint32_t b_w0 = round16((uint32_t)nloc * 8u);  // stays inside the padded rows
    const uint32_t b_cg = (uint32_t)nloc * 32u;
    const uint32_t b_ct = (uint32_t)MC * T * 2u;
    mbar_expect_tx(bar, b_state + b_rec + b_ct);
    const uint64_t once = l2_evict_first();
    bulk_g2s(b.st, a.qin + 3 * (size_t)c0, b_state, bar);
    bulk_g2s_hint(b.rec, a.tile_rec + rec_off, b_rec, bar, once);
    bulk_g2s_hint(b.ct, a.tile_contrib + (size_t)tile * MC * T, b_ct, bar, once);
    for (int k = 0; k < 5; k++) bulk_prefetch_l2(a.w0 + (size_t)k * a.w0_stride + c0, b_w0);
    bulk_prefetch_l2(a.cgeo + c0, b_cg);
}

// Halo state i of the tile (global cell h) into st[nloc + i] with three 16-byte cp.async.
__device__ __forceinline__ void tile_gather_halo(const StageArgs &a, const TileBuf &b, int nloc, int i, int h) {
    const double2 *src = a.qin + 3 * (size_t)h;
    double2 *dst = b.st + 3 * (nloc + i);
    cp_async16(dst, src);
    cp_async16(dst + 1, src + 1);
    cp_async16(dst + 2, src + 2);
}

__device__ __forceinline__ Prim tile_prim(const double2 *st, int i) {
    const double2 x = st[3 * i], y = st[3 * i + 1], z = st[3 * i + 2];
    return Prim{x.x, x.y, y.x, y.y, z.x, z.y};
}

// One flux per tile face; F*S of face j replaces record j (fs[5 j + k] aliases b.rec[j]).  The fast
// path takes sqrt(rho) and rsqrt(gamma p rho) of both sides per face: a per-cell pass over the tile
// before the fluxes would cost a barrier phase and 16 bytes of shared memory per local cell, and
// measured slower on B200.
template <bool EXACT, int NT>
__device__ __forceinline__ void tile_fluxes(const StageArgs &a, const TileBuf &b, double *fs, int nf, int c0,
                                            int tid) {
    const double g = a.gamma;
    for (int j = tid; j < nf; j += NT) {
        const FaceRec fr = b.rec[j];
        const int l = fr.code & ((1 << kTileLocalBits) - 1);
        const int r = (fr.code >> kTileLocalBits) & ((1 << kTileLocalBits) - 1);
        const int tag = fr.code >> (2 * kTileLocalBits);
        const double4 fg = make_double4(fr.nx, fr.ny, fr.nz, fr.S);
        const Prim L = tile_prim(b.st, l);
        double F[5];
        if (tag == TAG_LEFT) {
            const Prim R = tile_prim(b.st, r);
            if (a.scheme == 1) {
                if (EXACT) ausm_exact(L, R, fg.x, fg.y, fg.z, g, F);
                else ausm_fast(L, R, rsqrt_nr(g * L.p * L.rho), rsqrt_nr(g * R.p * R.rho), fg.x, fg.y, fg.z, g, F);
            } else {
                if (EXACT) roe_exact(L, R, fg.x, fg.y, fg.z, g, F);
                else
                    roe_fast(L, R, L.rho * rsqrt_nr(L.rho), R.rho * rsqrt_nr(R.rho), rsqrt_nr(g * L.p * L.rho), fg.x,
                             fg.y, fg.z, g, F);
            }
        } else {
            Prim gs;
            double *gp = a.ghost + 8 * (size_t)fr.ghost;
            if (boundary_face(a, tag, gp, c0 + l, L, fg, F, gs)) {
                // the ghost's density and pressure are the interior cell's (mirror)
                if (a.scheme == 1) {
                    if (EXACT) ausm_exact(L, gs, fg.x, fg.y, fg.z, g, F);
                    else {
                        const double rl = rsqrt_nr(g * L.p * L.rho);
                        ausm_fast(L, gs, rl, rl, fg.x, fg.y, fg.z, g, F);
                    }
                } else {
                    if (EXACT) roe_exact(L, gs, fg.x, fg.y, fg.z, g, F);
                    else {
                        const double sl = L.rho * rsqrt_nr(L.rho);
                        roe_fast(L, gs, sl, sl, rsqrt_nr(g * L.p * L.rho), fg.x, fg.y, fg.z, g, F);
                    }
                }
            }
        }
        // the record is in registers; keep the compiler from moving its loads past the overwrite
        asm volatile("" ::: "memory");
#pragma unroll
        for (int k = 0; k < 5; k++) fs[5 * j + k] = F[k] * fg.w;
    }
}

// W0 and geometry of owned cell i (global memory, prefetched into L2 when the tile started).
// Streaming loads (ld.global.cs): the stage reads these rows once.
__device__ __forceinline__ void tile_load_cell(const StageArgs &a, int c0, int i, double W0[5], double4 &cg) {
#pragma unroll
    for (int k = 0; k < 5; k++) W0[k] = __ldcs(a.w0 + (size_t)k * a.w0_stride + c0 + i);
    const double2 *g = reinterpret_cast<const double2 *>(a.cgeo + c0 + i);
    const double2 g0 = __ldcs(g), g1 = __ldcs(g + 1);
    cg = make_double4(g0.x, g0.y, g1.x, g1.y);
}

// Cell i of the tile: sum of its contributions, then time step and update; returns R_rho^2 on
// the last stage.  W0 and the geometry come from the caller, which loads them before the barrier
// that ends the flux phase so that their latency overlaps the wait.
template <bool EXACT>
__device__ __forceinline__ double tile_update(const StageArgs &a, const TileBuf &b, const double *fs, int c0, int i,
                                              const double W0[5], const double4 &cg) {
    const int T = kTileCells;
    double R[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    unsigned short e[6];
#pragma unroll
    for (int k = 0; k < 6; k++) e[k] = k < a.max_contrib ? b.ct[k * T + i] : kNoContrib;
    const Prim me = tile_prim(b.st, i);
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (e[k] == kNoContrib) break;
        const int j = e[k] >> 1;
        // R -/+ F*S as one fused multiply-add by -/+1: the product is exact and the sum rounds once,
        // so these are the bits of R - F*S or R + F*S, without a branch the cells of a warp split on
        const double sg = (e[k] & 1) ? -1.0 : 1.0;
#pragma unroll
        for (int q = 0; q < 5; q++) R[q] = fma(sg, fs[5 * j + q], R[q]);
    }
    return finish_cell<EXACT>(a, c0 + i, me, EXACT ? 0.0 : rsqrt_nr(a.gamma * me.p * me.rho), R, W0, cg);
}

// Bounded wait on an mbarrier phase by every thread (a.wait_polls polls); on timeout the fault word
// is set.  Returns true for the whole block only if every thread saw the phase complete.
__device__ __forceinline__ bool tile_wait(const StageArgs &a, uint64_t *bar, uint32_t parity) {
    bool ok = false;
    for (int it = 0; it < a.wait_polls && !ok; it++) ok = mbar_try_wait(bar, parity);
    if (!ok) atomicExch(a.fault, 1);
    return !__syncthreads_or(!ok);
}

// After a wait gave up: let the bulk copies still in flight on bar land (bounded by kWaitLimit)
// before the block leaves, so that nothing writes this block's shared memory after it exits.
__device__ __forceinline__ void tile_drain(uint64_t *bar, uint32_t parity) {
    for (int it = 0; it < kWaitLimit && !mbar_try_wait(bar, parity); it++) {
    }
}

// ---- one block per tile, all loads issued at the start (variant 2)
// Shared memory: TileBuf (face fluxes over the records) | mbarrier
// The body is shared by tile_kernel (one solver) and tile_batch_kernel (several solvers in one
// grid): `tile` is the solver's own tile index, `partial` where its RMS partial goes.
template <bool EXACT>
__device__ __forceinline__ void tile_body(const StageArgs &a, int tile, double *partial, unsigned char *smem_raw) {
    const int LC = a.smem_cells, FC = a.smem_faces, MC = a.max_contrib, T = kTileCells;
    const TileBuf b = tile_buf_at(smem_raw, LC, FC, MC);
    size_t off = (tile_buf_bytes(LC, FC, MC) + 15) & ~(size_t)15;
    double *fs = reinterpret_cast<double *>(b.rec);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + off);

    const int c0 = tile * T;
    const int nloc = min(T, a.n_cells - c0);
    // Every load the copies depend on is issued before the first barrier, and none of them waits
    // for another (the halo entries sit at a fixed stride per tile), so the copies start one
    // memory latency after the block does.  The run's done flag is read alongside them.
    const int *hrow = a.tile_halo + (size_t)tile * a.halo_stride;
    const int i0 = threadIdx.x, i1 = threadIdx.x + T;
    const int hx0 = i0 < a.halo_stride ? hrow[i0] : -1;
    const int hx1 = i1 < a.halo_stride ? hrow[i1] : -1;
    const int fp0 = a.tile_face_ptr[tile], fp1 = a.tile_face_ptr[tile + 1];
    const long long rec_off = a.tile_rec_off[tile];
    const bool done = !a.residual_only && a.ctl->done;
    const int nf = fp1 - fp0;

    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (done) return;  // uniform across the block (the run stopped: this stage leaves the state)
    if (threadIdx.x == 0) tile_issue_bulk(a, tile, nf, rec_off, b, bar);
    if (hx0 >= 0) tile_gather_halo(a, b, nloc, i0, hx0);
    if (hx1 >= 0) tile_gather_halo(a, b, nloc, i1, hx1);
    for (int i = threadIdx.x + 2 * T; i < a.halo_stride; i += T) {
        const int h = hrow[i];
        if (h >= 0) tile_gather_halo(a, b, nloc, i, h);
    }
    cp_async_wait_all();
    if (!tile_wait(a, bar, 0)) {
        tile_drain(bar, 0);
        return;
    }
    tile_fluxes<EXACT, kStageThreads>(a, b, fs, nf, c0, threadIdx.x);
    double W0[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double4 cg = make_double4(0.0, 0.0, 0.0, 0.0);
    if ((int)threadIdx.x < nloc) tile_load_cell(a, c0, threadIdx.x, W0, cg);
    __syncthreads();
    double r2 = 0.0;
    if ((int)threadIdx.x < nloc) r2 = tile_update<EXACT>(a, b, fs, c0, threadIdx.x, W0, cg);
    if (a.last_stage && !a.residual_only) block_sum_store(r2, partial);
}

template <bool EXACT, int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) tile_kernel(StageArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tile_body<EXACT>(a, blockIdx.x, a.partials + blockIdx.x, smem_raw);
}

// ---- several solvers ("members") in one grid
// The face tiles of every member are concatenated into one launch: block k handles tile
// table[k].y of member table[k].x with that member's own arguments (mesh, state buffers, flow
// conditions, CFL, run control).  Members are independent, so each one computes exactly what its
// own tile_kernel launch would: the same tiles, the same per-cell face order and the same RMS
// partials.  A member whose run has stopped (its done flag) costs its blocks one load.
struct BatchStage {
    const StageArgs *__restrict__ args;  // member m reading state buffer b: args[2 * m + b]
    const int2 *__restrict__ table;      // block -> (member, tile of that member)
    const int *__restrict__ n_entries;   // valid table entries; later blocks return at once
    double alpha;
    int first_stage, last_stage, parity;
    int ws_buffers, ws_stride;           // tile_ws_batch_kernel: buffers, bytes per buffer
};
static_assert(sizeof(StageArgs) % 4 == 0, "StageArgs is copied in 4-byte words");

// The block's member arguments into shared memory, with the stage's own alpha and flags written in
// place of the member's as the words are copied (one barrier).
__device__ __forceinline__ int2 batch_stage_args(const BatchStage &bs, StageArgs *sa) {
    const int2 e = bs.table[blockIdx.x];
    const uint32_t *src = reinterpret_cast<const uint32_t *>(bs.args + 2 * e.x + bs.parity);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sa);
    constexpr int kAlpha = (int)(offsetof(StageArgs, alpha) / 4), kFirst = (int)(offsetof(StageArgs, first_stage) / 4);
    constexpr int kLast = (int)(offsetof(StageArgs, last_stage) / 4);
    constexpr int kResidual = (int)(offsetof(StageArgs, residual_only) / 4);
    const unsigned long long alpha = (unsigned long long)__double_as_longlong(bs.alpha);
    for (int i = threadIdx.x; i < (int)(sizeof(StageArgs) / 4); i += blockDim.x) {
        uint32_t v = src[i];
        if (i == kAlpha) v = (uint32_t)alpha;
        else if (i == kAlpha + 1) v = (uint32_t)(alpha >> 32);
        else if (i == kFirst) v = (uint32_t)bs.first_stage;
        else if (i == kLast) v = (uint32_t)bs.last_stage;
        else if (i == kResidual) v = 0u;
        dst[i] = v;
    }
    __syncthreads();
    return e;
}

template <bool EXACT, int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) tile_batch_kernel(BatchStage bs) {
    if ((int)blockIdx.x >= *bs.n_entries) return;  // uniform across the block
    __shared__ __align__(16) StageArgs sa;
    const int2 e = batch_stage_args(bs, &sa);
    if (sa.ctl->done) return;  // uniform across the member's blocks
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tile_body<EXACT>(sa, e.y, sa.partials + e.y, smem_raw);
}

// ---- update phase of a split stage
// One thread per cell: the time step and the update of finish_cell from the residual in r_dev
// (smoothed between the residual phase and this one).  Blocks of kStageThreads cells, so the RMS
// partials line up with those of the stage kernels.
template <bool EXACT>
__global__ void __launch_bounds__(kStageThreads) update_kernel(StageArgs a) {
    if (a.ctl->done) return;  // uniform across the grid
    const int c = blockIdx.x * kStageThreads + threadIdx.x;
    double r2 = 0.0;
    if (c < a.n_cells) {
        const Prim me = load_prim(a.qin, c);
        const size_t st = (size_t)a.w0_stride;
        double R[5], W0[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            R[k] = a.r_dev[k * st + c];
            W0[k] = a.w0[k * st + c];
        }
        const double r_me = EXACT ? 0.0 : rsqrt_nr(a.gamma * me.p * me.rho);
        r2 = finish_cell<EXACT>(a, c, me, r_me, R, W0, a.cgeo[c]);
    }
    if (a.last_stage) block_sum_store(r2, a.partials + blockIdx.x);
}

// Dynamic shared memory of tile_kernel.
inline size_t tile_smem_bytes(int smem_cells, int smem_faces, int max_contrib) {
    const size_t bb = (tile_buf_bytes(smem_cells, smem_faces, max_contrib) + 15) & ~(size_t)15;
    return bb + 16;  // + its mbarrier
}

}  // namespace e3d
