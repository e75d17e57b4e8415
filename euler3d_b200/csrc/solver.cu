// Solver handle of the euler3d_b200 library: device layout construction, the RK5 run loop with
// on-device stop control, state exchange in the reference's numbering, and the solver half of
// the C ABI (include/euler3d_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "common.hpp"
#include "euler3d_b200.h"
#include "solver.hpp"
#include "stage_ws.cuh"

namespace e3d {


// ------------------------------------------------------------------------------ small kernels

// Sum of the per-block partials in a fixed order, RMS, and the stop tests of
// EulerSolver::Run (src/solver/EulerSolver.cpp:96-112).  One block per solver; `sh` is the block's
// kReduceThreads-entry scratch.
__device__ __forceinline__ void finalize_body(const FinalizeArgs &f, double *sh) {
    Control *ctl = f.ctl;
    if (ctl->done) return;
    if (ctl->fault) {  // a stage kernel's bounded wait gave up: its cells kept their old state, so stop
        if (threadIdx.x == 0) {
            ctl->done = 1;
            ctl->stop_reason = E3D_STOP_MAX_ITER;
        }
        return;
    }
    if (f.rsq) {
        // FP64_EXACT: EulerSolver::computeRMS's own order, one running sum over the cells in
        // reference order (src/solver/EulerSolver.cpp:382-389)
        if (threadIdx.x != 0) return;
        double s = 0.0;
        for (int i = 0; i < f.n_cells; i++) s += f.rsq[i];
        sh[0] = s;
    } else {
        double v = 0.0;
        for (int i = threadIdx.x; i < f.n_part; i += kReduceThreads) v += f.partials[i];
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int s = kReduceThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x != 0) return;
    }
    double rms = sqrt(sh[0] / f.n_domain);
    if (ctl->n_rms < ctl->hist_cap) f.hist[ctl->n_rms] = rms;
    if (ctl->n_rms == 0) ctl->rms0 = rms;
    ctl->n_rms += 1;
    ctl->last_rms = rms;
    ctl->minit_valid = 0;
    ctl->sample_now = 0;
    if (!isfinite(rms)) {  // the reference would spin to MAX_ITER on a NaN; stop and report it
        ctl->nonfinite = 1;
        ctl->done = 1;
        ctl->stop_reason = E3D_STOP_MAX_ITER;
        return;
    }
    if (rms < ctl->min_res || (ctl->min_drop > 0.0 && rms < ctl->min_drop * ctl->rms0)) {
        ctl->done = 1;
        ctl->stop_reason = E3D_STOP_RESIDUAL;
        return;
    }
    if (ctl->stall_window > 0 && (ctl->stall_below <= 0.0 || rms < ctl->stall_below * ctl->rms0)) {
        // the residual has stopped falling (a precision floor)
        if (ctl->best_rms == 0.0 || rms < ctl->best_rms) {
            ctl->best_rms = rms;
            ctl->since_best = 0;
        } else if (++ctl->since_best >= ctl->stall_window) {
            ctl->done = 1;
            ctl->stop_reason = E3D_STOP_STALL;
            return;
        }
    }
    ctl->it += 1;
    if (ctl->it % ctl->sampling == 0) {
        ctl->sample_now = 1;
    } else if (ctl->it >= ctl->max_iter) {
        ctl->done = 1;
        ctl->stop_reason = E3D_STOP_MAX_ITER;
    }
}

__global__ void __launch_bounds__(kReduceThreads) finalize_kernel(FinalizeArgs f) {
    __shared__ double sh[kReduceThreads];
    finalize_body(f, sh);
}

// Block m: member m of a batch.
__global__ void __launch_bounds__(kReduceThreads) finalize_batch_kernel(const FinalizeArgs *__restrict__ f,
                                                                        const int *__restrict__ n_members) {
    if ((int)blockIdx.x >= *n_members) return;
    __shared__ double sh[kReduceThreads];
    const FinalizeArgs a = f[blockIdx.x];
    finalize_body(a, sh);
}

__device__ __forceinline__ double wall_pressure(const CoeffArgs &a, int c) {
    if (!a.w0) return a.q[3 * c + 2].x;
    const size_t st = (size_t)a.w0_stride;
    const double rho = a.w0[c], mu = a.w0[st + c], mv = a.w0[2 * st + c], mw = a.w0[3 * st + c];
    return (a.gamma - 1.0) * (a.w0[4 * st + c] - 0.5 * (mu * mu + mv * mv + mw * mw) / rho);
}

// AeroCoefficients::Update (src/solver/AeroCoefficients.cpp:38-52): face terms in parallel, summed
// by one thread in the reference's wall order so the sums are the reference's; then
// EulerSolver::ConvergenceCriteria and the CL/CD/CM selection (src/solver/EulerSolver.cpp:132-152, :253-279).
// One block per solver; `terms` is the block's 6 x kCoeffThreads scratch.
__device__ __forceinline__ void coeff_body(const CoeffArgs &a, double (*terms)[kCoeffThreads]) {
    Control *ctl = a.ctl;
    if (a.run_mode && (ctl->done || !ctl->sample_now)) return;
    double F[3] = {0, 0, 0}, CP[3] = {0, 0, 0};
    if (a.sequential) {
        // the reference's order: one running sum over the wall list
        for (int base = 0; base < a.n_wall; base += kCoeffThreads) {
            int i = base + threadIdx.x;
            if (i < a.n_wall) {
                double p = wall_pressure(a, a.cell[i]);
                double cp = a.cp_factor * (p - a.p_inf);
                if (a.cp_out) a.cp_out[i] = cp;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    double coeff = a.svec[3 * i + k] * cp * a.cref / a.sref;
                    terms[k][threadIdx.x] = coeff;
                    terms[3 + k][threadIdx.x] = coeff * a.center[3 * i + k];
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int n = min(kCoeffThreads, a.n_wall - base);
                for (int j = 0; j < n; j++) {
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        F[k] += terms[k][j];
                        CP[k] += terms[3 + k][j];
                    }
                }
            }
            __syncthreads();
        }
    } else {
        // fixed-shape tree: strided per-thread sums over wall faces t, t + T, t + 2T, ... in that
        // order (their loads issued four faces at a time), then a pairwise tree (deterministic)
        constexpr int U = 4;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int base = threadIdx.x; base < a.n_wall; base += U * kCoeffThreads) {
            double p[U], sv[U][3], ce[U][3];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = base + u * kCoeffThreads;
                if (i < a.n_wall) {
                    p[u] = wall_pressure(a, a.cell[i]);
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        sv[u][k] = a.svec[3 * i + k];
                        ce[u][k] = a.center[3 * i + k];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (base + u * kCoeffThreads >= a.n_wall) break;
                const double cp = a.cp_factor * (p[u] - a.p_inf);
                if (a.cp_out) a.cp_out[base + u * kCoeffThreads] = cp;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double coeff = sv[u][k] * cp * a.cref / a.sref;
                    acc[k] += coeff;
                    acc[3 + k] += coeff * ce[u][k];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 6; k++) terms[k][threadIdx.x] = acc[k];
        __syncthreads();
        for (int st = kCoeffThreads / 2; st > 0; st >>= 1) {
            if (threadIdx.x < st)
#pragma unroll
                for (int k = 0; k < 6; k++) terms[k][threadIdx.x] += terms[k][threadIdx.x + st];
            __syncthreads();
        }
        for (int k = 0; k < 3; k++) {
            F[k] = terms[k][0];
            CP[k] = terms[3 + k][0];
        }
    }
    if (threadIdx.x != 0) return;
    double lever[3] = {a.ref[0] - CP[0], a.ref[1] - CP[1], a.ref[2] - CP[2]};
    double M[3] = {(F[1] * lever[2] - F[2] * lever[1]) / a.cref, (F[2] * lever[0] - F[0] * lever[2]) / a.cref,
                   (F[0] * lever[1] - F[1] * lever[0]) / a.cref};
    if (!a.run_mode) {
        for (int k = 0; k < 3; k++) {
            a.out[k] = F[k];
            a.out[3 + k] = M[k];
        }
        return;
    }
    double cl = F[a.axis[0]] * a.sign[0], cd = F[a.axis[1]] * a.sign[1], cm = M[a.axis[2]] * a.sign[2];
    double tol = ctl->min_aero;
    bool ok = fabs(ctl->cl - cl) < tol && fabs(ctl->cd - cd) < tol && fabs(ctl->cm - cm) < tol;
    ctl->counter = ok ? ctl->counter + 1 : 0;
    if (a.samples && ctl->n_samples < ctl->sample_cap) {  // a residuals.dat row (EulerSolver::PrintInfo)
        double *s = a.samples + 7 * (size_t)ctl->n_samples;
        s[0] = ctl->it;
        for (int k = 0; k < 3; k++) {
            s[1 + k] = F[k];
            s[4 + k] = M[k];
        }
    }
    ctl->n_samples += 1;
    ctl->cl = cl;
    ctl->cd = cd;
    ctl->cm = cm;
    for (int k = 0; k < 3; k++) {
        ctl->force[k] = F[k];
        ctl->moment[k] = M[k];
    }
    if (ctl->counter >= 2) {
        ctl->done = 1;
        ctl->stop_reason = E3D_STOP_COEFFICIENTS;
    } else if (ctl->it >= ctl->max_iter) {
        ctl->done = 1;
        ctl->stop_reason = E3D_STOP_MAX_ITER;
    }
}

__global__ void __launch_bounds__(kCoeffThreads) coeff_kernel(CoeffArgs a) {
    __shared__ double terms[6][kCoeffThreads];
    coeff_body(a, terms);
}

// Block m: member m of a batch, its arguments for the state buffer `parity`.
__global__ void __launch_bounds__(kCoeffThreads) coeff_batch_kernel(const CoeffArgs *__restrict__ c,
                                                                    const int *__restrict__ n_members, int parity) {
    if ((int)blockIdx.x >= *n_members) return;
    __shared__ double terms[6][kCoeffThreads];
    const CoeffArgs a = c[2 * blockIdx.x + parity];
    coeff_body(a, terms);
}

// Control blocks of a batch's members into one array (read back with one copy).
__global__ void control_gather_kernel(Control *const *__restrict__ ctl, const int *__restrict__ n_members,
                                      Control *__restrict__ out) {
    const int m = blockIdx.x;
    if (m >= *n_members) return;
    const int *src = reinterpret_cast<const int *>(ctl[m]);
    int *dst = reinterpret_cast<int *>(out + m);
    for (int i = threadIdx.x; i < (int)(sizeof(Control) / 4); i += blockDim.x) dst[i] = src[i];
}

// One Jacobi pass of EulerSolver::smoothResiduals (src/solver/EulerSolver.cpp:483-518), one thread
// per cell:  out_c = (r0_c + sum_j 0.25 last_j) / (1 + 0.25 n_faces(c)), the sum over interior
// neighbours in element2element order, in the reference's operation order.  The reference's loop
// ends after at most two passes (its difference vector is cleared after the first pass, so the
// second measures no change): the first pass records its largest change (and any NaN, on which the
// reference exits the process); the second pass runs only if that change is above 1e-16 and
// otherwise copies the first pass's result, so the update always reads the second buffer.
constexpr int kSmoothThreads = 256;

__global__ void __launch_bounds__(kSmoothThreads) smooth_kernel(SmoothArgs a) {
    if (a.ctl->done) return;  // uniform across the grid
    const int c = blockIdx.x * kSmoothThreads + threadIdx.x;
    const size_t st = (size_t)a.stride;
    if (a.pass == 1) {
        if (a.flags[1]) {  // NaN in the first pass: stop the run as non-finite
            if (c == 0) {
                a.ctl->nonfinite = 1;
                a.ctl->stop_reason = E3D_STOP_MAX_ITER;
                a.ctl->done = 1;
            }
            return;
        }
        if (!(__longlong_as_double((long long)a.flags[0]) > 1e-16)) {
            if (c < a.n_cells)
                for (int q = 0; q < 5; q++) a.out[q * st + c] = a.last[q * st + c];
            return;
        }
    }
    double m = 0.0;
    int bad = 0;
    if (c < a.n_cells) {
        double sum[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int k = a.nb_ptr[c]; k < a.nb_ptr[c + 1]; k++) {
            const int j = a.nb[k];
#pragma unroll
            for (int q = 0; q < 5; q++) sum[q] += a.last[q * st + j] * 0.25;
        }
        const double d = a.den[c];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const double v = (a.r0[q * st + c] + sum[q]) / d;
            a.out[q * st + c] = v;
            const double ch = fabs(a.last[q * st + c] - v);
            if (isnan(ch)) bad = 1;
            else if (ch > m) m = ch;
        }
    }
    if (a.pass != 0) return;
    // block maximum of the change (non-negative doubles order like their bit patterns)
    __shared__ double sm[kSmoothThreads / 32];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        for (int w = 1; w < kSmoothThreads / 32; w++) m = fmax(m, sm[w]);
        m = fmax(m, sm[0]);
        atomicMax(&a.flags[0], (unsigned long long)__double_as_longlong(m));
        if (bad) atomicOr(&a.flags[1], 1ull);
    }
}

void launch_smooth(const SmoothArgs &a, cudaStream_t s) {
    smooth_kernel<<<(a.n_cells + kSmoothThreads - 1) / kSmoothThreads, kSmoothThreads, 0, s>>>(a);
}

void launch_finalize(const FinalizeArgs &f, cudaStream_t s) { finalize_kernel<<<1, kReduceThreads, 0, s>>>(f); }
void launch_coeff(const CoeffArgs &c, cudaStream_t s) { coeff_kernel<<<1, kCoeffThreads, 0, s>>>(c); }
void launch_finalize_batch(const FinalizeArgs *f, const int *n_members, int grid, cudaStream_t s) {
    finalize_batch_kernel<<<grid, kReduceThreads, 0, s>>>(f, n_members);
}
void launch_coeff_batch(const CoeffArgs *c, const int *n_members, int parity, int grid, cudaStream_t s) {
    coeff_batch_kernel<<<grid, kCoeffThreads, 0, s>>>(c, n_members, parity);
}
void launch_control_gather(Control *const *ctl, const int *n_members, Control *out, int grid, cudaStream_t s) {
    control_gather_kernel<<<grid, 64, 0, s>>>(ctl, n_members, out);
}

// Reference-ordered FlowField arrays (staging, 8 x T) -> device layout.
__global__ void load_state_kernel(const double *__restrict__ st, int64_t T, int n_cells, int n_ghosts,
                                  const int *__restrict__ new2old, const int *__restrict__ ghost_ref,
                                  double2 *__restrict__ q, double *__restrict__ w0, int w0_stride,
                                  double *__restrict__ ecell, double *__restrict__ minit, double *__restrict__ ghost) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)w0_stride;
    if (i < n_cells) {
        int o = new2old[i];
        double rho = st[o], u = st[T + o], v = st[2 * T + o], w = st[3 * T + o];
        double p = st[4 * T + o], E = st[5 * T + o], H = st[6 * T + o], M = st[7 * T + o];
        store_prim(q, i, Prim{rho, u, v, w, p, H});
        w0[0 * N + i] = rho;  // W0 as RungeKutta forms it (src/solver/EulerSolver.cpp:431-438)
        w0[1 * N + i] = u * rho;
        w0[2 * N + i] = v * rho;
        w0[3 * N + i] = w * rho;
        w0[4 * N + i] = E * rho;
        ecell[i] = E;
        minit[i] = M;
    } else if (i < n_cells + n_ghosts) {
        int g = i - n_cells;
        int r = ghost_ref[g];
        for (int k = 0; k < 8; k++) ghost[8 * (size_t)g + k] = st[k * T + r];
    }
}

// Device layout -> reference-ordered FlowField arrays (staging, 8 x T).  Interior Mach is
// FlowField's c/|u| (src/solver/FlowField.cpp:157) unless the loaded Mach still holds.
__global__ void store_state_kernel(double *__restrict__ st, int64_t T, int n_cells, int n_ghosts,
                                   const int *__restrict__ new2old, const int *__restrict__ ghost_ref,
                                   const double2 *__restrict__ q, const double *__restrict__ ecell,
                                   const double *__restrict__ minit, const double *__restrict__ ghost, double gamma,
                                   const Control *ctl) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_cells) {
        int o = new2old[i];
        Prim s = load_prim(q, i);
        double M = ctl->minit_valid ? minit[i] : __ddiv_rn(__dsqrt_rn(__dmul_rn(gamma, __ddiv_rn(s.p, s.rho))),
                                                           __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(s.u, s.u),
                                                                                          __dmul_rn(s.v, s.v)),
                                                                                __dmul_rn(s.w, s.w))));
        st[o] = s.rho;
        st[T + o] = s.u;
        st[2 * T + o] = s.v;
        st[3 * T + o] = s.w;
        st[4 * T + o] = s.p;
        st[5 * T + o] = ecell[i];
        st[6 * T + o] = s.H;
        st[7 * T + o] = M;
    } else if (i < n_cells + n_ghosts) {
        int g = i - n_cells;
        int r = ghost_ref[g];
        for (int k = 0; k < 8; k++) st[k * T + r] = ghost[8 * (size_t)g + k];
    }
}

// FP32_FLUX mode: reference-ordered FlowField arrays -> float cell records and double W0.
__global__ void load_state_f32_kernel(const double *__restrict__ st, int64_t T, int n_cells, int n_ghosts,
                                      const int *__restrict__ new2old, const int *__restrict__ ghost_ref,
                                      float4 *__restrict__ q32, double *__restrict__ w0, int w0_stride,
                                      double *__restrict__ ecell, double *__restrict__ minit,
                                      double *__restrict__ ghost, double gamma) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)w0_stride;
    if (i < n_cells) {
        int o = new2old[i];
        double rho = st[o], u = st[T + o], v = st[2 * T + o], w = st[3 * T + o];
        double p = st[4 * T + o], E = st[5 * T + o], H = st[6 * T + o], M = st[7 * T + o];
        make_rec32(q32 + 2 * (size_t)i, rho, u, v, w, p, H, gamma);
        w0[0 * N + i] = rho;
        w0[1 * N + i] = u * rho;
        w0[2 * N + i] = v * rho;
        w0[3 * N + i] = w * rho;
        w0[4 * N + i] = E * rho;
        ecell[i] = E;
        minit[i] = M;
    } else if (i < n_cells + n_ghosts) {
        int g = i - n_cells;
        int r = ghost_ref[g];
        for (int k = 0; k < 8; k++) ghost[8 * (size_t)g + k] = st[k * T + r];
    }
}

// FP32_FLUX mode: the state is the double conservative W0 (updated at every completed RK step).
__global__ void store_state_f32_kernel(double *__restrict__ st, int64_t T, int n_cells, int n_ghosts,
                                       const int *__restrict__ new2old, const int *__restrict__ ghost_ref,
                                       const double *__restrict__ w0, int w0_stride,
                                       const double *__restrict__ minit, const double *__restrict__ ghost,
                                       double gamma, const Control *ctl) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)w0_stride;
    if (i < n_cells) {
        int o = new2old[i];
        double rho = w0[i], u = w0[N + i] / rho, v = w0[2 * N + i] / rho, w = w0[3 * N + i] / rho;
        double E = w0[4 * N + i] / rho;
        double q2 = u * u + v * v + w * w;
        double p = (gamma - 1) * rho * (E - q2 / 2.0);
        double H = E + p / rho;
        double M = ctl->minit_valid ? minit[i] : sqrt(gamma * (p / rho)) / sqrt(q2);
        st[o] = rho;
        st[T + o] = u;
        st[2 * T + o] = v;
        st[3 * T + o] = w;
        st[4 * T + o] = p;
        st[5 * T + o] = E;
        st[6 * T + o] = H;
        st[7 * T + o] = M;
    } else if (i < n_cells + n_ghosts) {
        int g = i - n_cells;
        int r = ghost_ref[g];
        for (int k = 0; k < 8; k++) st[k * T + r] = ghost[8 * (size_t)g + k];
    }
}

// ------------------------------------------------------------------------------ host handle


// Reverse Cuthill-McKee order of the interior cell graph (each connected component from a
// minimum-degree start, neighbours visited by increasing degree, whole order reversed).
static std::vector<int> rcm_order(int n, const std::vector<int> &adj_ptr, const std::vector<int> &adj) {
    std::vector<int> deg(n), order;
    order.reserve(n);
    for (int i = 0; i < n; i++) deg[i] = adj_ptr[i + 1] - adj_ptr[i];
    std::vector<int> by_deg(n);
    std::iota(by_deg.begin(), by_deg.end(), 0);
    std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    std::vector<char> seen(n, 0);
    std::vector<int> nb;
    for (int start : by_deg) {
        if (seen[start]) continue;
        size_t head = order.size();
        order.push_back(start);
        seen[start] = 1;
        while (head < order.size()) {
            int v = order[head++];
            nb.clear();
            for (int k = adj_ptr[v]; k < adj_ptr[v + 1]; k++)
                if (!seen[adj[k]]) nb.push_back(adj[k]);
            std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            for (int x : nb) {
                seen[x] = 1;
                order.push_back(x);
            }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}



static void check_desc(const e3d_mesh_desc *d) {
    if (!d) throw Error(E3D_ERR_INVALID_ARG, "mesh descriptor is NULL");
    if (d->n_cells <= 0 || d->n_faces <= 0 || d->n_faces_int < 0 || d->n_faces_int > d->n_faces)
        throw Error(E3D_ERR_INVALID_ARG, "mesh sizes are inconsistent");
    if (!d->face2cell || !d->face_unit_normal || !d->face_normal || !d->face_area || !d->face_center ||
        !d->cell_volume || !d->cell2face_ptr || !d->cell2face)
        throw Error(E3D_ERR_INVALID_ARG, "a mesh descriptor array is NULL");
    if ((int64_t)d->n_cells + (d->n_faces - d->n_faces_int) >= ((int64_t)1 << (31 - kTagBits)))
        throw Error(E3D_ERR_INVALID_ARG, "mesh too large for the device index encoding");
    auto chk_list = [&](int n, const int32_t *g, const int32_t *in, const int32_t *f, const char *what) {
        if (n < 0 || (n > 0 && (!g || !in || !f))) throw Error(E3D_ERR_INVALID_ARG, std::string(what) + " list is invalid");
    };
    chk_list(d->n_wall, d->wall_ghost, d->wall_interior, d->wall_face, "wall");
    chk_list(d->n_farfield, d->farfield_ghost, d->farfield_interior, d->farfield_face, "farfield");
    chk_list(d->n_sym, d->sym_ghost, d->sym_interior, d->sym_face, "symmetry");
}

// Order of a tile's interior face records for the flux phase.  Eight consecutive threads (a
// quarter-warp) load their faces' cell states in 16-byte pieces together, and cell x's pieces sit in
// 16-byte bank groups 3x + k (mod 8) of a 48-byte state array (2x + k of the 32-byte FP32 records):
// the eight meet no bank conflict when their left cells differ mod 8 and so do their right cells.
// Faces are drawn from 64 buckets by (left mod 8, right mod 8), eight at a time with distinct left
// and right classes where the buckets allow, the fullest bucket first.  The order changes no
// arithmetic: each face's flux is the same and every cell still sums its faces in its own order.
static void bank_order(const FaceRec *rec, int n, std::vector<int> &order, std::vector<int> &sorted) {
    const int mask = (1 << kTileLocalBits) - 1;
    auto cls = [&](int i) {
        const int l = rec[i].code & mask, r = (rec[i].code >> kTileLocalBits) & mask;
        return (l & 7) * 8 + (r & 7);
    };
    // the faces sorted by class, in their own order within a class (a counting sort into one array)
    int start[65] = {}, head[64];
    for (int i = 0; i < n; i++) start[cls(i) + 1]++;
    for (int k = 0; k < 64; k++) start[k + 1] += start[k];
    for (int k = 0; k < 64; k++) head[k] = start[k];
    sorted.resize(n);
    for (int i = 0; i < n; i++) sorted[head[cls(i)]++] = i;
    for (int k = 0; k < 64; k++) head[k] = start[k];
    auto count = [&](int k) { return start[k + 1] - head[k]; };
    order.clear();
    int left = n, rot = 0;
    while (left > 0) {
        unsigned used_l = 0, used_r = 0;
        for (int s = 0; s < 8 && left > 0; s++, rot++) {
            int chosen = -1;
            for (int da = 0; da < 8 && chosen < 0; da++) {
                const int a = (rot + da) & 7;
                if (used_l >> a & 1) continue;
                int best = 0;
                for (int b = 0; b < 8; b++)
                    if (!(used_r >> b & 1) && count(a * 8 + b) > best) {
                        best = count(a * 8 + b);
                        chosen = a * 8 + b;
                    }
            }
            if (chosen < 0) {  // no conflict-free choice left in this group: the fullest bucket
                int best = 0;
                for (int k = 0; k < 64; k++)
                    if (count(k) > best) {
                        best = count(k);
                        chosen = k;
                    }
            }
            order.push_back(sorted[head[chosen]++]);
            used_l |= 1u << (chosen / 8);
            used_r |= 1u << (chosen % 8);
            left--;
        }
    }
}

// Face-colouring classes (stage variants 5 and 6), from the device's own connectivity: every
// interior face once (from its left cell's list) and every boundary face, each given the smallest
// class that neither of its cells has taken yet, visited in device cell order.  A class keeps its
// faces in that order (ascending left cell), so its state gathers walk memory forwards.  On a mesh
// whose cells have at most k faces a face meets at most 2k - 2 others, so 2k - 1 classes suffice
// (11 for hexahedra); 32 are available.
void build_colours(Solver *S) {
    if (S->colours_built()) return;
    const int N = S->N;
    cudaStream_t s = S->stream;
    std::vector<int> cptr(N + 1);
    std::vector<int2> cf(S->cf.n);
    std::vector<double4> fgeo(S->fgeo.n);
    E3D_CUDA(cudaMemcpyAsync(cptr.data(), S->cptr.p, cptr.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    E3D_CUDA(cudaMemcpyAsync(cf.data(), S->cf.p, cf.size() * sizeof(int2), cudaMemcpyDeviceToHost, s));
    E3D_CUDA(cudaMemcpyAsync(fgeo.data(), S->fgeo.p, fgeo.size() * sizeof(double4), cudaMemcpyDeviceToHost, s));
    E3D_CUDA(cudaStreamSynchronize(s));
    const int mask = (1 << kTagBits) - 1;
    std::vector<uint32_t> used(N, 0u);
    std::vector<unsigned char> cls(cf.size(), 0xff);  // class of entry e (0xff: the right cell's entry)
    int n_cls = 0;
    std::vector<int> count(33, 0);
    for (int c = 0; c < N; c++)
        for (int e = cptr[c]; e < cptr[c + 1]; e++) {
            const int tag = cf[e].x & mask, idx = cf[e].x >> kTagBits;
            if (tag == TAG_RIGHT) continue;
            const bool inter = tag == TAG_LEFT;
            const uint32_t busy = used[c] | (inter ? used[idx] : 0u);
            if (busy == 0xffffffffu) throw Error(E3D_ERR_MESH, "face colouring needs more than 32 classes");
            const int k = __builtin_ctz(~busy);
            used[c] |= 1u << k;
            if (inter) used[idx] |= 1u << k;
            cls[e] = (unsigned char)k;
            count[k + 1]++;
            n_cls = std::max(n_cls, k + 1);
        }
    for (int k = 0; k < 32; k++) count[k + 1] += count[k];
    std::vector<ColourFace> faces(count[n_cls]);
    std::vector<int> head(count.begin(), count.begin() + n_cls);
    for (int c = 0; c < N; c++)
        for (int e = cptr[c]; e < cptr[c + 1]; e++) {
            if (cls[e] == 0xff) continue;
            const double4 g = fgeo[cf[e].y];
            faces[head[cls[e]]++] = ColourFace{c, cf[e].x >> kTagBits, cf[e].x & mask, 0, g.x, g.y, g.z, g.w};
        }
    S->colour_ptr.assign(count.begin(), count.begin() + n_cls + 1);
    S->n_colours = n_cls;
    S->colour_faces.upload(faces, s);
    S->colour_r.alloc(3 * (size_t)N);
    E3D_CUDA(cudaStreamSynchronize(s));
}

// Face tiles for tile_kernel.  Tile t owns cells [t*T, t*T + T); its local cells are the owned
// ones followed by the halo (outside neighbours, ascending); its faces are every interior face with
// an owned cell (once, interior ones before boundary ones) and its owned cells' boundary faces; each
// owned cell lists its faces in the order of its gather list (ascending reference face id).  Tiles
// whose local cells or faces exceed the entry encoding leave the variant disabled.
static void build_tiles(Solver *S, const std::vector<int> &cptr, const std::vector<int2> &cf,
                        const std::vector<double4> &fgeo, int Fint) {
    const int N = S->N, T = kTileCells;
    const int n_tiles = (N + T - 1) / T;
    std::vector<int> halo_ptr(n_tiles + 1, 0), halo, face_ptr(n_tiles + 1, 0);
    std::vector<long long> rec_off(n_tiles + 1, 0);
    std::vector<FaceRec> tface;
    int max_contrib = 0;
    for (int c = 0; c < N; c++) max_contrib = std::max(max_contrib, cptr[c + 1] - cptr[c]);
    std::vector<unsigned short> contrib((size_t)n_tiles * max_contrib * T, kNoContrib);
    std::vector<int> face_local(Fint, -1), face_tile(Fint, -1);
    int max_cells = 0, max_faces = 0;
    bool ok = max_contrib > 0;
    std::vector<int> hl, bnd, inter_slot, order, sorted;
    std::vector<FaceRec> inter;
    for (int t = 0; t < n_tiles && ok; t++) {
        const int c0 = t * T, c1 = std::min(N, c0 + T);
        hl.clear();
        for (int c = c0; c < c1; c++)
            for (int e = cptr[c]; e < cptr[c + 1]; e++) {
                int tag = cf[e].x & ((1 << kTagBits) - 1);
                int nb = cf[e].x >> kTagBits;
                if (tag <= TAG_RIGHT && (nb < c0 || nb >= c1)) hl.push_back(nb);
            }
        std::sort(hl.begin(), hl.end());
        hl.erase(std::unique(hl.begin(), hl.end()), hl.end());
        auto local = [&](int cell) {
            if (cell >= c0 && cell < c1) return cell - c0;
            return (c1 - c0) + (int)(std::lower_bound(hl.begin(), hl.end(), cell) - hl.begin());
        };
        const int nloc = (c1 - c0) + (int)hl.size();
        if (nloc > (1 << kTileLocalBits)) {
            ok = false;
            break;
        }
        const int fbase = (int)tface.size();  // tile blocks are padded, so fbase is rec_off[t] / 40
        bnd.clear();
        // interior faces first (one entry per face, in bank_order), boundary faces after
        inter.clear();
        inter_slot.clear();
        for (int c = c0; c < c1; c++)
            for (int e = cptr[c]; e < cptr[c + 1]; e++) {
                int tag = cf[e].x & ((1 << kTagBits) - 1);
                int slot = cf[e].y;
                if (tag > TAG_RIGHT) {
                    bnd.push_back(e);
                    continue;
                }
                if (face_tile[slot] == t) continue;
                face_tile[slot] = t;
                int nb = cf[e].x >> kTagBits;
                int l = tag == TAG_LEFT ? local(c) : local(nb);
                int r = tag == TAG_LEFT ? local(nb) : local(c);
                const double4 gq = fgeo[slot];
                inter.push_back(FaceRec{l | (r << kTileLocalBits) | (TAG_LEFT << (2 * kTileLocalBits)), -1, gq.x, gq.y,
                                        gq.z, gq.w});
                inter_slot.push_back(slot);
            }
        bank_order(inter.data(), (int)inter.size(), order, sorted);
        for (int i : order) {
            face_local[inter_slot[i]] = (int)tface.size() - fbase;
            tface.push_back(inter[i]);
        }
        std::vector<int> bnd_local(bnd.size());
        for (size_t b = 0; b < bnd.size(); b++) {
            int e = bnd[b];
            int tag = cf[e].x & ((1 << kTagBits) - 1);
            int c = (int)(std::upper_bound(cptr.begin(), cptr.end(), e) - cptr.begin()) - 1;
            bnd_local[b] = (int)tface.size() - fbase;
            const double4 gq = fgeo[cf[e].y];
            tface.push_back(FaceRec{local(c) | (tag << (2 * kTileLocalBits)), cf[e].y - Fint, gq.x, gq.y, gq.z, gq.w});
        }
        const int nfaces = (int)tface.size() - fbase;
        if (nfaces >= (1 << 15)) {
            ok = false;
            break;
        }
        // contributions in gather-list order
        size_t bi = 0;
        for (int c = c0; c < c1; c++) {
            int k = 0;
            for (int e = cptr[c]; e < cptr[c + 1]; e++, k++) {
                int tag = cf[e].x & ((1 << kTagBits) - 1);
                int jl = tag > TAG_RIGHT ? bnd_local[bi++] : face_local[cf[e].y];
                contrib[((size_t)t * max_contrib + k) * T + (c - c0)] =
                    (unsigned short)((jl << 1) | (tag == TAG_RIGHT ? 1 : 0));
            }
        }
        halo.insert(halo.end(), hl.begin(), hl.end());
        halo_ptr[t + 1] = (int)halo.size();
        face_ptr[t + 1] = face_ptr[t] + nfaces;
        while ((tface.size() * sizeof(FaceRec)) % 16) tface.push_back(FaceRec{0, -1, 0, 0, 0, 0});  // 16-byte blocks
        rec_off[t + 1] = (long long)(tface.size() * sizeof(FaceRec));
        max_cells = std::max(max_cells, nloc);
        max_faces = std::max(max_faces, nfaces);
    }
    const size_t smem = tile_smem_bytes(max_cells, max_faces, max_contrib);
    S->n_tiles = n_tiles;
    S->tiles_ok = ok && smem <= 200 * 1024;
    int max_halo = 0;
    for (int t = 0; t < n_tiles; t++) max_halo = std::max(max_halo, halo_ptr[t + 1] - halo_ptr[t]);
    // the warp-specialised kernel's ring: as many tile buffers as fit (at most eight, at least two)
    const int ws_prec = S->prm.precision == E3D_PREC_FP32_FLUX ? WS_F32 : S->prm.precision == E3D_PREC_FP64 ? WS_FAST : WS_EXACT;
    const size_t ws_stride = ws_buffer_bytes(ws_prec, max_cells, max_faces, max_contrib);
    S->ws_buffers = ws_buffers_for(ws_stride);
    S->pipe_ok = ok && S->ws_buffers >= 2;
    S->pipe_smem = S->pipe_ok ? ws_smem_for(ws_stride, S->ws_buffers) : 0;
    if (!S->tiles_ok) return;
    cudaStream_t s = S->stream;
    // halo lists at a fixed stride per tile, padded with -1: a block reads its entries without
    // first reading where they start
    S->halo_stride = std::max(max_halo, 1);
    std::vector<int> halo_pad((size_t)n_tiles * S->halo_stride, -1);
    for (int t = 0; t < n_tiles; t++)
        std::copy(halo.begin() + halo_ptr[t], halo.begin() + halo_ptr[t + 1], halo_pad.begin() + (size_t)t * S->halo_stride);
    S->tile_halo_ptr.upload(halo_ptr, s);
    S->tile_halo.upload(halo_pad, s);
    S->tile_face_ptr.upload(face_ptr, s);
    S->tile_rec.upload(tface, s);
    S->tile_rec_off.upload(rec_off, s);
    if (S->prm.precision == E3D_PREC_FP32_FLUX) {  // the same faces as 24-byte records, 16-byte blocks
        std::vector<FaceRec32> r32;
        std::vector<long long> off32(n_tiles + 1, 0);
        r32.reserve(tface.size());
        for (int t = 0; t < n_tiles; t++) {
            const size_t f0 = (size_t)(rec_off[t] / (long long)sizeof(FaceRec));
            for (int j = 0; j < face_ptr[t + 1] - face_ptr[t]; j++) {
                const FaceRec &f = tface[f0 + j];
                r32.push_back(FaceRec32{f.code, f.ghost, (float)f.nx, (float)f.ny, (float)f.nz, (float)f.S});
            }
            while ((r32.size() * sizeof(FaceRec32)) % 16) r32.push_back(FaceRec32{0, -1, 0, 0, 0, 0});
            off32[t + 1] = (long long)(r32.size() * sizeof(FaceRec32));
        }
        S->tile_rec32.upload(r32, s);
        S->tile_rec32_off.upload(off32, s);
        S->tile32_smem = tile32_smem_bytes(max_cells, max_faces, max_contrib);
    }
    S->tile_contrib.upload(contrib, s);
    S->max_contrib = max_contrib;
    S->smem_cells = max_cells;
    S->smem_faces = max_faces;
    S->tile_smem = smem;
    S->tile_faces_total = (int64_t)tface.size();
}

// Morton order of approximate cell centres (mean of the cell's face centres): consecutive cells
// form spatially compact groups, which keeps the halo of a face tile small.
static std::vector<int> spatial_order(const e3d_mesh_desc *d) {
    const int N = d->n_cells;
    std::vector<double> cx(3 * (size_t)N);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < N; c++) {
        double s[3] = {0, 0, 0};
        int n = d->cell2face_ptr[c + 1] - d->cell2face_ptr[c];
        for (int k = d->cell2face_ptr[c]; k < d->cell2face_ptr[c + 1]; k++)
            for (int q = 0; q < 3; q++) s[q] += d->face_center[3 * (size_t)d->cell2face[k] + q];
        for (int q = 0; q < 3; q++) {
            cx[3 * (size_t)c + q] = s[q] / std::max(n, 1);
            lo[q] = std::min(lo[q], cx[3 * (size_t)c + q]);
            hi[q] = std::max(hi[q], cx[3 * (size_t)c + q]);
        }
    }
    double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
    std::vector<std::pair<uint64_t, int>> key(N);
    for (int c = 0; c < N; c++) {
        uint64_t qv[3];
        for (int q = 0; q < 3; q++) {
            double u = (cx[3 * (size_t)c + q] - lo[q]) / ext;
            qv[q] = (uint64_t)std::min(std::max(u, 0.0) * 2097151.0, 2097151.0);
        }
        uint64_t m = 0;
        for (int b = 0; b < 21; b++)
            for (int q = 0; q < 3; q++) m |= ((qv[q] >> b) & 1ull) << (3 * b + q);
        key[c] = {m, c};
    }
    std::sort(key.begin(), key.end());
    std::vector<int> order(N);
    for (int c = 0; c < N; c++) order[c] = key[c].second;
    return order;
}

static void create_solver(const e3d_mesh_desc *d, const e3d_flow_params *p, Solver *S) {
    check_desc(d);
    if (!p) throw Error(E3D_ERR_INVALID_ARG, "flow parameters are NULL");
    if (p->precision != E3D_PREC_FP64_EXACT && p->precision != E3D_PREC_FP64 && p->precision != E3D_PREC_FP32_FLUX)
        throw Error(E3D_ERR_INVALID_ARG, "unknown precision mode");
    if (p->scheme != E3D_SCHEME_ROE && p->scheme != E3D_SCHEME_AUSM) throw Error(E3D_ERR_INVALID_ARG, "unknown flux scheme");
    if (p->ordering != E3D_ORDER_NATIVE && p->ordering != E3D_ORDER_RCM && p->ordering != E3D_ORDER_SPATIAL)
        throw Error(E3D_ERR_INVALID_ARG, "unknown cell ordering");
    if (!(p->gamma > 1.0) || !(p->cfl > 0.0) || !(p->mach >= 0.0) || !(p->cref != 0.0) || !(p->sref != 0.0))
        throw Error(E3D_ERR_INVALID_ARG, "flow parameters out of range (gamma > 1, cfl > 0, mach >= 0, cref, sref != 0)");
    for (int ax : {p->cl_axis, p->cd_axis, p->cm_axis})
        if (ax < 0 || ax > 2) throw Error(E3D_ERR_INVALID_ARG, "coefficient axis must be 0, 1 or 2");
    if (p->integrator != E3D_INTEGRATOR_RK5 && p->integrator != E3D_INTEGRATOR_EULER)
        throw Error(E3D_ERR_INVALID_ARG, "unknown integrator (E3D_INTEGRATOR_RK5 or E3D_INTEGRATOR_EULER)");
    if (p->residual_smoothing != 0 && p->residual_smoothing != 1)
        throw Error(E3D_ERR_INVALID_ARG, "residual_smoothing must be 0 or 1");
    if (p->precision == E3D_PREC_FP32_FLUX && (p->integrator != E3D_INTEGRATOR_RK5 || p->residual_smoothing))
        throw Error(E3D_ERR_INVALID_ARG, "FP32_FLUX mode runs RK5 without residual smoothing only");

    int ndev = 0;
    E3D_CUDA(cudaGetDeviceCount(&ndev));
    if (p->device < 0 || p->device >= ndev) throw Error(E3D_ERR_CUDA, "CUDA device ordinal out of range");
    cudaDeviceProp prop;
    E3D_CUDA(cudaGetDeviceProperties(&prop, p->device));
    if (prop.major != 10) throw Error(E3D_ERR_CUDA, "this library is built for sm_100a (B200); device is sm_" +
                                                        std::to_string(prop.major) + std::to_string(prop.minor));
    E3D_CUDA(cudaSetDevice(p->device));
    S->device = p->device;
    S->prm = *p;
    S->n_sm = prop.multiProcessorCount;
    if (p->stream) {
        S->stream = (cudaStream_t)p->stream;
    } else {
        E3D_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
        S->own_stream = true;
    }
    const int N = d->n_cells, F = d->n_faces, Fint = d->n_faces_int, G = F - Fint;
    S->N = N;
    S->F = F;
    S->Fint = Fint;
    S->G = G;

    // ---- validate connectivity and boundary lists
    for (int f = 0; f < F; f++) {
        int L = d->face2cell[2 * f], R = d->face2cell[2 * f + 1];
        if (L < 0 || L >= N) throw Error(E3D_ERR_INVALID_ARG, "face2cell left index out of range at face " + std::to_string(f));
        if (f < Fint ? (R < 0 || R >= N || R == L) : (R != N + (f - Fint)))
            throw Error(E3D_ERR_INVALID_ARG, "face2cell right index is not the reference numbering at face " + std::to_string(f));
    }
    std::vector<int8_t> bc(G, TAG_FROZEN);
    auto mark = [&](int n, const int32_t *gh, const int32_t *in, const int32_t *fc, int tag) {
        for (int i = 0; i < n; i++) {
            int f = fc[i];
            if (f < Fint || f >= F || gh[i] != N + (f - Fint) || in[i] != d->face2cell[2 * f])
                throw Error(E3D_ERR_INVALID_ARG, "boundary list entry inconsistent with face2cell");
            if (bc[f - Fint] != TAG_FROZEN) throw Error(E3D_ERR_INVALID_ARG, "boundary face listed twice");
            bc[f - Fint] = (int8_t)tag;
        }
    };
    mark(d->n_wall, d->wall_ghost, d->wall_interior, d->wall_face, TAG_WALL);
    mark(d->n_sym, d->sym_ghost, d->sym_interior, d->sym_face, TAG_SYM);
    mark(d->n_farfield, d->farfield_ghost, d->farfield_interior, d->farfield_face, TAG_FAR);
    if (d->cell2face_ptr[0] != 0) throw Error(E3D_ERR_INVALID_ARG, "cell2face_ptr[0] must be 0");
    for (int c = 0; c < N; c++)
        if (d->cell2face_ptr[c + 1] < d->cell2face_ptr[c]) throw Error(E3D_ERR_INVALID_ARG, "cell2face_ptr decreasing");
    for (int k = 0; k < d->cell2face_ptr[N]; k++)
        if (d->cell2face[k] < 0 || d->cell2face[k] >= F) throw Error(E3D_ERR_INVALID_ARG, "cell2face index out of range");

    // ---- cell order
    std::vector<int> new2old(N), old2new(N);
    if (p->ordering == E3D_ORDER_RCM) {
        std::vector<int> aptr(N + 1, 0), adj(2 * (size_t)Fint);
        for (int f = 0; f < Fint; f++) {
            aptr[d->face2cell[2 * f] + 1]++;
            aptr[d->face2cell[2 * f + 1] + 1]++;
        }
        for (int c = 0; c < N; c++) aptr[c + 1] += aptr[c];
        std::vector<int> cur(aptr.begin(), aptr.end() - 1);
        for (int f = 0; f < Fint; f++) {
            int L = d->face2cell[2 * f], R = d->face2cell[2 * f + 1];
            adj[cur[L]++] = R;
            adj[cur[R]++] = L;
        }
        new2old = rcm_order(N, aptr, adj);
    } else if (p->ordering == E3D_ORDER_SPATIAL) {
        new2old = spatial_order(d);
    } else {
        std::iota(new2old.begin(), new2old.end(), 0);
    }
    for (int c = 0; c < N; c++) old2new[new2old[c]] = c;

    // ---- per-cell face lists in ascending reference face id (old cell numbering first)
    std::vector<int> cnt(N + 1, 0);
    for (int f = 0; f < F; f++) {
        cnt[d->face2cell[2 * f] + 1]++;
        if (f < Fint) cnt[d->face2cell[2 * f + 1] + 1]++;
    }
    std::vector<int> optr(N + 1, 0);
    for (int c = 0; c < N; c++) optr[c + 1] = optr[c] + cnt[c + 1];
    const int64_t M = optr[N];
    std::vector<int> lst_face(M), lst_code(M);
    {
        std::vector<int> fill(optr.begin(), optr.end() - 1);
        for (int f = 0; f < F; f++) {
            int L = d->face2cell[2 * f], R = d->face2cell[2 * f + 1];
            if (f < Fint) {
                lst_face[fill[L]] = f;
                lst_code[fill[L]++] = (old2new[R] << kTagBits) | TAG_LEFT;
                lst_face[fill[R]] = f;
                lst_code[fill[R]++] = (old2new[L] << kTagBits) | TAG_RIGHT;
            } else {
                lst_face[fill[L]] = f;
                lst_code[fill[L]++] = bc[f - Fint];  // ghost slot filled in below
            }
        }
    }
    // ---- device order: cells by new index; interior faces and ghosts by first use in that order;
    // the geometry of boundary face with ghost slot g sits at slot Fint + g
    std::vector<int> cptr(N + 1, 0);
    std::vector<int2> cf(M);
    std::vector<int> face_slot(F, -1);
    std::vector<double4> fgeo(F), cgeo(N);
    std::vector<int> ghost_ref(G);
    int nf = 0, ng = 0;
    for (int c = 0; c < N; c++) {
        int o = new2old[c];
        cptr[c + 1] = cptr[c] + (optr[o + 1] - optr[o]);
        for (int k = optr[o], j = cptr[c]; k < optr[o + 1]; k++, j++) {
            int f = lst_face[k];
            int code = lst_code[k];
            if (face_slot[f] < 0) {
                if (f < Fint) {
                    face_slot[f] = nf++;
                } else {
                    int g = ng++;
                    ghost_ref[g] = N + (f - Fint);
                    face_slot[f] = Fint + g;
                }
                fgeo[face_slot[f]] = make_double4(d->face_unit_normal[3 * (size_t)f], d->face_unit_normal[3 * (size_t)f + 1],
                                                  d->face_unit_normal[3 * (size_t)f + 2], d->face_area[f]);
            }
            if (f >= Fint) code = ((face_slot[f] - Fint) << kTagBits) | code;
            cf[j] = make_int2(code, face_slot[f]);
        }
        // spectral-radius face sums in the reference's element-to-face order (TimeIntegration.cpp:209-215)
        double sx = 0, sy = 0, sz = 0;
        for (int k = d->cell2face_ptr[o]; k < d->cell2face_ptr[o + 1]; k++) {
            const double *Sv = d->face_normal + 3 * (size_t)d->cell2face[k];
            sx += std::fabs(Sv[0]);
            sy += std::fabs(Sv[1]);
            sz += std::fabs(Sv[2]);
        }
        cgeo[c] = make_double4(sx, sy, sz, d->cell_volume[o]);
    }
    if (nf != Fint || ng != G) throw Error(E3D_ERR_INVALID_ARG, "faces not reached from any cell");

    // ---- face tiles (tile_kernel): kTileCells consecutive cells, their halo, faces, contributions
    build_tiles(S, cptr, cf, fgeo, Fint);

    // ---- freestream, FlowField::Initialize (src/solver/FlowField.cpp:68-101)
    const double PI = 3.141592653589793238;
    Freestream fs;
    fs.rho = 1.0;
    fs.p = 1.0;
    fs.M = p->mach;
    fs.u = p->mach * std::sqrt(p->gamma) * std::cos(p->aoa_deg * (PI / 180));
    fs.v = p->mach * std::sqrt(p->gamma) * std::sin(p->aoa_deg * (PI / 180));
    fs.w = 0.0;
    fs.E = fs.p / ((p->gamma - 1) * fs.rho) + ((fs.u * fs.u + fs.v * fs.v + fs.w * fs.w) / 2.0);
    fs.H = fs.E + (fs.p / fs.rho);
    S->fs = fs;
    double u2 = fs.u * fs.u + fs.v * fs.v + fs.w * fs.w;
    S->cp_factor = 1 / (0.5 * fs.rho * u2);  // AeroCoefficients ctor, src/solver/AeroCoefficients.cpp:25

    // ---- wall list for the force coefficients (reference wall order)
    S->n_wall = d->n_wall;
    std::vector<int> wcell(d->n_wall);
    std::vector<double> wsv(3 * (size_t)d->n_wall), wct(3 * (size_t)d->n_wall);
    for (int i = 0; i < d->n_wall; i++) {
        wcell[i] = old2new[d->wall_interior[i]];
        for (int k = 0; k < 3; k++) {
            wsv[3 * i + k] = d->face_normal[3 * (size_t)d->wall_face[i] + k];
            wct[3 * i + k] = d->face_center[3 * (size_t)d->wall_face[i] + k];
        }
    }

    // ---- upload
    cudaStream_t s = S->stream;
    S->cptr.upload(cptr, s);
    S->cf.upload(cf, s);
    S->fgeo.upload(fgeo, s);
    S->cgeo.upload(cgeo, s);
    S->new2old_d.upload(new2old, s);
    S->ghost_ref_d.upload(ghost_ref, s);
    S->wall_cell.upload(wcell, s);
    S->wall_svec.upload(wsv, s);
    S->wall_center.upload(wct, s);
    S->wall_cp.alloc(std::max(d->n_wall, 1));
    E3D_CUDA(cudaMemsetAsync(S->wall_cp.p, 0, S->wall_cp.n * sizeof(double), s));
    // AeroCoefficients' sum of the wall face vectors (src/solver/AeroCoefficients.cpp:29-33)
    for (int i = 0; i < d->n_wall; i++)
        for (int k = 0; k < 3; k++) S->wall_sum[k] += wsv[3 * i + k];
    S->wall_center_host = wct;
    S->f32 = p->precision == E3D_PREC_FP32_FLUX;
    if (S->f32) {
        if (!S->tiles_ok) throw Error(E3D_ERR_INVALID_ARG, "FP32_FLUX mode needs face tiles this mesh cannot form");
        S->q32[0].alloc(2 * (size_t)N);
        S->q32[1].alloc(2 * (size_t)N);
        std::vector<float4> cg32(N);
        for (int c = 0; c < N; c++)
            cg32[c] = make_float4((float)cgeo[c].x, (float)cgeo[c].y, (float)cgeo[c].z, (float)cgeo[c].w);
        S->cgeo32.upload(cg32, s);
    } else {
        S->q[0].alloc(3 * (size_t)N);
        S->q[1].alloc(3 * (size_t)N);
    }
    S->w0_stride = (N + 31) / 32 * 32;
    S->w0.alloc(5 * (size_t)S->w0_stride);
    if (p->precision == E3D_PREC_FP64_EXACT) S->rsq.alloc(N);
    if (p->residual_smoothing) {
        // interior neighbours of each device cell in the reference's element2face order (which is
        // its element2element order, src/connectivity/Connectivity.cpp:184-218), and 1 + 0.25 n
        // with n counting every face (EulerSolver.cpp:500-504)
        std::vector<int> nptr(N + 1, 0), nbl;
        std::vector<double> den(N);
        nbl.reserve(d->cell2face_ptr[N]);
        for (int c = 0; c < N; c++) {
            const int o = new2old[c];
            for (int k = d->cell2face_ptr[o]; k < d->cell2face_ptr[o + 1]; k++) {
                const int f = d->cell2face[k];
                const int j = d->face2cell[2 * f] == o ? d->face2cell[2 * f + 1] : d->face2cell[2 * f];
                if (j < N) nbl.push_back(old2new[j]);
            }
            nptr[c + 1] = (int)nbl.size();
            den[c] = 1 + (d->cell2face_ptr[o + 1] - d->cell2face_ptr[o]) * 0.25;
        }
        S->smoothing = true;
        S->nb_ptr.upload(nptr, s);
        S->nb.upload(nbl, s);
        S->den.upload(den, s);
        S->rbuf.alloc(3 * 5 * (size_t)S->w0_stride);
        S->smooth_flags.alloc(2);
        E3D_CUDA(cudaMemsetAsync(S->rbuf.p, 0, S->rbuf.n * sizeof(double), s));
    }
    S->ecell.alloc(N);
    S->minit.alloc(N);
    S->ghost.alloc(8 * (size_t)std::max(G, 1));
    S->n_blocks = (N + kStageThreads - 1) / kStageThreads;
    S->partials.alloc(S->n_blocks);
    S->staging.alloc(8 * (size_t)S->state_size());
    S->scratch.alloc(6);
    E3D_CUDA(cudaMalloc(&S->ctl, sizeof(Control)));
    E3D_CUDA(cudaHostAlloc(&S->ctl_host, sizeof(Control), cudaHostAllocDefault));
    E3D_CUDA(cudaMemsetAsync(S->ctl, 0, sizeof(Control), s));
    E3D_CUDA(cudaEventCreate(&S->ev0));
    E3D_CUDA(cudaEventCreate(&S->ev1));
    S->new2old = std::move(new2old);
    S->ghost_ref = std::move(ghost_ref);
    E3D_CUDA(cudaStreamSynchronize(s));
}

static void upload_state(Solver *S, const double *const *arr) {
    const int64_t T = S->state_size();
    for (int k = 0; k < 8; k++) {
        if (!arr[k]) throw Error(E3D_ERR_INVALID_ARG, "state array is NULL");
        E3D_CUDA(cudaMemcpyAsync(S->staging.p + k * T, arr[k], T * sizeof(double), cudaMemcpyHostToDevice, S->stream));
    }
    int threads = 256, blocks = (int)((T + threads - 1) / threads);
    if (S->f32)
        load_state_f32_kernel<<<blocks, threads, 0, S->stream>>>(S->staging.p, T, S->N, S->G, S->new2old_d.p,
                                                                 S->ghost_ref_d.p, S->q32[0].p, S->w0.p,
                                                                 S->w0_stride, S->ecell.p, S->minit.p, S->ghost.p,
                                                                 S->prm.gamma);
    else
        load_state_kernel<<<blocks, threads, 0, S->stream>>>(S->staging.p, T, S->N, S->G, S->new2old_d.p,
                                                             S->ghost_ref_d.p, S->q[0].p, S->w0.p, S->w0_stride,
                                                             S->ecell.p, S->minit.p, S->ghost.p);
    E3D_CUDA(cudaGetLastError());
    S->cur = 0;
    Control init{};
    init.minit_valid = 1;
    std::memcpy(S->ctl_host, &init, sizeof init);
    E3D_CUDA(cudaMemcpyAsync(S->ctl, S->ctl_host, sizeof(Control), cudaMemcpyHostToDevice, S->stream));
    E3D_CUDA(cudaStreamSynchronize(S->stream));
}

static void set_freestream(Solver *S) {
    const int64_t T = S->state_size();
    std::vector<double> buf(8 * (size_t)T);
    const double v[8] = {S->fs.rho, S->fs.u, S->fs.v, S->fs.w, S->fs.p, S->fs.E, S->fs.H, S->fs.M};
    for (int k = 0; k < 8; k++) std::fill(buf.begin() + k * T, buf.begin() + (k + 1) * T, v[k]);
    const double *arr[8];
    for (int k = 0; k < 8; k++) arr[k] = buf.data() + k * T;
    upload_state(S, arr);
}

}  // namespace e3d

using namespace e3d;

namespace e3d {

// A solver that is not a member of a batch (the batch owns its members' state and run).
static Solver *solo(e3d_solver *s) {
    Solver *S = as_solver(s);
    if (S->batch) throw Error(E3D_ERR_INVALID_ARG, "solver is a member of a batch (retire or remove it first)");
    return S;
}

// A fresh control block for a run -- a new EulerSolver's counters (_nbInteration = 0,
// _CL = _CD = _CM = 0, src/solver/EulerSolver.cpp:21-58) -- keeping whether the loaded interior
// Mach still holds.  Reads the old block back first (synchronises stream s once).
static void init_control(Solver *S, const e3d_run_params *rp, int max_iter, int hist_cap, int sample_cap,
                         cudaStream_t s) {
    E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, s));
    E3D_CUDA(cudaStreamSynchronize(s));
    Control init{};
    init.minit_valid = S->ctl_host->minit_valid;
    init.max_iter = max_iter;
    init.sampling = rp->sampling;
    init.hist_cap = hist_cap;
    init.min_res = rp->min_residual;
    init.min_aero = rp->min_aerocoeff_error;
    init.min_drop = rp->min_residual_drop;
    init.sample_cap = sample_cap;
    init.stall_window = std::max(rp->stall_window, 0);
    init.stall_below = rp->stall_below;
    init.done = max_iter == 0;
    std::memcpy(S->ctl_host, &init, sizeof init);
    E3D_CUDA(cudaMemcpyAsync(S->ctl, S->ctl_host, sizeof(Control), cudaMemcpyHostToDevice, s));
}

// Runs start from state buffer 0 (their graphs and launch sequences assume it).
static void state_to_buffer0(Solver *S, cudaStream_t s) {
    if (S->cur == 0) return;
    if (S->f32)
        E3D_CUDA(cudaMemcpyAsync(S->q32[0].p, S->q32[1].p, 2 * (size_t)S->N * sizeof(float4), cudaMemcpyDeviceToDevice,
                                 s));
    else
        E3D_CUDA(cudaMemcpyAsync(S->q[0].p, S->q[1].p, 3 * (size_t)S->N * sizeof(double2), cudaMemcpyDeviceToDevice,
                                 s));
    S->cur = 0;
}

void begin_run(Solver *S, const e3d_run_params *rp, cudaStream_t s) {
    if (rp->sampling <= 0) throw Error(E3D_ERR_INVALID_ARG, "sampling must be a positive integer");
    if (!(rp->min_residual_drop >= 0.0)) throw Error(E3D_ERR_INVALID_ARG, "min_residual_drop must be >= 0");
    const int max_iter = std::max(rp->max_iter, 0);
    // The history and sample buffers grow geometrically from a floor, so that a short run (a
    // warm-up, a first chunk) leaves room for the next one: a reallocation also throws away the
    // instantiated graph, whose finalize and coefficient kernels hold these pointers.
    auto grown = [](int need, int cap, int floor_) {
        return (int)std::min<int64_t>(INT32_MAX, std::max<int64_t>({need, 2 * (int64_t)cap, floor_}));
    };
    if (S->hist_cap < max_iter || !S->hist.p) {
        E3D_CUDA(cudaStreamSynchronize(s));
        const int cap = grown(max_iter, S->hist_cap, 1024);
        S->hist.release();
        S->hist.alloc(cap);
        S->hist_cap = cap;
        if (S->graph) {  // the captured finalize kernels hold the old history pointer
            cudaGraphExecDestroy(S->graph);
            S->graph = nullptr;
        }
    }
    // one sample every `sampling` iterations: max_iter / sampling rows at most
    const int need = max_iter / rp->sampling + 1;
    if (S->sample_cap < need || !S->samples.p) {
        E3D_CUDA(cudaStreamSynchronize(s));
        const int cap = grown(need, S->sample_cap, 256);
        S->samples.release();
        S->samples.alloc(7 * (size_t)cap);
        S->sample_cap = cap;
        if (S->graph) {  // the captured coefficient kernels hold the old pointer
            cudaGraphExecDestroy(S->graph);
            S->graph = nullptr;
        }
    }
    // a fresh AeroCoefficients: Cp of every wall face zero until the first sample
    if (S->n_wall) E3D_CUDA(cudaMemsetAsync(S->wall_cp.p, 0, S->n_wall * sizeof(double), s));
    init_control(S, rp, max_iter, S->hist_cap, S->sample_cap, s);
    state_to_buffer0(S, s);
    S->records_valid = true;
}

void stats_from_control(const Control &c, e3d_run_stats *st) {
    st->iterations = c.it;
    st->stop_reason = c.stop_reason;
    st->n_rms = c.n_rms;
    st->last_rms = c.last_rms;
    st->cl = c.cl;
    st->cd = c.cd;
    st->cm = c.cm;
    for (int k = 0; k < 3; k++) {
        st->force[k] = c.force[k];
        st->moment[k] = c.moment[k];
    }
}

}  // namespace e3d

extern "C" {

e3d_status e3d_solver_create(const e3d_mesh_desc *mesh, const e3d_flow_params *params, e3d_solver **out) {
    if (!out) {
        set_last_error("output handle pointer is NULL");
        return E3D_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<Solver> S(new (std::nothrow) Solver());
    if (!S) {
        set_last_error("host allocation failed");
        return E3D_ERR_OOM;
    }
    e3d_status st = guarded([&] {
        create_solver(mesh, params, S.get());
        set_freestream(S.get());
        if (params->no_autotune) S->use_default_variant();
        else S->autotune();
    });
    if (st == E3D_OK) *out = reinterpret_cast<e3d_solver *>(S.release());
    return st;
}

void e3d_solver_destroy(e3d_solver *solver) {
    if (!solver) return;
    Solver *S = as_solver(solver);
    cudaSetDevice(S->device);
    batch_detach(S);
    if (S->stream) cudaStreamSynchronize(S->stream);
    delete S;
}

e3d_status e3d_solver_info_get(const e3d_solver *solver, e3d_solver_info *info) {
    return guarded([&] {
        if (!solver || !info) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        const Solver *S = reinterpret_cast<const Solver *>(solver);
        std::memset(info, 0, sizeof *info);
        info->n_cells = S->N;
        info->n_ghosts = S->G;
        info->n_faces = S->F;
        info->stage_variant = S->variant;
        info->n_variants = kStageVariants;
        for (int v = 0; v < kStageVariants; v++) info->variant_ms[v] = S->variant_ms[v];
        info->tile_smem_bytes = (int32_t)(S->f32 ? S->tile32_smem : S->tile_smem);
        info->device_bytes = S->device_bytes();
    });
}

int64_t e3d_solver_state_size(const e3d_solver *solver) {
    return solver ? reinterpret_cast<const Solver *>(solver)->state_size() : -1;
}

e3d_status e3d_solver_set_state(e3d_solver *solver, const double *const state[8]) {
    return guarded([&] {
        if (!solver || !state) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        upload_state(S, state);
    });
}

e3d_status e3d_solver_set_freestream(e3d_solver *solver) {
    return guarded([&] {
        if (!solver) throw Error(E3D_ERR_INVALID_ARG, "NULL solver");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        set_freestream(S);
    });
}

e3d_status e3d_solver_get_state(e3d_solver *solver, double *const state[8]) {
    return guarded([&] {
        if (!solver || !state) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        for (int k = 0; k < 8; k++)
            if (!state[k]) throw Error(E3D_ERR_INVALID_ARG, "state array is NULL");
        E3D_CUDA(cudaSetDevice(S->device));
        const int64_t T = S->state_size();
        int threads = 256, blocks = (int)((T + threads - 1) / threads);
        if (S->f32)
            store_state_f32_kernel<<<blocks, threads, 0, S->stream>>>(S->staging.p, T, S->N, S->G, S->new2old_d.p,
                                                                      S->ghost_ref_d.p, S->w0.p, S->w0_stride,
                                                                      S->minit.p, S->ghost.p, S->prm.gamma, S->ctl);
        else
            store_state_kernel<<<blocks, threads, 0, S->stream>>>(S->staging.p, T, S->N, S->G, S->new2old_d.p,
                                                                  S->ghost_ref_d.p, S->q[S->cur].p, S->ecell.p,
                                                                  S->minit.p, S->ghost.p, S->prm.gamma, S->ctl);
        E3D_CUDA(cudaGetLastError());
        for (int k = 0; k < 8; k++)
            E3D_CUDA(cudaMemcpyAsync(state[k], S->staging.p + k * T, T * sizeof(double), cudaMemcpyDeviceToHost,
                                     S->stream));
        E3D_CUDA(cudaStreamSynchronize(S->stream));
    });
}

e3d_status e3d_solver_residual(e3d_solver *solver, double *residual, double *dt) {
    return guarded([&] {
        if (!solver) throw Error(E3D_ERR_INVALID_ARG, "NULL solver");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        const size_t N = (size_t)S->N;
        if (S->staging.n < 6 * N) throw Error(E3D_ERR_INVALID_ARG, "staging buffer too small");
        StageArgs a = S->stage_args(S->cur, 0.0, 1, 0);
        a.residual_only = 1;
        a.r_out = S->staging.p;
        a.dt_out = S->staging.p + 5 * N;
        a.qout = nullptr;
        S->launch_stage(a);
        E3D_CUDA(cudaGetLastError());
        if (residual)
            E3D_CUDA(cudaMemcpyAsync(residual, S->staging.p, 5 * N * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
        if (dt) E3D_CUDA(cudaMemcpyAsync(dt, S->staging.p + 5 * N, N * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
        E3D_CUDA(cudaStreamSynchronize(S->stream));
    });
}

e3d_status e3d_solver_coefficients(e3d_solver *solver, double force[3], double moment[3]) {
    return guarded([&] {
        if (!solver || !force || !moment) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        launch_coeff(S->coeff_args(S->cur, 0, S->scratch.p), S->stream);
        E3D_CUDA(cudaGetLastError());
        double h[6];
        E3D_CUDA(cudaMemcpyAsync(h, S->scratch.p, sizeof h, cudaMemcpyDeviceToHost, S->stream));
        E3D_CUDA(cudaStreamSynchronize(S->stream));
        for (int k = 0; k < 3; k++) {
            force[k] = h[k];
            moment[k] = h[3 + k];
        }
    });
}

e3d_status e3d_solver_run(e3d_solver *solver, const e3d_run_params *rp, e3d_run_stats *stats) {
    return guarded([&] {
        if (!solver || !rp) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        if (rp->sampling <= 0) throw Error(E3D_ERR_INVALID_ARG, "sampling must be a positive integer");
        e3d_run_stats st{};
        const int max_iter = std::max(rp->max_iter, 0);
        begin_run(S, rp, S->stream);
        if (rp->stage_kernel > 0) {
            const int v = rp->stage_kernel - 1;
            if (!S->variant_ok(v))
                throw Error(E3D_ERR_INVALID_ARG, "stage kernel variant not available for this mesh and precision");
            if (v >= kColourVariant) build_colours(S);
            if (S->f32) prepare_tile_f32(S->tile32_smem, S->pipe_smem);
            else if (v >= 2 && S->prm.precision == E3D_PREC_FP64_EXACT) prepare_tile_exact(S->tile_smem, S->pipe_smem);
            else if (v >= 2) prepare_tile_fast(S->tile_smem, S->pipe_smem);
            if (v != S->variant && S->graph) {
                cudaGraphExecDestroy(S->graph);
                S->graph = nullptr;
            }
            S->variant = v;
        }
        int64_t launches = 0;
        double stage_ms = 0.0;
        int64_t stage_launches = 0;
        if (rp->profile_stages < 0 || rp->profile_stages > 2) throw Error(E3D_ERR_INVALID_ARG, "profile_stages must be 0, 1 or 2");
        if (rp->profile_stages != 1) {
            int every = rp->check_every > 0 ? rp->check_every : 32;
            every += every & 1;  // whole graphs start and end on buffer 0
            const bool timed = rp->profile_stages == 2;
            S->build_graph(every, timed);
            E3D_CUDA(cudaEventRecord(S->ev0, S->stream));
            int launched_iters = 0;
            int n_before = 0;  // iterations done before this graph launch (the control block's RMS count)
            while (max_iter > 0) {
                E3D_CUDA(cudaGraphLaunch(S->graph, S->stream));
                launches += (int64_t)S->kernels_per_iteration() * every;
                launched_iters += every;
                E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S->stream));
                E3D_CUDA(cudaStreamSynchronize(S->stream));
                if (timed) {  // the stage kernels of the iterations that ran (later ones return at once)
                    const int ran = std::min(every, S->ctl_host->n_rms - n_before);
                    const int ns = S->n_stages();
                    for (int i = 0; i < ran; i++)
                        for (int st_i = 0; st_i < ns; st_i++) {
                            const cudaEvent_t *e = S->graph_ev.data() + 2 * ((size_t)ns * i + st_i);
                            float ems = 0.f;
                            E3D_CUDA(cudaEventElapsedTime(&ems, e[0], e[1]));
                            stage_ms += ems;
                        }
                    stage_launches += (int64_t)ran * ns;
                    n_before = S->ctl_host->n_rms;
                }
                if (S->ctl_host->done) break;
                if (launched_iters > max_iter + every)
                    throw Error(E3D_ERR_TIMEOUT, "run did not reach its stop condition");
            }
        } else {
            // direct launches, an event pair around every stage (its kernels)
            if (!S->prof_ev[0]) {
                for (auto &e : S->prof_ev) E3D_CUDA(cudaEventCreate(&e));
            }
            E3D_CUDA(cudaEventRecord(S->ev0, S->stream));
            int b = 0;
            for (int it = 0; it < max_iter; it++) {
                const int ns = S->n_stages();
                for (int st_i = 0; st_i < ns; st_i++) {
                    E3D_CUDA(cudaEventRecord(S->prof_ev[2 * st_i], S->stream));
                    S->enqueue_stage(b, st_i, S->partials.p);
                    E3D_CUDA(cudaEventRecord(S->prof_ev[2 * st_i + 1], S->stream));
                    b = 1 - b;
                }
                launch_finalize(S->finalize_args(S->partials.p, S->hist.p), S->stream);
                launch_coeff(S->coeff_args(b, 1, nullptr), S->stream);
                E3D_CUDA(cudaGetLastError());
                launches += S->kernels_per_iteration();
                E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S->stream));
                E3D_CUDA(cudaStreamSynchronize(S->stream));
                for (int st_i = 0; st_i < ns; st_i++) {
                    float ms = 0.f;
                    E3D_CUDA(cudaEventElapsedTime(&ms, S->prof_ev[2 * st_i], S->prof_ev[2 * st_i + 1]));
                    stage_ms += ms;
                }
                stage_launches += ns;
                if (S->ctl_host->done) break;
            }
        }
        E3D_CUDA(cudaEventRecord(S->ev1, S->stream));
        E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S->stream));
        E3D_CUDA(cudaStreamSynchronize(S->stream));
        float ms = 0.f;
        E3D_CUDA(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
        const Control &c = *S->ctl_host;
        S->cur = c.n_rms & 1;
        stats_from_control(c, &st);
        st.device_ms = ms;
        st.kernel_launches = launches;
        st.stage_ms = stage_ms;
        st.stage_launches = stage_launches;
        if (stats) *stats = st;
        if (c.fault) throw Error(E3D_ERR_TIMEOUT, "a bounded device wait gave up (asynchronous copy did not complete)");
        if (c.nonfinite)
            throw Error(E3D_ERR_NONFINITE, "density residual became NaN/Inf at iteration " + std::to_string(c.it));
    });
}

// ---------------------------------------------------------------------------------------------
// Allocation-free run.  The RMS partials and the RMS history of e3d_solver_run_noalloc live in this
// file-scope device array instead of handle buffers, and the iterations are launched directly
// (instantiating a CUDA graph allocates), so the call allocates no memory.  The array is 1.5 MiB,
// exists on every device that loads the library until the process exits, and is shared by every
// call: calls that overlap on the GPU race on it.
constexpr int kNoAllocMaxBlocks = 131072;  // RMS partials -> at most 131072 x 128 = 16,777,216 cells
constexpr int kNoAllocMaxIter = 65536;    // RMS history entries -> at most 65536 iterations per call
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks + kNoAllocMaxIter];

namespace {
std::mutex g_noalloc_mutex;
double *g_noalloc_ptr[64] = {};  // device address of g_noalloc_scratch, per device ordinal
}  // namespace

// Device address of the scratch array on the current device.  Host code may not use the symbol's
// name as a pointer (it names the host-side stand-in), so the address is looked up once per device
// with that device current, on the first call made on it.
static double *noalloc_scratch(int device) {
    if (device < 0 || device >= 64) throw Error(E3D_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        double *p = nullptr;
        cudaError_t err = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p)
            throw Error(E3D_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                          cudaGetErrorString(err));
        g_noalloc_ptr[device] = p;
    }
    return g_noalloc_ptr[device];
}

e3d_status e3d_solver_run_noalloc(e3d_solver *solver, const e3d_run_params *rp, e3d_run_stats *stats,
                                  double *rms_history, int32_t history_capacity) {
    return guarded([&] {
        if (!solver || !rp) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        if (rp->sampling <= 0) throw Error(E3D_ERR_INVALID_ARG, "sampling must be a positive integer");
        const int max_iter = std::max(rp->max_iter, 0);
        if (max_iter > kNoAllocMaxIter)
            throw Error(E3D_ERR_INVALID_ARG, "max_iter " + std::to_string(max_iter) + " exceeds the no-alloc limit of " +
                                                 std::to_string(kNoAllocMaxIter) + " iterations per call");
        if (S->n_blocks > kNoAllocMaxBlocks)
            throw Error(E3D_ERR_INVALID_ARG, "mesh of " + std::to_string(S->N) + " cells exceeds the no-alloc limit of " +
                                                 std::to_string(kNoAllocMaxBlocks * kStageThreads) + " cells");
        if (rp->stage_kernel != 0) throw Error(E3D_ERR_INVALID_ARG, "the no-alloc run uses the handle's stage kernel");
        if (S->euler() || S->smoothing)
            throw Error(E3D_ERR_INVALID_ARG, "the no-alloc run supports RK5 without residual smoothing only");
        if (!(rp->min_residual_drop >= 0.0)) throw Error(E3D_ERR_INVALID_ARG, "min_residual_drop must be >= 0");
        double *partials = noalloc_scratch(S->device);
        double *hist = partials + kNoAllocMaxBlocks;
        // the history region starts cleared, so no entry of an earlier call can be read back
        E3D_CUDA(cudaMemsetAsync(hist, 0, (size_t)std::max(max_iter, 1) * sizeof(double), S->stream));
        // a fresh AeroCoefficients, as e3d_solver_run starts one: wall Cp zero until the first sample
        if (S->n_wall) E3D_CUDA(cudaMemsetAsync(S->wall_cp.p, 0, S->n_wall * sizeof(double), S->stream));
        init_control(S, rp, max_iter, kNoAllocMaxIter, 0, S->stream);
        state_to_buffer0(S, S->stream);
        // the handle's RMS history and sample record still hold an earlier run's: this run keeps
        // neither there (its RMS history goes to rms_history), so the queries of them report none
        S->records_valid = false;
        static const double alphas[5] = {0.0533, 0.1263, 0.2375, 0.4414, 1.0};
        const int every = rp->check_every > 0 ? rp->check_every : 32;
        int64_t launches = 0;
        E3D_CUDA(cudaEventRecord(S->ev0, S->stream));
        int b = 0;
        for (int it = 0; it < max_iter; it++) {
            for (int st_i = 0; st_i < 5; st_i++) {
                StageArgs a = S->stage_args(b, alphas[st_i], st_i == 0, st_i == 4);
                a.partials = partials;
                S->launch_stage(a);
                b = 1 - b;
            }
            launch_finalize(S->finalize_args(partials, hist), S->stream);
            launch_coeff(S->coeff_args(b, 1, nullptr), S->stream);
            E3D_CUDA(cudaGetLastError());
            launches += 5 * S->stage_launches(S->variant) + 2;
            if ((it + 1) % every == 0 || it + 1 == max_iter) {
                E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S->stream));
                E3D_CUDA(cudaStreamSynchronize(S->stream));
                if (S->ctl_host->done) break;
            }
        }
        E3D_CUDA(cudaEventRecord(S->ev1, S->stream));
        E3D_CUDA(cudaMemcpyAsync(S->ctl_host, S->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S->stream));
        E3D_CUDA(cudaStreamSynchronize(S->stream));
        float ms = 0.f;
        E3D_CUDA(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
        const Control &c = *S->ctl_host;
        S->cur = c.n_rms & 1;
        e3d_run_stats st{};
        stats_from_control(c, &st);
        st.device_ms = ms;
        st.kernel_launches = launches;
        if (stats) *stats = st;
        if (rms_history && history_capacity > 0 && c.n_rms > 0)
            E3D_CUDA(cudaMemcpy(rms_history, hist, std::min(c.n_rms, history_capacity) * sizeof(double),
                                cudaMemcpyDeviceToHost));
        if (c.fault) throw Error(E3D_ERR_TIMEOUT, "a bounded device wait gave up (asynchronous copy did not complete)");
        if (c.nonfinite)
            throw Error(E3D_ERR_NONFINITE, "density residual became NaN/Inf at iteration " + std::to_string(c.it));
    });
}

e3d_status e3d_fast_reciprocals(int32_t device, const double *x, int64_t n, double *out) {
    return guarded([&] {
        if (n < 0 || (n > 0 && (!x || !out))) throw Error(E3D_ERR_INVALID_ARG, "NULL argument or negative count");
        if (n == 0) return;
        E3D_CUDA(cudaSetDevice(device));
        struct Bufs {  // released on every exit
            DevBuf<double> x, out;
            ~Bufs() {
                x.release();
                out.release();
            }
        } d;
        d.x.alloc((size_t)n);
        d.out.alloc(4 * (size_t)n);
        E3D_CUDA(cudaMemcpy(d.x.p, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
        launch_fast_reciprocals(d.x.p, n, d.out.p, 0);
        E3D_CUDA(cudaGetLastError());
        E3D_CUDA(cudaMemcpy(out, d.out.p, 4 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

e3d_status e3d_solver_set_wait_limit(e3d_solver *solver, int32_t polls) {
    return guarded([&] {
        if (!solver) throw Error(E3D_ERR_INVALID_ARG, "NULL solver");
        Solver *S = as_solver(solver);
        if (S->batch) throw Error(E3D_ERR_INVALID_ARG, "solver is a member of a batch (retire or remove it first)");
        const int v = polls < 0 ? kWaitLimit : std::min<int>(polls, kWaitLimit);
        if (v != S->wait_polls && S->graph) {  // the captured launches hold the old limit
            E3D_CUDA(cudaSetDevice(S->device));
            E3D_CUDA(cudaStreamSynchronize(S->stream));
            cudaGraphExecDestroy(S->graph);
            S->graph = nullptr;
        }
        S->wait_polls = v;
    });
}

e3d_status e3d_solver_rms_history(e3d_solver *solver, double *out, int32_t capacity, int32_t *count) {
    return guarded([&] {
        if (!solver || !count) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = solo(solver);
        E3D_CUDA(cudaSetDevice(S->device));
        int n = S->records_valid ? std::min(S->ctl_host->n_rms, S->hist_cap) : 0;
        *count = n;
        if (out && capacity > 0 && n > 0)
            E3D_CUDA(cudaMemcpy(out, S->hist.p, std::min(n, capacity) * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"
