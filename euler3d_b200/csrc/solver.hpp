// Host-side solver handle of the euler3d_b200 library, shared by the single-solver entry points
// (solver.cu) and the batch of solvers (batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "common.hpp"
#include "euler3d_b200.h"
#include "stage.cuh"

namespace e3d {

void launch_stage_exact(const StageArgs &a, cudaStream_t s, int variant);
void launch_stage_fast(const StageArgs &a, cudaStream_t s, int variant);
void prepare_tile_exact(size_t smem_bytes, size_t pipe_smem_bytes);
void prepare_tile_fast(size_t smem_bytes, size_t pipe_smem_bytes);
void launch_stage_f32(const StageArgs &a, cudaStream_t s, int variant);
void prepare_tile_f32(size_t smem_bytes, size_t ws_smem_bytes);
// gather (two register budgets), face tiles, warp-specialised persistent face tiles, face tiles at 7 blocks/SM,
// face colouring at 128 and at 512 faces per block
constexpr int kStageVariants = 7;
constexpr int kColourVariant = 5;  // variants 5 and 6
void launch_colour_fast(const StageArgs &a, const ColourFace *faces, int n, double2 *rc, int per_block, cudaStream_t s);
void launch_colour_finish_fast(const StageArgs &a, const double2 *rc, cudaStream_t s);
struct Solver;
void build_colours(Solver *S);

constexpr int kReduceThreads = 256;
constexpr int kCoeffThreads = 512;
void launch_update_exact(const StageArgs &a, cudaStream_t s);
void launch_fast_reciprocals(const double *x, int64_t n, double *out, cudaStream_t s);
void launch_update_fast(const StageArgs &a, cudaStream_t s);
void prepare_batch_exact(size_t smem_bytes, size_t ws_smem_bytes);
void prepare_batch_fast(size_t smem_bytes, size_t ws_smem_bytes);
void prepare_batch_f32(size_t smem_bytes, size_t ws_smem_bytes);
void launch_batch_exact(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);
void launch_batch_fast(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);
void launch_batch_f32(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);
void launch_batch_ws_exact(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);
void launch_batch_ws_fast(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);
void launch_batch_ws_f32(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s);

struct CoeffArgs {
    int n_wall;
    const int *__restrict__ cell;       // device cell of each wall face, reference wall order
    const double *__restrict__ svec;    // 3 per wall face: full face normal
    const double *__restrict__ center;  // 3 per wall face: face centre
    const double2 *__restrict__ q;
    const double *__restrict__ w0;      // FP32_FLUX mode: pressure from the double conservative state
    int w0_stride;
    double gamma;
    double p_inf, cp_factor, cref, sref, ref[3];
    int axis[3], sign[3];
    Control *ctl;
    int run_mode;                       // 1: sampled inside e3d_solver_run, apply the stop test
    int sequential;                     // 1: sum in the reference's wall order (FP64_EXACT)
    double *__restrict__ out;           // 6 doubles (force, moment) when not in run mode
    double *__restrict__ cp_out;        // [n_wall] Cp of every wall face (AeroCoefficients::_cp), or null
    double *__restrict__ samples;       // run mode: 7 doubles (iteration, force, moment) per sample, or null
};

// Arguments of the RMS / stop-test kernel of one solver.
struct FinalizeArgs {
    const double *partials;  // per-tile (per-block) sums of R_rho^2
    int n_part;
    double n_domain;         // interior cells
    double *hist;            // RMS history
    Control *ctl;
    const double *rsq;       // FP64_EXACT: R_rho^2 per cell in reference order, summed sequentially
    int n_cells;
};

// Residual smoothing (EulerSolver::smoothResiduals, src/solver/EulerSolver.cpp:483-518): one Jacobi
// pass over every cell.
struct SmoothArgs {
    int n_cells, stride;                 // stride: row stride of the [5 x stride] residual arrays
    const int *__restrict__ nb_ptr;      // interior neighbours of each cell, element2face order
    const int *__restrict__ nb;
    const double *__restrict__ den;      // 1 + 0.25 x (faces of the cell, ghosts included)
    const double *__restrict__ r0;       // the stage's residual
    const double *__restrict__ last;     // this pass's input
    double *__restrict__ out;
    unsigned long long *flags;           // [0] largest change of the first pass (bits), [1] NaN seen
    Control *ctl;
    int pass;                            // 0 first pass, 1 second pass
};

// Kernels of solver.cu, launched through these.
void launch_finalize(const FinalizeArgs &f, cudaStream_t s);
void launch_coeff(const CoeffArgs &c, cudaStream_t s);
void launch_finalize_batch(const FinalizeArgs *f, const int *n_members, int grid, cudaStream_t s);
void launch_coeff_batch(const CoeffArgs *c, const int *n_members, int parity, int grid, cudaStream_t s);
void launch_control_gather(Control *const *ctl, const int *n_members, Control *out, int grid, cudaStream_t s);
void launch_smooth(const SmoothArgs &a, cudaStream_t s);

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        n = count;
        if (count) E3D_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void upload(const std::vector<T> &v, cudaStream_t s) {
        alloc(v.size());
        if (n) E3D_CUDA(cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
    }
};

struct Batch;

struct Solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int N = 0, G = 0, F = 0, Fint = 0;
    e3d_flow_params prm{};
    Freestream fs{};
    double cp_factor = 0;
    int n_wall = 0;
    int n_blocks = 0;

    std::vector<int> new2old, ghost_ref;  // host copies of the maps

    DevBuf<int> cptr, new2old_d, ghost_ref_d, wall_cell, tile_halo_ptr, tile_halo, tile_face_ptr;
    DevBuf<FaceRec> tile_rec;
    DevBuf<long long> tile_rec_off;
    bool f32 = false;                  // FP32_FLUX mode
    DevBuf<float4> q32[2], cgeo32;
    DevBuf<FaceRec32> tile_rec32;
    DevBuf<long long> tile_rec32_off;
    size_t tile32_smem = 0;
    DevBuf<unsigned short> tile_contrib;
    int w0_stride = 0;
    int halo_stride = 0;        // entries per tile of tile_halo
    bool tiles_ok = false, pipe_ok = false;
    size_t pipe_smem = 0;      // dynamic shared memory of the warp-specialised kernel
    int ws_buffers = 0;        // its tile buffers
    int n_tiles = 0, n_sm = 0;
    int max_contrib = 0, smem_cells = 0, smem_faces = 0;
    size_t tile_smem = 0;
    int64_t tile_faces_total = 0;
    DevBuf<int2> cf;
    DevBuf<double4> fgeo, cgeo;
    DevBuf<double2> q[2];
    DevBuf<double> w0, ecell, minit, ghost, partials, staging, wall_svec, wall_center, hist, scratch;
    // residual smoothing: interior neighbours (element2face order), denominators, residual arrays
    // r0 (the stage's residual), r1, r2 (after the first / second Jacobi pass), pass flags
    bool smoothing = false;
    // output files: the last run's coefficient samples, the wall Cp of the last sample, and host
    // copies of the wall geometry (reference wall order)
    DevBuf<double> samples, wall_cp;
    int sample_cap = 0;
    double wall_sum[3] = {0, 0, 0};
    std::vector<double> wall_center_host;
    DevBuf<int> nb_ptr, nb;
    DevBuf<double> rsq;                 // FP64_EXACT: per-cell R_rho^2 in reference order
    DevBuf<double> den, rbuf;
    DevBuf<unsigned long long> smooth_flags;
    Control *ctl = nullptr;        // device
    Control *ctl_host = nullptr;   // pinned mirror
    int cur = 0;                   // q buffer holding the current state
    int hist_cap = 0;
    // the RMS history and coefficient samples on the device are the last run's (false after an
    // e3d_solver_run_noalloc, which keeps neither in the handle)
    bool records_valid = true;
    int wait_polls = kWaitLimit;   // polls of the stage kernels' data waits (e3d_solver_set_wait_limit)

    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    bool graph_timed = false;             // the graph records graph_ev around its stage kernels
    std::vector<cudaEvent_t> graph_ev;    // [iteration][stage][begin, end] of a timed graph
    Batch *batch = nullptr;        // the batch running this solver, if any (batch.cu)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t prof_ev[10] = {};

    ~Solver() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto e : prof_ev)
            if (e) cudaEventDestroy(e);
        for (auto e : graph_ev) cudaEventDestroy(e);
        DevBuf<int> *ib[] = {&cptr, &new2old_d, &ghost_ref_d, &wall_cell, &tile_halo_ptr, &tile_halo, &tile_face_ptr};
        for (auto *b : ib) b->release();
        tile_rec.release();
        tile_rec_off.release();
        q32[0].release();
        q32[1].release();
        cgeo32.release();
        tile_rec32.release();
        tile_rec32_off.release();
        tile_contrib.release();
        release_colours();
        cf.release();
        fgeo.release();
        cgeo.release();
        q[0].release();
        q[1].release();
        DevBuf<double> *db[] = {&w0, &ecell, &minit, &ghost, &partials, &staging, &wall_svec, &wall_center, &hist,
                                &scratch, &den, &rbuf};
        nb_ptr.release();
        nb.release();
        rsq.release();
        samples.release();
        wall_cp.release();
        smooth_flags.release();
        for (auto *b : db) b->release();
        if (ctl) cudaFree(ctl);
        if (ctl_host) cudaFreeHost(ctl_host);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    int64_t state_size() const { return (int64_t)N + G; }

    // Face colouring (variants 5 and 6, FP64 mode): the faces grouped in classes that share no cell,
    // class k at [colour_ptr[k], colour_ptr[k + 1]), and the residual accumulator.  Built on first
    // use (build_colours), released when the autotuner picks another variant.
    DevBuf<ColourFace> colour_faces;
    std::vector<int> colour_ptr;
    DevBuf<double2> colour_r;  // 3 per cell
    int n_colours = 0;
    void release_colours() {
        colour_faces.release();
        colour_r.release();
        colour_faces.n = colour_r.n = 0;
        colour_ptr.clear();
        n_colours = 0;
    }
    bool colours_built() const { return colour_faces.p != nullptr; }

    int64_t device_bytes() const {
        return (int64_t)(cptr.n + new2old_d.n + ghost_ref_d.n + wall_cell.n + tile_halo_ptr.n + tile_halo.n +
                         tile_face_ptr.n) * 4 + (int64_t)cf.n * 8 + (int64_t)tile_rec.n * 40 + (int64_t)tile_rec_off.n * 8 +
               (int64_t)tile_contrib.n * 2 + (int64_t)(q32[0].n + q32[1].n + cgeo32.n) * 16 + (int64_t)tile_rec32.n * 24 +
               (int64_t)tile_rec32_off.n * 8 +
               (int64_t)(fgeo.n + cgeo.n) * 32 + (int64_t)(q[0].n + q[1].n) * 16 +
               (int64_t)(w0.n + ecell.n + minit.n + ghost.n + partials.n + staging.n + wall_svec.n + wall_center.n +
                         hist.n + scratch.n + den.n + rbuf.n + smooth_flags.n + samples.n + wall_cp.n + rsq.n) * 8 +
               (int64_t)(nb_ptr.n + nb.n) * 4 + (int64_t)colour_faces.n * 48 + (int64_t)colour_r.n * 16 +
               (int64_t)sizeof(Control);
    }

    StageArgs stage_args(int in_buf, double alpha, int first, int last) {
        StageArgs a{};
        a.n_cells = N;
        a.n_ghosts = G;
        a.cptr = cptr.p;
        a.cf = cf.p;
        a.fgeo = fgeo.p;
        a.cgeo = cgeo.p;
        a.qin = q[in_buf].p;
        a.qout = q[1 - in_buf].p;
        a.w0 = w0.p;
        a.ecell = ecell.p;
        a.minit = minit.p;
        a.ghost = ghost.p;
        a.partials = partials.p;
        a.ctl = ctl;
        a.fs = fs;
        a.gamma = prm.gamma;
        a.cfl = prm.cfl;
        a.alpha = alpha;
        a.scheme = prm.scheme;
        a.first_stage = first;
        a.last_stage = last;
        a.new2old = new2old_d.p;
        a.tile_halo_ptr = tile_halo_ptr.p;
        a.tile_halo = tile_halo.p;
        a.tile_face_ptr = tile_face_ptr.p;
        a.tile_rec = reinterpret_cast<const char *>(tile_rec.p);
        a.tile_rec_off = tile_rec_off.p;
        a.tile_contrib = tile_contrib.p;
        a.max_contrib = max_contrib;
        a.smem_cells = smem_cells;
        a.smem_faces = smem_faces;
        a.w0_stride = w0_stride;
        a.fault = &ctl->fault;
        a.halo_stride = halo_stride;
        a.n_tiles = n_tiles;
        a.pipe_grid = std::min(n_tiles, n_sm);
        a.ws_buffers = ws_buffers;
        a.q32in = q32[in_buf].p;
        a.q32out = q32[1 - in_buf].p;
        a.tile_rec32 = reinterpret_cast<const char *>(tile_rec32.p);
        a.tile_rec32_off = tile_rec32_off.p;
        a.cgeo32 = cgeo32.p;
        a.integrator = prm.integrator;
        a.split = 0;
        a.r_dev = nullptr;
        a.rsq = rsq.p;
        a.wait_polls = wait_polls;
        return a;
    }

    int variant = 0;                // stage-kernel variant picked by autotune()
    float variant_ms[kStageVariants] = {};

    // Variants compiled for this precision and possible on this mesh.  FP32_FLUX mode has face-tile
    // kernels only (2 and 4 are its two register budgets, 3 the warp-specialised one); variant 4 is
    // the seven-blocks-per-SM face-tile kernel in FP64 (in FP64_EXACT it would spill).
    bool variant_ok(int v) const {
        if (v < 0 || v >= kStageVariants) return false;
        if (f32) return v == 2 || v == 4 || (v == 3 && pipe_ok);
        if (v == 2) return tiles_ok;
        if (v == 3) return pipe_ok;
        if (v == 4) return tiles_ok && prm.precision == E3D_PREC_FP64;
        if (v >= kColourVariant) return prm.precision == E3D_PREC_FP64;
        return true;
    }

    // The launches of one stage with variant v (face colouring: one per class and the update).
    int stage_launches(int v) const { return v >= kColourVariant ? n_colours + 1 : 1; }

    void launch_stage(const StageArgs &a, int v = -1) {
        if (v < 0) v = variant;
        if (v >= kColourVariant) {  // the accumulator is cleared, every class adds, the update reads it
            E3D_CUDA(cudaMemsetAsync(colour_r.p, 0, colour_r.n * sizeof(double2), stream));
            const int per_block = v == kColourVariant ? 128 : 512;
            for (int k = 0; k < n_colours; k++)
                launch_colour_fast(a, colour_faces.p + colour_ptr[k], colour_ptr[k + 1] - colour_ptr[k], colour_r.p,
                                   per_block, stream);
            launch_colour_finish_fast(a, colour_r.p, stream);
            return;
        }
        if (f32) launch_stage_f32(a, stream, v);
        else if (prm.precision == E3D_PREC_FP64_EXACT) launch_stage_exact(a, stream, v);
        else launch_stage_fast(a, stream, v);
    }

    // Time every stage-kernel variant on this mesh and keep the fastest.  The trial launches
    // read the current state and write only scratch: the other state buffer (overwritten by the
    // next real stage anyway) and a copy of the ghost cells; W0, E and the RMS partials are
    // untouched (not a last stage), so results do not depend on the tuning.
    void autotune() {
        DevBuf<double> ghost_copy;
        ghost_copy.alloc(ghost.n);
        E3D_CUDA(cudaMemcpyAsync(ghost_copy.p, ghost.p, ghost.n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        StageArgs a = stage_args(cur, 0.0533, 1, 0);
        a.ghost = ghost_copy.p;
        const int reps = N > 200000 ? 3 : 10;
        float best = 1e30f;
        if (f32) {
            prepare_tile_f32(tile32_smem, pipe_smem);
        } else if (tiles_ok) {
            if (prm.precision == E3D_PREC_FP64_EXACT) prepare_tile_exact(tile_smem, pipe_smem);
            else prepare_tile_fast(tile_smem, pipe_smem);
        }
        if (variant_ok(kColourVariant)) build_colours(this);
        for (int v = 0; v < kStageVariants; v++) {
            variant_ms[v] = -1.0f;
            if (!variant_ok(v)) continue;
            launch_stage(a, v);  // warm
            E3D_CUDA(cudaEventRecord(ev0, stream));
            for (int r = 0; r < reps; r++) launch_stage(a, v);
            E3D_CUDA(cudaEventRecord(ev1, stream));
            E3D_CUDA(cudaEventSynchronize(ev1));
            float ms = 0.f;
            E3D_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
            variant_ms[v] = ms / reps;
            if (variant_ms[v] < best) {
                best = variant_ms[v];
                variant = v;
            }
        }
        E3D_CUDA(cudaGetLastError());
        ghost_copy.release();
        if (variant < kColourVariant) {
            E3D_CUDA(cudaStreamSynchronize(stream));
            release_colours();
        }
    }

    // Without tuning: the face-tile kernel (seven blocks per SM in FP64, eight in FP32_FLUX), or the
    // gather kernel when the mesh does not fit the tiles.
    void use_default_variant() {
        for (auto &m : variant_ms) m = -1.0f;
        if (f32) {
            variant = 4;
            prepare_tile_f32(tile32_smem, pipe_smem);
        } else if (tiles_ok) {
            variant = prm.precision == E3D_PREC_FP64 ? 4 : 2;
            if (prm.precision == E3D_PREC_FP64_EXACT) prepare_tile_exact(tile_smem, pipe_smem);
            else prepare_tile_fast(tile_smem, pipe_smem);
        } else {
            variant = 1;
        }
    }

    CoeffArgs coeff_args(int buf, int run_mode, double *out) {
        CoeffArgs c{};
        c.n_wall = n_wall;
        c.cell = wall_cell.p;
        c.svec = wall_svec.p;
        c.center = wall_center.p;
        c.q = q[buf].p;
        c.p_inf = fs.p;
        c.cp_factor = cp_factor;
        c.cref = prm.cref;
        c.sref = prm.sref;
        for (int k = 0; k < 3; k++) c.ref[k] = prm.ref_point[k];
        c.axis[0] = prm.cl_axis;
        c.axis[1] = prm.cd_axis;
        c.axis[2] = prm.cm_axis;
        c.sign[0] = prm.cl_sign;
        c.sign[1] = prm.cd_sign;
        c.sign[2] = prm.cm_sign;
        c.ctl = ctl;
        c.run_mode = run_mode;
        c.sequential = prm.precision == E3D_PREC_FP64_EXACT;
        c.w0 = f32 ? w0.p : nullptr;
        c.w0_stride = w0_stride;
        c.gamma = prm.gamma;
        c.out = out;
        c.cp_out = wall_cp.p;
        c.samples = run_mode ? samples.p : nullptr;
        return c;
    }

    FinalizeArgs finalize_args(const double *part, double *h) const {
        return FinalizeArgs{part, n_blocks, (double)N, h, ctl, rsq.p, N};
    }

    bool euler() const { return prm.integrator == E3D_INTEGRATOR_EULER; }
    // Stages per iteration (RK5: 5; explicit Euler: 1) and kernels per stage and per iteration.
    int n_stages() const { return euler() ? 1 : 5; }
    int kernels_per_stage() const { return stage_launches(variant) + (smoothing ? 3 : 0); }
    int kernels_per_iteration() const { return n_stages() * kernels_per_stage() + 2; }

    // Stage s of an iteration from q[b] (EulerSolver::RungeKutta, src/solver/EulerSolver.cpp:425-472,
    // or EulerSolver::EulerExplicit, :419-423).  Without smoothing one fused kernel; with it the
    // residual phase writes R, two Jacobi passes smooth it (EulerSolver::smoothResiduals, :483-518,
    // called by Run() :91-93 for the first stage and by RungeKutta :456-458 for the others) and the
    // update kernel applies it.
    void enqueue_stage(int b, int s, double *part) {
        static const double alphas[5] = {0.0533, 0.1263, 0.2375, 0.4414, 1.0};
        StageArgs a = stage_args(b, euler() ? 1.0 : alphas[s], s == 0, euler() || s == 4);
        a.partials = part;
        if (!smoothing) {
            launch_stage(a);
            return;
        }
        const size_t n5 = 5 * (size_t)w0_stride;
        double *r0 = rbuf.p, *r1 = rbuf.p + n5, *r2 = rbuf.p + 2 * n5;
        StageArgs ar = a;
        ar.split = 1;
        ar.ghost_out = a.last_stage;  // the residual phase of the last stage leaves the ghosts
        ar.last_stage = 0;
        ar.r_dev = r0;
        launch_stage(ar);
        E3D_CUDA(cudaMemsetAsync(smooth_flags.p, 0, 2 * sizeof(unsigned long long), stream));
        SmoothArgs sa{N, w0_stride, nb_ptr.p, nb.p, den.p, r0, r0, r1, smooth_flags.p, ctl, 0};
        launch_smooth(sa, stream);
        sa.last = r1;
        sa.out = r2;
        sa.pass = 1;
        launch_smooth(sa, stream);
        a.r_dev = r2;
        if (prm.precision == E3D_PREC_FP64_EXACT) launch_update_exact(a, stream);
        else launch_update_fast(a, stream);
    }

    // One iteration of EulerSolver::Run (src/solver/EulerSolver.cpp:84-153) starting from q[in_buf];
    // returns the kernels launched.  With ev, event pair ev[2 s], ev[2 s + 1] brackets stage s (as
    // external event-record nodes when the stream is being captured).
    int enqueue_iteration(int in_buf, const cudaEvent_t *ev = nullptr) {
        int b = in_buf;
        for (int s = 0; s < n_stages(); s++) {
            if (ev) E3D_CUDA(cudaEventRecordWithFlags(ev[2 * s], stream, cudaEventRecordExternal));
            enqueue_stage(b, s, partials.p);
            if (ev) E3D_CUDA(cudaEventRecordWithFlags(ev[2 * s + 1], stream, cudaEventRecordExternal));
            b = 1 - b;
        }
        launch_finalize(finalize_args(partials.p, hist.p), stream);
        launch_coeff(coeff_args(b, 1, nullptr), stream);
        return kernels_per_iteration();
    }

    // A graph of `iters` iterations; with `timed`, an event pair around every stage kernel (see
    // e3d_run_params.profile_stages = 2).
    void build_graph(int iters, bool timed = false) {
        if (graph && graph_iters == iters && graph_timed == timed) return;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        const size_t n_ev = timed ? 2 * (size_t)n_stages() * iters : 0;
        while (graph_ev.size() < n_ev) {
            cudaEvent_t e;
            E3D_CUDA(cudaEventCreate(&e));
            graph_ev.push_back(e);
        }
        cudaGraph_t g;
        E3D_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int b = 0;
        for (int i = 0; i < iters; i++) {
            enqueue_iteration(b, timed ? graph_ev.data() + 2 * (size_t)n_stages() * i : nullptr);
            b = 1 - b;  // five stages flip the buffer once per iteration
        }
        cudaError_t cap = cudaStreamEndCapture(stream, &g);
        E3D_CUDA(cap);
        cudaError_t inst = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        E3D_CUDA(inst);
        graph_iters = iters;
        graph_timed = timed;
    }
};

inline Solver *as_solver(e3d_solver *s) { return reinterpret_cast<Solver *>(s); }

// Start of a run (e3d_solver_run and e3d_batch_add): history capacity, a fresh control block
// and the current state moved to buffer 0, all enqueued on stream s.
void begin_run(Solver *S, const e3d_run_params *rp, cudaStream_t s);
// Run statistics from a control block read back from the device.
void stats_from_control(const Control &c, e3d_run_stats *st);
// Take a solver out of the batch that holds it (e3d_solver_destroy of a member).
void batch_detach(Solver *S);

}  // namespace e3d
