// Batches of solvers advanced in shared launches: the e3d_batch_* half of the C ABI
// (include/euler3d_b200.h).
//
// Device tables of a batch (sized to capacities that only change when the membership outgrows
// them, so that one captured CUDA graph serves many membership changes):
//   args[2m + b]    StageArgs of member m reading state buffer b (its own mesh, buffers, flow)
//   cargs[2m + b]   CoeffArgs of member m for state buffer b
//   fargs[m]        FinalizeArgs of member m (its RMS partials, history and control block)
//   table[k]        (member, tile) of stage-kernel block k, running members only
//   counts          [0] table entries, [1] members
// One iteration = 5 stage launches over the table + one finalize and one coefficient launch of
// one block per member; a step = `iters` iterations + a gather of the members' control blocks and
// one copy of them to the host, all in one graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "solver.hpp"
#include "stage_ws.cuh"

namespace e3d {

struct Member {
    Solver *S = nullptr;
    bool stopped = false;  // its run has stopped (seen in the last control read-back)
    bool fault = false;    // a bounded device wait gave up, or the run overran its stop condition
    Control last{};        // control block as of the last step
    double ms = 0.0;       // device time of the steps it took part in
    int64_t launches = 0;  // kernels of the steps it took part in
    int64_t iters = 0;     // iterations launched for it
};

struct Batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int precision = -1;  // E3D_PREC_* of the members (set by the first one)
    std::vector<Member> members;
    std::mutex mu;

    DevBuf<StageArgs> args;
    DevBuf<CoeffArgs> cargs;
    DevBuf<FinalizeArgs> fargs;
    DevBuf<Control *> ctlp;
    DevBuf<int2> table;
    DevBuf<int> counts;
    DevBuf<Control> ctl_all;
    Control *ctl_host = nullptr;  // pinned, member_cap entries
    int *one_host = nullptr;      // pinned constant 1 (sets a member's done flag)
    int member_cap = 0, tile_cap = 0;
    size_t smem_cap = 0;
    // stage kernel: E3D_BATCH_KERNEL_TILES (one block per table entry) or E3D_BATCH_KERNEL_WS (the
    // warp-specialised persistent kernel walking the table); its ring of buffers
    int kernel = E3D_BATCH_KERNEL_TILES;
    int n_sm = 0;
    int ws_buffers = 0;
    size_t ws_stride = 0, ws_smem = 0;
    int n_entries = 0;
    bool dirty = true;

    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    int graph_builds = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int64_t launches = 0;

    ~Batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        args.release();
        cargs.release();
        fargs.release();
        ctlp.release();
        table.release();
        counts.release();
        ctl_all.release();
        if (ctl_host) cudaFreeHost(ctl_host);
        if (one_host) cudaFreeHost(one_host);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }

    static int grow(int need, int floor_) {
        int c = floor_;
        while (c < need) c *= 2;
        return c;
    }

    size_t member_smem(const Solver *S) const { return S->f32 ? S->tile32_smem : S->tile_smem; }

    // Rebuild the device tables for the current membership; resize (and drop the graph) when a
    // capacity no longer fits or the tile table has shrunk well below its capacity.
    void refresh() {
        const int nm = (int)members.size();
        std::vector<StageArgs> A(2 * (size_t)nm);
        std::vector<CoeffArgs> C(2 * (size_t)nm);
        std::vector<FinalizeArgs> Fa(nm);
        std::vector<Control *> P(nm);
        std::vector<int2> T;
        size_t smem = 0;
        for (int m = 0; m < nm; m++) {
            Solver *S = members[m].S;
            for (int b = 0; b < 2; b++) {
                A[2 * m + b] = S->stage_args(b, 0.0, 0, 0);  // alpha and stage flags come per launch
                C[2 * m + b] = S->coeff_args(b, 1, nullptr);
            }
            Fa[m] = S->finalize_args(S->partials.p, S->hist.p);
            P[m] = S->ctl;
            smem = std::max(smem, member_smem(S));
            if (!members[m].stopped)
                for (int t = 0; t < S->n_tiles; t++) T.push_back(make_int2(m, t));
        }
        n_entries = (int)T.size();
        const int mcap = grow(std::max(nm, 1), 8);
        int tcap = tile_cap;
        if (n_entries > tile_cap || n_entries * 4 < tile_cap) tcap = grow(std::max(n_entries, 1), 64);
        if (mcap > member_cap) {
            drop_graph();
            args.release();
            cargs.release();
            fargs.release();
            ctlp.release();
            ctl_all.release();
            if (ctl_host) cudaFreeHost(ctl_host);
            ctl_host = nullptr;
            args.alloc(2 * (size_t)mcap);
            cargs.alloc(2 * (size_t)mcap);
            fargs.alloc(mcap);
            ctlp.alloc(mcap);
            ctl_all.alloc(mcap);
            E3D_CUDA(cudaMallocHost(&ctl_host, (size_t)mcap * sizeof(Control)));
            member_cap = mcap;
        }
        if (tcap != tile_cap) {
            drop_graph();
            table.release();
            table.alloc(tcap);
            tile_cap = tcap;
        }
        if (smem > smem_cap) {
            drop_graph();
            smem_cap = smem;
        }
        // the warp-specialised kernel's buffers: the largest member's tile data plus its arguments
        size_t stride = 0;
        for (const Member &m : members) {
            const int wp = m.S->f32 ? WS_F32 : m.S->prm.precision == E3D_PREC_FP64 ? WS_FAST : WS_EXACT;
            stride = std::max(stride, kWsArgsSlot + ws_buffer_bytes(wp, m.S->smem_cells, m.S->smem_faces, m.S->max_contrib));
        }
        if (stride > ws_stride) {
            drop_graph();
            ws_stride = stride;
            ws_buffers = ws_buffers_for(ws_stride);
            ws_smem = ws_buffers ? ws_smem_for(ws_stride, ws_buffers) : 0;
        }
        if (!counts.p) counts.alloc(2);
        if (nm) {
            E3D_CUDA(cudaMemcpyAsync(args.p, A.data(), A.size() * sizeof(StageArgs), cudaMemcpyHostToDevice, stream));
            E3D_CUDA(cudaMemcpyAsync(cargs.p, C.data(), C.size() * sizeof(CoeffArgs), cudaMemcpyHostToDevice, stream));
            E3D_CUDA(cudaMemcpyAsync(fargs.p, Fa.data(), Fa.size() * sizeof(FinalizeArgs), cudaMemcpyHostToDevice,
                                     stream));
            E3D_CUDA(cudaMemcpyAsync(ctlp.p, P.data(), P.size() * sizeof(Control *), cudaMemcpyHostToDevice, stream));
        }
        if (n_entries)
            E3D_CUDA(cudaMemcpyAsync(table.p, T.data(), T.size() * sizeof(int2), cudaMemcpyHostToDevice, stream));
        const int cnt[2] = {n_entries, nm};
        E3D_CUDA(cudaMemcpyAsync(counts.p, cnt, sizeof cnt, cudaMemcpyHostToDevice, stream));
        E3D_CUDA(cudaStreamSynchronize(stream));  // the host vectors go out of scope
        dirty = false;
    }

    bool use_ws() const { return kernel == E3D_BATCH_KERNEL_WS && ws_buffers >= 2; }

    void launch_stage(BatchStage bs) {
        if (use_ws()) {
            bs.ws_buffers = ws_buffers;
            bs.ws_stride = (int)ws_stride;
            const int grid = std::max(1, std::min(tile_cap, n_sm));
            if (precision == E3D_PREC_FP32_FLUX) launch_batch_ws_f32(bs, grid, ws_smem, stream);
            else if (precision == E3D_PREC_FP64_EXACT) launch_batch_ws_exact(bs, grid, ws_smem, stream);
            else launch_batch_ws_fast(bs, grid, ws_smem, stream);
            return;
        }
        if (precision == E3D_PREC_FP32_FLUX) launch_batch_f32(bs, tile_cap, smem_cap, stream);
        else if (precision == E3D_PREC_FP64_EXACT) launch_batch_exact(bs, tile_cap, smem_cap, stream);
        else launch_batch_fast(bs, tile_cap, smem_cap, stream);
    }

    // `iters` iterations (even, so every running member ends on state buffer 0) + the control
    // read-back, as one graph.
    void build_graph(int iters) {
        drop_graph();
        const size_t wss = use_ws() ? ws_smem : 0;
        if (precision == E3D_PREC_FP32_FLUX) prepare_batch_f32(smem_cap, wss);
        else if (precision == E3D_PREC_FP64_EXACT) prepare_batch_exact(smem_cap, wss);
        else prepare_batch_fast(smem_cap, wss);
        static const double alphas[5] = {0.0533, 0.1263, 0.2375, 0.4414, 1.0};
        cudaGraph_t g;
        E3D_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < iters; i++) {
            const int p = i & 1;
            for (int s = 0; s < 5; s++) {
                BatchStage bs{};
                bs.args = args.p;
                bs.table = table.p;
                bs.n_entries = counts.p;
                bs.alpha = alphas[s];
                bs.first_stage = s == 0;
                bs.last_stage = s == 4;
                bs.parity = p ^ (s & 1);
                launch_stage(bs);
            }
            launch_finalize_batch(fargs.p, counts.p + 1, member_cap, stream);
            launch_coeff_batch(cargs.p, counts.p + 1, 1 - p, member_cap, stream);
        }
        launch_control_gather(ctlp.p, counts.p + 1, ctl_all.p, member_cap, stream);
        cudaMemcpyAsync(ctl_host, ctl_all.p, (size_t)member_cap * sizeof(Control), cudaMemcpyDeviceToHost, stream);
        cudaError_t cap = cudaStreamEndCapture(stream, &g);
        E3D_CUDA(cap);
        cudaError_t inst = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        E3D_CUDA(inst);
        graph_iters = iters;
        graph_builds++;
    }

    int running() const {
        int n = 0;
        for (const Member &m : members) n += !m.stopped;
        return n;
    }

    // Stop a member on the device (its later kernels return at once).
    void halt(Member &m) { E3D_CUDA(cudaMemcpyAsync(&m.S->ctl->done, one_host, sizeof(int), cudaMemcpyHostToDevice, stream)); }

    void step(int iters) {
        if (running() == 0) return;
        const int every = std::max(2, iters + (iters & 1));
        if (dirty) refresh();
        if (!graph || graph_iters != every) build_graph(every);
        E3D_CUDA(cudaEventRecord(ev0, stream));
        E3D_CUDA(cudaGraphLaunch(graph, stream));
        E3D_CUDA(cudaEventRecord(ev1, stream));
        E3D_CUDA(cudaStreamSynchronize(stream));
        float ms = 0.f;
        E3D_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        const int64_t step_launches = 7LL * every + 1;
        launches += step_launches;
        bool halted = false;
        for (size_t k = 0; k < members.size(); k++) {
            Member &m = members[k];
            if (m.stopped) continue;
            m.last = ctl_host[k];
            m.ms += ms;
            m.launches += step_launches;
            m.iters += every;
            if (m.last.fault || (!m.last.done && m.iters > (int64_t)m.last.max_iter + every)) {
                m.fault = true;
                halt(m);
                halted = true;
            }
            if (m.last.done || m.fault) {
                m.stopped = true;
                dirty = true;
            }
        }
        if (halted) E3D_CUDA(cudaStreamSynchronize(stream));
    }

    // Hand a member's solver back: stats and status as e3d_solver_run would give them.
    e3d_status release(Member &m, e3d_run_stats *stats) {
        Solver *S = m.S;
        e3d_run_stats st{};
        stats_from_control(m.last, &st);
        st.device_ms = m.ms;
        st.kernel_launches = m.launches;
        if (stats) *stats = st;
        std::memcpy(S->ctl_host, &m.last, sizeof(Control));
        S->cur = m.last.n_rms & 1;
        S->batch = nullptr;
        if (m.fault || m.last.fault) return E3D_ERR_TIMEOUT;
        if (m.last.nonfinite) return E3D_ERR_NONFINITE;
        return E3D_OK;
    }

    int find(const Solver *S) const {
        for (size_t k = 0; k < members.size(); k++)
            if (members[k].S == S) return (int)k;
        return -1;
    }
};

static Batch *as_batch(e3d_batch *b) { return reinterpret_cast<Batch *>(b); }

void batch_detach(Solver *S) {
    Batch *B = S->batch;
    if (!B) return;
    std::lock_guard<std::mutex> lock(B->mu);
    const int k = B->find(S);
    if (k >= 0) {
        B->release(B->members[k], nullptr);
        B->members.erase(B->members.begin() + k);
        B->dirty = true;
    }
    S->batch = nullptr;
}

}  // namespace e3d

using namespace e3d;

extern "C" {

e3d_status e3d_batch_create(int32_t device, void *stream, e3d_batch **out) {
    return guarded([&] {
        if (!out) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        *out = nullptr;
        int n = 0;
        E3D_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Error(E3D_ERR_INVALID_ARG, "device ordinal out of range");
        E3D_CUDA(cudaSetDevice(device));
        auto B = std::make_unique<Batch>();
        B->device = device;
        if (stream) {
            B->stream = static_cast<cudaStream_t>(stream);
        } else {
            E3D_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
            B->own_stream = true;
        }
        E3D_CUDA(cudaDeviceGetAttribute(&B->n_sm, cudaDevAttrMultiProcessorCount, device));
        E3D_CUDA(cudaEventCreate(&B->ev0));
        E3D_CUDA(cudaEventCreate(&B->ev1));
        E3D_CUDA(cudaMallocHost(&B->one_host, sizeof(int)));
        *B->one_host = 1;
        *out = reinterpret_cast<e3d_batch *>(B.release());
    });
}

void e3d_batch_destroy(e3d_batch *batch) {
    if (!batch) return;
    Batch *B = as_batch(batch);
    cudaSetDevice(B->device);
    {
        std::lock_guard<std::mutex> lock(B->mu);
        cudaStreamSynchronize(B->stream);
        for (Member &m : B->members) B->release(m, nullptr);
        B->members.clear();
    }
    delete B;
}

e3d_status e3d_batch_add(e3d_batch *batch, e3d_solver *solver, const e3d_run_params *rp) {
    return guarded([&] {
        if (!batch || !solver || !rp) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Batch *B = as_batch(batch);
        Solver *S = as_solver(solver);
        std::lock_guard<std::mutex> lock(B->mu);
        if (S->batch) throw Error(E3D_ERR_INVALID_ARG, "solver is already a member of a batch");
        if (S->device != B->device) throw Error(E3D_ERR_INVALID_ARG, "solver and batch are on different devices");
        if (B->precision >= 0 && S->prm.precision != B->precision)
            throw Error(E3D_ERR_INVALID_ARG, "solver precision differs from the batch's members");
        if (!S->tiles_ok)
            throw Error(E3D_ERR_INVALID_ARG, "the solver's mesh does not fit the face-tile kernel a batch runs");
        if (S->euler() || S->smoothing)
            throw Error(E3D_ERR_INVALID_ARG, "batch members run RK5 without residual smoothing");
        E3D_CUDA(cudaSetDevice(B->device));
        E3D_CUDA(cudaStreamSynchronize(S->stream));  // the solver's own pending work (state uploads)
        begin_run(S, rp, B->stream);
        Member m;
        m.S = S;
        std::memcpy(&m.last, S->ctl_host, sizeof(Control));
        m.stopped = m.last.done != 0;  // max_iter 0: nothing to run
        B->members.push_back(m);
        B->precision = S->prm.precision;
        S->batch = B;
        B->dirty = true;
    });
}

e3d_status e3d_batch_step(e3d_batch *batch, int32_t iterations, int32_t *n_active) {
    return guarded([&] {
        if (!batch) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        if (iterations <= 0) throw Error(E3D_ERR_INVALID_ARG, "iterations must be positive");
        Batch *B = as_batch(batch);
        std::lock_guard<std::mutex> lock(B->mu);
        E3D_CUDA(cudaSetDevice(B->device));
        B->step(iterations);
        if (n_active) *n_active = B->running();
    });
}

e3d_status e3d_batch_retire(e3d_batch *batch, e3d_solver **solvers, e3d_run_stats *stats, e3d_status *status,
                            int32_t capacity, int32_t *count) {
    return guarded([&] {
        if (!batch || !count || (capacity > 0 && !solvers)) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Batch *B = as_batch(batch);
        std::lock_guard<std::mutex> lock(B->mu);
        int n = 0;
        std::vector<Member> keep;
        keep.reserve(B->members.size());
        for (Member &m : B->members) {
            if (m.stopped && n < capacity) {
                solvers[n] = reinterpret_cast<e3d_solver *>(m.S);
                const e3d_status st = B->release(m, stats ? stats + n : nullptr);
                if (status) status[n] = st;
                n++;
            } else {
                keep.push_back(m);
            }
        }
        if (n) {
            B->members.swap(keep);
            B->dirty = true;
        }
        *count = n;
    });
}

e3d_status e3d_batch_remove(e3d_batch *batch, e3d_solver *solver, e3d_run_stats *stats) {
    return guarded([&] {
        if (!batch || !solver) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Batch *B = as_batch(batch);
        Solver *S = as_solver(solver);
        std::lock_guard<std::mutex> lock(B->mu);
        const int k = B->find(S);
        if (k < 0) throw Error(E3D_ERR_INVALID_ARG, "solver is not a member of this batch");
        B->release(B->members[k], stats);
        B->members.erase(B->members.begin() + k);
        B->dirty = true;
    });
}

e3d_status e3d_batch_set_kernel(e3d_batch *batch, int32_t kernel) {
    return guarded([&] {
        if (!batch) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        if (kernel != E3D_BATCH_KERNEL_TILES && kernel != E3D_BATCH_KERNEL_WS)
            throw Error(E3D_ERR_INVALID_ARG, "unknown batch stage kernel");
        Batch *B = as_batch(batch);
        std::lock_guard<std::mutex> lock(B->mu);
        if (kernel != B->kernel) {
            E3D_CUDA(cudaSetDevice(B->device));
            E3D_CUDA(cudaStreamSynchronize(B->stream));
            B->drop_graph();
            B->kernel = kernel;
        }
    });
}

e3d_status e3d_batch_info_get(const e3d_batch *batch, e3d_batch_info *info) {
    return guarded([&] {
        if (!batch || !info) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Batch *B = const_cast<Batch *>(reinterpret_cast<const Batch *>(batch));
        std::lock_guard<std::mutex> lock(B->mu);
        e3d_batch_info r{};
        r.n_members = (int32_t)B->members.size();
        r.n_running = B->running();
        r.n_tiles = B->n_entries;
        r.graph_builds = B->graph_builds;
        for (const Member &m : B->members) r.member_device_bytes += m.S->device_bytes();
        r.device_bytes = (int64_t)(B->args.n * sizeof(StageArgs) + B->cargs.n * sizeof(CoeffArgs) +
                                   B->fargs.n * sizeof(FinalizeArgs) + B->ctlp.n * sizeof(Control *) +
                                   B->table.n * sizeof(int2) + B->counts.n * sizeof(int) + B->ctl_all.n * sizeof(Control));
        r.last_step_ms = B->last_ms;
        r.kernel_launches = B->launches;
        *info = r;
    });
}

}  // extern "C"
