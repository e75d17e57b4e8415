// Warp-specialised persistent stage kernel (stage-kernel variant 3), for every precision and for
// batches.
//
// One block per SM: a producer warp and up to kWsGroups consumer groups of kTileCells threads, each
// group with a ring of D tile buffers of its own in shared memory.  The block walks its work items
// blockIdx.x, + gridDim.x, ...; its k-th item goes to group g = k % Gc, whose j-th item (j = k / Gc)
// fills the group's buffer j % D.  A buffer has one consumer, which takes its fills in order, so a
// parity wait on its barriers always refers to the next phase.  The producer warp streams items
// ahead of the consumers: for each item it waits until the item's buffer is free (empty barrier),
// then issues every copy the tile needs onto the buffer's full barrier -- the owned cell records,
// face records and contribution lists as bulk copies (no multicast), the halo records as 16-byte
// cp.async by the 32 lanes, each lane's completion arriving on the barrier
// (cp.async.mbarrier.arrive.noinc), and L2 prefetches of the W0 rows and the cell geometry.  A consumer
// group waits for its item's full barrier, evaluates the fluxes and the update exactly as the
// one-block-per-tile kernels do (the same functions), with a named barrier of its own between the
// phases, and hands the buffer back.  So copies for the next tiles are in flight while every group
// computes, with no block launch, barrier initialisation or index chase between tiles.
//
// Every wait is bounded: a consumer that gives up sets the fault word of its item's solver and
// leaves; the producer stops issuing once that fault word is set or its own wait gives up, and lets
// every copy it issued land before it leaves.
#pragma once
#include "stage.cuh"
#include "stage_f32.cuh"

namespace e3d {

constexpr int kWsGroups = 5;
constexpr int kWsThreads = 32 + kWsGroups * kTileCells;
// Halo entries per producer lane loaded one item ahead (the first 32 x kWsPreHalo of a tile's halo).
constexpr int kWsPreHalo = 8;
// Bytes ahead of a batch buffer's tile data that hold the member's StageArgs.
constexpr size_t kWsArgsSlot = (sizeof(StageArgs) + 127) & ~(size_t)127;
static_assert(sizeof(StageArgs) % 16 == 0, "StageArgs is bulk-copied");

// Precision of a warp-specialised instantiation.
enum : int { WS_EXACT = 0, WS_FAST = 1, WS_F32 = 2 };

// Bytes of one tile buffer (128-byte multiple) for the precision's layout.
__host__ __device__ __forceinline__ size_t ws_buffer_bytes(int prec, int LC, int FC, int MC) {
    const size_t b = prec == WS_F32 ? tile32_buf_bytes(LC, FC, MC) : tile_buf_bytes(LC, FC, MC);
    return (b + 127) & ~(size_t)127;
}

// Dynamic shared memory with B buffers of `stride` bytes: the buffers, a full and an empty mbarrier
// per buffer, four doubles per consumer group for its RMS partial, and per buffer the face count of
// the tile in it (an int, 16 bytes reserved).
__host__ __device__ __forceinline__ size_t ws_smem_for(size_t stride, int buffers) {
    return (size_t)buffers * stride + 16 * (size_t)buffers + 32 * (size_t)kWsGroups + 16 * (size_t)buffers;
}

// Consumer groups for B buffers: one buffer per group up to kWsGroups groups, then more per group.
__host__ __device__ __forceinline__ int ws_groups_for(int buffers) {
    return buffers < kWsGroups ? buffers : kWsGroups;
}

// Buffers of `stride` bytes for the block: as many as fit its 227 KB (at most two per group), made a
// multiple of the group count; 0 when not even three fit.
inline int ws_buffers_for(size_t stride) {
    int fit = 0;
    for (int nb = 2 * kWsGroups; nb >= 1 && !fit; nb--)
        if (ws_smem_for(stride, nb) <= 227 * 1024) fit = nb;
    if (fit < 3) return 0;
    const int g = ws_groups_for(fit);
    return g * (fit / g);
}

// Halo records of an item: 16-byte cp.async by the producer's lanes.
__device__ __forceinline__ void ws_halo_gather(char *dst, const char *src, uint32_t bytes) {
    for (uint32_t o = 0; o < bytes; o += 16) cp_async16(dst + o, src + o);
}

// This lane's cp.async operations issued so far arrive on bar when they complete (one arrival,
// counted in the barrier's expected arrivals).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void named_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Named barrier of `threads` threads that also returns, to all of them, whether any passed true.
__device__ __forceinline__ bool named_sync_or(int id, int threads, bool v) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(threads)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Body of the warp-specialised kernels.  Solo (BATCH false): work item k of the block is tile
// blockIdx.x + k gridDim.x of the one solver whose arguments `solo` holds.  Batch (BATCH true): work
// item k is entry blockIdx.x + k gridDim.x of the batch's (member, tile) table; the producer copies
// the member's StageArgs into the buffer beside the tile's data, and the consumer group sets the
// stage's alpha and flags in that copy before it reads it -- so each member computes what its solo
// run computes.  A stopped member's items carry only the arguments, which the consumers skip.  A
// wait that gives up sets the fault word of the member whose item it waited for.
template <int PREC, bool BATCH>
__device__ __forceinline__ void ws_body(const StageArgs &solo, const BatchStage &bs, unsigned char *smem_raw) {
    constexpr bool F32 = PREC == WS_F32, EXACT = PREC == WS_EXACT;
    constexpr uint32_t kState = F32 ? 32u : 48u;   // bytes of a cell record
    constexpr uint32_t kRec = F32 ? 24u : 40u;     // bytes of a face record
    constexpr uint32_t kGeo = F32 ? 16u : 32u;     // bytes of a cell's geometry
    const int T = kTileCells, G = gridDim.x;
    const int B = BATCH ? bs.ws_buffers : solo.ws_buffers;
    const int Gc = ws_groups_for(B), D = B / Gc;  // consumer groups, buffers per group
    // buffer and fill number of the block's k-th item
    auto buffer_of = [&](int k, int &fill) {
        const int j = k / Gc;
        fill = j / D;
        return (k % Gc) * D + j % D;
    };
    const int n_items = BATCH ? *bs.n_entries : solo.n_tiles;
    const size_t slot = BATCH ? kWsArgsSlot : 0;  // the member's arguments, ahead of the tile's data
    const size_t bb = BATCH ? (size_t)bs.ws_stride
                            : ws_buffer_bytes(PREC, solo.smem_cells, solo.smem_faces, solo.max_contrib);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + (size_t)B * bb);
    uint64_t *empty = full + B;
    double *gsum = reinterpret_cast<double *>(empty + B);  // [kWsGroups][4]
    // face count of the tile in buffer b, written by the producer before its arrival on the buffer's
    // full barrier (release) and read by the consumer after its wait on it (acquire)
    int *meta = reinterpret_cast<int *>(gsum + 4 * kWsGroups);
    // the arguments (in global memory, or the kernel's own) of work item `item`, and its tile
    auto item_args = [&](int item, int &tile) -> const StageArgs * {
        if (!BATCH) {
            tile = item;
            return &solo;
        }
        const int2 e = bs.table[item];
        tile = e.y;
        return bs.args + 2 * e.x + bs.parity;
    };
    // where the tile's cell records, face records and contribution lists sit in a buffer
    auto layout = [&](unsigned char *p, const StageArgs &a, void *&st, void *&rec, unsigned short *&ct) {
        if (F32) {
            const Tile32 t = tile32_at(p, a.smem_cells, a.smem_faces);
            st = t.st, rec = t.rec, ct = t.ct;
        } else {
            const TileBuf t = tile_buf_at(p, a.smem_cells, a.smem_faces, a.max_contrib);
            st = t.st, rec = t.rec, ct = t.ct;
        }
    };
    if (threadIdx.x == 0) {
        for (int k = 0; k < B; k++) {
            mbar_init(&full[k], 1 + 32);  // the producer's expect-tx arrival + one per lane's cp.async
            mbar_init(&empty[k], 1);
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {  // ------------------------------------------------ producer
        // Everything an item's copies depend on -- its tile, sizes and source addresses, and this
        // lane's first kWsPreHalo halo entries -- is loaded one item ahead, before the producer waits
        // for the buffer of the item it issues now, so those global-memory round trips overlap that
        // wait and the copies it issues, instead of running back to back once per tile.
        struct Pre {
            const StageArgs *a;
            const char *st_src, *rec_src, *geo_src;
            const unsigned short *ct_src;
            const int *hrow;
            const double *w0;
            int tile, c0, nloc, nf, hs, w0_stride, lc, fc, mc;
            bool skip;
            int hidx[kWsPreHalo];
        };
        auto prepare = [&](int item, Pre &p) {
            int tile;
            const StageArgs &a = *item_args(item, tile);
            p.a = &a;
            p.tile = tile;
            p.skip = BATCH && a.ctl->done;  // a stopped member: its arguments only
            p.c0 = tile * T;
            p.nloc = min(T, a.n_cells - p.c0);
            p.lc = a.smem_cells, p.fc = a.smem_faces, p.mc = a.max_contrib;
            const char *qsrc = F32 ? reinterpret_cast<const char *>(a.q32in) : reinterpret_cast<const char *>(a.qin);
            p.st_src = qsrc;
            p.nf = p.skip ? 0 : a.tile_face_ptr[tile + 1] - a.tile_face_ptr[tile];
            p.rec_src = p.skip ? nullptr : (F32 ? a.tile_rec32 + a.tile_rec32_off[tile] : a.tile_rec + a.tile_rec_off[tile]);
            p.ct_src = a.tile_contrib + (size_t)tile * a.max_contrib * T;
            p.w0 = a.w0;
            p.w0_stride = a.w0_stride;
            p.geo_src = F32 ? reinterpret_cast<const char *>(a.cgeo32) : reinterpret_cast<const char *>(a.cgeo);
            // halo entries sit at a fixed stride per tile, padded with -1: no count needed to load them
            p.hs = p.skip ? 0 : a.halo_stride;
            p.hrow = a.tile_halo + (size_t)tile * a.halo_stride;
#pragma unroll
            for (int m = 0; m < kWsPreHalo; m++) {
                const int i = lane + 32 * m;
                p.hidx[m] = i < p.hs ? p.hrow[i] : -1;
            }
        };
        auto issue = [&](const Pre &p, int bi) {
            unsigned char *base = smem_raw + (size_t)bi * bb;
            void *st, *rec;
            unsigned short *ct;
            if (F32) {
                const Tile32 t = tile32_at(base + slot, p.lc, p.fc);
                st = t.st, rec = t.rec, ct = t.ct;
            } else {
                const TileBuf t = tile_buf_at(base + slot, p.lc, p.fc, p.mc);
                st = t.st, rec = t.rec, ct = t.ct;
            }
            if (lane == 0) {
                meta[bi] = p.nf;
                const uint32_t b_ct = (uint32_t)p.mc * T * 2u;
                const uint32_t tile_bytes =
                    p.skip ? 0u : (uint32_t)p.nloc * kState + round16(kRec * (uint32_t)p.nf) + b_ct;
                mbar_expect_tx(&full[bi], tile_bytes + (BATCH ? (uint32_t)sizeof(StageArgs) : 0u));
                if (BATCH) bulk_g2s(base, p.a, (uint32_t)sizeof(StageArgs), &full[bi]);
                if (!p.skip) {
                    bulk_g2s(st, p.st_src + (size_t)kState * p.c0, (uint32_t)p.nloc * kState, &full[bi]);
                    bulk_g2s(rec, p.rec_src, round16(kRec * (uint32_t)p.nf), &full[bi]);
                    bulk_g2s(ct, p.ct_src, b_ct, &full[bi]);
                    const uint32_t b_w0 = round16((uint32_t)p.nloc * 8u);
                    for (int q = 0; q < 5; q++) bulk_prefetch_l2(p.w0 + (size_t)q * p.w0_stride + p.c0, b_w0);
                    bulk_prefetch_l2(p.geo_src + (size_t)kGeo * p.c0, (uint32_t)p.nloc * kGeo);
                }
            }
            if (!p.skip) {
                char *hdst = static_cast<char *>(st) + (size_t)kState * p.nloc;
#pragma unroll
                for (int m = 0; m < kWsPreHalo; m++)
                    if (p.hidx[m] >= 0)
                        ws_halo_gather(hdst + (size_t)kState * (lane + 32 * m), p.st_src + (size_t)kState * p.hidx[m],
                                       kState);
                for (int i = lane + 32 * kWsPreHalo; i < p.hs; i += 32) {  // larger halos: the rest
                    const int h = p.hrow[i];
                    if (h >= 0) ws_halo_gather(hdst + (size_t)kState * i, p.st_src + (size_t)kState * h, kState);
                }
            }
            cp_async_arrive_noinc(&full[bi]);  // every lane, with or without halo copies
        };
        int issued = 0;  // items whose copies were issued
        bool stopped = false;
        Pre cur{}, nxt{};
        if ((int)blockIdx.x < n_items) prepare(blockIdx.x, cur);
        for (int k = 0, item = blockIdx.x; item < n_items; k++, item += G) {
            if (item + G < n_items) prepare(item + G, nxt);  // in flight while this item waits
            int fill;
            const int bi = buffer_of(k, fill);
            if (fill >= 1) {  // the buffer's previous item (k - B) has been handed back
                // lane 0 waits and the warp follows its answer, so every decision is warp-uniform
                int ok = 0;
                if (lane == 0) {
                    int prev_tile;
                    int *prev_fault = item_args(item - B * G, prev_tile)->fault;
                    const uint32_t par = (uint32_t)((fill - 1) & 1);
                    for (int it = 0; it < kWaitLimit && !ok; it++) {
                        ok = mbar_try_wait(&empty[bi], par);
                        if (!ok && (it & 255) == 255 && *(volatile int *)prev_fault) break;
                    }
                    if (!ok) atomicExch(prev_fault, 1);
                }
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    stopped = true;
                    break;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            issue(cur, bi);
            issued = k + 1;
            cur = nxt;
        }
        // every copy issued must land before the block can leave (the consumers wait for them when
        // the walk completes; after a give-up they may not have)
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (lane == 0 && stopped) {
            for (int k = (issued > B ? issued - B : 0); k < issued; k++) {
                int fill;
                const int bi = buffer_of(k, fill);
                tile_drain(&full[bi], (uint32_t)(fill & 1));
            }
        }
        return;
    }

    // ------------------------------------------------------------------ consumer group
    const int grp = (threadIdx.x - 32) / T;
    const int tid = (threadIdx.x - 32) % T;
    if (grp >= Gc) return;  // fewer groups than the block has (large tiles: fewer buffers)
    const int bar_id = 1 + grp;
    double *fsum = gsum + 4 * grp;
    for (int k = grp, item = blockIdx.x + grp * G; item < n_items; k += Gc, item += Gc * G) {
        int fill;
        const int bi = buffer_of(k, fill);
        unsigned char *base = smem_raw + (size_t)bi * bb;
        int tile;
        const StageArgs *ag = item_args(item, tile);  // global (batch) or the kernel's own arguments
        bool ok = false;
        const int polls = ag->wait_polls;
        for (int it = 0; it < polls && !ok; it++) ok = mbar_try_wait(&full[bi], (uint32_t)(fill & 1));
        if (!ok) atomicExch(ag->fault, 1);
        if (BATCH && ok && tid == 0) {  // this stage's alpha and flags in the member's arguments
            StageArgs *sa = reinterpret_cast<StageArgs *>(base);
            sa->alpha = bs.alpha;
            sa->first_stage = bs.first_stage;
            sa->last_stage = bs.last_stage;
            sa->residual_only = 0;
        }
        if (named_sync_or(bar_id, T, !ok)) return;  // the same decision for the whole group
        const StageArgs &a = BATCH ? *reinterpret_cast<const StageArgs *>(base) : solo;
        const bool run = !BATCH || !a.ctl->done;  // the member of a batch item may have stopped
        double r2 = 0.0;
        if (run) {
            const int c0 = tile * T, nloc = min(T, a.n_cells - c0);
            const int nf = meta[bi];  // the producer's, instead of a global-memory round trip
            if (F32) {
                const Tile32 b = tile32_at(base + slot, a.smem_cells, a.smem_faces);
                tile_fluxes_f32(a, b, nf, c0, tid, T);
                double W0[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                float4 cg = make_float4(0.f, 0.f, 0.f, 0.f);
                if (tid < nloc) tile_load_cell_f32(a, c0 + tid, W0, cg);
                named_sync(bar_id, T);
                if (tid < nloc) r2 = tile_update_f32(a, b, c0, tid, W0, cg);
            } else {
                const TileBuf b = tile_buf_at(base + slot, a.smem_cells, a.smem_faces, a.max_contrib);
                double *fs = reinterpret_cast<double *>(b.rec);
                tile_fluxes<EXACT, kTileCells>(a, b, fs, nf, c0, tid);
                double W0[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                double4 cg = make_double4(0.0, 0.0, 0.0, 0.0);
                if (tid < nloc) tile_load_cell(a, c0, tid, W0, cg);
                named_sync(bar_id, T);
                if (tid < nloc) r2 = tile_update<EXACT>(a, b, fs, c0, tid, W0, cg);
            }
        }
        const bool sum = run && a.last_stage && !a.residual_only;  // uniform across the group
        double *partial = sum ? a.partials + tile : nullptr;
        if (sum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
            if ((tid & 31) == 0) fsum[tid >> 5] = r2;
        }
        named_sync(bar_id, T);  // every read of the buffer (the arguments included) is done
        if (tid == 0) {
            // the order of block_sum_store's last shuffle tree, so every kernel writes the same partial
            if (sum) *partial = (fsum[0] + fsum[2]) + (fsum[1] + fsum[3]);
            mbar_arrive(&empty[bi]);
        }
        if (sum) named_sync(bar_id, T);  // fsum is reused by the next item
    }
}

template <int PREC>
__global__ void __launch_bounds__(kWsThreads, 1) tile_ws_kernel(StageArgs a) {
    if (!a.residual_only && a.ctl->done) return;  // uniform across the grid
    extern __shared__ __align__(128) unsigned char smem_raw[];
    ws_body<PREC, false>(a, BatchStage{}, smem_raw);
}

// Several solvers in one persistent grid: the batch's (member, tile) table walked as above.
template <int PREC>
__global__ void __launch_bounds__(kWsThreads, 1) tile_ws_batch_kernel(BatchStage bs) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    ws_body<PREC, true>(StageArgs{}, bs, smem_raw);
}

}  // namespace e3d
