// FP64 instantiations of the stage kernels: restructured arithmetic, fused multiply-adds where the
// source writes fma() (built with -fmad=false, so nothing else is contracted).
#include "common.hpp"
#include "stage_ws.cuh"

namespace e3d {

// Dynamic shared memory the tile kernels may use (raised before their first launch).
void prepare_tile_fast(size_t smem_bytes, size_t pipe_smem_bytes) {
    raise_smem_limit((const void *)tile_kernel<false, 4>, smem_bytes);
    raise_smem_limit((const void *)tile_kernel<false, 7>, smem_bytes);
    if (pipe_smem_bytes) raise_smem_limit((const void *)tile_ws_kernel<WS_FAST>, pipe_smem_bytes);
}

void prepare_batch_fast(size_t smem_bytes, size_t ws_smem_bytes) {
    raise_smem_limit((const void *)tile_batch_kernel<false, 6>, smem_bytes);
    if (ws_smem_bytes) raise_smem_limit((const void *)tile_ws_batch_kernel<WS_FAST>, ws_smem_bytes);
}

// Update phase of a split stage (residual smoothing between residual and update).
void launch_update_fast(const StageArgs &a, cudaStream_t s) {
    update_kernel<false><<<(a.n_cells + kStageThreads - 1) / kStageThreads, kStageThreads, 0, s>>>(a);
}

// One stage of every member of a batch: `grid` blocks over the (member, tile) table.
void launch_batch_fast(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_batch_kernel<false, 6><<<grid, kStageThreads, smem_bytes, s>>>(bs);
}

// The same stage with the warp-specialised persistent kernel: `grid` blocks walk the table.
void launch_batch_ws_fast(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_ws_batch_kernel<WS_FAST><<<grid, kWsThreads, smem_bytes, s>>>(bs);
}

// The FP64 mode's reciprocal and reciprocal square root beside CUDA's own double-precision
// operations, for their accuracy check: out[4 i .. 4 i + 3] = rcp_nr(x), 1.0 / x, rsqrt_nr(x), rsqrt(x).
__global__ void fast_reciprocals_kernel(const double *__restrict__ x, int64_t n, double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = x[i];
        out[4 * i] = rcp_nr(v);
        out[4 * i + 1] = 1.0 / v;
        out[4 * i + 2] = rsqrt_nr(v);
        out[4 * i + 3] = rsqrt(v);
    }
}

void launch_fast_reciprocals(const double *x, int64_t n, double *out, cudaStream_t s) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4096);
    fast_reciprocals_kernel<<<blocks, 256, 0, s>>>(x, n, out);
}

// One colour class of a face-colouring stage: n faces, `per_block` (128 or 512) faces per block.
void launch_colour_fast(const StageArgs &a, const ColourFace *faces, int n, double2 *rc, int per_block,
                        cudaStream_t s) {
    if (n <= 0) return;
    if (per_block == 512) colour_kernel<512><<<(n + 511) / 512, 512, 0, s>>>(a, faces, n, rc);
    else colour_kernel<128><<<(n + 127) / 128, 128, 0, s>>>(a, faces, n, rc);
}

// The update after the last colour class.
void launch_colour_finish_fast(const StageArgs &a, const double2 *rc, cudaStream_t s) {
    colour_finish_kernel<><<<(a.n_cells + kStageThreads - 1) / kStageThreads, kStageThreads, 0, s>>>(a, rc);
}

// variant 0: gather kernel, registers for 4 blocks/SM; 1: gather kernel, 5 blocks/SM;
// 2: face tiles, one block per tile (4 blocks/SM); 3: face tiles, persistent and warp-specialised;
// 4: face tiles with registers for 7 blocks/SM
void launch_stage_fast(const StageArgs &a, cudaStream_t s, int variant) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    if (variant == 4) {
        const size_t smem = tile_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
        tile_kernel<false, 7><<<blocks, kStageThreads, smem, s>>>(a);
    } else if (variant == 3) {
        const size_t smem = ws_smem_for(ws_buffer_bytes(WS_FAST, a.smem_cells, a.smem_faces, a.max_contrib), a.ws_buffers);
        tile_ws_kernel<WS_FAST><<<a.pipe_grid, kWsThreads, smem, s>>>(a);
    } else if (variant == 2) {
        const size_t smem = tile_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
        tile_kernel<false, 4><<<blocks, kStageThreads, smem, s>>>(a);
    } else if (variant == 1) {
        stage_kernel<false, 5><<<blocks, kStageThreads, 0, s>>>(a);
    } else {
        stage_kernel<false, 4><<<blocks, kStageThreads, 0, s>>>(a);
    }
}

}  // namespace e3d
