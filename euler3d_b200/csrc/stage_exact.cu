// FP64_EXACT instantiations of the stage kernels.  Built with -fmad=false so that every double
// operation rounds exactly as the reference's source order does.
#include "common.hpp"
#include "stage_ws.cuh"

namespace e3d {

// Dynamic shared memory the tile kernels may use (raised before their first launch).
void prepare_tile_exact(size_t smem_bytes, size_t pipe_smem_bytes) {
    raise_smem_limit((const void *)tile_kernel<true, 4>, smem_bytes);
    if (pipe_smem_bytes) raise_smem_limit((const void *)tile_ws_kernel<WS_EXACT>, pipe_smem_bytes);
}

void prepare_batch_exact(size_t smem_bytes, size_t ws_smem_bytes) {
    raise_smem_limit((const void *)tile_batch_kernel<true, 4>, smem_bytes);
    if (ws_smem_bytes) raise_smem_limit((const void *)tile_ws_batch_kernel<WS_EXACT>, ws_smem_bytes);
}

// Update phase of a split stage (residual smoothing between residual and update).
void launch_update_exact(const StageArgs &a, cudaStream_t s) {
    update_kernel<true><<<(a.n_cells + kStageThreads - 1) / kStageThreads, kStageThreads, 0, s>>>(a);
}

// One stage of every member of a batch: `grid` blocks over the (member, tile) table.
void launch_batch_exact(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_batch_kernel<true, 4><<<grid, kStageThreads, smem_bytes, s>>>(bs);
}

// The same stage with the warp-specialised persistent kernel: `grid` blocks walk the table.
void launch_batch_ws_exact(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_ws_batch_kernel<WS_EXACT><<<grid, kWsThreads, smem_bytes, s>>>(bs);
}

// variant 0: gather kernel, registers for 2 blocks/SM; 1: gather kernel, 4 blocks/SM;
// 2: face tiles, one block per tile (4 blocks/SM); 3: face tiles, persistent and warp-specialised
void launch_stage_exact(const StageArgs &a, cudaStream_t s, int variant) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    if (variant == 3) {
        const size_t smem = ws_smem_for(ws_buffer_bytes(WS_EXACT, a.smem_cells, a.smem_faces, a.max_contrib), a.ws_buffers);
        tile_ws_kernel<WS_EXACT><<<a.pipe_grid, kWsThreads, smem, s>>>(a);
    } else if (variant == 2) {
        const size_t smem = tile_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
        tile_kernel<true, 4><<<blocks, kStageThreads, smem, s>>>(a);
    } else if (variant == 1) {
        stage_kernel<true, 4><<<blocks, kStageThreads, 0, s>>>(a);
    } else {
        stage_kernel<true, 2><<<blocks, kStageThreads, 0, s>>>(a);
    }
}

}  // namespace e3d
