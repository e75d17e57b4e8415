// FP32_FLUX instantiations of the face-tile stage kernel.
#include "common.hpp"
#include "stage_ws.cuh"

namespace e3d {

void prepare_tile_f32(size_t smem_bytes, size_t ws_smem_bytes) {
    raise_smem_limit((const void *)tile_kernel_f32<4>, smem_bytes);
    raise_smem_limit((const void *)tile_kernel_f32<8>, smem_bytes);
    if (ws_smem_bytes) raise_smem_limit((const void *)tile_ws_kernel<WS_F32>, ws_smem_bytes);
}

void prepare_batch_f32(size_t smem_bytes, size_t ws_smem_bytes) {
    raise_smem_limit((const void *)tile_batch_kernel_f32<8>, smem_bytes);
    if (ws_smem_bytes) raise_smem_limit((const void *)tile_ws_batch_kernel<WS_F32>, ws_smem_bytes);
}

// One stage of every member of a batch with the warp-specialised persistent kernel.
void launch_batch_ws_f32(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_ws_batch_kernel<WS_F32><<<grid, kWsThreads, smem_bytes, s>>>(bs);
}

// One stage of every member of a batch: `grid` blocks over the (member, tile) table.
void launch_batch_f32(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_batch_kernel_f32<8><<<grid, kStageThreads, smem_bytes, s>>>(bs);
}

// variant 2: face tiles with registers for four blocks/SM; 3: warp-specialised persistent face
// tiles; 4: face tiles at eight blocks/SM
void launch_stage_f32(const StageArgs &a, cudaStream_t s, int variant) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    const size_t smem = tile32_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
    if (variant == 3) {
        const size_t ws = ws_smem_for(ws_buffer_bytes(WS_F32, a.smem_cells, a.smem_faces, a.max_contrib), a.ws_buffers);
        tile_ws_kernel<WS_F32><<<a.pipe_grid, kWsThreads, ws, s>>>(a);
    } else if (variant == 4) {
        tile_kernel_f32<8><<<blocks, kStageThreads, smem, s>>>(a);
    } else {
        tile_kernel_f32<4><<<blocks, kStageThreads, smem, s>>>(a);
    }
}

}  // namespace e3d
