// FP32_FLUX instantiations of the face-tile stage kernel.
#include "common.hpp"
#include "stage_f32.cuh"

namespace e3d {

void prepare_tile_f32(size_t smem_bytes) {
    raise_smem_limit((const void *)tile_kernel_f32<4>, smem_bytes);
    raise_smem_limit((const void *)tile_kernel_f32<8>, smem_bytes);
}

void prepare_batch_f32(size_t smem_bytes, size_t) { raise_smem_limit((const void *)tile_batch_kernel_f32<7>, smem_bytes); }

// One stage of every member of a batch: `grid` blocks over the (member, tile) table.
void launch_batch_f32(const BatchStage &bs, int grid, size_t smem_bytes, cudaStream_t s) {
    tile_batch_kernel_f32<7><<<grid, kStageThreads, smem_bytes, s>>>(bs);
}

// variant 2: registers for four blocks/SM; 3: eight blocks/SM
void launch_stage_f32(const StageArgs &a, cudaStream_t s, int variant) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    const size_t smem = tile32_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
    if (variant == 3) tile_kernel_f32<8><<<blocks, kStageThreads, smem, s>>>(a);
    else tile_kernel_f32<4><<<blocks, kStageThreads, smem, s>>>(a);
}

}  // namespace e3d
