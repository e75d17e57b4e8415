// FP32_FLUX instantiations of the face-tile stage kernel.
#include "stage_f32.cuh"

namespace e3d {

void prepare_tile_f32(size_t smem_bytes) {
    cudaFuncSetAttribute(tile_kernel_f32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    cudaFuncSetAttribute(tile_kernel_f32<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}

// variant 2: two blocks/SM register budget; 3: three blocks/SM
void launch_stage_f32(const StageArgs &a, cudaStream_t s, int variant) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    const size_t smem = tile32_smem_bytes(a.smem_cells, a.smem_faces, a.max_contrib);
    if (variant == 3) tile_kernel_f32<3><<<blocks, kStageThreads, smem, s>>>(a);
    else tile_kernel_f32<2><<<blocks, kStageThreads, smem, s>>>(a);
}

}  // namespace e3d
