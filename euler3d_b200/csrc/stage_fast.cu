// FP64 instantiation of the stage kernel: restructured arithmetic, FMA contraction allowed.
#include "stage.cuh"

namespace e3d {

void launch_stage_fast(const StageArgs &a, cudaStream_t s) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    stage_kernel<false><<<blocks, kStageThreads, 0, s>>>(a);
}

}  // namespace e3d
