// FP64_EXACT instantiation of the stage kernel.  Built with -fmad=false so that every double
// operation rounds exactly as the reference's source order does.
#include "stage.cuh"

namespace e3d {

void launch_stage_exact(const StageArgs &a, cudaStream_t s) {
    const int blocks = (a.n_cells + kStageThreads - 1) / kStageThreads;
    stage_kernel<true><<<blocks, kStageThreads, 0, s>>>(a);
}

}  // namespace e3d
