// FP64 instantiation of the row-pipelined step (step_tma.cuh).  Compiled
// with -fmad=false: the collision keeps the reference's rounding.
#include "step_tma.cuh"

namespace dnslbm {

int tma_prepare_f64(size_t smem) { return tma_set_smem_attr<double>(smem); }
int tma_occupancy_f64(int threads, size_t smem) { return tma_occupancy<double>(threads, smem); }
void launch_tma_f64(const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd, bool textured,
                    cudaStream_t s)
{
    launch_tma<double>(p, t, grid, threads, smem, odd, textured, s);
}

}  // namespace dnslbm
