// FP64 instantiation of the row-pipelined step (step_tma.cuh) and of the
// persistent batch kernel (step_persist.cuh).  Compiled with -fmad=false: the
// collision keeps the reference's rounding.
#include "step_persist.cuh"

namespace dnslbm {

int tma_prepare_f64(size_t smem) { return tma_set_smem_attr<double>(smem); }
int tma_occupancy_f64(int threads, size_t smem, bool const_q) { return tma_occupancy<double>(threads, smem, const_q); }
void launch_tma_f64(const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd, int tex,
                    cudaStream_t s)
{
    launch_tma<double>(p, t, grid, threads, smem, odd, tex, s);
}

int tma_batch_prepare_f64(size_t smem) { return tma_batch_set_smem_attr<double>(smem); }
int tma_batch_occupancy_f64(int threads, size_t smem) { return tma_batch_occupancy<double>(threads, smem); }
void launch_tma_batch_f64(const ChannelLaunch *chans, int nchan, int grid, int threads, size_t smem, bool odd,
                          cudaStream_t s)
{
    launch_tma_batch<double>(chans, nchan, grid, threads, smem, odd, s);
}


void launch_links_f64(const LinksLaunch *tab, int n, int blocks, bool odd, cudaStream_t s)
{
    launch_links_pass<double>(tab, n, blocks, odd, s);
}

int persist_prepare_f64(size_t smem) { return persist_set_smem_attr<double>(smem); }
int persist_occupancy_f64(int threads, size_t smem, bool any_q) { return persist_occupancy<double>(threads, smem, any_q); }
cudaError_t launch_persist_f64(const PersistArgs &a, int grid, int threads, size_t smem, bool any_q, cudaStream_t s)
{
    return launch_persist<double>(a, grid, threads, smem, any_q, s);
}

}  // namespace dnslbm
