// FP32 / FP16 instantiations of the row-pipelined step (step_tma.cuh) and of
// the persistent batch kernel (step_persist.cuh).
#include "step_persist.cuh"

namespace dnslbm {

int tma_prepare_lp(int precision, size_t smem)
{
    return precision == 32 ? tma_set_smem_attr<float>(smem) : tma_set_smem_attr<__half>(smem);
}
int tma_occupancy_lp(int precision, int threads, size_t smem, bool const_q)
{
    return precision == 32 ? tma_occupancy<float>(threads, smem, const_q) : tma_occupancy<__half>(threads, smem, const_q);
}
void launch_tma_lp(int precision, const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd,
                   int tex, cudaStream_t s)
{
    if (precision == 32) launch_tma<float>(p, t, grid, threads, smem, odd, tex, s);
    else launch_tma<__half>(p, t, grid, threads, smem, odd, tex, s);
}

int tma_batch_prepare_lp(int precision, size_t smem)
{
    return precision == 32 ? tma_batch_set_smem_attr<float>(smem) : tma_batch_set_smem_attr<__half>(smem);
}
int tma_batch_occupancy_lp(int precision, int threads, size_t smem)
{
    return precision == 32 ? tma_batch_occupancy<float>(threads, smem) : tma_batch_occupancy<__half>(threads, smem);
}
void launch_tma_batch_lp(int precision, const ChannelLaunch *chans, int nchan, int grid, int threads, size_t smem,
                         bool odd, cudaStream_t s)
{
    if (precision == 32) launch_tma_batch<float>(chans, nchan, grid, threads, smem, odd, s);
    else launch_tma_batch<__half>(chans, nchan, grid, threads, smem, odd, s);
}


void launch_links_lp(int precision, const LinksLaunch *tab, int n, int blocks, bool odd, cudaStream_t s)
{
    if (precision == 32) launch_links_pass<float>(tab, n, blocks, odd, s);
    else launch_links_pass<__half>(tab, n, blocks, odd, s);
}

int persist_prepare_lp(int precision, size_t smem)
{
    return precision == 32 ? persist_set_smem_attr<float>(smem) : persist_set_smem_attr<__half>(smem);
}
int persist_occupancy_lp(int precision, int threads, size_t smem, bool any_q)
{
    return precision == 32 ? persist_occupancy<float>(threads, smem, any_q)
                           : persist_occupancy<__half>(threads, smem, any_q);
}
cudaError_t launch_persist_lp(int precision, const PersistArgs &a, int grid, int threads, size_t smem, bool any_q,
                              cudaStream_t s)
{
    return precision == 32 ? launch_persist<float>(a, grid, threads, smem, any_q, s)
                           : launch_persist<__half>(a, grid, threads, smem, any_q, s);
}

}  // namespace dnslbm
