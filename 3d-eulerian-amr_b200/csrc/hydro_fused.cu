// Fused persistent hydro substep, FP64 reconstruction and flux (no FMA
// contraction: bitwise equal to the one-launch-per-step path).
#include "hydro_fused.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace amr {

namespace {
int fused_blocks(const void* kernel, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, FUSED_BLOCK, smem) != cudaSuccess || per <= 0)
        return -1;
    return sms * per;
}
}  // namespace

cudaError_t launch_substep_fused_f64(const FusedArgs& a, int blocks_per_sm_cap, cudaStream_t s, int* blocks_used) {
    const size_t smem = fused_smem_bytes<double>();
    const void* k = (const void*)k_substep_fused<double>;
    int blocks = fused_blocks(k, smem);
    if (blocks <= 0) return cudaErrorInvalidConfiguration;
    if (blocks_per_sm_cap > 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        blocks = std::min(blocks, sms * blocks_per_sm_cap);
    }
    blocks = std::min(blocks, std::max(a.nwork, 1));
    if (blocks_used) *blocks_used = blocks;
    launch_k(k_substep_fused<double>, blocks, FUSED_BLOCK, smem, s, a);
    return cudaGetLastError();
}

}  // namespace amr
