// Mixed-precision hydro: the KT reconstruction and flux in FP32 (FMA
// allowed in this translation unit), fluxes stored in FP64 for the FP64
// coarse-fine correction and conservative update.
#include "flux_kernel.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace amr {

template <int R>
__global__ void k_flux_f32(Geom g, DevState st, const int* __restrict__ slots) {
    flux_pencils<float, R>(g, st, slots[blockIdx.x]);
}

void launch_flux_f32(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (g.recon == RECON_PPM)
        launch_k(k_flux_f32<RECON_PPM>, n, 3 * g.nx * g.nx, 0, s, g, st, slots);
    else
        launch_k(k_flux_f32<RECON_MINMOD>, n, 3 * g.nx * g.nx, 0, s, g, st, slots);
}

}  // namespace amr
