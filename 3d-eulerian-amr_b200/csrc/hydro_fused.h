// Fused persistent hydro substep (hydro_fused.cuh): arguments and launches.
#pragma once

#include <cuda_runtime.h>

#include "amr_internal.h"

namespace amr {

struct FusedArgs {
    Geom g;
    BrickTable bt;
    const double* Uin;  // state at the start of the substep (interiors read)
    const double* U0;   // RK store
    double* Uout;       // updated state (interiors written)
    const int2* work;   // (slot, item-range entry or -1), finest level first
    int nwork;
    unsigned int* next;  // work counter, zero at launch
    int* done;           // [cap] epoch stamp once a brick's faces are published
    int epoch;
    const unsigned char* pubmask;  // [cap] faces to publish: bit 2 dir + (upper)
    double* pub;                   // [cap][6][nf][nx*nx] published face fluxes
    const RefluxItem* vitems;      // coarse-fine items grouped by coarse brick
    const int* vranges;            // [4 entry + 0..3]: first x, y, z item, end
    double dt, beta;
    int root;
    double* Fx;  // the root's face fluxes (for the domain flow-off)
    double* Fy;
    double* Fz;
    int* err;  // bit 0: a wait for a child ran out; bit 1: ghost chain too deep
    unsigned long long wait_limit;  // polls of one wait for a child's faces before bit 0 is set
};

// Launch over a.nwork bricks; blocks_per_sm_cap > 0 limits the resident
// blocks per SM (0: as many as fit).  *blocks_used receives the grid size.
cudaError_t launch_substep_fused_f64(const FusedArgs& a, int blocks_per_sm_cap, cudaStream_t s, int* blocks_used);
cudaError_t launch_substep_fused_f32(const FusedArgs& a, int blocks_per_sm_cap, cudaStream_t s, int* blocks_used);

}  // namespace amr
