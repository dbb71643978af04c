// Launch wrappers of the device kernels (host-callable).
#pragma once

#include <cuda_runtime.h>

#include "amr_internal.h"

namespace amr {

// hydro_kernels.cu
void launch_ghost_fill(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                       cudaStream_t s);
void launch_flux(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s);
// hydro_mixed.cu: FP32 reconstruction + flux (used by launch_flux when g.precision is mixed)
void launch_flux_f32(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s);
void launch_reflux(const Geom& g, const DevState& st, const RefluxItem* items, int n, cudaStream_t s);
// dtp: when non-null the step is read from device memory (captured graphs)
void launch_add_difs(const Geom& g, const DevState& st, const int* slots, int n, const double* hs, double dt,
                     double beta, int gravity, cudaStream_t s, const double* dtp = nullptr);
void launch_flow_off(const Geom& g, const DevState& st, int root, double h, double dt, double beta, double* fo,
                     cudaStream_t s, const double* dtp = nullptr);
void launch_inject(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                   cudaStream_t s);
void launch_prolong(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                    cudaStream_t s);
void launch_max_dt(const Geom& g, const DevState& st, const int* slots, int n, const double* hs, double* dt_out,
                   cudaStream_t s);
void launch_refine_flags(const Geom& g, const DevState& st, const int* slots, int n, double thr,
                         unsigned char* flags, cudaStream_t s);
void launch_state_max(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n, int field,
                      double* out, cudaStream_t s);

}  // namespace amr

namespace amr {
void launch_gather(const double* src, const int* slots, int n, int count, double* dst, cudaStream_t s);
void launch_scatter(const double* src, const int* slots, int n, int count, double* dst, cudaStream_t s);
}  // namespace amr
