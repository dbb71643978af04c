// Storage type of the multigrid correction: the FP64 form keeps dphi and
// dphi1 in FP64 (DevState::dphi, dphi1); the mixed form keeps them in FP32
// (DevState::fdphi, fdphi1) while the residual and the potential stay FP64.
#pragma once

#include "amr_internal.h"

namespace amr {

template <typename CT>
struct Corr;

template <>
struct Corr<double> {
    static __host__ __device__ __forceinline__ double* dphi(const DevState& s) { return s.dphi; }
    static __host__ __device__ __forceinline__ double* dphi1(const DevState& s) { return s.dphi1; }
};

template <>
struct Corr<float> {
    static __host__ __device__ __forceinline__ float* dphi(const DevState& s) { return s.fdphi; }
    static __host__ __device__ __forceinline__ float* dphi1(const DevState& s) { return s.fdphi1; }
};

}  // namespace amr
