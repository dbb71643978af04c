// Helmholtz EOS: device table and launch wrappers (helm_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "helm_b200.h"

namespace amr {

constexpr int HELM_NODE = 10;  // doubles per table node (9 values + pad)

// code <- cgs factors of helmholtz_set_cgs_units / eos_from_code
// (helmeos.cpp:132-162): x_code = x_cgs / f_x
struct HelmUnits {
    double f_p, f_e, f_T, f_cs, f_cv, f_rho, f_s, f_dsdt;
};

struct HelmTable {
    const double* node;  // [JMAX][IMAX][HELM_NODE]
    const double* tj;    // [JMAX][8]: t, dt, dt^2, 1/dt, 1/dt^2
    const double* di;    // [IMAX][8]: d, dd, dd^2, 1/dd, 1/dd^2
    double tlo, tstpi, dlo, dstpi;
    double t_first, t_last, d_first, d_last;
    HelmUnits u;
};

struct HelmPoint {
    double p, e, cs, cv, s, dsdt, rho, T;
    int status;
};

// helm_point / helm_invert_point: helm_device.cuh

// the device table of a context (helm_host.cpp)
const HelmTable* helm_table_of(const helm_ctx* c);

void launch_helm_eos(const HelmTable& H, long long n, const double* rho, const double* T, const double* abar,
                     const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                     int* status, cudaStream_t st);
void launch_helm_invert(const HelmTable& H, long long n, const double* rho, const double* target,
                        const double* abar, const double* zbar, int from_entropy, double* T, double* p, double* e,
                        double* cs, double* cv, double* s, int* iters, int* status, cudaStream_t st);
void launch_helm_ztwd(long long n, const double* zbar, const double* rho, double* p, double* e, cudaStream_t st);

}  // namespace amr
