// Helmholtz EOS kernels (helmholtz/helmeos.cpp), FP64, one thread per point
// (device code of one point in helm_device.cuh).
//
// Table in HBM (L2-resident, 35 MB): node[j][i][10] = f, f_d, f_t, f_dd, f_tt,
// f_dt, f_ddt, f_dtt, f_ddtt, pad -- the two density neighbours of a row are
// one contiguous 160-byte run read as 16-byte vectors; tj[j][8] = t, dt, dt^2,
// 1/dt, 1/dt^2 and di[i][8] = d, dd, dd^2, 1/dd, 1/dd^2 (computed on the host
// exactly as read_helm_table does, helmeos.cpp:100-129).
#include <cuda_runtime.h>

#include "helm_device.cuh"
#include "launch.cuh"

namespace amr {

namespace {

__global__ void __launch_bounds__(128) k_helm_eos(HelmTable H, long long n, const double* __restrict__ rho,
                                                  const double* __restrict__ T, const double* __restrict__ abar,
                                                  const double* __restrict__ zbar, double* p, double* e, double* cs,
                                                  double* cv, double* s, double* dsdt, int* __restrict__ status) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        HelmPoint o;
        helm_point(H, rho[q], T[q], abar[q], zbar[q], o);
        status[q] = o.status;
        if (o.status == 1) continue;
        if (p) p[q] = o.p;
        if (e) e[q] = o.e;
        if (cs) cs[q] = o.cs;
        if (cv) cv[q] = o.cv;
        if (s) s[q] = o.s;
        if (dsdt) dsdt[q] = o.dsdt;
    }
}

// helmholtz_compute_T (helmeos.cpp:436-486), one point per thread
__global__ void __launch_bounds__(128) k_helm_invert(HelmTable H, long long n, const double* __restrict__ rho,
                                                     const double* __restrict__ target,
                                                     const double* __restrict__ abar,
                                                     const double* __restrict__ zbar, int from_entropy,
                                                     double* __restrict__ T, double* p, double* e, double* cs,
                                                     double* cv, double* s, int* iters_out,
                                                     int* __restrict__ status) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        double Tq = T[q];
        HelmPoint o;
        int iters;
        const int st = helm_invert_point(H, rho[q], target[q], abar[q], zbar[q], from_entropy, Tq, o, &iters);
        status[q] = st;
        if (iters_out) iters_out[q] = iters;
        if (st == 1 && iters == 0) continue;  // outside the table at the floor temperature
        T[q] = Tq;
        if (st == 1) continue;
        if (p) p[q] = o.p;
        if (e) e[q] = o.e;
        if (cs) cs[q] = o.cs;
        if (cv) cv[q] = o.cv;
        if (s) s[q] = o.s;
    }
}

// helmholtz_ztwd (helmeos.cpp:423-434)
__global__ void k_helm_ztwd(long long n, const double* __restrict__ zbar, const double* __restrict__ rho,
                            double* __restrict__ p, double* __restrict__ e) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double A = 6.023e+22;
        const double B = 9.7595e+5 * zbar[q];
        const double x = pow(rho[q] / B, 1.0 / 3.0);
        double pv;
        if (x > 0.1) {
            pv = A * (x * (2.0 * x * x - 3.0) * sqrt(x * x + 1.0) + 3.0 * log(x + sqrt(x * x + 1.0)));
        } else {
            pv = A * 1.6 * pow(x, 5);
        }
        p[q] = pv;
        e[q] = A * (8.0 * pow(x, 3) * (sqrt(x * x + 1.0) - 1.0)) - pv / rho[q];
    }
}

int grid_for(long long n) {
    // grid-stride loops over at most 148 SMs x 16 blocks of 128 threads
    const long long want = (n + 127) / 128;
    return (int)(want < 148LL * 16 ? (want > 0 ? want : 1) : 148LL * 16);
}

}  // namespace

void launch_helm_eos(const HelmTable& H, long long n, const double* rho, const double* T, const double* abar,
                     const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                     int* status, cudaStream_t st) {
    if (n <= 0) return;
    launch_k(k_helm_eos, grid_for(n), 128, 0, st, H, n, rho, T, abar, zbar, p, e, cs, cv, s, dsdt, status);
}

void launch_helm_invert(const HelmTable& H, long long n, const double* rho, const double* target,
                        const double* abar, const double* zbar, int from_entropy, double* T, double* p, double* e,
                        double* cs, double* cv, double* s, int* iters, int* status, cudaStream_t st) {
    if (n <= 0) return;
    launch_k(k_helm_invert, grid_for(n), 128, 0, st, H, n, rho, target, abar, zbar, from_entropy, T, p, e, cs, cv, s,
             iters, status);
}

void launch_helm_ztwd(long long n, const double* zbar, const double* rho, double* p, double* e, cudaStream_t st) {
    if (n <= 0) return;
    launch_k(k_helm_ztwd, grid_for(n), 128, 0, st, n, zbar, rho, p, e);
}

}  // namespace amr
