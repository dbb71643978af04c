// Euler state algebra on one cell (device), in the reference's exact
// operation order so the FP64 instantiation reproduces the CPU path to
// round-off; the FP32 instantiation is the mixed form's reconstruction and
// flux arithmetic.  Fields: 0 d, 1 sx, 2 sy, 3 sz, 4 et, 5 tau
// (euler/state.cpp:12-17).
#pragma once

#include "amr_internal.h"

namespace amr {

constexpr int NF_EULER = 6;

// real.h:21-73
template <typename T>
__device__ __forceinline__ T r_max(T a, T b) {
    return a > b ? a : b;
}
template <typename T>
__device__ __forceinline__ T r_min(T a, T b) {
    return a > b ? b : a;
}
template <typename T>
__device__ __forceinline__ T r_sgn(T a) {
    return a > T(0) ? T(1) : (a < T(0) ? T(-1) : T(0));
}
template <typename T>
__device__ __forceinline__ T minmod2(T a, T b) {
    return T(0.5) * (r_sgn(a) + r_sgn(b)) * r_min(fabs(a), fabs(b));
}
template <typename T>
__device__ __forceinline__ T minmod3(T a, T b, T c) {
    return minmod2(a, minmod2(b, c));
}
// vector.h:195-202: minmod(theta*up, theta*um, 0.5*(up+um))
template <typename T>
__device__ __forceinline__ T minmod_theta(T up, T um, T th) {
    return minmod3(th * up, th * um, T(0.5) * (up + um));
}

// State::ek (euler/state.cpp:181-183)
template <typename T>
__device__ __forceinline__ T st_ek(const T* u) {
    return T(0.5) * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
}
// State::pg (euler/state.cpp:189-196): dual-energy switch on tau.
template <typename T>
__device__ __forceinline__ T st_pg(const T* u, T gamma) {
    const T ei0 = u[4] - st_ek(u);
    if (ei0 < T(0.001) * u[4]) return (gamma - T(1)) * pow(u[5], gamma);
    return (gamma - T(1)) * ei0;
}
// State::to_prim / to_con (euler/state.cpp:246-258)
template <typename T>
__device__ __forceinline__ void st_to_prim(T* u) {
    u[4] -= st_ek(u);
    u[1] /= u[0];
    u[2] /= u[0];
    u[3] /= u[0];
}
template <typename T>
__device__ __forceinline__ void st_to_con(T* u) {
    u[1] *= u[0];
    u[2] *= u[0];
    u[3] *= u[0];
    u[4] += st_ek(u);
}
// State::floor (euler/state.cpp:86-92)
__device__ __forceinline__ void st_floor(double* u, double gamma, double rho_floor, double ei_floor) {
    u[0] = r_max(u[0], rho_floor);
    const double ei0 = u[4] - st_ek(u);
    if (ei0 > 0.1 * u[4]) u[5] = pow(r_max(ei0, ei_floor), 1.0 / gamma);
}
// State::x_flux/y_flux/z_flux and max_abs_*_eigen (euler/state.cpp:198-244)
// for direction d (0,1,2); returns the eigenvalue |v| + cs.
template <typename T>
__device__ __forceinline__ T st_flux(const T* u, int d, T gamma, T* f) {
    const T v = u[1 + d] / u[0];
    const T p = st_pg(u, gamma);
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) f[l] = u[l] * v;
    f[1 + d] += p;
    f[4] += v * p;
    const T cs = sqrt(gamma * p / u[0]);
    return fabs(v) + cs;
}
template <typename T>
__device__ __forceinline__ T st_eigen(const T* u, int d, T gamma) {
    const T v = u[1 + d] / u[0];
    return fabs(v) + sqrt(gamma * st_pg(u, gamma) / u[0]);
}
// State::enforce_outflow (euler/state.cpp:45-84); `bface` is the face of
// the boundary proxy (the inverse of the brick face it serves).
__device__ __forceinline__ void st_enforce_outflow(double* u, int bface) {
    const int m = 1 + (bface >> 1);
    bool zero;
    if (bface == ZU || bface == ZL) {
        zero = (bface == ZU) ? (u[3] > 0.0) : (u[3] < 0.0);
    } else {
        const double v = u[m] / u[0];
        zero = (bface & 1) ? (v > 0.0) : (v < 0.0);
    }
    if (zero) {
        u[4] = u[4] - 0.5 * u[m] * u[m] / u[0];
        u[m] = 0.0;
    }
}

}  // namespace amr
