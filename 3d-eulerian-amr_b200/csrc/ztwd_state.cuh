// The ZTWD binary state (binary/state_ztwd.cpp, binary/state.h) on one cell
// or face, in the reference's operation order (include only from
// translation units compiled without FMA contraction).  The functions the
// flux uses are templates over the arithmetic type T: FP64 in the plain
// form (every cast below is then the identity), FP32 for the face states
// and fluxes of the mixed form, whose EOS calls stay FP64 (zt_eos_of).
//
// Fields (state_ztwd.cpp:16-26): 0 rho, 1 rho_acc, 2 rho_don, 3 sr (radial
// momentum), 4 lz (inertial angular momentum), 5 sz, 6 pot, 7 et, 8 tau
// (internal energy when it dominates), 9 T, 10..12 species densities
// (abar 4, 14.12, 17.52, state_ztwd.cpp:27).  Positions are cell or face
// centres in the rotating frame; R is the cylindrical radius.  Pressure and
// sound speed come from the Helmholtz EOS (helm_device.cuh) at (rho, T) with
// abar and zbar of the species mix (State::compute_eos, :176-185).
#pragma once

#include "helm_device.cuh"
#include "ztwd.h"

namespace amr {

constexpr int ZT_NF = ZTWD_NF;
constexpr int ZT_D = 0, ZT_ACC = 1, ZT_DON = 2, ZT_SR = 3, ZT_LZ = 4, ZT_SZ = 5, ZT_POT = 6, ZT_ET = 7, ZT_TAU = 8,
              ZT_T = 9, ZT_SPECIE = 10, ZT_NSPECIES = 3;

// real.h max/min: a > b ? a : b / a > b ? b : a
__device__ __forceinline__ double zmax(double a, double b) { return a > b ? a : b; }

template <typename T>
__device__ __forceinline__ T zt_R(const T* X) { return sqrt(X[0] * X[0] + X[1] * X[1]); }

// State::A, State::Z (state_ztwd.cpp:33-45)
template <typename T>
__device__ __forceinline__ T zt_abar(const ZtwdPar& P, const T* u) {
    T sum = T(0.0);
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) sum += u[ZT_SPECIE + i] / T(P.abar[i]);
    sum = u[ZT_D] / sum;
    return sum;
}

// State::st (:241-243): lz/R - rho R Omega
template <typename T>
__device__ __forceinline__ T zt_st(const ZtwdPar& P, const T* u, const T* X) {
    return u[ZT_LZ] / zt_R(X) - u[ZT_D] * zt_R(X) * T(P.omega);
}
template <typename T>
__device__ __forceinline__ T zt_vx(const ZtwdPar& P, const T* u, const T* X) {
    return (X[0] * u[ZT_SR] - X[1] * zt_st(P, u, X)) / zt_R(X) / u[ZT_D];
}
template <typename T>
__device__ __forceinline__ T zt_vy(const ZtwdPar& P, const T* u, const T* X) {
    return (X[1] * u[ZT_SR] + X[0] * zt_st(P, u, X)) / zt_R(X) / u[ZT_D];
}
template <typename T>
__device__ __forceinline__ T zt_vz(const T* u) { return u[ZT_SZ] / u[ZT_D]; }
// normal velocity of direction d (State::vx/vy/vz, :249-267)
template <typename T>
__device__ __forceinline__ T zt_v(const ZtwdPar& P, const T* u, const T* X, int d) {
    return d == 0 ? zt_vx(P, u, X) : (d == 1 ? zt_vy(P, u, X) : zt_vz(u));
}
// State::ek (:158-160)
template <typename T>
__device__ __forceinline__ T zt_ek(const ZtwdPar& P, const T* u, const T* X) {
    const T st = zt_st(P, u, X);
    return T(0.5) * (u[ZT_SR] * u[ZT_SR] + st * st + u[ZT_SZ] * u[ZT_SZ]) / u[ZT_D];
}
// State::ei (:140-156): et - ek, or tau when that is below 0.001 et
__device__ __forceinline__ double zt_ei(const ZtwdPar& P, const double* u, const double* X) {
    const double e = u[ZT_ET] - zt_ek(P, u, X);
    if (e < u[ZT_ET] * 0.001) return u[ZT_TAU];
    return e;
}

// State::compute_eos (:176-185): p and cs of the cell (status != 0 where the
// reference aborts)
__device__ __forceinline__ int zt_eos(const ZtwdPar& P, const double* u, double* p, double* cs) {
    const double A = zt_abar(P, u);
    HelmPoint o;
    helm_point(P.H, u[ZT_D], u[ZT_T], A, A / 2.0, o);
    *p = o.p;
    *cs = o.cs;
    return o.status;
}

// State::compute_eos in FP64 for a state held in T: the EOS inputs (rho,
// T, the species mix) are widened to FP64 first
template <typename T>
__device__ __forceinline__ int zt_eos_of(const ZtwdPar& P, const T* u, T* p, T* cs) {
    double w[ZT_NF];
#pragma unroll
    for (int l = 0; l < ZT_NF; l++) w[l] = double(u[l]);
    double pd, csd;
    const int st = zt_eos(P, w, &pd, &csd);
    *p = T(pd);
    *cs = T(csd);
    return st;
}

// State::to_con (:560-585) at position X
template <typename T>
__device__ __forceinline__ void zt_to_con(const ZtwdPar& P, T* u, const T* X) {
    const T R = zt_R(X);
    u[ZT_SZ] *= u[ZT_D];
    u[ZT_POT] *= u[ZT_D];
    u[ZT_SR] *= u[ZT_D];
    u[ZT_LZ] += T(P.omega) * R;
    u[ZT_LZ] *= u[ZT_D] * R;
    u[ZT_ET] += zt_ek(P, u, X);
    T sum = T(0.0);
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) sum += u[ZT_SPECIE + i];
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] /= sum;
    sum = T(0.0);
    sum += u[ZT_DON];
    sum += u[ZT_ACC];
    u[ZT_DON] /= sum;
    u[ZT_ACC] /= sum;
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] *= u[ZT_D];
    u[ZT_DON] *= u[ZT_D];
    u[ZT_ACC] *= u[ZT_D];
}

// State::to_prim (:587-599) at position X
__device__ __forceinline__ void zt_to_prim(const ZtwdPar& P, double* u, const double* X) {
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] /= u[ZT_D];
    u[ZT_DON] /= u[ZT_D];
    u[ZT_ACC] /= u[ZT_D];
    u[ZT_ET] -= zt_ek(P, u, X);
    const double R = zt_R(X);
    u[ZT_SR] /= u[ZT_D];
    u[ZT_LZ] /= u[ZT_D] * R;
    u[ZT_LZ] -= P.omega * R;
    u[ZT_SZ] /= u[ZT_D];
    u[ZT_POT] /= u[ZT_D];
}

// State::x_flux / y_flux / z_flux (:360-396) for direction d with pressure p
template <typename T>
__device__ __forceinline__ void zt_flux(const ZtwdPar& P, const T* u, const T* X, int d, T p, T* f) {
    const T v = zt_v(P, u, X, d);
#pragma unroll
    for (int i = 0; i < ZT_NF; i++) f[i] = v * u[i];
    if (d == 0) {
        f[ZT_SR] += X[0] * p / zt_R(X);
        f[ZT_LZ] -= X[1] * p;
        f[ZT_ET] += (v + (-X[1] * T(P.omega - P.omega0))) * p;
    } else if (d == 1) {
        f[ZT_SR] += X[1] * p / zt_R(X);
        f[ZT_LZ] += X[0] * p;
        f[ZT_ET] += (v + X[0] * T(P.omega - P.omega0)) * p;
    } else {
        f[ZT_SZ] += p;
        f[ZT_ET] += v * p;
    }
}

// State::enforce_outflow (:398-443); bface is the face of the boundary
// proxy (the inverse of the brick face), X the boundary face centre of the
// copied cell (grid_phys_bound.cpp:27-54)
__device__ __forceinline__ void zt_enforce_outflow(const ZtwdPar& P, double* u, const double* X, int bface) {
    u[ZT_ET] = zt_ei(P, u, X);
    double v0;
    switch (bface) {
        case XU:
        case XL: {
            const double vx = zt_vx(P, u, X);
            if (bface == XU ? vx > 0.0 : vx < 0.0) {
                v0 = zt_vy(P, u, X);
                u[ZT_LZ] = (X[0] * (v0 + X[0] * P.omega)) * u[ZT_D];
                u[ZT_SR] = X[1] * v0 * u[ZT_D] / zt_R(X);
            }
            break;
        }
        case YU:
        case YL: {
            const double vy = zt_vy(P, u, X);
            if (bface == YU ? vy > 0.0 : vy < 0.0) {
                v0 = zt_vx(P, u, X);
                u[ZT_LZ] = (-X[1] * (v0 - X[1] * P.omega)) * u[ZT_D];
                u[ZT_SR] = X[0] * v0 * u[ZT_D] / zt_R(X);
            }
            break;
        }
        case ZU:
            if (u[ZT_SZ] > 0.0) u[ZT_SZ] = 0.0;
            break;
        default:
            if (u[ZT_SZ] < 0.0) u[ZT_SZ] = 0.0;
            break;
    }
    const double st = zt_st(P, u, X);
    u[ZT_ET] += 0.5 * (u[ZT_SR] * u[ZT_SR] + st * st + u[ZT_SZ] * u[ZT_SZ]) / u[ZT_D];
}

// State::floor (:482-554, not SCF_CODE): species and the two star
// densities made non-negative and renormalised to rho, then T from the
// internal energy by Newton (helmholtz_compute_T) and tau reset when the
// internal energy dominates.  Returns the EOS status.
__device__ __forceinline__ int zt_floor(const ZtwdPar& P, double* u, const double* X) {
    if (u[ZT_D] < P.rho_floor) {
        u[ZT_D] = P.rho_floor;
        u[ZT_ACC] = P.rho_floor * 0.5;
        u[ZT_DON] = P.rho_floor * 0.5;
        u[ZT_SPECIE + 0] = P.rho_floor;
#pragma unroll
        for (int i = 1; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] = 0.0;
    } else {
#pragma unroll
        for (int i = 0; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] = zmax(u[ZT_SPECIE + i], 0.0);
        u[ZT_DON] = zmax(u[ZT_DON], P.rho_floor / 2.0);
        u[ZT_ACC] = zmax(u[ZT_ACC], P.rho_floor / 2.0);
    }
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < ZT_NSPECIES; i++) sum += u[ZT_SPECIE + i];
    if (sum != 0.0) {
#pragma unroll
        for (int i = 0; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] *= u[ZT_D] / sum;
    } else {
        u[ZT_SPECIE] = u[ZT_D];
#pragma unroll
        for (int i = 1; i < ZT_NSPECIES; i++) u[ZT_SPECIE + i] = 0.0;
    }
    sum = 0.0;
    sum += u[ZT_DON];
    sum += u[ZT_ACC];
    if (sum != 0.0) {
        u[ZT_DON] *= u[ZT_D] / sum;
        u[ZT_ACC] *= u[ZT_D] / sum;
    } else {
        u[ZT_DON] = u[ZT_D] / 2.0;
        u[ZT_ACC] = u[ZT_D] / 2.0;
    }
    const double d = u[ZT_D];
    const double ui = zt_ei(P, u, X);
    const double A = zt_abar(P, u);
    double T = u[ZT_T];
    HelmPoint o;
    int iters;
    const int st = helm_invert_point(P.H, d, ui / d, A, A / 2.0, 0, T, o, &iters);
    if (!(st == 1 && iters == 0)) u[ZT_T] = T;
    if (ui > 0.1 * u[ZT_ET]) u[ZT_TAU] = ui;
    return st;
}

// State::source (:347-358, not SCF_CODE): pressure and centrifugal term of
// the radial momentum plus the centre-of-mass correction force; added to D
__device__ __forceinline__ int zt_add_source(const ZtwdPar& P, const double* u, const double* X, double* D) {
    double p, cs;
    const int st = zt_eos(P, u, &p, &cs);
    const double R = zt_R(X);
    const double lr = u[ZT_LZ] / R;
    double s_sr = (p + lr * lr / u[ZT_D]) / R;
    const double theta = atan2(X[1], X[0]);
    const double c = cos(theta - P.ftheta), s = sin(theta - P.ftheta);
    s_sr += u[ZT_D] * P.fR * c;
    double s_lz = 0.0;
    s_lz -= u[ZT_D] * P.fR * s * R;
    double s_et = 0.0;
    s_et += u[ZT_SR] * P.fR * c;
    s_et -= zt_st(P, u, X) * P.fR * s * R;
    D[ZT_SR] += s_sr;
    D[ZT_LZ] += s_lz;
    D[ZT_ET] += s_et;
    return st;
}

}  // namespace amr
