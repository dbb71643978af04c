// Helmholtz EOS at one point, device side (helmholtz/helmeos.cpp), shared by
// the batched EOS kernels (helm_kernels.cu) and the ZTWD hydro kernels
// (ztwd_kernels.cu).  FP64; include only from translation units compiled
// without FMA contraction, so every sum rounds as the reference's x86-64
// build does.
//
// The electron-positron free energy is a biquintic Hermite interpolant in
// (ye*rho, T) of the tabulated F and its derivatives; the six sums F, F_d,
// F_t, F_dd, F_tt, F_dt share the 36 node values and are accumulated in the
// reference's term order (helmeos.cpp:20-37).
#pragma once

#include <cuda_runtime.h>

#include "helm_internal.h"

namespace amr {

namespace {

// physical constants of helmholtz/const.h
constexpr double C_PI = 3.1415926535897932384e0;
constexpr double C_H = 6.6260689633e-27;
constexpr double C_AVO = 6.0221417930e23;
constexpr double C_KERG = 1.380650424e-16;
constexpr double C_AMU = 1.66053878283e-24;

__device__ __forceinline__ double hmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double hmin(double a, double b) { return a < b ? a : b; }

// quintic Hermite basis functions and their derivatives (helmeos.cpp:17-25)
__device__ __forceinline__ void psi_all(double z, double* p, double* dp, double* ddp) {
    p[0] = z * z * z * (z * (-6.0 * z + 15.0) - 10.0) + 1.0;
    dp[0] = z * z * (z * (-30.0 * z + 60.0) - 30.0);
    ddp[0] = z * (z * (-120.0 * z + 180.0) - 60.0);
    p[1] = z * (z * z * (z * (-3.0 * z + 8.0) - 6.0) + 1.0);
    dp[1] = z * z * (z * (-15.0 * z + 32.0) - 18.0) + 1.0;
    ddp[1] = z * (z * (-60.0 * z + 96.0) - 36.0);
    p[2] = 0.5 * z * z * (z * (z * (-z + 3.0) - 3.0) + 1.0);
    dp[2] = 0.5 * z * (z * (z * (-5.0 * z + 12.0) - 9.0) + 2.0);
    ddp[2] = 0.5 * (z * (z * (-20.0 * z + 36.0) - 18.0) + 2.0);
}

// Weights of one axis (helmeos.cpp:272-324): W[deriv][order][side], side 0 =
// the lower node (argument x), side 1 = the upper node (argument 1 - x).
struct AxisWeights {
    double W[3][3][2];
};

__device__ __forceinline__ void axis_weights(double x, double h, double h2, double hi, double h2i, AxisWeights& a) {
    double p[3], dp[3], ddp[3], pm[3], dpm[3], ddpm[3];
    const double mx = 1.0 - x;
    psi_all(x, p, dp, ddp);
    psi_all(mx, pm, dpm, ddpm);
    a.W[0][0][0] = p[0];
    a.W[0][1][0] = p[1] * h;
    a.W[0][2][0] = p[2] * h2;
    a.W[0][0][1] = pm[0];
    a.W[0][1][1] = -pm[1] * h;
    a.W[0][2][1] = pm[2] * h2;
    a.W[1][0][0] = dp[0] * hi;
    a.W[1][1][0] = dp[1];
    a.W[1][2][0] = dp[2] * h;
    a.W[1][0][1] = -dpm[0] * hi;
    a.W[1][1][1] = dpm[1];
    a.W[1][2][1] = -dpm[2] * h;
    a.W[2][0][0] = ddp[0] * h2i;
    a.W[2][1][0] = ddp[1] * hi;
    a.W[2][2][0] = ddp[2];
    a.W[2][0][1] = ddpm[0] * h2i;
    a.W[2][1][1] = -ddpm[1] * hi;
    a.W[2][2][1] = ddpm[2];
}

// The 36 terms in the reference's order: block b (4 corners each) reads table
// column COL[b] with density-weight order OD[b] and temperature-weight order
// OT[b]; corner c: density side c & 1, temperature side c >> 1.
__device__ constexpr int COL[9] = {0, 2, 4, 1, 3, 5, 6, 7, 8};
__device__ constexpr int OD[9] = {0, 0, 0, 1, 2, 1, 2, 1, 2};
__device__ constexpr int OT[9] = {0, 1, 2, 0, 0, 1, 1, 2, 2};

}  // namespace

// helmholtz_eos (helmeos.cpp:164-421) at one point in code units.
__device__ __forceinline__ void helm_point(const HelmTable& H, double rho_code, double T_code, double abar, double zbar,
                           HelmPoint& o) {
    const double den = rho_code * H.u.f_rho;  // eos_from_code (helmeos.cpp:153-162)
    const double Tc = T_code * H.u.f_T;
    o.rho = den / H.u.f_rho;  // eos_to_code applied to the inputs (helmeos.cpp:142-151)
    o.T = Tc / H.u.f_T;
    const double temp = hmax(Tc, HELM_TMIN);
    const double ytot1 = 1.0 / abar;
    const double ye = hmax(1.0 - 16, ytot1 * zbar);  // the reference writes 1.0d - 16
    const double deni = 1.0 / den;
    const double kt = C_KERG * temp;
    // ion section
    const double xni = C_AVO * ytot1 * den;
    const double dxnidd = C_AVO * ytot1;
    const double pion = xni * kt;
    const double dpiondd = dxnidd * kt;
    const double dpiondt = xni * C_KERG;
    const double eion = 1.5 * pion * deni;
    const double deiondt = 1.5 * dpiondt * deni;
    // Sackur-Tetrode ion entropy
    double x = abar * abar * sqrt(abar) * deni / C_AVO;
    const double s = ((2.0 * C_PI * C_AMU * C_KERG) / (C_H * C_H)) * temp;
    const double z = x * s * sqrt(s);
    const double y = log(z);
    const double tempi = 1.0 / temp;
    const double sion = (pion * deni + eion) * tempi + C_KERG * C_AVO * ytot1 * y;
    const double dsiondt = (dpiondt * deni + deiondt) * tempi - (pion * deni + eion) * tempi * tempi +
                           1.5 * C_KERG * C_AVO * tempi * ytot1;
    // electron-positron section: enter the table with ye*den
    const double din = ye * den;
    if ((temp > H.t_last) || (temp < H.t_first) || (din > H.d_last) || (din < H.d_first)) {
        o.status = 1;  // the reference aborts here
        o.p = o.e = o.cs = o.cv = o.s = o.dsdt = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    int jat = int((log10(temp) - H.tlo) * H.tstpi) + 1;
    jat = (int)hmax(1, hmin(jat, HELM_JMAX - 1));
    int iat = int((log10(din) - H.dlo) * H.dstpi) + 1;
    iat = (int)hmax(1, hmin(iat, HELM_IMAX - 1));
    --jat;
    --iat;
    const double* tj = H.tj + 8 * jat;
    const double* di = H.di + 8 * iat;
    const double t_j = __ldg(tj + 0), dt = __ldg(tj + 1), dt2 = __ldg(tj + 2), dti = __ldg(tj + 3),
                 dt2i = __ldg(tj + 4);
    const double d_i = __ldg(di + 0), dd = __ldg(di + 1), dd2 = __ldg(di + 2), ddi = __ldg(di + 3),
                 dd2i = __ldg(di + 4);
    const double xt = hmax((temp - t_j) * dti, 0.0);
    const double xd = hmax((din - d_i) * ddi, 0.0);
    AxisWeights wt, wd;
    axis_weights(xt, dt, dt2, dti, dt2i, wt);
    axis_weights(xd, dd, dd2, ddi, dd2i, wd);
    // node values of the four corners: rows j and j+1, each a 20-double run
    // (two nodes of 10) starting at node (iat, row)
    const double2* r0 = reinterpret_cast<const double2*>(H.node + ((size_t)jat * HELM_IMAX + iat) * HELM_NODE);
    const double2* r1 = reinterpret_cast<const double2*>(H.node + ((size_t)(jat + 1) * HELM_IMAX + iat) * HELM_NODE);
    double v0[2 * HELM_NODE], v1[2 * HELM_NODE];
#pragma unroll
    for (int q = 0; q < HELM_NODE; q++) {
        const double2 a = __ldg(r0 + q), b = __ldg(r1 + q);
        v0[2 * q] = a.x;
        v0[2 * q + 1] = a.y;
        v1[2 * q] = b.x;
        v1[2 * q + 1] = b.y;
    }
    // the six biquintic sums (helmeos.cpp:327-354), term by term in order
    double free = 0.0, df_d = 0.0, df_t = 0.0, df_dd = 0.0, df_tt = 0.0, df_dt = 0.0;
    bool first = true;
#pragma unroll
    for (int b = 0; b < 9; b++) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int sd = c & 1, st = c >> 1;
            const double fi = (st ? v1 : v0)[sd * HELM_NODE + COL[b]];
            const double a0 = fi * wd.W[0][OD[b]][sd] * wt.W[0][OT[b]][st];
            const double a1 = fi * wd.W[1][OD[b]][sd] * wt.W[0][OT[b]][st];
            const double a2 = fi * wd.W[0][OD[b]][sd] * wt.W[1][OT[b]][st];
            const double a3 = fi * wd.W[2][OD[b]][sd] * wt.W[0][OT[b]][st];
            const double a4 = fi * wd.W[0][OD[b]][sd] * wt.W[2][OT[b]][st];
            const double a5 = fi * wd.W[1][OD[b]][sd] * wt.W[1][OT[b]][st];
            if (first) {
                free = a0, df_d = a1, df_t = a2, df_dd = a3, df_tt = a4, df_dt = a5;
                first = false;
            } else {
                free += a0, df_d += a1, df_t += a2, df_dd += a3, df_tt += a4, df_dt += a5;
            }
        }
    }
    // electron-positron thermodynamics (helmeos.cpp:386-404)
    x = din * din;
    const double pele = x * df_d;
    const double dpepdd = ye * (x * df_dd + 2.0 * din * df_d);
    const double dpepdt = x * df_dt;
    const double sele = -df_t * ye;
    const double dsepdt = -df_tt * ye;
    const double eele = ye * free + temp * sele;
    const double deepdt = temp * dsepdt;
    const double p = pele + pion;
    const double e = eele + eion;
    const double sv = sele + sion;
    const double dsdt = dsiondt + dsepdt;
    const double cv = deiondt + deepdt;
    const double dpgasdd = dpiondd + dpepdd;
    const double dpgasdt = dpiondt + dpepdt;
    x = (p * deni * deni) * (dpgasdt / cv) + dpgasdd;
    o.status = 0;
    double cs = 0.0;
    if (cv < 0.0) {
        o.status = 2;
    } else if (x < 0.0) {
        o.status = 3;
    } else {
        cs = sqrt(x);
    }
    o.p = p / H.u.f_p;
    o.e = e / H.u.f_e;
    o.cs = cs / H.u.f_cs;
    o.cv = cv / H.u.f_cv;
    o.s = sv / H.u.f_s;
    o.dsdt = dsdt / H.u.f_dsdt;
}

// helmholtz_compute_T (helmeos.cpp:436-486) at one point: Newton on e(T) (or
// s(T)) from the guess T (in/out), at most 100 iterations, step damped by 0.9
// every 10 iterations, T kept above the midpoint of the last T and the floor.
// o holds the EOS at the final temperature; returns the point's status
// (0 ok, 1 outside the table, 2 cv < 0, 3 cs^2 < 0, 4 no convergence,
// 5 below the temperature floor); *iters_out gets the iteration count.
__device__ __forceinline__ int helm_invert_point(const HelmTable& H, double r, double e0, double ab, double zb,
                                                 int from_entropy, double& Tq, HelmPoint& o, int* iters_out) {
    double T0 = Tq;
    helm_point(H, r, HELM_TMIN, ab, zb, o);
    r = o.rho;
    int st = o.status;
    int iters = 0;
    if (st == 1) {  // outside the table at the floor temperature
        *iters_out = 0;
        return st;
    }
    if ((from_entropy ? o.s : o.e) >= e0) {
        Tq = HELM_TMIN;
    } else {
        double a = 1.0;
        for (;;) {
            T0 = hmax(Tq, HELM_TMIN);
            helm_point(H, r, Tq, ab, zb, o);
            r = o.rho;
            Tq = o.T;
            if (!st) st = o.status;
            const double f = (from_entropy ? o.s : o.e) - e0;
            const double dT = -f / (from_entropy ? o.dsdt : o.cv);
            Tq += a * dT;
            Tq = hmax(Tq, (T0 + HELM_TMIN) / 2.0);
            iters++;
            if (iters % 10 == 0) a *= 0.9;
            if (Tq < HELM_TMIN) {
                if (!st) st = 5;
                break;
            }
            if (!(fabs(f / e0) >= 1.0e-9 && iters < 100)) break;
        }
        helm_point(H, r, Tq, ab, zb, o);
        r = o.rho;
        Tq = o.T;
        if (!st) st = o.status;
        if (iters >= 100 && !st) st = 4;
    }
    if (Tq < HELM_TMIN && !st) st = 5;
    *iters_out = iters;
    return st;
}

}  // namespace amr
