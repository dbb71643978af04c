// KT/Rusanov face fluxes, Grid::compute_{x,y,z}_flux (grid.cpp:215-302),
// with minmod-theta reconstruction (reconstruct.cpp:60-71), templated on the
// arithmetic type: double is the plain form (instantiated in
// hydro_kernels.cu, no FMA contraction), float the mixed form's FP32
// reconstruction and flux (hydro_mixed.cu) whose fluxes are stored in FP64
// and accumulated in FP64 by the conservative update.
//
// Block = one brick, 3*nx*nx threads: thread = (direction, pencil).  A pencil
// walks its GNX cells keeping a four-cell window of primitives.
#pragma once

#include "euler_state.cuh"

namespace amr {

// index of flux array element for direction d: face index fi (0..nx) along d,
// transverse interior indices t1 (lower axis) and t2 (higher axis).
__device__ __forceinline__ int flux_index(int d, int nx, int fi, int t1, int t2) {
    if (d == 0) return (t2 * nx + t1) * (nx + 1) + fi;
    if (d == 1) return (t2 * (nx + 1) + fi) * nx + t1;
    return (fi * nx + t2) * nx + t1;
}

__device__ __forceinline__ int cell_index(int gnx, int i, int j, int k) { return (k * gnx + j) * gnx + i; }

template <typename T, int d>
__device__ __forceinline__ void flux_pencil_dir(const Geom& g, const DevState& st, int b, int p);

// The direction is made a compile-time constant per thread, so the state
// arrays indexed by it (normal velocity, normal momentum flux) stay in
// registers.
template <typename T>
__device__ __forceinline__ void flux_pencils(const Geom& g, const DevState& st, int b) {
    const int npen = g.nx * g.nx;
    const int d = threadIdx.x / npen;
    const int p = threadIdx.x % npen;
    if (d == 0)
        flux_pencil_dir<T, 0>(g, st, b, p);
    else if (d == 1)
        flux_pencil_dir<T, 1>(g, st, b, p);
    else if (d == 2)
        flux_pencil_dir<T, 2>(g, st, b, p);
}

template <typename T, int d>
__device__ __forceinline__ void flux_pencil_dir(const Geom& g, const DevState& st, int b, int p) {
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const int npen = nx * nx;
    const int t1 = p % nx, t2 = p / nx;  // interior transverse indices
    const double* U = st.U + (size_t)b * g.ucount;
    int stride, base;
    if (d == 0) {
        stride = 1;
        base = cell_index(gnx, 0, t1 + bw, t2 + bw);
    } else if (d == 1) {
        stride = gnx;
        base = cell_index(gnx, t1 + bw, 0, t2 + bw);
    } else {
        stride = gnx * gnx;
        base = cell_index(gnx, t1 + bw, t2 + bw, 0);
    }
    double* F = (d == 0 ? st.Fx : (d == 1 ? st.Fy : st.Fz)) + (size_t)b * g.nf * npen * (nx + 1);
    const int fstride = npen * (nx + 1);
    const T th = (T)g.theta, gam = (T)g.gamma;

    T w[4][NF_EULER];  // primitives of cells f-2 .. f+1
    for (int n = 0; n < 3; n++) {
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) w[n + 1][l] = (T)U[l * g.gnx3 + base + n * stride];
        st_to_prim(w[n + 1]);
    }
    T sR[NF_EULER];
    // for bw > 2 advance the window up to face bw
    for (int n = 3; n < bw + 1; n++) {
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) w[m][l] = w[m + 1][l];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) w[3][l] = (T)U[l * g.gnx3 + base + n * stride];
        st_to_prim(w[3]);
    }
    // now w[1..3] hold cells bw-2 .. bw; sR = slope at cell bw-1
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) sR[l] = minmod_theta(w[3][l] - w[2][l], w[2][l] - w[1][l], th);
    for (int f = bw; f <= gnx - bw; f++) {
        // shift window: w[0..3] = cells f-2, f-1, f, f+1
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) w[m][l] = w[m + 1][l];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) w[3][l] = (T)U[l * g.gnx3 + base + (f + 1) * stride];
        st_to_prim(w[3]);
        T ql[NF_EULER], qr[NF_EULER], sL[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            sL[l] = sR[l];                                                   // s[f-1]
            sR[l] = minmod_theta(w[3][l] - w[2][l], w[2][l] - w[1][l], th);  // s[f]
            ql[l] = w[1][l] + sL[l] / T(2);
            qr[l] = w[2][l] - sR[l] / T(2);
        }
        st_to_con(ql);
        st_to_con(qr);
        T fl[NF_EULER], fr[NF_EULER];
        const T al = st_flux(ql, d, gam, fl);
        const T ar = st_flux(qr, d, gam, fr);
        const T a = r_max(al, ar);
        const int fi = flux_index(d, nx, f - bw, t1, t2);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++)
            F[l * fstride + fi] = (double)(((fl[l] + fr[l]) - (qr[l] - ql[l]) * a) * T(0.5));
    }
}

}  // namespace amr
