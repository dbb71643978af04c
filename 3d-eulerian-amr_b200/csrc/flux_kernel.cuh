// KT/Rusanov face fluxes, Grid::compute_{x,y,z}_flux (grid.cpp:215-302),
// with minmod-theta (reconstruct.cpp:60-71) or PPM (reconstruct.cpp:22-58)
// reconstruction, templated on the arithmetic type: double is the plain form
// (instantiated in hydro_kernels.cu, no FMA contraction), float the mixed
// form's FP32 reconstruction and flux (hydro_mixed.cu) whose fluxes are
// stored in FP64 and accumulated in FP64 by the conservative update.
//
// Block = one brick, 3*nx*nx threads: thread = (direction, pencil).  A pencil
// walks its GNX cells streaming the reconstruction (recon.cuh).
#pragma once

#include "recon.cuh"

namespace amr {

// index of flux array element for direction d: face index fi (0..nx) along d,
// transverse interior indices t1 (lower axis) and t2 (higher axis).
__device__ __forceinline__ int flux_index(int d, int nx, int fi, int t1, int t2) {
    if (d == 0) return (t2 * nx + t1) * (nx + 1) + fi;
    if (d == 1) return (t2 * (nx + 1) + fi) * nx + t1;
    return (fi * nx + t2) * nx + t1;
}

__device__ __forceinline__ int cell_index(int gnx, int i, int j, int k) { return (k * gnx + j) * gnx + i; }

// Primitives of cell n of one pencil (conserved state read as T, then
// State::to_prim).
template <typename T>
struct PencilLoad {
    const double* U;
    int base, stride, gnx3;
    __device__ __forceinline__ void operator()(int n, T* q) const {
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) q[l] = (T)U[l * gnx3 + base + n * stride];
        st_to_prim(q);
    }
};

// pencil p (interior transverse t1 + nx*t2) of direction d in brick b
template <typename T, int d>
__device__ __forceinline__ PencilLoad<T> pencil_load(const Geom& g, const double* Ub, int p) {
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const int t1 = p % nx, t2 = p / nx;
    PencilLoad<T> L;
    L.U = Ub;
    L.gnx3 = g.gnx3;
    if (d == 0) {
        L.stride = 1;
        L.base = cell_index(gnx, 0, t1 + bw, t2 + bw);
    } else if (d == 1) {
        L.stride = gnx;
        L.base = cell_index(gnx, t1 + bw, 0, t2 + bw);
    } else {
        L.stride = gnx * gnx;
        L.base = cell_index(gnx, t1 + bw, t2 + bw, 0);
    }
    return L;
}

template <typename T, int d, int R>
__device__ __forceinline__ void flux_pencil_dir(const Geom& g, const DevState& st, int b, int p) {
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const int npen = nx * nx;
    const int t1 = p % nx, t2 = p / nx;
    PencilLoad<T> load = pencil_load<T, d>(g, st.U + (size_t)b * g.ucount, p);
    double* F = (d == 0 ? st.Fx : (d == 1 ? st.Fy : st.Fz)) + (size_t)b * g.nf * npen * (nx + 1);
    const int fstride = npen * (nx + 1);
    const T gam = (T)g.gamma;
    PencilRecon<T, R> rec;
    rec.begin(load, bw, (T)g.theta);
    for (int f = bw; f <= gnx - bw; f++) {
        T ql[NF_EULER], qr[NF_EULER];
        rec.next(load, f, ql, qr);
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

// The direction is made a compile-time constant per thread, so the state
// arrays indexed by it (normal velocity, normal momentum flux) stay in
// registers.
template <typename T, int R>
__device__ __forceinline__ void flux_pencils(const Geom& g, const DevState& st, int b) {
    const int npen = g.nx * g.nx;
    const int d = threadIdx.x / npen;
    const int p = threadIdx.x % npen;
    if (d == 0)
        flux_pencil_dir<T, 0, R>(g, st, b, p);
    else if (d == 1)
        flux_pencil_dir<T, 1, R>(g, st, b, p);
    else if (d == 2)
        flux_pencil_dir<T, 2, R>(g, st, b, p);
}

// Largest face eigenvalue max(lambda(ql), lambda(qr)) over the faces of
// pencil p of direction d (Grid::max_dt's inner loop, grid.cpp:430-470).
template <int d, int R>
__device__ __forceinline__ double max_eigen_pencil(const Geom& g, const DevState& st, int b, int p, double lam) {
    PencilLoad<double> load = pencil_load<double, d>(g, st.U + (size_t)b * g.ucount, p);
    PencilRecon<double, R> rec;
    rec.begin(load, g.bw, g.theta);
    for (int f = g.bw; f <= g.gnx - g.bw; f++) {
        double ql[NF_EULER], qr[NF_EULER];
        rec.next(load, f, ql, qr);
        st_to_con(ql);
        st_to_con(qr);
        lam = r_max(lam, r_max(st_eigen(ql, d, g.gamma), st_eigen(qr, d, g.gamma)));
    }
    return lam;
}

}  // namespace amr
