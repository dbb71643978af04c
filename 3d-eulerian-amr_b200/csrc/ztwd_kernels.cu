// Hydro kernels of the ZTWD binary state (BINARY build of the reference:
// binary/state_ztwd.cpp, binary/binary.cpp), plain FP64, no FMA
// contraction.  Same layouts as the Euler kernels (hydro_kernels.cu) with
// NF = 13, plus
//   W  [slot][13][gnx^3]  primitives at cell centres (the cells the flux
//                         pencils read), rebuilt before every flux or CFL pass
//   Vx/Vy/Vz [slot][nx][nx][nx+1] ...  normal velocity of the face-averaged
//                         state (ql+qr)/2, the SAVE_RECONSTRUCTIONS face states
//                         Uxf/Uyf/Uzf of grid.cpp:232-234 as Binary::add_difs
//                         uses them (binary.cpp:228-235)
// The reference aborts where the EOS leaves its table or fails; here the
// first such status is kept in an error word and the host returns
// AMR_ERR_RANGE.
#include "euler_state.cuh"
#include "flux_kernel.cuh"
#include "launch.cuh"
#include "poisson_ops.cuh"
#include "ztwd.h"
#include "ztwd_state.cuh"

namespace amr {

namespace {

__device__ __forceinline__ void zt_fail(int* err, int st) {
    if (st) atomicCAS(err, 0, st);
}

// Grid::xf/yf/zf (grid/grid.cpp:512-526) and the centres xf + h/2
__device__ __forceinline__ double grid_face(const Geom& g, int axis, int off, double h, int gi) {
    if (axis < 2) return double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0 - g.origin[axis];
    if (g.z_reflect) return double(off + gi) * h - double(g.bw) * g.h0 - g.origin[2];
    return double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0;
}
__device__ __forceinline__ double grid_centre(const Geom& g, int axis, int off, double h, int gi) {
    return grid_face(g, axis, off, h, gi) + 0.5 * h;
}
__device__ __forceinline__ void cell_X(const Geom& g, const BrickTable& bt, int b, int i, int j, int k, double* X) {
    const double h = bt.h[b];
    X[0] = grid_centre(g, 0, bt.off[3 * b + 0], h, i);
    X[1] = grid_centre(g, 1, bt.off[3 * b + 1], h, j);
    X[2] = grid_centre(g, 2, bt.off[3 * b + 2], h, k);
}

__device__ __forceinline__ void load_cell(const Geom& g, const double* Ub, int ci, double* u) {
#pragma unroll
    for (int l = 0; l < ZT_NF; l++) u[l] = Ub[l * g.gnx3 + ci];
}
__device__ __forceinline__ void store_cell(const Geom& g, double* Ub, int ci, const double* u) {
#pragma unroll
    for (int l = 0; l < ZT_NF; l++) Ub[l * g.gnx3 + ci] = u[l];
}

// ---------------------------------------------------------------------------
// ghost zones: GridNode::enforce_boundaries (grid_node.cpp:59-112) with the
// ZTWD physical boundaries (grid_phys_bound.cpp:27-54: outflow at the
// boundary face centre of the copied cell, State::reflect_on_z).
// grid = (bricks of one level, 6 faces); thread per ghost cell of the slab.
// ---------------------------------------------------------------------------
__global__ void k_zt_ghost_fill(Geom g, BrickTable bt, DevState st, ZtwdPar P, const int* __restrict__ slots) {
    const int b = slots[blockIdx.x];
    const int face = blockIdx.y;
    const int ax = face >> 1, upper = face & 1;
    const int bw = g.bw, gnx = g.gnx, nx = g.nx;
    const int kind = bt.ftype[6 * b + face];
    const int nbr = bt.fnbr[6 * b + face];
    double* U = st.U + (size_t)b * g.ucount;
    for (int t = threadIdx.x; t < bw * nx * nx; t += blockDim.x) {
        const int n = t % bw;
        const int t1 = (t / bw) % nx + bw;
        const int t2 = (t / bw) / nx + bw;
        const int gi = upper ? gnx - bw + n : n;
        int c[3];
        c[ax] = gi;
        c[ax == 0 ? 1 : 0] = t1;
        c[ax == 2 ? 1 : 2] = t2;
        const int dst = cell_index(gnx, c[0], c[1], c[2]);
        double u[ZT_NF];
        if (kind == FACE_SIB) {
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = upper ? gi - (gnx - 2 * bw) : gi + (gnx - 2 * bw);
            load_cell(g, st.U + (size_t)nbr * g.ucount, cell_index(gnx, s[0], s[1], s[2]), u);
        } else if (kind == FACE_OUTFLOW) {
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = upper ? gnx - bw - 1 : bw;
            load_cell(g, U, cell_index(gnx, s[0], s[1], s[2]), u);
            const double h = bt.h[b];
            double X[3];
#pragma unroll
            for (int d = 0; d < 3; d++)
                X[d] = d == ax ? grid_face(g, d, bt.off[3 * b + d], h, upper ? gnx - bw : bw)
                               : grid_centre(g, d, bt.off[3 * b + d], h, c[d]);
            zt_enforce_outflow(P, u, X, face ^ 1);
        } else if (kind == FACE_REFLECT) {
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = 2 * bw - 1 - gi;
            load_cell(g, U, cell_index(gnx, s[0], s[1], s[2]), u);
            u[ZT_SZ] = -u[ZT_SZ];
        } else {
            // GridAMRBound (grid_amr_bound.cpp:27-78), field by field
            const double* Pp = st.U + (size_t)nbr * g.ucount;
            int pi[3], par = 0;
            for (int d = 0; d < 3; d++) {
                const int fine = bt.off[3 * b + d] - 2 * bt.off[3 * nbr + d] + c[d];
                pi[d] = fine / 2;
                if (d == ax) par = fine % 2;
            }
            int pp[3] = {pi[0], pi[1], pi[2]}, pm[3] = {pi[0], pi[1], pi[2]};
            pp[ax] += 1;
            pm[ax] -= 1;
            const int i0 = cell_index(gnx, pi[0], pi[1], pi[2]);
            const int ip = cell_index(gnx, pp[0], pp[1], pp[2]);
            const int im = cell_index(gnx, pm[0], pm[1], pm[2]);
#pragma unroll
            for (int l = 0; l < ZT_NF; l++) {
                const double uc = Pp[l * g.gnx3 + i0];
                double m = minmod2(Pp[l * g.gnx3 + ip] - uc, uc - Pp[l * g.gnx3 + im]);
                if (par == 1) m = -m;
                u[l] = uc - m * 0.25;
            }
        }
        store_cell(g, U, dst, u);
    }
}

// ---------------------------------------------------------------------------
// primitives of the cells the flux pencils read (interior, and the six
// ghost slabs' transverse-interior cells): State::to_prim at the cell centre
// (the q0[i].to_prim(X(i, j, k)) of grid.cpp:226-229)
// ---------------------------------------------------------------------------
__global__ void k_zt_prim(Geom g, BrickTable bt, DevState st, ZtwdPar P, const int* __restrict__ slots) {
    const int b = slots[blockIdx.x];
    const int gnx = g.gnx, bw = g.bw;
    const double* U = st.U + (size_t)b * g.ucount;
    double* W = st.W + (size_t)b * g.ucount;
    for (int t = threadIdx.x; t < g.gnx3; t += blockDim.x) {
        const int i = t % gnx, j = (t / gnx) % gnx, k = t / (gnx * gnx);
        const int out = (i < bw || i >= gnx - bw) + (j < bw || j >= gnx - bw) + (k < bw || k >= gnx - bw);
        if (out > 1) continue;  // edge and corner ghosts: never read
        double u[ZT_NF], X[3];
        load_cell(g, U, t, u);
        cell_X(g, bt, b, i, j, k, X);
        zt_to_prim(P, u, X);
        store_cell(g, W, t, u);
    }
}

// Colella-Woodward monotonisation of one cell's edges (reconstruct.cpp:40-53)
template <typename T>
__device__ __forceinline__ void cw_mono(T q0, T& lo, T& hi) {
    const T six = T(1.0) / T(6.0);
    const T tmp1 = hi - lo;
    const T tmp2 = hi + lo;
    if ((hi - q0) * (q0 - lo) <= T(0.0)) {
        hi = lo = q0;
    } else if (tmp1 * (q0 - T(0.5) * tmp2) > six * tmp1 * tmp1) {
        lo = T(3.0) * q0 - T(2.0) * hi;
    } else if (-six * tmp1 * tmp1 > tmp1 * (q0 - T(0.5) * tmp2)) {
        hi = T(3.0) * q0 - T(2.0) * lo;
    }
}

// Face f (grid index along d) of pencil (t1, t2): left and right primitive
// states by Reconstruct::ppm as called (reconstruct.cpp:22-58, 94) from the
// primitives of cells f-3 .. f+2; the potential is a low-order and smooth
// field (state_ztwd.cpp:50-56): plain interface average, no monotonisation.
template <typename T>
__device__ __forceinline__ void zt_face_states(const Geom& g, const double* W, int base, int stride, int f, T* ql,
                                               T* qr) {
    const T six = T(1.0) / T(6.0);
#pragma unroll
    for (int l = 0; l < ZT_NF; l++) {
        const double* w = W + l * g.gnx3 + base;
        T q[6];
#pragma unroll
        for (int m = 0; m < 6; m++) q[m] = T(w[(f - 3 + m) * stride]);
        if (l == ZT_POT) {
            const T I = (q[2] + q[3]) * T(0.5);
            ql[l] = I;
            qr[l] = I;
            continue;
        }
        T s[5];
#pragma unroll
        for (int m = 1; m <= 4; m++) s[m] = minmod_theta(q[m + 1] - q[m], q[m] - q[m - 1], T(2.0));
        T I[4];
#pragma unroll
        for (int m = 1; m <= 3; m++) {
            I[m] = (q[m] + q[m + 1]) * T(0.5);
            I[m] += (s[m] - s[m + 1]) * six;
        }
        T lo1 = I[1], hi1 = I[2];  // cell f-1
        cw_mono(q[2], lo1, hi1);
        T lo2 = I[2], hi2 = I[3];  // cell f
        cw_mono(q[3], lo2, hi2);
        ql[l] = hi1;
        qr[l] = lo2;
    }
}

// decode face r of direction d (flux_index layout) into (fi, t1, t2)
__device__ __forceinline__ void face_decode(int d, int nx, int r, int& fi, int& t1, int& t2) {
    if (d == 0) {
        fi = r % (nx + 1);
        t1 = (r / (nx + 1)) % nx;
        t2 = r / ((nx + 1) * nx);
    } else if (d == 1) {
        t1 = r % nx;
        fi = (r / nx) % (nx + 1);
        t2 = r / (nx * (nx + 1));
    } else {
        t1 = r % nx;
        t2 = (r / nx) % nx;
        fi = r / (nx * nx);
    }
}

// pencil base cell and stride of direction d at interior transverse (t1, t2)
__device__ __forceinline__ void pencil_of(const Geom& g, int d, int t1, int t2, int& base, int& stride) {
    const int gnx = g.gnx, bw = g.bw;
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
}

// centre of face f along d at transverse (t1, t2): Grid::Xfx/Xfy/Xfz
__device__ __forceinline__ void face_X(const Geom& g, const BrickTable& bt, int b, int d, int f, int t1, int t2,
                                       double* X) {
    const double h = bt.h[b];
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    X[d] = grid_face(g, d, bt.off[3 * b + d], h, f);
    X[a1] = grid_centre(g, a1, bt.off[3 * b + a1], h, t1 + g.bw);
    X[a2] = grid_centre(g, a2, bt.off[3 * b + a2], h, t2 + g.bw);
}

// ---------------------------------------------------------------------------
// KT fluxes of the ZTWD state: Grid::compute_{x,y,z}_flux (grid.cpp:215-302)
// with PPM, the face states to_con'd at the face centre, p and cs from one
// EOS call per face state, and the face-averaged normal velocity.
// Binary::compute_*_flux's adjust_rho_fluxes (binary.cpp:1171-1235) has an
// empty body (state_ztwd.cpp:445-480).  Block = one brick, thread per face.
// T = double: the plain form.  T = float: the mixed form's reconstruction,
// to_con and KT combination in FP32 from the FP64 primitives, the EOS in
// FP64 (zt_eos_of), the fluxes and face velocities stored in FP64 for the
// FP64 flux correction and conservative update.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_zt_flux(Geom g, BrickTable bt, DevState st, ZtwdPar P,
                                                 const int* __restrict__ slots, int* err) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, bw = g.bw;
    const int fstride = nx * nx * (nx + 1);
    const double* W = st.W + (size_t)b * g.ucount;
    for (int q = threadIdx.x; q < 3 * fstride; q += blockDim.x) {
        const int d = q / fstride, r = q % fstride;
        int fi, t1, t2, base, stride;
        face_decode(d, nx, r, fi, t1, t2);
        pencil_of(g, d, t1, t2, base, stride);
        const int f = fi + bw;
        T ql[ZT_NF], qr[ZT_NF], X[3];
        zt_face_states(g, W, base, stride, f, ql, qr);
        {
            double Xd[3];
            face_X(g, bt, b, d, f, t1, t2, Xd);
#pragma unroll
            for (int e = 0; e < 3; e++) X[e] = T(Xd[e]);
        }
        zt_to_con(P, ql, X);
        zt_to_con(P, qr, X);
        T pl, csl, pr, csr;
        zt_fail(err, zt_eos_of(P, ql, &pl, &csl));
        zt_fail(err, zt_eos_of(P, qr, &pr, &csr));
        const T al = fabs(zt_v(P, ql, X, d)) + csl;
        const T ar = fabs(zt_v(P, qr, X, d)) + csr;
        const T a = al > ar ? al : ar;
        T avg[ZT_NF];
#pragma unroll
        for (int l = 0; l < ZT_NF; l++) avg[l] = (ql[l] + qr[l]) * T(0.5);
        double* F = (d == 0 ? st.Fx : (d == 1 ? st.Fy : st.Fz)) + (size_t)b * g.nf * fstride;
        double* V = (d == 0 ? st.Vx : (d == 1 ? st.Vy : st.Vz)) + (size_t)b * fstride;
        V[r] = double(zt_v(P, avg, X, d));
        T fl[ZT_NF], fr[ZT_NF];
        zt_flux(P, ql, X, d, pl, fl);
        zt_flux(P, qr, X, d, pr, fr);
#pragma unroll
        for (int l = 0; l < ZT_NF; l++)
            F[l * fstride + r] = double(((fl[l] + fr[l]) - (qr[l] - ql[l]) * a) * T(0.5));
    }
}

// Grid::max_dt (grid.cpp:422-483) with the ZTWD eigenvalues |v| + cs
__global__ void __launch_bounds__(128) k_zt_max_dt(Geom g, BrickTable bt, DevState st, ZtwdPar P,
                                                   const int* __restrict__ slots, double* __restrict__ dt_out,
                                                   int* err) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, bw = g.bw;
    const int fstride = nx * nx * (nx + 1);
    const double* W = st.W + (size_t)b * g.ucount;
    __shared__ double red[32];
    double lam = 0.0;
    for (int q = threadIdx.x; q < 3 * fstride; q += blockDim.x) {
        const int d = q / fstride, r = q % fstride;
        int fi, t1, t2, base, stride;
        face_decode(d, nx, r, fi, t1, t2);
        pencil_of(g, d, t1, t2, base, stride);
        const int f = fi + bw;
        double ql[ZT_NF], qr[ZT_NF], X[3];
        zt_face_states(g, W, base, stride, f, ql, qr);
        face_X(g, bt, b, d, f, t1, t2, X);
        zt_to_con(P, ql, X);
        zt_to_con(P, qr, X);
        double pl, csl, pr, csr;
        zt_fail(err, zt_eos(P, ql, &pl, &csl));
        zt_fail(err, zt_eos(P, qr, &pr, &csr));
        const double al = fabs(zt_v(P, ql, X, d)) + csl;
        const double ar = fabs(zt_v(P, qr, X, d)) + csr;
        lam = zmax(lam, zmax(al, ar));
    }
    for (int o = 16; o > 0; o >>= 1) lam = zmax(lam, __shfl_xor_sync(0xffffffffu, lam, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lam;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) m = zmax(m, red[w]);
        double dtinv = m / bt.h[b];
        if (dtinv == 0.0) dtinv = 1.0E-10;
        double dt = 1.0 / dtinv;
        dt *= g.cfl;
        dt_out[b] = dt;
    }
}

// ---------------------------------------------------------------------------
// clear_difs + sum_{x,y,z}_difs (grid.cpp:201-213, 304-344), the cell part
// of Binary::add_difs (binary.cpp:205-245: gravity source from the mean face
// forces, -p div u from the face-averaged velocities, D[pot] = D[T] = 0),
// then Grid::add_difs (grid.cpp:406-420: State::source, RK combine,
// State::floor).  Block = one brick, thread per interior cell.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_zt_add_difs(Geom g, BrickTable bt, DevState st, ZtwdPar P,
                                                     const int* __restrict__ slots, double dt, double beta,
                                                     int* err) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, pnx = g.pnx;
    const int npen = nx * nx, fstride = npen * (nx + 1);
    const double h = bt.h[b];
    const double hinv = 1.0 / h;
    const double* Fx = st.Fx + (size_t)b * g.nf * fstride;
    const double* Fy = st.Fy + (size_t)b * g.nf * fstride;
    const double* Fz = st.Fz + (size_t)b * g.nf * fstride;
    const double* Vx = st.Vx + (size_t)b * fstride;
    const double* Vy = st.Vy + (size_t)b * fstride;
    const double* Vz = st.Vz + (size_t)b * fstride;
    double* U = st.U + (size_t)b * g.ucount;
    const double* U0 = st.U0 + (size_t)b * g.ucount;
    const size_t pb = (size_t)b * g.pnx3;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx, j = (t / nx) % nx, k = t / npen;
        double D[ZT_NF];
        const int a0 = flux_index(0, nx, i, j, k), a1 = flux_index(0, nx, i + 1, j, k);
        const int b0 = flux_index(1, nx, j, i, k), b1 = flux_index(1, nx, j + 1, i, k);
        const int c0 = flux_index(2, nx, k, i, j), c1 = flux_index(2, nx, k + 1, i, j);
#pragma unroll
        for (int l = 0; l < ZT_NF; l++) {
            double v = 0.0;
            v -= (Fx[l * fstride + a1] - Fx[l * fstride + a0]) * hinv;
            v -= (Fy[l * fstride + b1] - Fy[l * fstride + b0]) * hinv;
            v -= (Fz[l * fstride + c1] - Fz[l * fstride + c0]) * hinv;
            D[l] = v;
        }
        const int ci = cell_index(gnx, i + bw, j + bw, k + bw);
        double u[ZT_NF], X[3];
        load_cell(g, U, ci, u);
        cell_X(g, bt, b, i + bw, j + bw, k + bw, X);
        // Poisson frame: cell (i+1, j+1, k+1); fx(i) is the face below cell i
        const int pc = ((k + 1) * pnx + (j + 1)) * pnx + (i + 1);
        double gf[3];
        gf[0] = 0.5 * (st.fx[pb + pc] + st.fx[pb + pc + 1]);
        gf[1] = 0.5 * (st.fy[pb + pc] + st.fy[pb + pc + pnx]);
        gf[2] = 0.5 * (st.fz[pb + pc] + st.fz[pb + pc + pnx * pnx]);
        {  // State::gravity_source (state_ztwd.cpp:276-288), D read before the update
            const double dd = u[ZT_D];
            const double R = zt_R(X);
            const double s_sr = dd * (X[0] * gf[0] + X[1] * gf[1]) / R;
            const double s_lz = dd * (X[0] * gf[1] - X[1] * gf[0]);
            const double s_sz = dd * gf[2];
            double s_et = 0.0;
            s_et += D[ZT_POT];
            s_et -= D[ZT_D] * u[ZT_POT] / dd;
            const double dvx = -X[1] * (P.omega - P.omega0), dvy = X[0] * (P.omega - P.omega0);
            s_et += u[ZT_D] * (dvx * gf[0] + dvy * gf[1]);
            D[ZT_SR] += s_sr;
            D[ZT_LZ] += s_lz;
            D[ZT_SZ] += s_sz;
            D[ZT_ET] += s_et;
        }
        double du = 0.0;
        du += Vx[a1];
        du += Vy[b1];
        du += Vz[c1];
        du -= Vx[a0];
        du -= Vy[b0];
        du -= Vz[c0];
        du /= h;
        double p, cs;
        zt_fail(err, zt_eos(P, u, &p, &cs));
        D[ZT_TAU] += -p * du;  // State::internal_energy_source (state_ztwd.cpp:269-274)
        D[ZT_POT] = 0.0;
        D[ZT_T] = 0.0;
        zt_fail(err, zt_add_source(P, u, X, D));
#pragma unroll
        for (int l = 0; l < ZT_NF; l++) u[l] = (u[l] + D[l] * dt) * beta + U0[l * g.gnx3 + ci] * (1.0 - beta);
        zt_fail(err, zt_floor(P, u, X));
        store_cell(g, U, ci, u);
    }
}

// ---------------------------------------------------------------------------
// GridNode::inject_from_children (grid_node.cpp:1035-1074) with the ZTWD
// floor at the parent cell centre
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_zt_inject(Geom g, BrickTable bt, DevState st, ZtwdPar P,
                                                  const int* __restrict__ slots, int* err) {
    const int p = slots[blockIdx.x];
    const int c = blockIdx.y;
    const int ch = bt.child[8 * p + c];
    if (ch < 0) return;
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, half = nx / 2;
    const int t = threadIdx.x;
    if (t >= half * half * half) return;
    const int a = t % half, bb = (t / half) % half, cc = t / (half * half);
    const int i = bw + 2 * a, j = bw + 2 * bb, k = bw + 2 * cc;
    const int i0 = bw + a + (c & 1) * half, j0 = bw + bb + ((c >> 1) & 1) * half, k0 = bw + cc + ((c >> 2) & 1) * half;
    const double* C = st.U + (size_t)ch * g.ucount;
    double* Pp = st.U + (size_t)p * g.ucount;
    double u[ZT_NF];
#pragma unroll
    for (int l = 0; l < ZT_NF; l++) {
        const double* Cl = C + l * g.gnx3;
        double s = 0.0;
        s += Cl[cell_index(gnx, i + 0, j + 0, k + 0)];
        s += Cl[cell_index(gnx, i + 1, j + 0, k + 0)];
        s += Cl[cell_index(gnx, i + 0, j + 1, k + 0)];
        s += Cl[cell_index(gnx, i + 1, j + 1, k + 0)];
        s += Cl[cell_index(gnx, i + 0, j + 0, k + 1)];
        s += Cl[cell_index(gnx, i + 1, j + 0, k + 1)];
        s += Cl[cell_index(gnx, i + 0, j + 1, k + 1)];
        s += Cl[cell_index(gnx, i + 1, j + 1, k + 1)];
        u[l] = s * 0.125;
    }
    double X[3];
    cell_X(g, bt, p, i0, j0, k0, X);
    zt_fail(err, zt_floor(P, u, X));
    store_cell(g, Pp, cell_index(gnx, i0, j0, k0), u);
}

// ---------------------------------------------------------------------------
// GridNode::inject_from_parent (grid_node.cpp:193-233) for new bricks, ZTWD
// floor at each child cell centre
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_zt_prolong(Geom g, BrickTable bt, DevState st, ZtwdPar P,
                                                   const int* __restrict__ slots, int* err) {
    const int b = slots[blockIdx.x];
    const int p = bt.parent[b];
    const int c = bt.cidx[b];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, half = nx / 2;
    const int t = threadIdx.x;
    if (t >= half * half * half) return;
    const int a = t % half, bb = (t / half) % half, cc = t / (half * half);
    const int i = bw + 2 * a, j = bw + 2 * bb, k = bw + 2 * cc;
    const int i0 = bw + a + (c & 1) * half, j0 = bw + bb + ((c >> 1) & 1) * half, k0 = bw + cc + ((c >> 2) & 1) * half;
    const double* Pp = st.U + (size_t)p * g.ucount;
    double* C = st.U + (size_t)b * g.ucount;
    for (int o = 0; o < 8; o++) {
        double u[ZT_NF];
#pragma unroll
        for (int l = 0; l < ZT_NF; l++) {
            const double* Pl = Pp + l * g.gnx3;
            const double v = Pl[cell_index(gnx, i0, j0, k0)];
            const double s1 = minmod2(Pl[cell_index(gnx, i0 + 1, j0, k0)] - v, v - Pl[cell_index(gnx, i0 - 1, j0, k0)]);
            const double s2 = minmod2(Pl[cell_index(gnx, i0, j0 + 1, k0)] - v, v - Pl[cell_index(gnx, i0, j0 - 1, k0)]);
            const double s3 = minmod2(Pl[cell_index(gnx, i0, j0, k0 + 1)] - v, v - Pl[cell_index(gnx, i0, j0, k0 - 1)]);
            switch (o) {
                case 0: u[l] = v - (s1 + s2 + s3) * 0.25; break;
                case 1: u[l] = v + (s1 - s2 - s3) * 0.25; break;
                case 2: u[l] = v - (s1 - s2 + s3) * 0.25; break;
                case 3: u[l] = v + (s1 + s2 - s3) * 0.25; break;
                case 4: u[l] = v - (s1 + s2 - s3) * 0.25; break;
                case 5: u[l] = v + (s1 - s2 + s3) * 0.25; break;
                case 6: u[l] = v - (s1 - s2 - s3) * 0.25; break;
                default: u[l] = v + (s1 + s2 + s3) * 0.25; break;
            }
        }
        const int ii = i + (o & 1), jj = j + ((o >> 1) & 1), kk = k + ((o >> 2) & 1);
        double X[3];
        cell_X(g, bt, b, ii, jj, kk, X);
        zt_fail(err, zt_floor(P, u, X));
        store_cell(g, C, cell_index(gnx, ii, jj, kk), u);
    }
}

// ---------------------------------------------------------------------------
// potential <-> state (binary.cpp:825-936), interior cells in the Poisson
// frame (i = 1..PNX-2 <-> grid index i + BW - 1).  mode 0 pot_to_grid:
// pot = rho (phi - R^2 Omega0^2 / 2); 1 pot_from_grid: phi = pot / rho +
// R^2 Omega0^2 / 2; 2 add_pot_et: et += pot - phi rho / 2; 3 sub_pot_et.
// ---------------------------------------------------------------------------
__global__ void k_zt_pot(Geom g, BrickTable bt, DevState st, ZtwdPar P, const int* __restrict__ slots, int mode) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, pnx = g.pnx;
    double* U = st.U + (size_t)b * g.ucount;
    double* phi = st.phi + (size_t)b * g.pnx3;
    const double O = P.omega0;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int i0 = i + bw - 1, j0 = j + bw - 1, k0 = k + bw - 1;
        const int ci = cell_index(gnx, i0, j0, k0);
        const int pc = (k * pnx + j) * pnx + i;
        const double d = U[ZT_D * g.gnx3 + ci];
        if (mode == 0 || mode == 1) {
            double X[3];
            cell_X(g, bt, b, i0, j0, k0, X);
            const double R2 = X[0] * X[0] + X[1] * X[1];
            if (mode == 0)
                U[ZT_POT * g.gnx3 + ci] = d * (phi[pc] - 0.5 * R2 * O * O);
            else
                phi[pc] = (U[ZT_POT * g.gnx3 + ci] / d + 0.5 * R2 * O * O);
        } else {
            double e = U[ZT_ET * g.gnx3 + ci];
            if (mode == 2)
                e += U[ZT_POT * g.gnx3 + ci] - 0.5 * phi[pc] * d;
            else
                e -= U[ZT_POT * g.gnx3 + ci] - 0.5 * phi[pc] * d;
            U[ZT_ET * g.gnx3 + ci] = e;
        }
    }
}

}  // namespace

void launch_zt_ghost_fill(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                          const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_zt_ghost_fill, dim3(n, 6), 128, 0, s, g, bt, st, P, slots);
}
void launch_zt_flux(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                    int n, int* err, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_zt_prim, n, 256, 0, s, g, bt, st, P, slots);
    if (g.flux32)
        launch_k(k_zt_flux<float>, n, 128, 0, s, g, bt, st, P, slots, err);
    else
        launch_k(k_zt_flux<double>, n, 128, 0, s, g, bt, st, P, slots, err);
}
void launch_zt_max_dt(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                      int n, double* dt_out, int* err, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_zt_prim, n, 256, 0, s, g, bt, st, P, slots);
    launch_k(k_zt_max_dt, n, 128, 0, s, g, bt, st, P, slots, dt_out, err);
}
void launch_zt_add_difs(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                        const int* slots, int n, double dt, double beta, int* err, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_zt_add_difs, n, 128, 0, s, g, bt, st, P, slots, dt, beta, err);
}
void launch_zt_inject(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                      const int* slots, int n, int* err, cudaStream_t s) {
    if (n <= 0) return;
    const int half = g.nx / 2;
    launch_k(k_zt_inject, dim3(n, 8), ((half * half * half + 31) / 32) * 32, 0, s, g, bt, st, P, slots, err);
}
void launch_zt_prolong(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                       const int* slots, int n, int* err, cudaStream_t s) {
    if (n <= 0) return;
    const int half = g.nx / 2;
    launch_k(k_zt_prolong, n, ((half * half * half + 31) / 32) * 32, 0, s, g, bt, st, P, slots, err);
}
void launch_zt_pot(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                   int n, int mode, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_zt_pot, n, 256, 0, s, g, bt, st, P, slots, mode);
}

}  // namespace amr
