// Hydro kernels, plain FP64 form.  One CUDA block per brick (or per brick
// face / correction item); bricks of any level run in one launch wherever
// the reference's recursion order does not create a dependency.
//
// Layouts (see amr_internal.h):
//   U  [slot][f][k][j][i], GNX^3 per field, ghosts included
//   Fx [slot][f][k'][j'][i'] faces i'=0..nx (grid face bw+i'), j',k' interior
//   Fy [slot][f][k'][j'][i'] faces j'=0..nx
//   Fz [slot][f][k'][j'][i'] faces k'=0..nx
#include "euler_state.cuh"
#include "flux_kernel.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace amr {

// ---------------------------------------------------------------------------
// ghost zones: GridNode::enforce_boundaries (grid_node.cpp:59-112) with the
// three kinds of face source (same level, GridAMRBound, GridPhysBound).
// grid = (bricks of one level, 6 faces); thread per ghost cell of the face
// slab (bw x nx x nx, transverse interior only; edges/corners untouched).
// ---------------------------------------------------------------------------
__global__ void k_ghost_fill(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    const int b = slots[blockIdx.x];
    const int face = blockIdx.y;
    const int ax = face >> 1, upper = face & 1;
    const int bw = g.bw, gnx = g.gnx, nx = g.nx;
    const int kind = bt.ftype[6 * b + face];
    const int nbr = bt.fnbr[6 * b + face];
    double* U = st.U + (size_t)b * g.ucount;
    for (int t = threadIdx.x; t < bw * nx * nx; t += blockDim.x) {
        const int n = t % bw;             // depth into the ghost layer
        const int t1 = (t / bw) % nx + bw;  // lower transverse axis
        const int t2 = (t / bw) / nx + bw;  // higher transverse axis
        const int gi = upper ? gnx - bw + n : n;  // ghost index along ax
        int c[3];
        c[ax] = gi;
        c[ax == 0 ? 1 : 0] = t1;
        c[ax == 2 ? 1 : 2] = t2;
        const int dst = cell_index(gnx, c[0], c[1], c[2]);
        double u[NF_EULER];
        if (kind == FACE_SIB) {
            // (*sib)(GNX-2bw+i, j, k) for the lower face, (i-GNX+2bw) upper.
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = upper ? gi - (gnx - 2 * bw) : gi + (gnx - 2 * bw);
            const double* V = st.U + (size_t)nbr * g.ucount;
            const int src = cell_index(gnx, s[0], s[1], s[2]);
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) u[l] = V[l * g.gnx3 + src];
        } else if (kind == FACE_OUTFLOW) {
            // GridPhysBound map (grid_phys_bound.cpp:60-169): copy the first
            // interior cell, then enforce_outflow with the proxy's face.
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = upper ? gnx - bw - 1 : bw;
            const int src = cell_index(gnx, s[0], s[1], s[2]);
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) u[l] = U[l * g.gnx3 + src];
            st_enforce_outflow(u, face ^ 1);
        } else if (kind == FACE_REFLECT) {
            // Z_REFLECT at z=0: ghost k <- cell 2*bw-1-k, sz -> -sz
            // (grid_phys_bound.cpp:140-155, State::reflect_on_z).
            int s[3] = {c[0], c[1], c[2]};
            s[ax] = 2 * bw - 1 - gi;
            const int src = cell_index(gnx, s[0], s[1], s[2]);
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) u[l] = U[l * g.gnx3 + src];
            u[3] = -u[3];
        } else {
            // GridAMRBound::operator() (grid_amr_bound.cpp:27-78): parent cell
            // at half the fine index, minus a quarter of the face-normal
            // minmod slope, sign by the fine cell's parity.
            const double* P = st.U + (size_t)nbr * g.ucount;
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
            for (int l = 0; l < NF_EULER; l++) {
                const double uc = P[l * g.gnx3 + i0];
                double m = minmod2(P[l * g.gnx3 + ip] - uc, uc - P[l * g.gnx3 + im]);
                if (par == 1) m = -m;
                u[l] = uc - m * 0.25;
            }
        }
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) U[l * g.gnx3 + dst] = u[l];
    }
}

// ---------------------------------------------------------------------------
// KT/Rusanov fluxes, Grid::compute_{x,y,z}_flux (grid.cpp:215-302) with
// minmod-theta (reconstruct.cpp:60-71) or PPM (reconstruct.cpp:22-58)
// reconstruction.  Block = one brick, 3*nx*nx threads: thread = (direction,
// pencil).  A pencil walks its GNX cells streaming the reconstruction.
// ---------------------------------------------------------------------------
template <int R>
__global__ void k_flux(Geom g, DevState st, const int* __restrict__ slots) {
    flux_pencils<double, R>(g, st, slots[blockIdx.x]);
}

// ---------------------------------------------------------------------------
// Coarse-fine flux correction, GridNode::adjust_{x,y,z}_flux
// (grid_node.cpp:1076-1274): the coarse face quadrant takes the mean of the
// child's four faces.  One block per item, thread per (field, face cell).
// Items of one coarse level run after every finer level is final.
// ---------------------------------------------------------------------------
__global__ void k_reflux(Geom g, DevState st, const RefluxItem* __restrict__ items) {
    const RefluxItem it = items[blockIdx.x];
    const int nx = g.nx, bw = g.bw, gnx = g.gnx;
    const int half = nx / 2;
    const int t = threadIdx.x;
    if (t >= g.nf * half * half) return;
    const int l = t / (half * half);
    const int q = t % (half * half);
    const int a = q % half, c = q / half;      // by2 indexer: j = bw+2a, k = bw+2c
    const int j = 2 * a, k = 2 * c;            // child interior offsets
    const int j0 = a + it.cj * half, k0 = c + it.ck * half;  // coarse interior offsets
    const int npen = nx * nx, fstride = npen * (nx + 1);
    double* Fbase = (it.dir == 0 ? st.Fx : (it.dir == 1 ? st.Fy : st.Fz));
    const double* Fc = Fbase + (size_t)it.child * g.nf * fstride + l * fstride;
    double* Fp = Fbase + (size_t)it.coarse * g.nf * fstride + l * fstride;
    const int ic = it.ic - bw, i0 = it.i0 - bw;
    double v = +Fc[flux_index(it.dir, nx, ic, j, k)];
    v += Fc[flux_index(it.dir, nx, ic, j + 1, k)];
    v += Fc[flux_index(it.dir, nx, ic, j, k + 1)];
    v += Fc[flux_index(it.dir, nx, ic, j + 1, k + 1)];
    v *= 0.25;
    Fp[flux_index(it.dir, nx, i0, j0, k0)] = v;
    (void)gnx;
}

// ---------------------------------------------------------------------------
// Flux differences + RK combine + floor: clear_difs, sum_{x,y,z}_difs and
// Grid::add_difs (grid.cpp:201-213, 304-344, 406-420).  With gravity the
// ZSTAR energy work term and the momentum sources of the restated coupling
// (single/single.cpp:49-97, 304-383) are added in the reference order.
// Block = one brick, thread per interior cell.
// ---------------------------------------------------------------------------
__global__ void k_add_difs(Geom g, DevState st, const int* __restrict__ slots, const double* __restrict__ hs,
                           double dt_arg, const double* __restrict__ dtp, double beta, int gravity) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, pnx = g.pnx;
    const int npen = nx * nx, fstride = npen * (nx + 1);
    const double dt = dtp ? *dtp : dt_arg;  // device-computed step in captured graphs
    const double h = hs[b];
    const double hinv = 1.0 / h;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx, j = (t / nx) % nx, k = t / npen;
        double D[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) D[l] = 0.0;
        const double* Fx = st.Fx + (size_t)b * g.nf * fstride;
        const double* Fy = st.Fy + (size_t)b * g.nf * fstride;
        const double* Fz = st.Fz + (size_t)b * g.nf * fstride;
        // Poisson frame: pi = i + 1 (grid index i+bw == pi + BW - 1)
        const size_t pb = (size_t)b * g.pnx3;
        const int pc = ((k + 1) * pnx + (j + 1)) * pnx + (i + 1);
        const int a0 = flux_index(0, nx, i, j, k), a1 = flux_index(0, nx, i + 1, j, k);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) D[l] -= (Fx[l * fstride + a1] - Fx[l * fstride + a0]) * hinv;
        if (gravity) {
            D[4] += 0.5 * st.fx[pb + pc] * (Fx[a0]);
            D[4] += 0.5 * st.fx[pb + pc + 1] * (Fx[a1]);
        }
        const int b0 = flux_index(1, nx, j, i, k), b1 = flux_index(1, nx, j + 1, i, k);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) D[l] -= (Fy[l * fstride + b1] - Fy[l * fstride + b0]) * hinv;
        if (gravity) {
            D[4] += 0.5 * st.fy[pb + pc] * (Fy[b0]);
            D[4] += 0.5 * st.fy[pb + pc + pnx] * (Fy[b1]);
        }
        const int c0 = flux_index(2, nx, k, i, j), c1 = flux_index(2, nx, k + 1, i, j);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) D[l] -= (Fz[l * fstride + c1] - Fz[l * fstride + c0]) * hinv;
        if (gravity) {
            D[4] += 0.5 * st.fz[pb + pc] * (Fz[c0]);
            D[4] += 0.5 * st.fz[pb + pc + pnx * pnx] * (Fz[c1]);
        }
        const int ci = cell_index(gnx, i + bw, j + bw, k + bw);
        double* U = st.U + (size_t)b * g.ucount;
        const double* U0 = st.U0 + (size_t)b * g.ucount;
        double u[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) u[l] = U[l * g.gnx3 + ci];
        if (gravity) {
            const double fx0 = 0.5 * u[0] * (st.fx[pb + pc] + st.fx[pb + pc + 1]);
            const double fy0 = 0.5 * u[0] * (st.fy[pb + pc] + st.fy[pb + pc + pnx]);
            const double fz0 = 0.5 * u[0] * (st.fz[pb + pc] + st.fz[pb + pc + pnx * pnx]);
            D[3] += fz0;
            D[1] += fx0;
            D[2] += fy0;
        }
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            D[l] += 0.0;  // State::source() is zero for the Euler state
            u[l] = (u[l] + D[l] * dt) * beta + U0[l * g.gnx3 + ci] * (1.0 - beta);
        }
        st_floor(u, g.gamma, g.rho_floor, g.ei_floor);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) U[l * g.gnx3 + ci] = u[l];
    }
}

// Root flow-off: Grid::sum_{x,y,z}_flow_off (grid.cpp:346-404) in the
// sequential order of a one-thread OpenMP run, then FO update of
// Grid::add_difs (grid.cpp:419).  fo = [FO(nf), FO0(nf)].  One thread/field.
__global__ void k_flow_off(Geom g, DevState st, int root, double h, double dt_arg, const double* __restrict__ dtp,
                           double beta, double* fo) {
    const int l = threadIdx.x;
    const double dt = dtp ? *dtp : dt_arg;
    if (l >= g.nf) return;
    const int nx = g.nx, npen = nx * nx, fstride = npen * (nx + 1);
    const double* Fx = st.Fx + (size_t)root * g.nf * fstride + l * fstride;
    const double* Fy = st.Fy + (size_t)root * g.nf * fstride + l * fstride;
    const double* Fz = st.Fz + (size_t)root * g.nf * fstride + l * fstride;
    double dfo = 0.0;
    for (int t2 = 0; t2 < nx; t2++)
        for (int t1 = 0; t1 < nx; t1++)
            dfo += (Fx[flux_index(0, nx, nx, t1, t2)] - Fx[flux_index(0, nx, 0, t1, t2)]) * h * h;
    for (int t2 = 0; t2 < nx; t2++)
        for (int t1 = 0; t1 < nx; t1++)
            dfo += (Fy[flux_index(1, nx, nx, t1, t2)] - Fy[flux_index(1, nx, 0, t1, t2)]) * h * h;
    for (int t2 = 0; t2 < nx; t2++)
        for (int t1 = 0; t1 < nx; t1++) {
            if (g.z_reflect)
                dfo += (Fz[flux_index(2, nx, nx, t1, t2)]) * h * h;
            else
                dfo += (Fz[flux_index(2, nx, nx, t1, t2)] - Fz[flux_index(2, nx, 0, t1, t2)]) * h * h;
        }
    fo[l] = (fo[l] + dfo * dt) * beta + fo[g.nf + l] * (1.0 - beta);
}

// ---------------------------------------------------------------------------
// Restriction, GridNode::inject_from_children (grid_node.cpp:1035-1074):
// covered parent cell := mean of its 8 child cells, then floor.
// grid = (parents of one level, 8 children); thread per parent cell.
// ---------------------------------------------------------------------------
__global__ void k_inject(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
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
    double* P = st.U + (size_t)p * g.ucount;
    double u[NF_EULER];
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) {
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
    st_floor(u, g.gamma, g.rho_floor, g.ei_floor);
    const int dst = cell_index(gnx, i0, j0, k0);
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) P[l * g.gnx3 + dst] = u[l];
}

// ---------------------------------------------------------------------------
// Prolongation of new bricks, GridNode::inject_from_parent
// (grid_node.cpp:193-233): parent cell +- a quarter of the three minmod
// slopes, then floor.  Thread per parent cell of the child's octant.
// ---------------------------------------------------------------------------
__global__ void k_prolong(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    const int b = slots[blockIdx.x];
    const int p = bt.parent[b];
    const int c = bt.cidx[b];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, half = nx / 2;
    const int t = threadIdx.x;
    if (t >= half * half * half) return;
    const int a = t % half, bb = (t / half) % half, cc = t / (half * half);
    const int i = bw + 2 * a, j = bw + 2 * bb, k = bw + 2 * cc;
    const int i0 = bw + a + (c & 1) * half, j0 = bw + bb + ((c >> 1) & 1) * half, k0 = bw + cc + ((c >> 2) & 1) * half;
    const double* P = st.U + (size_t)p * g.ucount;
    double* C = st.U + (size_t)b * g.ucount;
    double out[8][NF_EULER];
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) {
        const double* Pl = P + l * g.gnx3;
        const double u = Pl[cell_index(gnx, i0, j0, k0)];
        const double s1 = minmod2(Pl[cell_index(gnx, i0 + 1, j0, k0)] - u, u - Pl[cell_index(gnx, i0 - 1, j0, k0)]);
        const double s2 = minmod2(Pl[cell_index(gnx, i0, j0 + 1, k0)] - u, u - Pl[cell_index(gnx, i0, j0 - 1, k0)]);
        const double s3 = minmod2(Pl[cell_index(gnx, i0, j0, k0 + 1)] - u, u - Pl[cell_index(gnx, i0, j0, k0 - 1)]);
        out[0][l] = u - (s1 + s2 + s3) * 0.25;
        out[1][l] = u + (s1 - s2 - s3) * 0.25;
        out[2][l] = u - (s1 - s2 + s3) * 0.25;
        out[3][l] = u + (s1 + s2 - s3) * 0.25;
        out[4][l] = u - (s1 + s2 - s3) * 0.25;
        out[5][l] = u + (s1 - s2 + s3) * 0.25;
        out[6][l] = u - (s1 - s2 - s3) * 0.25;
        out[7][l] = u + (s1 + s2 + s3) * 0.25;
    }
#pragma unroll
    for (int o = 0; o < 8; o++) {
        st_floor(out[o], g.gamma, g.rho_floor, g.ei_floor);
        const int dst = cell_index(gnx, i + (o & 1), j + ((o >> 1) & 1), k + ((o >> 2) & 1));
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) C[l * g.gnx3 + dst] = out[o][l];
    }
}

// ---------------------------------------------------------------------------
// CFL time step, Grid::max_dt (grid.cpp:422-483): largest face eigenvalue of
// the reconstructed states over all three directions; per-brick dt out.
// ---------------------------------------------------------------------------
template <int R>
__global__ void k_max_dt(Geom g, DevState st, const int* __restrict__ slots, const double* __restrict__ hs,
                         double* __restrict__ dt_out) {
    const int b = slots[blockIdx.x];
    const int npen = g.nx * g.nx;
    __shared__ double red[32];
    double lam = 0.0;
    for (int t = threadIdx.x; t < 3 * npen; t += blockDim.x) {
        const int d = t / npen, p = t % npen;
        if (d == 0)
            lam = max_eigen_pencil<0, R>(g, st, b, p, lam);
        else if (d == 1)
            lam = max_eigen_pencil<1, R>(g, st, b, p, lam);
        else
            lam = max_eigen_pencil<2, R>(g, st, b, p, lam);
    }
    // block max (max is exact, order-free)
    for (int o = 16; o > 0; o >>= 1) lam = r_max(lam, __shfl_xor_sync(0xffffffffu, lam, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lam;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) m = r_max(m, red[w]);
        double dtinv = m / hs[b];
        if (dtinv == 0.0) dtinv = 1.0E-10;
        double dt = 1.0 / dtinv;
        dt *= g.cfl;
        dt_out[b] = dt;
    }
}

// ---------------------------------------------------------------------------
// Density test of GridNode::set_refine_flags (grid_node.cpp:649-671):
// flag octant c when an interior cell of it has rho > threshold.
// ---------------------------------------------------------------------------
__global__ void k_refine_flags(Geom g, DevState st, const int* __restrict__ slots, double thr,
                               unsigned char* __restrict__ flags) {
    const int b = slots[blockIdx.x];
    __shared__ int f8[8];
    if (threadIdx.x < 8) f8[threadIdx.x] = 0;
    __syncthreads();
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const double* R = st.U + (size_t)b * g.ucount;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + bw, j = (t / nx) % nx + bw, k = t / (nx * nx) + bw;
        if (R[cell_index(gnx, i, j, k)] > thr) {
            const int c = (2 * i / gnx) | ((2 * j / gnx) << 1) | ((2 * k / gnx) << 2);
            f8[c] = 1;
        }
    }
    __syncthreads();
    if (threadIdx.x < 8) flags[8 * blockIdx.x + threadIdx.x] = (unsigned char)f8[threadIdx.x];
}

// Per-brick max of one field over uncovered interior cells
// (GridNode::state_max, grid_node.cpp:1529-1558).
__global__ void k_state_max(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots, int field,
                            double* __restrict__ out) {
    const int b = slots[blockIdx.x];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const double* R = st.U + (size_t)b * g.ucount + field * g.gnx3;
    __shared__ double red[32];
    double m = -1.0E+99;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + bw, j = (t / nx) % nx + bw, k = t / (nx * nx) + bw;
        const int c = (2 * i / gnx) | ((2 * j / gnx) << 1) | ((2 * k / gnx) << 2);
        if (bt.child[8 * b + c] < 0) m = r_max(R[cell_index(gnx, i, j, k)], m);
    }
    for (int o = 16; o > 0; o >>= 1) m = r_max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = -1.0E+99;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) r = r_max(red[w], r);
        out[blockIdx.x] = r;
    }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
void launch_ghost_fill(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                       cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_ghost_fill, dim3(n, 6), 128, 0, s, g, bt, st, slots);
}
void launch_flux(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (g.flux32) {
        launch_flux_f32(g, st, slots, n, s);
        return;
    }
    if (g.recon == RECON_PPM)
        launch_k(k_flux<RECON_PPM>, n, 3 * g.nx * g.nx, 0, s, g, st, slots);
    else
        launch_k(k_flux<RECON_MINMOD>, n, 3 * g.nx * g.nx, 0, s, g, st, slots);
}
void launch_reflux(const Geom& g, const DevState& st, const RefluxItem* items, int n, cudaStream_t s) {
    if (n <= 0) return;
    const int half = g.nx / 2;
    launch_k(k_reflux, n, ((g.nf * half * half + 31) / 32) * 32, 0, s, g, st, items);
}
void launch_add_difs(const Geom& g, const DevState& st, const int* slots, int n, const double* hs, double dt,
                     double beta, int gravity, cudaStream_t s, const double* dtp) {
    if (n <= 0) return;
    launch_k(k_add_difs, n, 256, 0, s, g, st, slots, hs, dt, dtp, beta, gravity);
}
void launch_flow_off(const Geom& g, const DevState& st, int root, double h, double dt, double beta, double* fo,
                     cudaStream_t s, const double* dtp) {
    launch_k(k_flow_off, 1, 32, 0, s, g, st, root, h, dt, dtp, beta, fo);
}
void launch_inject(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                   cudaStream_t s) {
    if (n <= 0) return;
    const int half = g.nx / 2;
    launch_k(k_inject, dim3(n, 8), ((half * half * half + 31) / 32) * 32, 0, s, g, bt, st, slots);
}
void launch_prolong(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                    cudaStream_t s) {
    if (n <= 0) return;
    const int half = g.nx / 2;
    launch_k(k_prolong, n, ((half * half * half + 31) / 32) * 32, 0, s, g, bt, st, slots);
}
void launch_max_dt(const Geom& g, const DevState& st, const int* slots, int n, const double* hs, double* dt_out,
                   cudaStream_t s) {
    if (n <= 0) return;
    if (g.recon == RECON_PPM)
        launch_k(k_max_dt<RECON_PPM>, n, 192, 0, s, g, st, slots, hs, dt_out);
    else
        launch_k(k_max_dt<RECON_MINMOD>, n, 192, 0, s, g, st, slots, hs, dt_out);
}
void launch_refine_flags(const Geom& g, const DevState& st, const int* slots, int n, double thr,
                         unsigned char* flags, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_refine_flags, n, 256, 0, s, g, st, slots, thr, flags);
}
void launch_state_max(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n, int field,
                      double* out, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_state_max, n, 256, 0, s, g, bt, st, slots, field, out);
}

}  // namespace amr

namespace amr {
// Host transfer helpers: pack the listed bricks into / out of a contiguous
// staging buffer (count doubles per brick).
__global__ void k_gather(const double* __restrict__ src, const int* __restrict__ slots, int count,
                         double* __restrict__ dst) {
    const int e = blockIdx.y;
    const double* s = src + (size_t)slots[e] * count;
    double* d = dst + (size_t)e * count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) d[t] = s[t];
}
__global__ void k_scatter(const double* __restrict__ src, const int* __restrict__ slots, int count,
                          double* __restrict__ dst) {
    const int e = blockIdx.y;
    const double* s = src + (size_t)e * count;
    double* d = dst + (size_t)slots[e] * count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) d[t] = s[t];
}
void launch_gather(const double* src, const int* slots, int n, int count, double* dst, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_gather, dim3((count + 255) / 256, n), 256, 0, s, src, slots, count, dst);
}
void launch_scatter(const double* src, const int* slots, int n, int count, double* dst, cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_scatter, dim3((count + 255) / 256, n), 256, 0, s, src, slots, count, dst);
}
}  // namespace amr
