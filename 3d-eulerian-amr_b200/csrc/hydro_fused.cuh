// One hydro substep of every brick in one persistent launch: ghost zones,
// minmod-theta reconstruction, KT flux, coarse-fine flux correction, flux
// differences and the RK combination with floor, fused per brick.
//
// The reference runs this as level-ordered ghost fills
// (GridNode::enforce_boundaries, grid_node.cpp:59-112), Grid::compute_*_flux
// (grid.cpp:215-302) and the coarse-fine corrections (grid_node.cpp:1076-1274),
// then Grid::add_difs (grid.cpp:304-420).  Here each block takes bricks from
// a device work list, finest level first:
//  * ghost cells are not stored: a pencil's two ghost cells at each end are
//    computed where they are needed, from the neighbour's interior, the
//    parent's cells with the minmod slope (a parent ghost cell resolved the
//    same way), or the brick's own cells at a domain face -- the values the
//    level-ordered ghost fill would have written;
//  * a brick whose faces a coarser brick corrects publishes those face fluxes
//    and stamps itself done; the coarse brick waits (bounded) for the stamp
//    and replaces its own face flux by the mean of the four child faces;
//  * the updated state goes to a second state array, so no block reads a
//    brick another block is writing.
// The arithmetic of every value is that of the one-launch-per-step kernels,
// so with FT = double the result is bitwise that of amr_sub_step.
#pragma once

#include "euler_state.cuh"
#include "flux_kernel.cuh"
#include "hydro_fused.h"

namespace amr {

constexpr int FUSED_THREADS = 192;  // 3 directions x 64 pencils
constexpr unsigned long long FUSED_WAIT_SPINS = 1ull << 24;

__device__ __forceinline__ void fused_load(const FusedArgs& A, int b, const int* c, double* u) {
    const double* U = A.Uin + (size_t)b * A.g.ucount + cell_index(A.g.gnx, c[0], c[1], c[2]);
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) u[l] = U[(size_t)l * A.g.gnx3];
}

// Cell c (GNX frame) of brick b: the interior value, or the face-ghost value
// k_ghost_fill would store there (at most one coordinate outside the
// interior).  DEPTH bounds the coarse-fine hops.
template <int DEPTH>
__device__ bool fused_cell(const FusedArgs& A, int b, const int* c, double* u) {
    const Geom& g = A.g;
    const int bw = g.bw, gnx = g.gnx;
    int ax = -1, upper = 0;
    for (int d = 0; d < 3; d++) {
        if (c[d] < bw) ax = d, upper = 0;
        else if (c[d] >= gnx - bw) ax = d, upper = 1;
    }
    if (ax < 0) {
        fused_load(A, b, c, u);
        return true;
    }
    const int face = 2 * ax + upper;
    const int kind = A.bt.ftype[6 * b + face];
    const int nbr = A.bt.fnbr[6 * b + face];
    const int gi = c[ax];
    int s[3] = {c[0], c[1], c[2]};
    if (kind == FACE_SIB) {
        s[ax] = upper ? gi - (gnx - 2 * bw) : gi + (gnx - 2 * bw);
        fused_load(A, nbr, s, u);
        return true;
    }
    if (kind == FACE_OUTFLOW) {
        s[ax] = upper ? gnx - bw - 1 : bw;
        fused_load(A, b, s, u);
        st_enforce_outflow(u, face ^ 1);
        return true;
    }
    if (kind == FACE_REFLECT) {
        s[ax] = 2 * bw - 1 - gi;
        fused_load(A, b, s, u);
        u[3] = -u[3];
        return true;
    }
    if constexpr (DEPTH == 0) {
        atomicOr(A.err, 2);
        for (int l = 0; l < NF_EULER; l++) u[l] = 0.0;
        return false;
    } else {
        // GridAMRBound::operator() (grid_amr_bound.cpp:27-78)
        int pi[3], par = 0;
        for (int d = 0; d < 3; d++) {
            const int fine = A.bt.off[3 * b + d] - 2 * A.bt.off[3 * nbr + d] + c[d];
            pi[d] = fine / 2;
            if (d == ax) par = fine % 2;
        }
        int pp[3] = {pi[0], pi[1], pi[2]}, pm[3] = {pi[0], pi[1], pi[2]};
        pp[ax] += 1;
        pm[ax] -= 1;
        double uc[NF_EULER], up[NF_EULER], um[NF_EULER];
        bool ok = fused_cell<DEPTH - 1>(A, nbr, pi, uc);
        ok &= fused_cell<DEPTH - 1>(A, nbr, pp, up);
        ok &= fused_cell<DEPTH - 1>(A, nbr, pm, um);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            double m = minmod2(up[l] - uc[l], uc[l] - um[l]);
            if (par == 1) m = -m;
            u[l] = uc[l] - m * 0.25;
        }
        return ok;
    }
}

__device__ __forceinline__ void fused_wait(const FusedArgs& A, int child) {
    unsigned long long spins = 0;
    while (*(volatile const int*)(A.done + child) != A.epoch) {
        if (++spins > FUSED_WAIT_SPINS) {
            atomicOr(A.err, 1);
            break;
        }
        __nanosleep(64);
    }
    __threadfence();
}

// Phase 1 of brick b for pencil thread t < 192: the pencil's nine face
// fluxes in FT (stored in FP64), the coarse-fine replacements, the brick's
// published faces, and the pencil's flux differences into T[d][l][cell].
template <typename FT>
__device__ __forceinline__ void fused_pencil(const FusedArgs& A, int b, int vr, double* T) {
    const Geom& g = A.g;
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, npen = nx * nx, half = nx / 2;
    const int d = threadIdx.x / npen;
    const int p = threadIdx.x % npen;
    const int t1 = p % nx, t2 = p / nx;
    const double hinv = 1.0 / A.bt.h[b];
    const FT th = (FT)g.theta, gam = (FT)g.gamma;
    // coarse-fine faces of this pencil (at most one per child boundary)
    int ov_fi[3], ov_child[3], ov_side[3], ov_a[3], ov_c[3], nov = 0;
    if (vr >= 0) {
        const int* rg = A.vranges + 4 * vr;
        for (int q = rg[d]; q < rg[d + 1] && nov < 3; q++) {
            const RefluxItem it = A.vitems[q];
            const int a = t1 - it.cj * half, c = t2 - it.ck * half;
            if (a < 0 || a >= half || c < 0 || c >= half) continue;
            ov_fi[nov] = it.i0 - bw;
            ov_child[nov] = it.child;
            ov_side[nov] = it.ic == bw ? 0 : 1;
            ov_a[nov] = a;
            ov_c[nov] = c;
            nov++;
        }
    }
    int cell[3];
    cell[d == 0 ? 1 : 0] = t1 + bw;
    cell[d == 2 ? 1 : 2] = t2 + bw;
    auto load = [&](int n, FT* w) {
        double u[NF_EULER];
        cell[d] = n;
        if (n >= bw && n < gnx - bw)
            fused_load(A, b, cell, u);
        else
            fused_cell<3>(A, b, cell, u);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) w[l] = (FT)u[l];
        st_to_prim(w);
    };
    FT w[4][NF_EULER];
    for (int n = 0; n < 3; n++) load(n, w[n + 1]);
    FT sR[NF_EULER];
    for (int n = 3; n < bw + 1; n++) {
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) w[m][l] = w[m + 1][l];
        load(n, w[3]);
    }
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) sR[l] = minmod_theta(w[3][l] - w[2][l], w[2][l] - w[1][l], th);
    const unsigned char pm = A.pubmask[b];
    double* pubb = A.pub + (size_t)b * 6 * NF_EULER * npen;
    double Fprev[NF_EULER];
    for (int f = bw; f <= gnx - bw; f++) {
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) w[m][l] = w[m + 1][l];
        load(f + 1, w[3]);
        FT ql[NF_EULER], qr[NF_EULER], sL[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            sL[l] = sR[l];
            sR[l] = minmod_theta(w[3][l] - w[2][l], w[2][l] - w[1][l], th);
            ql[l] = w[1][l] + sL[l] / FT(2);
            qr[l] = w[2][l] - sR[l] / FT(2);
        }
        st_to_con(ql);
        st_to_con(qr);
        FT fl[NF_EULER], fr[NF_EULER];
        const FT al = st_flux(ql, d, gam, fl);
        const FT ar = st_flux(qr, d, gam, fr);
        const FT a = r_max(al, ar);
        const int fi = f - bw;
        double F[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) F[l] = (double)(((fl[l] + fr[l]) - (qr[l] - ql[l]) * a) * FT(0.5));
        // coarse-fine correction: mean of the child's four faces
        for (int o = 0; o < nov; o++) {
            if (ov_fi[o] != fi) continue;
            fused_wait(A, ov_child[o]);
            const double* Fc = A.pub + ((size_t)ov_child[o] * 6 + 2 * d + ov_side[o]) * NF_EULER * npen;
            const int j = 2 * ov_a[o], k = 2 * ov_c[o];
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) {
                const double* C = Fc + l * npen;
                double v = +__ldcg(C + k * nx + j);
                v += __ldcg(C + k * nx + j + 1);
                v += __ldcg(C + (k + 1) * nx + j);
                v += __ldcg(C + (k + 1) * nx + j + 1);
                F[l] = v * 0.25;
            }
        }
        if (fi == 0 && (pm & (1u << (2 * d))))
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) pubb[(2 * d * NF_EULER + l) * npen + p] = F[l];
        if (fi == nx && (pm & (1u << (2 * d + 1))))
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) pubb[((2 * d + 1) * NF_EULER + l) * npen + p] = F[l];
        if (b == A.root) {
            double* Fr = (d == 0 ? A.Fx : (d == 1 ? A.Fy : A.Fz)) + (size_t)b * g.nf * npen * (nx + 1);
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) Fr[l * npen * (nx + 1) + flux_index(d, nx, fi, t1, t2)] = F[l];
        }
        if (fi > 0) {
            // cell fi-1 along the pencil: (F(fi) - F(fi-1)) / h
            const int i = fi - 1;
            const int x = d == 0 ? i : t1, y = d == 1 ? i : (d == 0 ? t1 : t2), z = d == 2 ? i : t2;
            const int cc = (z * nx + y) * nx + x;
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) T[(d * NF_EULER + l) * nx * nx * nx + cc] = (F[l] - Fprev[l]) * hinv;
        }
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) Fprev[l] = F[l];
    }
}

template <typename FT>
__global__ void __launch_bounds__(FUSED_THREADS) k_substep_fused(FusedArgs A) {
    extern __shared__ double T[];  // [3][nf][nx^3] flux differences
    __shared__ int s_item;
    const Geom& g = A.g;
    const int nx = g.nx, bw = g.bw, gnx = g.gnx;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(A.next, 1u);
        __syncthreads();
        const int w = s_item;
        if (w >= A.nwork) break;
        const int b = A.work[w].x, vr = A.work[w].y;
        fused_pencil<FT>(A, b, vr, T);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0 && A.pubmask[b]) atomicExch(A.done + b, A.epoch);
        // Grid::add_difs (grid.cpp:406-420) with the x, y, z differences
        const double dt = A.dt, beta = A.beta;
        const double* U = A.Uin + (size_t)b * g.ucount;
        const double* U0 = A.U0 + (size_t)b * g.ucount;
        double* Uo = A.Uout + (size_t)b * g.ucount;
        for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
            const int i = t % nx, j = (t / nx) % nx, k = t / (nx * nx);
            const int ci = cell_index(gnx, i + bw, j + bw, k + bw);
            double u[NF_EULER];
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) {
                double D = 0.0;
                D -= T[(0 * NF_EULER + l) * nx * nx * nx + t];
                D -= T[(1 * NF_EULER + l) * nx * nx * nx + t];
                D -= T[(2 * NF_EULER + l) * nx * nx * nx + t];
                D += 0.0;  // State::source() is zero for the Euler state
                u[l] = (U[(size_t)l * g.gnx3 + ci] + D * dt) * beta + U0[(size_t)l * g.gnx3 + ci] * (1.0 - beta);
            }
            st_floor(u, g.gamma, g.rho_floor, g.ei_floor);
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) Uo[(size_t)l * g.gnx3 + ci] = u[l];
        }
        __syncthreads();
    }
}

}  // namespace amr
