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


// Six conserved fields of one cell, indexed only by compile-time constants
// (stays in registers).
struct Cell6 {
    double v[NF_EULER];
};

// State::enforce_outflow (euler/state.cpp:45-84) on a register cell, the
// same arithmetic as st_enforce_outflow without a run-time array index.
__device__ __forceinline__ void fused_outflow(Cell6& u, int bface) {
    const int m = 1 + (bface >> 1);
    const double um = m == 1 ? u.v[1] : (m == 2 ? u.v[2] : u.v[3]);
    bool zero;
    if (bface == ZU || bface == ZL) {
        zero = (bface == ZU) ? (u.v[3] > 0.0) : (u.v[3] < 0.0);
    } else {
        const double v = um / u.v[0];
        zero = (bface & 1) ? (v > 0.0) : (v < 0.0);
    }
    if (zero) {
        u.v[4] = u.v[4] - 0.5 * um * um / u.v[0];
        if (m == 1) u.v[1] = 0.0;
        else if (m == 2) u.v[2] = 0.0;
        else u.v[3] = 0.0;
    }
}

__device__ __forceinline__ int axis_of(int x, int y, int z, int a) { return a == 0 ? x : (a == 1 ? y : z); }

__device__ __forceinline__ void fused_load(const FusedArgs& A, int b, int x, int y, int z, Cell6& u) {
    const double* U = A.Uin + (size_t)b * A.g.ucount + cell_index(A.g.gnx, x, y, z);
#pragma unroll
    for (int l = 0; l < NF_EULER; l++) u.v[l] = U[(size_t)l * A.g.gnx3];
}

// Cell (x, y, z) (GNX frame) of brick b: the interior value, or the
// face-ghost value k_ghost_fill would store there (at most one coordinate
// outside the interior).  DEPTH bounds the coarse-fine hops: a coarse-fine
// ghost reads the parent's cells, whose ghosts across the same face are
// same-level or domain ghosts under proper nesting, so DEPTH = 1 suffices;
// a deeper chain sets err bit 1.
template <int DEPTH>
__device__ __forceinline__ void fused_cell(const FusedArgs& A, int b, int x, int y, int z, Cell6& u) {
    const int bw = 2, gnx = 12;
    const int ax = (x < bw || x >= gnx - bw) ? 0 : ((y < bw || y >= gnx - bw) ? 1 : ((z < bw || z >= gnx - bw) ? 2 : -1));
    if (ax < 0) {
        fused_load(A, b, x, y, z, u);
        return;
    }
    const int gi = axis_of(x, y, z, ax);
    const int upper = gi >= gnx - bw ? 1 : 0;
    const int face = 2 * ax + upper;
    const int kind = A.bt.ftype[6 * b + face];
    const int nbr = A.bt.fnbr[6 * b + face];
    int sx = x, sy = y, sz = z, src = b;
    int s;
    if (kind == FACE_SIB) {
        s = upper ? gi - (gnx - 2 * bw) : gi + (gnx - 2 * bw);
        src = nbr;
    } else if (kind == FACE_OUTFLOW) {
        s = upper ? gnx - bw - 1 : bw;
    } else if (kind == FACE_REFLECT) {
        s = 2 * bw - 1 - gi;
    } else {
        s = -1;
    }
    if (s >= 0) {
        if (ax == 0) sx = s;
        else if (ax == 1) sy = s;
        else sz = s;
        fused_load(A, src, sx, sy, sz, u);
        if (kind == FACE_OUTFLOW) fused_outflow(u, face ^ 1);
        if (kind == FACE_REFLECT) u.v[3] = -u.v[3];
        return;
    }
    if constexpr (DEPTH == 0) {
        atomicOr(A.err, 2);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) u.v[l] = 0.0;
    } else {
        // GridAMRBound::operator() (grid_amr_bound.cpp:27-78)
        const int fx = A.bt.off[3 * b + 0] - 2 * A.bt.off[3 * nbr + 0] + x;
        const int fy = A.bt.off[3 * b + 1] - 2 * A.bt.off[3 * nbr + 1] + y;
        const int fz = A.bt.off[3 * b + 2] - 2 * A.bt.off[3 * nbr + 2] + z;
        const int px = fx / 2, py = fy / 2, pz = fz / 2;
        const int par = axis_of(fx, fy, fz, ax) % 2;
        const int dx = ax == 0, dy = ax == 1, dz = ax == 2;
        Cell6 uc, up, um;
        fused_cell<DEPTH - 1>(A, nbr, px, py, pz, uc);
        fused_cell<DEPTH - 1>(A, nbr, px + dx, py + dy, pz + dz, up);
        fused_cell<DEPTH - 1>(A, nbr, px - dx, py - dy, pz - dz, um);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            double m = minmod2(up.v[l] - uc.v[l], uc.v[l] - um.v[l]);
            if (par == 1) m = -m;
            u.v[l] = uc.v[l] - m * 0.25;
        }
    }
}

__device__ __forceinline__ void fused_wait(const FusedArgs& A, int child) {
    unsigned long long spins = 0;
    while (*(volatile const int*)(A.done + child) != A.epoch) {
        if (++spins > A.wait_limit) {
            atomicOr(A.err, 1);
            break;
        }
        __nanosleep(64);
    }
    __threadfence();
}

// Block layout: 512 threads; per brick the "cross" -- the 8^3 interior and
// the six 2-deep ghost slabs the dimension-split stencil reads -- is held in
// shared memory as primitives (FT), and one direction's 9 x 64 face fluxes
// (FP64) at a time.
constexpr int FUSED_BLOCK = 256;  // two cells per thread in the per-cell phases
constexpr int CROSS = 512 + 6 * 2 * 64;  // interior + ghost slabs
constexpr int FACES = 9 * 64;            // faces of one direction

// cross index of the cell at position n (0..11) along direction d of pencil
// (t1, t2): interior (z*8 + y)*8 + x, or slab ((face*2 + depth)*8 + t2)*8 + t1
__device__ __forceinline__ int cross_index(int d, int n, int t1, int t2) {
    if (n < 2) return 512 + (((2 * d) * 2 + n) * 8 + t2) * 8 + t1;
    if (n >= 10) return 512 + (((2 * d + 1) * 2 + (n - 10)) * 8 + t2) * 8 + t1;
    const int i = n - 2;
    const int x = d == 0 ? i : t1, y = d == 1 ? i : (d == 0 ? t1 : t2), z = d == 2 ? i : t2;
    return (z * 8 + y) * 8 + x;
}

template <typename FT>
__device__ __forceinline__ void fused_brick(const FusedArgs& A, int b, int vr, FT* P, double* Fs) {
    const Geom& g = A.g;
    const int nx = 8, gnx = 12, bw = 2, npen = 64, half = 4;
    const int tid = threadIdx.x;
    // (a) the cross as primitives: interior cells, then ghost cells resolved
    //     as the level-ordered ghost fill would have set them
    for (int q = tid; q < CROSS; q += FUSED_BLOCK) {
        Cell6 u;
        if (q < 512) {
            fused_load(A, b, q % 8 + bw, (q / 8) % 8 + bw, q / 64 + bw, u);
        } else {
            const int r = q - 512, t1 = r % 8 + bw, t2 = (r / 8) % 8 + bw, depth = (r / 64) % 2, face = r / 128;
            const int ax = face >> 1;
            const int n = (face & 1) ? gnx - bw + depth : depth;
            if (ax == 0)
                fused_cell<1>(A, b, n, t1, t2, u);
            else if (ax == 1)
                fused_cell<1>(A, b, t1, n, t2, u);
            else
                fused_cell<1>(A, b, t1, t2, n, u);
        }
        FT w[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) w[l] = (FT)u.v[l];
        st_to_prim(w);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) P[l * CROSS + q] = w[l];
    }
    __syncthreads();
    const double hinv = 1.0 / A.bt.h[b];
    const FT th = (FT)g.theta, gam = (FT)g.gamma;
    const unsigned char pm = A.pubmask[b];
    double* pubb = A.pub + (size_t)b * 6 * NF_EULER * npen;
    const int* rg = vr >= 0 ? A.vranges + 4 * vr : nullptr;
    double D[2][NF_EULER];  // this thread's cells tid, tid + 256: flux differences, x then y then z
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) D[h][l] = 0.0;
    // unrolled: the direction is a compile-time constant in each copy, so the
    // state arrays indexed by it (normal velocity, normal momentum flux) stay
    // in registers
#pragma unroll
    for (int d = 0; d < 3; d++) {
        // (b) face fluxes of direction d, one thread per face
        for (int q = tid; q < FACES; q += FUSED_BLOCK) {
            const int p = q % npen, fi = q / npen;
            const int t1 = p % nx, t2 = p / nx;
            FT w[4][NF_EULER];  // cells f-2 .. f+1 (f = fi + bw)
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int ci = cross_index(d, fi + m, t1, t2);
#pragma unroll
                for (int l = 0; l < NF_EULER; l++) w[m][l] = P[l * CROSS + ci];
            }
            FT ql[NF_EULER], qr[NF_EULER];
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) {
                const FT sL = minmod_theta(w[2][l] - w[1][l], w[1][l] - w[0][l], th);  // slope of cell f-1
                const FT sR = minmod_theta(w[3][l] - w[2][l], w[2][l] - w[1][l], th);  // slope of cell f
                ql[l] = w[1][l] + sL / FT(2);
                qr[l] = w[2][l] - sR / FT(2);
            }
            st_to_con(ql);
            st_to_con(qr);
            FT fl[NF_EULER], fr[NF_EULER];
            const FT al = st_flux(ql, d, gam, fl);
            const FT ar = st_flux(qr, d, gam, fr);
            const FT a = r_max(al, ar);
            double F[NF_EULER];
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) F[l] = (double)(((fl[l] + fr[l]) - (qr[l] - ql[l]) * a) * FT(0.5));
            // coarse-fine correction: mean of the child's four faces
            if (rg) {
                for (int it_q = rg[d]; it_q < rg[d + 1]; it_q++) {
                    const RefluxItem it = A.vitems[it_q];
                    const int aa = t1 - it.cj * half, cc = t2 - it.ck * half;
                    if (it.i0 - bw != fi || aa < 0 || aa >= half || cc < 0 || cc >= half) continue;
                    fused_wait(A, it.child);
                    const int side = it.ic == bw ? 0 : 1;
                    const double* Fc = A.pub + ((size_t)it.child * 6 + 2 * d + side) * NF_EULER * npen;
                    const int j = 2 * aa, k = 2 * cc;
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
#pragma unroll
            for (int l = 0; l < NF_EULER; l++) Fs[l * FACES + q] = F[l];
        }
        __syncthreads();
        // (c) this thread's cell: D -= (F(i+1) - F(i)) / h along d
        {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int cc = tid + h * FUSED_BLOCK;
                const int x = cc % 8, y = (cc / 8) % 8, z = cc / 64;
                const int i = d == 0 ? x : (d == 1 ? y : z);
                const int p = d == 0 ? z * 8 + y : (d == 1 ? z * 8 + x : y * 8 + x);
#pragma unroll
                for (int l = 0; l < NF_EULER; l++)
                    D[h][l] -= (Fs[l * FACES + (i + 1) * npen + p] - Fs[l * FACES + i * npen + p]) * hinv;
            }
        }
        __syncthreads();
    }
    // faces published: stamp the brick done for the coarser bricks
    __threadfence();
    __syncthreads();
    if (tid == 0 && pm) atomicExch(A.done + b, A.epoch);
    // (d) Grid::add_difs (grid.cpp:406-420) for this thread's cells
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int cc = tid + h * FUSED_BLOCK;
        const int x = cc % 8, y = (cc / 8) % 8, z = cc / 64;
        const int ci = cell_index(gnx, x + bw, y + bw, z + bw);
        const double* U = A.Uin + (size_t)b * g.ucount;
        const double* U0 = A.U0 + (size_t)b * g.ucount;
        double* Uo = A.Uout + (size_t)b * g.ucount;
        double u[NF_EULER];
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            const double Dl = D[h][l] + 0.0;  // State::source() is zero for the Euler state
            u[l] = (U[(size_t)l * g.gnx3 + ci] + Dl * A.dt) * A.beta + U0[(size_t)l * g.gnx3 + ci] * (1.0 - A.beta);
        }
        st_floor(u, g.gamma, g.rho_floor, g.ei_floor);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) Uo[(size_t)l * g.gnx3 + ci] = u[l];
    }
}

template <typename FT>
__global__ void __launch_bounds__(FUSED_BLOCK, 2) k_substep_fused(FusedArgs A) {
    extern __shared__ double smem[];  // [nf][CROSS] primitives (FT), then [nf][FACES] fluxes (FP64)
    FT* P = reinterpret_cast<FT*>(smem);
    double* Fs = smem + (NF_EULER * CROSS * sizeof(FT) + sizeof(double) - 1) / sizeof(double);
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(A.next, 1u);
        __syncthreads();
        const int w = s_item;
        if (w >= A.nwork) break;
        fused_brick<FT>(A, A.work[w].x, A.work[w].y, P, Fs);
        __syncthreads();
    }
}

template <typename FT>
constexpr size_t fused_smem_bytes() {
    return ((NF_EULER * CROSS * sizeof(FT) + sizeof(double) - 1) / sizeof(double)) * sizeof(double) +
           sizeof(double) * NF_EULER * FACES;
}

}  // namespace amr
