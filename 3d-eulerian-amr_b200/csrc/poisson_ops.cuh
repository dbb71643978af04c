// Per-brick bodies of the multigrid Poisson kernels (poisson/poisson.cpp and
// its ghost proxies poisson_amr_bound.cpp / poisson_phys_bound.cpp) as
// device functions, shared by the one-launch-per-step kernels
// (poisson_kernels.cu) and the persistent solve (persistent.cu), so both run
// the same arithmetic.  op_X(..., b, t0, nt): brick b, this thread's first
// work index t0 and the stride nt.
//
// Poisson arrays live on the PNX^3 frame of every brick (PNX = nx + 2: the
// interior plus one ghost layer); Poisson index p <-> grid index p + BW - 1.
#pragma once

#include "amr_internal.h"
#include "corr.cuh"
#include "euler_state.cuh"

namespace amr {

constexpr int MAX_NEST = 16;  // refinement levels 0..12 (amr_create rejects deeper trees)

__device__ __forceinline__ int pidx(int pnx, int i, int j, int k) { return (k * pnx + j) * pnx + i; }

// Grid::xf/yf/zf + h/2 (grid/grid.cpp:500-526) for grid index gi.
__device__ __forceinline__ double cell_centre(const Geom& g, int axis, int off, double h, int gi) {
    double f;
    if (axis < 2) {
        f = double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0 - g.origin[axis];
    } else if (g.z_reflect) {
        f = double(off + gi) * h - double(g.bw) * g.h0 - g.origin[2];
    } else {
        f = double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0;
    }
    return f + 0.5 * h;
}

// 1-D quadratic interpolation weights at +1/4 from the nodes -1, 0, +1;
// their tensor product is the 27-point table of poisson_amr_bound.cpp:23-29
// (every product is an exact dyadic double).
__device__ __forceinline__ double w27(int l) { return l == 0 ? -0.09375 : (l == 1 ? 0.9375 : 0.15625); }

// 4x4x4 restriction weights of poisson.cpp:12-15: 11 on the 2x2x2 core,
// -1 where exactly one index is outside the core, 0 elsewhere.
__device__ __forceinline__ double w64(int n, int o, int p) {
    const int out = (n == 0 || n == 3) + (o == 0 || o == 3) + (p == 0 || p == 3);
    return out == 0 ? 11.0 : (out == 1 ? -1.0 : 0.0);
}

// Array3d::divergence (array3d.h:139-150)
__device__ __forceinline__ double divergence(const double* a, int pnx, int i, int j, int k) {
    const int c = pidx(pnx, i, j, k);
    return (a[c + 1] + a[c - 1] + a[c + pnx] + a[c - pnx] + a[c + pnx * pnx] + a[c - pnx * pnx]) - (a[c] * 6.0);
}

// Array3d::oct_avg (array3d.h:151-161)
template <typename T>
__device__ __forceinline__ T oct_avg(const T* a, int pnx, int i, int j, int k) {
    const int c = pidx(pnx, i, j, k);
    const int s = pnx * pnx;
    return (a[c] + a[c + 1] + a[c + pnx] + a[c + pnx + 1] + a[c + s] + a[c + s + 1] + a[c + s + pnx] +
            a[c + s + pnx + 1]) *
           T(0.125);
}

// ---------------------------------------------------------------------------
// sources and domain boundary
// ---------------------------------------------------------------------------
// Poisson::set_source (poisson.cpp:950-966): S = 4 pi G rho over PNX^3.
__device__ __forceinline__ void op_set_source(const Geom& g, const DevState& st, int b, int t0, int nt) {
    const int pnx = g.pnx, gnx = g.gnx, off = g.bw - 1;
    const double* R = st.U + (size_t)b * g.ucount;
    double* S = st.S + (size_t)b * g.pnx3;
    for (int t = t0; t < g.pnx3; t += nt) {
        const int i = t % pnx, j = (t / pnx) % pnx, k = t / (pnx * pnx);
        const double rho = R[((k + off) * gnx + (j + off)) * gnx + (i + off)];
        S[t] = 4.0 * M_PI * g.grav_g * rho;
    }
}


// Domain-face potential, PoissonPhysBound::compute_boundaries
// (poisson_phys_bound.cpp:70-81) evaluating Single::compute_phi
// (single/single.cpp:219-243): the recursive sum over all bricks of
// -alpha m / r over their octant monopoles, with each brick's own sum formed
// first and the children's sums added after it in child order.  Two kernels:
// every (point, brick) own sum in parallel into a scratch matrix [brick][point],
// then one thread per point accumulates them with the nesting of the
// recursion (a stack of partial sums indexed by level).
__device__ __forceinline__ void bound_point(const Geom& g, const BrickTable& bt, const int* bfaces, int p, double* xyz,
                                            int* where) {
    const int pnx = g.pnx;
    const int fe = p / (pnx * pnx), pt = p % (pnx * pnx);
    const int b = bfaces[2 * fe], face = bfaces[2 * fe + 1];
    const int a = pt / pnx, cc = pt % pnx;  // table[a][cc]: lower, higher transverse
    const int ax = face >> 1;
    int pi[3];
    pi[ax] = (face & 1) ? pnx - 1 : 0;
    pi[ax == 0 ? 1 : 0] = a;
    pi[ax == 2 ? 1 : 2] = cc;
    const double h = bt.h[b];
    for (int d = 0; d < 3; d++) xyz[d] = cell_centre(g, d, bt.off[3 * b + d], h, pi[d] + g.bw - 1);
    if (where) *where = ((b * 6 + face) * pnx * pnx) + a * pnx + cc;
}

// Potential at point xyz of one brick's eight octant monopoles
// (PoissonPhysBound::compute_boundaries, poisson_phys_bound.cpp:70-81: a
// fully refined brick contributes 0).
__device__ __forceinline__ double own_term(const double* xyz, const double* __restrict__ m, bool ar,
                                           double alpha) {
    double sum = 0.0;
    for (int q = 0; q < 8; q++) {
        const double dx = xyz[0] - m[4 * q + 1], dy = xyz[1] - m[4 * q + 2], dz = xyz[2] - m[4 * q + 3];
        if (!ar) {
            sum -= alpha * m[4 * q + 0] / sqrt(dx * dx + dy * dy + dz * dz);
        } else {
            sum = 0.0;
        }
    }
    return sum;
}

// Nested sum of the reference's recursion: a brick's value is its own term
// plus its children's subtree values, added child by child in DFS order.
// acc[l] holds the running value of the open brick at level l.
struct NestStack {
    double acc[MAX_NEST];
    int depth = -1;
    __device__ __forceinline__ void push(int L, double v) {
        while (depth >= L) {
            acc[depth - 1] += acc[depth];
            depth--;
        }
        acc[L] = v;
        depth = L;
    }
    __device__ __forceinline__ double close(int L0) {
        while (depth > L0) {
            acc[depth - 1] += acc[depth];
            depth--;
        }
        return acc[L0];
    }
};



// ---------------------------------------------------------------------------
// ghost values seen through a brick face: PoissonInterface::get_phi /
// get_dphi of whatever sits there (a real brick, a PoissonAMRBound, a
// PoissonPhysBound).
// ---------------------------------------------------------------------------
struct PoissonAux {
    const double* bphi;  // [cap][6][pnx][pnx]
    int* err;            // set when a mirrored ghost is asked for an index the reference aborts on
};

// PoissonAMRBound::get_phi (poisson_amr_bound.cpp:39-109).
__device__ inline double amr_get_phi(const Geom& g, const BrickTable& bt, const DevState& st, int b, int face, int i, int j,
                              int k) {
    const int pnx = g.pnx;
    const int p0 = bt.fnbr[6 * b + face];  // parent
    const int ax = face >> 1;
    const int v = (face & 1) ? 1 : -1;
    int q[3] = {i, j, k}, par[3];
    for (int d = 0; d < 3; d++) {
        const int rel = bt.off[3 * b + d] + (d == ax ? v * (pnx - 2) : 0) - 2 * bt.off[3 * p0 + d] - (g.bw - 1);
        const int t = rel + q[d];
        par[d] = t % 2;
        q[d] = t / 2;
    }
    int P = p0;
    for (int d = 0; d < 3; d++) {
        if (q[d] > pnx - 2) {
            if (bt.ftype[6 * P + 2 * d + 1] != FACE_SIB) return 0.0;
            P = bt.fnbr[6 * P + 2 * d + 1];
            q[d] -= pnx - 2;
        } else if (q[d] < 1) {
            if (bt.ftype[6 * P + 2 * d] != FACE_SIB) return 0.0;
            P = bt.fnbr[6 * P + 2 * d];
            q[d] += pnx - 2;
        }
    }
    const double* phi = st.phi + (size_t)P * g.pnx3;
    double sum = 0.0;
    for (int l = 0; l < 3; l++)
        for (int n = 0; n < 3; n++)
            for (int m = 0; m < 3; m++) {
                const int i2 = q[0] + (l - 1) * (2 * par[0] - 1);
                const int j2 = q[1] + (n - 1) * (2 * par[1] - 1);
                const int k2 = q[2] + (m - 1) * (2 * par[2] - 1);
                sum += (w27(l) * w27(n) * w27(m)) * phi[pidx(pnx, i2, j2, k2)];
            }
    return sum;
}

__device__ inline double get_phi_from(const Geom& g, const BrickTable& bt, const DevState& st, const PoissonAux& aux, int b,
                               int face, int i, int j, int k) {
    const int pnx = g.pnx;
    const int kind = bt.ftype[6 * b + face];
    if (kind == FACE_SIB) return st.phi[(size_t)bt.fnbr[6 * b + face] * g.pnx3 + pidx(pnx, i, j, k)];
    if (kind == FACE_OUTFLOW) {
        // PoissonPhysBound::get_phi (poisson_phys_bound.cpp:86-98): the face
        // table indexed by the two transverse indices
        const int ax = face >> 1;
        const int a = ax == 0 ? j : i, c = ax == 2 ? j : k;
        return aux.bphi[((size_t)b * 6 + face) * pnx * pnx + a * pnx + c];
    }
    if (kind == FACE_REFLECT) {
        // mirrored plane z = 0 (poisson_phys_bound.cpp:99-126)
        const double* phi = st.phi + (size_t)b * g.pnx3;
        if (k == 1) return phi[pidx(pnx, i, j, pnx - 2)];
        if (k == pnx - 2) return phi[pidx(pnx, i, j, 1)];
        atomicExch(aux.err, 1);
        return 0.0;
    }
    return amr_get_phi(g, bt, st, b, face, i, j, k);
}

// get_dphi: neighbour copy; PoissonAMRBound::get_dphi (poisson_amr_bound.cpp
// :111-116) parent value without interpolation; 0 on a domain face; mirror.
template <typename CT>
__device__ CT get_dphi_from(const Geom& g, const BrickTable& bt, const DevState& st, const PoissonAux& aux, int b,
                            int face, int i, int j, int k) {
    const int pnx = g.pnx;
    const int kind = bt.ftype[6 * b + face];
    const int nbr = bt.fnbr[6 * b + face];
    const CT* D = Corr<CT>::dphi(st);
    if (kind == FACE_SIB) return D[(size_t)nbr * g.pnx3 + pidx(pnx, i, j, k)];
    if (kind == FACE_OUTFLOW) return CT(0);
    if (kind == FACE_REFLECT) {
        const CT* d = D + (size_t)b * g.pnx3;
        if (k == 1) return d[pidx(pnx, i, j, pnx - 2)];
        if (k == pnx - 2) return d[pidx(pnx, i, j, 1)];
        atomicExch(aux.err, 1);
        return CT(0);
    }
    const int ax = face >> 1;
    const int v = (face & 1) ? 1 : -1;
    const int q[3] = {i, j, k};
    int r[3];
    for (int d = 0; d < 3; d++) {
        const int rel = bt.off[3 * b + d] + (d == ax ? v * (pnx - 2) : 0) - 2 * bt.off[3 * nbr + d] - (g.bw - 1);
        r[d] = (rel + q[d]) / 2;
    }
    return D[(size_t)nbr * g.pnx3 + pidx(pnx, r[0], r[1], r[2])];
}

// ---------------------------------------------------------------------------
// ghost fills, Poisson::enforce_phi_boundaries (poisson.cpp:749-888) and
// enforce_dphi_boundaries (poisson.cpp:890-929), one level at a time.
// ---------------------------------------------------------------------------
// faces: phi(0,j,k) = sib(XL).get_phi(PNX-2,j,k), phi(PNX-1,j,k) =
// sib(XU).get_phi(1,j,k), ... over the transverse interior.
__device__ __forceinline__ void op_phi_faces(const Geom& g, const BrickTable& bt, const DevState& st,
                                             const PoissonAux& aux, int b, int face, int t0, int nt) {
    const int pnx = g.pnx, m = pnx - 2;
    const int ax = face >> 1;
    for (int t = t0; t < m * m; t += nt) {
        const int t1 = t % m + 1, t2 = t / m + 1;
        const int da = (face & 1) ? pnx - 1 : 0, sa = (face & 1) ? 1 : pnx - 2;  // ghost / source layer
        const int c0 = ax == 0 ? -1 : t1, c1 = ax == 1 ? -1 : (ax == 0 ? t1 : t2), c2 = ax == 2 ? -1 : t2;
        const double v = get_phi_from(g, bt, st, aux, b, face, c0 < 0 ? sa : c0, c1 < 0 ? sa : c1, c2 < 0 ? sa : c2);
        st.phi[(size_t)b * g.pnx3 + pidx(pnx, c0 < 0 ? da : c0, c1 < 0 ? da : c1, c2 < 0 ? da : c2)] = v;
    }
}

// the same face fill for the correction (enforce_dphi_boundaries)
template <typename CT>
__device__ __forceinline__ void op_dphi_faces(const Geom& g, const BrickTable& bt, const DevState& st,
                                              const PoissonAux& aux, int b, int face, int t0, int nt) {
    const int pnx = g.pnx, m = pnx - 2;
    const int ax = face >> 1;
    CT* D = Corr<CT>::dphi(st);
    for (int t = t0; t < m * m; t += nt) {
        const int t1 = t % m + 1, t2 = t / m + 1;
        const int da = (face & 1) ? pnx - 1 : 0, sa = (face & 1) ? 1 : pnx - 2;  // ghost / source layer
        const int c0 = ax == 0 ? -1 : t1, c1 = ax == 1 ? -1 : (ax == 0 ? t1 : t2), c2 = ax == 2 ? -1 : t2;
        const CT v = get_dphi_from<CT>(g, bt, st, aux, b, face, c0 < 0 ? sa : c0, c1 < 0 ? sa : c1, c2 < 0 ? sa : c2);
        D[(size_t)b * g.pnx3 + pidx(pnx, c0 < 0 ? da : c0, c1 < 0 ? da : c1, c2 < 0 ? da : c2)] = v;
    }
}

// edges: Poisson::enforce_phi_boundaries_edge (poisson.cpp:788-842).
// edge e (0..11) at position k = 1 .. PNX-2 along it; the source face is
// the x face pair when one of them is physical, else the y or z face, as in
// the reference.  Edges read face ghosts only (this level's faces are
// complete), so all edge cells are independent.
__device__ __forceinline__ void op_phi_edge(const Geom& g, const BrickTable& bt, const DevState& st,
                                            const PoissonAux& aux, int b, int e, int k) {
    const int pnx = g.pnx, N = pnx - 1, M = pnx - 2;
    auto phys = [&](int f) { const int t = bt.ftype[6 * b + f]; return t == FACE_OUTFLOW || t == FACE_REFLECT; };
    int f, i, j, kk, di, dj, dk;  // source face and cell; destination cell
    if (e < 8) {
        const int x = e < 4 ? 0 : N, r = e & 3;
        di = x;
        dj = r == 0 ? 0 : (r == 1 ? N : k);
        dk = r < 2 ? k : (r == 2 ? 0 : N);
        if (phys(XL) || phys(XU)) {
            f = e < 4 ? XL : XU;
            i = e < 4 ? M : 1;
            j = dj;
            kk = dk;
        } else if (r < 2) {
            f = r == 0 ? YL : YU;
            i = x;
            j = r == 0 ? M : 1;
            kk = k;
        } else {
            f = r == 2 ? ZL : ZU;
            i = x;
            j = k;
            kk = r == 2 ? M : 1;
        }
    } else {
        const int r = e - 8;
        di = k;
        dj = (r >> 1) ? N : 0;
        dk = (r & 1) ? N : 0;
        if (phys(YL) || phys(YU)) {
            f = r < 2 ? YL : YU;
            i = k;
            j = r < 2 ? M : 1;
            kk = dk;
        } else {
            f = (r & 1) ? ZU : ZL;
            i = k;
            j = dj;
            kk = (r & 1) ? 1 : M;
        }
    }
    st.phi[(size_t)b * g.pnx3 + pidx(pnx, di, dj, dk)] = get_phi_from(g, bt, st, aux, b, f, i, j, kk);
}

// vertices: Poisson::enforce_phi_boundaries_vertex (poisson.cpp:844-888).
// vertex c = x | y<<1 | z<<2; the source face is an x face when one of them
// is physical, else a y face when one of them is, else a z face.
__device__ __forceinline__ void op_phi_vertex(const Geom& g, const BrickTable& bt, const DevState& st,
                                              const PoissonAux& aux, int b, int c) {
    const int pnx = g.pnx, N = pnx - 1, M = pnx - 2;
    auto phys = [&](int f) { const int t = bt.ftype[6 * b + f]; return t == FACE_OUTFLOW || t == FACE_REFLECT; };
    const int x = c & 1, y = (c >> 1) & 1, z = (c >> 2) & 1;
    int f, i = x * N, j = y * N, k = z * N;
    if (phys(XL) || phys(XU)) {
        f = x ? XU : XL;
        i = x ? 1 : M;
    } else if (phys(YL) || phys(YU)) {
        f = y ? YU : YL;
        j = y ? 1 : M;
    } else {
        f = z ? ZU : ZL;
        k = z ? 1 : M;
    }
    st.phi[(size_t)b * g.pnx3 + pidx(pnx, x * N, y * N, z * N)] = get_phi_from(g, bt, st, aux, b, f, i, j, k);
}

// ---------------------------------------------------------------------------
// V-cycle pieces
// ---------------------------------------------------------------------------
// Poisson::phi_from_children (poisson.cpp:707-747): covered coarse phi :=
// 64-point weighted child stencil / 64.  grid = (parents, 8 children).
// parent p, child octant c, t < (nx/2)^3: one coarse cell
__device__ __forceinline__ void op_phi_from_children(const Geom& g, const BrickTable& bt, const DevState& st, int p,
                                                     int c, int t) {
    const int ch = bt.child[8 * p + c];
    if (ch < 0) return;
    const int pnx = g.pnx, half = (pnx - 2) / 2;
    if (t >= half * half * half) return;
    const int a = t % half, bb = (t / half) % half, cc = t / (half * half);
    const int i = 2 * a + 1, j = 2 * bb + 1, k = 2 * cc + 1;
    const int i0 = a + 1 + (c & 1) * half, j0 = bb + 1 + ((c >> 1) & 1) * half, k0 = cc + 1 + ((c >> 2) & 1) * half;
    const double* C = st.phi + (size_t)ch * g.pnx3;
    double sum = 0.0;
    for (int n = -1; n < 3; n++)
        for (int o = -1; o < 3; o++)
            for (int q = -1; q < 3; q++) sum += w64(n + 1, o + 1, q + 1) * C[pidx(pnx, i + q, j + o, k + n)];
    st.phi[(size_t)p * g.pnx3 + pidx(pnx, i0, j0, k0)] = sum / 64.0;
}

// Poisson::init_vcycle (poisson.cpp:931-948)
template <typename CT>
__device__ __forceinline__ void op_init_vcycle(const Geom& g, const DevState& st, int b, int t0, int nt) {
    const size_t base = (size_t)b * g.pnx3;
    CT* D = Corr<CT>::dphi(st);
    CT* D1 = Corr<CT>::dphi1(st);
    for (int t = t0; t < g.pnx3; t += nt) {
        D[base + t] = CT(0);
        D1[base + t] = CT(0);
    }
}

// Poisson::vcycle_down (poisson.cpp:989-1046) for one brick per block:
//  (a) residual/6 from phi and S on uncovered cells, child averages of dphi
//      and dphi1 on covered ones (poisson.cpp:989-1017);
//  (b) adjust_x_dphi, adjust_y_dphi, adjust_z_dphi (poisson.cpp:249-443):
//      on uncovered cells next to a face refined on one side, the coarse
//      minus the averaged fine potential difference /6 is added / subtracted;
//      this brick's items, x then y then z (an item touches only cells of
//      its coarse brick, so bricks are independent);
//  (c) dphi1 = dphi on uncovered cells (poisson.cpp:1021-1040).
// The residual and the corrections are formed in FP64 from phi; they are
// stored in the correction type CT.  ranges[4 q .. 4 q + 3] = first x, y, z
// item and end of the brick at list position q.
// Called by every thread of the block (block barriers inside); rg = the
// brick's four item offsets.
template <typename CT>
__device__ __forceinline__ void op_vdown(const Geom& g, const BrickTable& bt, const DevState& st, int b,
                                         const RefluxItem* __restrict__ items, const int* rg) {
    const int pnx = g.pnx, nx = pnx - 2, half = nx / 2;
    const double h = bt.h[b];
    const double h2 = h * h;
    const size_t base = (size_t)b * g.pnx3;
    CT* D = Corr<CT>::dphi(st);
    CT* D1 = Corr<CT>::dphi1(st);
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int oc = ((i - 1) / half) | (((j - 1) / half) << 1) | (((k - 1) / half) << 2);
        const int ch = bt.child[8 * b + oc];
        const int c = pidx(pnx, i, j, k);
        if (ch < 0) {
            D[base + c] = CT((divergence(st.phi + base, pnx, i, j, k) - h2 * st.S[base + c]) * (1.0 / 6.0));
        } else {
            const int ci = 2 * (i - (oc & 1) * half) - 1;
            const int cj = 2 * (j - ((oc >> 1) & 1) * half) - 1;
            const int ck = 2 * (k - ((oc >> 2) & 1) * half) - 1;
            const size_t cb = (size_t)ch * g.pnx3;
            D1[base + c] = oct_avg(D1 + cb, pnx, ci, cj, ck);
            D[base + c] = oct_avg(D + cb, pnx, ci, cj, ck);
        }
    }
    const int hh = half * half;
    auto refined = [&](int cell) {
        const int ci = cell % pnx, cj = (cell / pnx) % pnx, ck = cell / (pnx * pnx);
        const int oc = (2 * ci / pnx) | ((2 * cj / pnx) << 1) | ((2 * ck / pnx) << 2);
        return bt.child[8 * b + oc] >= 0;
    };
    for (int d = 0; d < 3; d++) {
        __syncthreads();
        const int i_beg = rg[d], i_end = rg[d + 1];
        for (int q = threadIdx.x; q < (i_end - i_beg) * hh; q += blockDim.x) {
            const RefluxItem it = items[i_beg + q / hh];
            const int a = (q % hh) % half, cc = (q % hh) / half;
            const int j = 2 * a + 1, k = 2 * cc + 1;                          // child transverse
            const int j0 = a + 1 + it.cj * half, k0 = cc + 1 + it.ck * half;  // coarse transverse
            const int i = it.ic - g.bw + 1, i0 = it.i0 - g.bw + 1;            // PNX frame
            auto at = [&](int nrm, int t1, int t2) {
                int qq[3];
                qq[d] = nrm;
                qq[d == 0 ? 1 : 0] = t1;
                qq[d == 2 ? 1 : 2] = t2;
                return pidx(pnx, qq[0], qq[1], qq[2]);
            };
            const double* C = st.phi + (size_t)it.child * g.pnx3;
            const double* P = st.phi + base;
            double v = +C[at(i, j, k)] - C[at(i - 1, j, k)];
            v += C[at(i, j + 1, k)] - C[at(i - 1, j + 1, k)];
            v += C[at(i, j, k + 1)] - C[at(i - 1, j, k + 1)];
            v += C[at(i, j + 1, k + 1)] - C[at(i - 1, j + 1, k + 1)];
            v *= 0.5;
            const double dd = (P[at(i0, j0, k0)] - P[at(i0 - 1, j0, k0)] - v) * (1.0 / 6.0);
            const int c1 = at(i0, j0, k0), c0 = at(i0 - 1, j0, k0);
            if (!refined(c1)) D[base + c1] = CT(double(D[base + c1]) + dd);
            if (!refined(c0)) D[base + c0] = CT(double(D[base + c0]) - dd);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int oc = ((i - 1) / half) | (((j - 1) / half) << 1) | (((k - 1) / half) << 2);
        if (bt.child[8 * b + oc] < 0) D1[base + pidx(pnx, i, j, k)] = D[base + pidx(pnx, i, j, k)];
    }
}


// Poisson::vcycle_coarse_correction (poisson.cpp:17-51): child dphi +=
// parent dphi - mean of the child's 2x2x2 group.
// t < (nx/2)^3: one 2x2x2 child group
template <typename CT>
__device__ __forceinline__ void op_coarse_correction(const Geom& g, const BrickTable& bt, const DevState& st, int b,
                                                     int t) {
    const int p = bt.parent[b];
    if (p < 0) return;
    const int c = bt.cidx[b];
    const int pnx = g.pnx, half = (pnx - 2) / 2;
    if (t >= half * half * half) return;
    const int a = t % half, bb = (t / half) % half, cc = t / (half * half);
    const int i = 2 * a + 1, j = 2 * bb + 1, k = 2 * cc + 1;
    const int i0 = a + 1 + (c & 1) * half, j0 = bb + 1 + ((c >> 1) & 1) * half, k0 = cc + 1 + ((c >> 2) & 1) * half;
    CT* D = Corr<CT>::dphi(st) + (size_t)b * g.pnx3;
    const CT av = Corr<CT>::dphi(st)[(size_t)p * g.pnx3 + pidx(pnx, i0, j0, k0)] - oct_avg(D, pnx, i, j, k);
    for (int o = 0; o < 8; o++) D[pidx(pnx, i + (o & 1), j + ((o >> 1) & 1), k + ((o >> 2) & 1))] += av;
}

// Poisson::vcycle_retire_dphi (poisson.cpp:1048-1067): phi += dphi, in FP64.
template <typename CT>
__device__ __forceinline__ void op_retire(const Geom& g, const DevState& st, int b, int t0, int nt) {
    const int pnx = g.pnx, nx = pnx - 2;
    const size_t base = (size_t)b * g.pnx3;
    const CT* D = Corr<CT>::dphi(st);
    for (int t = t0; t < nx * nx * nx; t += nt) {
        const int c = pidx(pnx, t % nx + 1, (t / nx) % nx + 1, t / (nx * nx) + 1);
        st.phi[base + c] += double(D[base + c]);
    }
}

// Poisson::compute_forces (poisson.cpp:223-247): face forces -grad phi for
// faces 1..PNX-1 on rows 1..PNX-1.
__device__ __forceinline__ void op_forces(const Geom& g, const BrickTable& bt, const DevState& st, int b, int t0,
                                          int nt) {
    const int pnx = g.pnx, m = pnx - 1;
    const double h = bt.h[b];
    const size_t base = (size_t)b * g.pnx3;
    const double* phi = st.phi + base;
    for (int t = t0; t < m * m * m; t += nt) {
        const int i = t % m + 1, j = (t / m) % m + 1, k = t / (m * m) + 1;
        const int c = pidx(pnx, i, j, k);
        st.fx[base + c] = -(phi[c] - phi[c - 1]) / h;
        st.fy[base + c] = -(phi[c] - phi[c - pnx]) / h;
        st.fz[base + c] = -(phi[c] - phi[c - pnx * pnx]) / h;
    }
}

// Poisson::adjust_{x,y,z}_force (poisson.cpp:445-635): coarse face force :=
// mean of the child's four face forces.
// t < (nx/2)^2: one coarse face of the item's quadrant
__device__ __forceinline__ void op_adjust_force(const Geom& g, const DevState& st, const RefluxItem& it, int t) {
    const int pnx = g.pnx, half = (pnx - 2) / 2;
    if (t >= half * half) return;
    const int a = t % half, cc = t / half;
    const int j = 2 * a + 1, k = 2 * cc + 1;
    const int j0 = a + 1 + it.cj * half, k0 = cc + 1 + it.ck * half;
    const int i = it.ic - g.bw + 1, i0 = it.i0 - g.bw + 1;
    const int d = it.dir;
    auto at = [&](int nrm, int t1, int t2) {
        int q[3];
        q[d] = nrm;
        q[d == 0 ? 1 : 0] = t1;
        q[d == 2 ? 1 : 2] = t2;
        return pidx(pnx, q[0], q[1], q[2]);
    };
    double* f = d == 0 ? st.fx : (d == 1 ? st.fy : st.fz);
    const double* C = f + (size_t)it.child * g.pnx3;
    double v = +C[at(i, j, k)];
    v += C[at(i, j + 1, k)];
    v += C[at(i, j, k + 1)];
    v += C[at(i, j + 1, k + 1)];
    f[(size_t)it.coarse * g.pnx3 + at(i0, j0, k0)] = v * 0.25;
}

// Poisson::solution_error (poisson.cpp:637-669): dphi := div f - S on
// uncovered cells (0 on covered), per-brick sum of |dphi| h^3.
// Called by every thread of the block; the first nt threads (a multiple of
// 32) take part, and the brick's sum is formed in their order whatever the
// block size; red = blockDim.x / 32 doubles of shared memory.
template <typename CT>
__device__ __forceinline__ void op_solution_error(const Geom& g, const BrickTable& bt, const DevState& st, int b,
                                                  double* __restrict__ out, double* red, int nt) {
    CT* D = Corr<CT>::dphi(st);
    const int pnx = g.pnx, nx = pnx - 2, half = nx / 2;
    const double h = bt.h[b];
    const double h3 = h * h * h, hinv = 1.0 / h;
    const size_t base = (size_t)b * g.pnx3;
    double sum = 0.0;
    for (int t = threadIdx.x; t < nx * nx * nx && (int)threadIdx.x < nt; t += nt) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int c = pidx(pnx, i, j, k);
        const int oc = ((i - 1) / half) | (((j - 1) / half) << 1) | (((k - 1) / half) << 2);
        if (bt.child[8 * b + oc] < 0) {
            double df = -(st.fx[base + c + 1] - st.fx[base + c]) * hinv;
            df -= (st.fy[base + c + pnx] - st.fy[base + c]) * hinv;
            df -= (st.fz[base + c + pnx * pnx] - st.fz[base + c]) * hinv;
            const double r = df - st.S[base + c];
            D[base + c] = CT(r);
            sum += fabs(r) * h3;
        } else {
            D[base + c] = CT(0);
        }
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nt / 32; w++) s += red[w];
        out[b] = s;
    }
}

}  // namespace amr
