// Multigrid Poisson kernels (poisson/poisson.cpp and its ghost proxies
// poisson_amr_bound.cpp / poisson_phys_bound.cpp): one launch per level or
// brick set; the per-brick bodies are in poisson_ops.cuh.
#include "context.h"
#include "poisson.h"
#include "poisson_ops.cuh"
#include "relax_brick.cuh"
#include "launch.cuh"

namespace amr {
// Octant monopoles of every brick (single/single.cpp:245-288, identical to
// binary/binary.cpp:977-1019): per octant without a child, sums of S h^3 and
// S x h^3 ... in the reference's cell order (k, j, i).  msrc[e][c] =
// {src_0, src_x, src_y, src_z} for DFS entry e.
__global__ void k_source_sums(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots,
                              double* __restrict__ msrc, int* __restrict__ allref) {
    const int e = blockIdx.x;
    const int b = slots[e];
    const int c = threadIdx.x;  // octant
    const int pnx = g.pnx, half = (pnx - 2) / 2;
    const double h = bt.h[b];
    const double h3 = h * h * h;
    __shared__ int uncovered;
    if (c == 0) uncovered = 0;
    __syncthreads();
    double s0 = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    if (c < 8 && bt.child[8 * b + c] < 0) {
        atomicOr(&uncovered, 1);
        const double* S = st.S + (size_t)b * g.pnx3;
        const int ox = (c & 1) * half, oy = ((c >> 1) & 1) * half, oz = ((c >> 2) & 1) * half;
        for (int k = 1 + oz; k <= half + oz; k++)
            for (int j = 1 + oy; j <= half + oy; j++)
                for (int i = 1 + ox; i <= half + ox; i++) {
                    const double s = S[pidx(pnx, i, j, k)];
                    s0 += s * h3;
                    sx += s * cell_centre(g, 0, bt.off[3 * b + 0], h, i + g.bw - 1) * h3;
                    sy += s * cell_centre(g, 1, bt.off[3 * b + 1], h, j + g.bw - 1) * h3;
                    sz += s * cell_centre(g, 2, bt.off[3 * b + 2], h, k + g.bw - 1) * h3;
                }
    }
    __syncthreads();
    if (c < 8) {
        const bool all_refined = uncovered == 0;
        double* m = msrc + ((size_t)e * 8 + c) * 4;
        if (!all_refined && s0 != 0.0) {
            m[1] = sx / s0;
            m[2] = sy / s0;
            m[3] = sz / s0;
            m[0] = s0 / (4.0 * M_PI);
        } else {
            m[0] = 0.0;
            m[1] = m[2] = m[3] = 1.0;
        }
        if (c == 0) allref[e] = all_refined ? 1 : 0;
    }
}
// Pass 1: thread (point p, subtree s) forms the nested sum of subtree s
// (DFS entries segs[2s] .. segs[2s+1]-1, a brick and all its descendants)
// and leaves it in part[s][p].
__global__ void k_phys_seg(Geom g, BrickTable bt, const int* __restrict__ bfaces, const int* __restrict__ order,
                           const int* __restrict__ segs, int p0, int np, const double* __restrict__ msrc,
                           const int* __restrict__ allref, double* __restrict__ part) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int sg = blockIdx.y;
    if (p >= np) return;
    double xyz[3];
    bound_point(g, bt, bfaces, p0 + p, xyz, nullptr);
    const double alpha = g.z_reflect ? 2.0 : 1.0;
    const int e0 = segs[2 * sg], e1 = segs[2 * sg + 1];
    const int L0 = bt.level[order[e0]];
    NestStack st;
    for (int e = e0; e < e1; e++)
        st.push(bt.level[order[e]], own_term(xyz, msrc + (size_t)e * 32, allref[e] != 0, alpha));
    part[(size_t)sg * np + p] = st.close(L0);
}
// Pass 2: thread p walks the bricks above the subtrees (own terms formed
// here) and the subtrees themselves (their sums from pass 1) in DFS order,
// giving the same additions in the same order as one walk over all bricks.
// top[t] >= 0: a DFS entry; top[t] < 0: subtree -top[t]-1.
__global__ void k_phys_top(Geom g, BrickTable bt, const int* __restrict__ bfaces, const int* __restrict__ order,
                           const int* __restrict__ segs, const int* __restrict__ top, int ntop, int p0, int np,
                           const double* __restrict__ msrc, const int* __restrict__ allref,
                           const double* __restrict__ part, double* __restrict__ bphi) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double xyz[3];
    int where;
    bound_point(g, bt, bfaces, p0 + p, xyz, &where);
    const double alpha = g.z_reflect ? 2.0 : 1.0;
    NestStack st;
    for (int t = 0; t < ntop; t++) {
        const int code = top[t];
        if (code >= 0) {
            st.push(bt.level[order[code]], own_term(xyz, msrc + (size_t)code * 32, allref[code] != 0, alpha));
        } else {
            const int sg = -code - 1;
            st.push(bt.level[order[segs[2 * sg]]], part[(size_t)sg * np + p]);
        }
    }
    bphi[where] = st.close(0);
}
// Poisson::vcycle_relax (poisson.cpp:88-130): Jacobi sweeps on one brick
// with its ghost dphi frozen, until the sweep's sum of squared updates drops
// below half the first sweep's or 16 sweeps.  Block = one brick
// (RelaxThreads<NX> threads), dphi staged in dynamic shared memory.
// out[e] = last sweep's sum.
template <int NX, typename CT>
__global__ void __launch_bounds__(RelaxThreads<NX>::value) k_relax(Geom g, DevState st, const int* __restrict__ slots,
                                                                   double* __restrict__ out) {
    constexpr int P = NX + 2, P3 = P * P * P, TH = RelaxThreads<NX>::value, K = NX * NX * NX / TH;
    RelaxSmem<NX, CT>& sm = *reinterpret_cast<RelaxSmem<NX, CT>*>(dyn_smem());
    const int b = slots[blockIdx.x];
    const size_t base = (size_t)b * P3;
    const int t = threadIdx.x;
    CT* D = Corr<CT>::dphi(st);
    int c[K];
    CT v[K];
    const double resid = relax_brick<NX, TH, CT>(sm, D + base, Corr<CT>::dphi1(st) + base, t, c, v, BlockSync{});
#pragma unroll
    for (int r = 0; r < K; r++) D[base + c[r]] = v[r];
    if (t == 0) out[b] = resid;
}
// Poisson::store_phi / restore_phi / restore_half_phi (poisson.cpp:166-221).
__global__ void k_phi_time(Geom g, DevState st, const int* __restrict__ slots, int mode) {
    const int b = slots[blockIdx.x];
    const int pnx = g.pnx, nx = pnx - 2;
    const size_t base = (size_t)b * g.pnx3;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const size_t c = base + pidx(pnx, t % nx + 1, (t / nx) % nx + 1, t / (nx * nx) + 1);
        if (mode == 0) {
            st.phi0[c] = st.phi[c];
        } else if (mode == 1) {
            st.phi[c] = st.phi0[c];
        } else {
            const double r = st.phi[c];
            st.phi[c] = (st.phi[c] + st.phi0[c]) * 0.5;
            st.phi0[c] = r;
        }
    }
}
// Poisson::Poisson() zeroes phi, dphi1, dphi, phi0 (poisson.cpp:671-685);
// S and the forces are zeroed here too.  Then Poisson::inject_from_parent
// (poisson.cpp:132-164): phi = phi0 = parent phi, piecewise constant.
__global__ void k_poisson_new(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    const int b = slots[blockIdx.x];
    const int pnx = g.pnx;
    const size_t base = (size_t)b * g.pnx3;
    for (int t = threadIdx.x; t < g.pnx3; t += blockDim.x) {
        st.phi[base + t] = 0.0;
        st.phi0[base + t] = 0.0;
        st.dphi[base + t] = 0.0;
        st.dphi1[base + t] = 0.0;
        st.S[base + t] = 0.0;
        st.fx[base + t] = 0.0;
        st.fy[base + t] = 0.0;
        st.fz[base + t] = 0.0;
        if (st.fdphi) {
            st.fdphi[base + t] = 0.0f;
            st.fdphi1[base + t] = 0.0f;
        }
    }
    __syncthreads();
    const int p = bt.parent[b];
    if (p < 0) return;
    const int c = bt.cidx[b];
    const int nx = pnx - 2, half = nx / 2;
    const size_t pbase = (size_t)p * g.pnx3;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int i0 = (i + 1) / 2 + (c & 1) * half;
        const int j0 = (j + 1) / 2 + ((c >> 1) & 1) * half;
        const int k0 = (k + 1) / 2 + ((c >> 2) & 1) * half;
        const double u = st.phi[pbase + pidx(pnx, i0, j0, k0)];
        st.phi[base + pidx(pnx, i, j, k)] = u;
        st.phi0[base + pidx(pnx, i, j, k)] = u;
    }
}

// ---------------------------------------------------------------------------
// one launch per level (or per brick set): block = brick
// ---------------------------------------------------------------------------
__global__ void k_set_source(Geom g, DevState st, const int* __restrict__ slots) {
    op_set_source(g, st, slots[blockIdx.x], threadIdx.x, blockDim.x);
}
__global__ void k_phi_faces(Geom g, BrickTable bt, DevState st, PoissonAux aux, const int* __restrict__ slots) {
    op_phi_faces(g, bt, st, aux, slots[blockIdx.x], blockIdx.y, threadIdx.x, blockDim.x);
}
template <typename CT>
__global__ void k_dphi_faces(Geom g, BrickTable bt, DevState st, PoissonAux aux, const int* __restrict__ slots) {
    op_dphi_faces<CT>(g, bt, st, aux, slots[blockIdx.x], blockIdx.y, threadIdx.x, blockDim.x);
}
// thread = (edge, position along it)
__global__ void k_phi_edges(Geom g, BrickTable bt, DevState st, PoissonAux aux, const int* __restrict__ slots) {
    const int m = g.pnx - 2;
    const int t = threadIdx.x;
    if (t < 12 * m) op_phi_edge(g, bt, st, aux, slots[blockIdx.x], t / m, t % m + 1);
}
// thread = vertex
__global__ void k_phi_vertices(Geom g, BrickTable bt, DevState st, PoissonAux aux, const int* __restrict__ slots) {
    if (threadIdx.x < 8) op_phi_vertex(g, bt, st, aux, slots[blockIdx.x], threadIdx.x);
}
__global__ void k_phi_from_children(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    op_phi_from_children(g, bt, st, slots[blockIdx.x], blockIdx.y, threadIdx.x);
}
template <typename CT>
__global__ void k_init_vcycle(Geom g, DevState st, const int* __restrict__ slots) {
    op_init_vcycle<CT>(g, st, slots[blockIdx.x], threadIdx.x, blockDim.x);
}
template <typename CT>
__global__ void k_vdown(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots,
                        const RefluxItem* __restrict__ items, const int* __restrict__ ranges) {
    op_vdown<CT>(g, bt, st, slots[blockIdx.x], items, ranges + 4 * blockIdx.x);
}
template <typename CT>
__global__ void k_coarse_correction(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    op_coarse_correction<CT>(g, bt, st, slots[blockIdx.x], threadIdx.x);
}
template <typename CT>
__global__ void k_retire(Geom g, DevState st, const int* __restrict__ slots) {
    op_retire<CT>(g, st, slots[blockIdx.x], threadIdx.x, blockDim.x);
}
__global__ void k_forces(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots) {
    op_forces(g, bt, st, slots[blockIdx.x], threadIdx.x, blockDim.x);
}
__global__ void k_adjust_force(Geom g, DevState st, const RefluxItem* __restrict__ items) {
    op_adjust_force(g, st, items[blockIdx.x], threadIdx.x);
}
template <typename CT>
__global__ void k_solution_error(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots,
                                 double* __restrict__ out) {
    __shared__ double red[32];
    op_solution_error<CT>(g, bt, st, slots[blockIdx.x], out, red, blockDim.x);
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
void launch_poisson_new_bricks(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                               cudaStream_t s) {
    if (n <= 0) return;
    launch_k(k_poisson_new, n, 256, 0, s, g, bt, st, slots);
}

}  // namespace amr

namespace amr {

void launch_set_source(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s) {
    if (n > 0) launch_k(k_set_source, n, 256, 0, s, g, st, slots);
}
void launch_source_sums(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                        double* msrc, int* allref, cudaStream_t s) {
    if (n > 0) launch_k(k_source_sums, n, 32, 0, s, g, bt, st, slots, msrc, allref);
}
int launch_phys_bound(const Geom& g, const BrickTable& bt, const int* bfaces, int nbf, const int* order,
                      const PhysWalk& w, const double* msrc, const int* allref, double* bphi, double* scratch,
                      size_t scratch_cap, cudaStream_t s) {
    if (nbf <= 0 || w.ntop <= 0) return 0;
    const int npts = nbf * g.pnx * g.pnx;
    const size_t per = (size_t)std::max(w.nseg, 1);
    if (scratch_cap < per) return -1;
    const int batch = (int)std::min<size_t>((size_t)npts, scratch_cap / per);
    for (int p0 = 0; p0 < npts; p0 += batch) {
        const int np = std::min(batch, npts - p0);
        if (w.nseg > 0)
            launch_k(k_phys_seg, dim3((np + 127) / 128, w.nseg), 128, 0, s, g, bt, bfaces, order, w.segs, p0, np, msrc,
                                                                      allref, scratch);
        launch_k(k_phys_top, (np + 63) / 64, 64, 0, s, g, bt, bfaces, order, w.segs, w.top, w.ntop, p0, np, msrc, allref,
                                                 scratch, bphi);
    }
    return 0;
}
void launch_phi_boundaries(const Geom& g, const BrickTable& bt, const DevState& st, const double* bphi, int* err,
                           const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    PoissonAux aux{bphi, err};
    launch_k(k_phi_faces, dim3(n, 6), 64, 0, s, g, bt, st, aux, slots);
    launch_k(k_phi_edges, n, ((12 * (g.pnx - 2) + 31) / 32) * 32, 0, s, g, bt, st, aux, slots);
    launch_k(k_phi_vertices, n, 32, 0, s, g, bt, st, aux, slots);
}
void launch_dphi_boundaries(const Geom& g, const BrickTable& bt, const DevState& st, const double* bphi, int* err,
                            const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    PoissonAux aux{bphi, err};
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_dphi_faces<float>, dim3(n, 6), 64, 0, s, g, bt, st, aux, slots);
    else
        launch_k(k_dphi_faces<double>, dim3(n, 6), 64, 0, s, g, bt, st, aux, slots);
}
void launch_phi_from_children(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                              cudaStream_t s) {
    const int half = (g.pnx - 2) / 2;
    if (n > 0) launch_k(k_phi_from_children, dim3(n, 8), ((half * half * half + 31) / 32) * 32, 0, s, g, bt, st, slots);
}
void launch_init_vcycle(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_init_vcycle<float>, n, 256, 0, s, g, st, slots);
    else
        launch_k(k_init_vcycle<double>, n, 256, 0, s, g, st, slots);
}
void launch_vdown(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                  const RefluxItem* items, const int* ranges, cudaStream_t s) {
    if (n <= 0) return;
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_vdown<float>, n, 256, 0, s, g, bt, st, slots, items, ranges);
    else
        launch_k(k_vdown<double>, n, 256, 0, s, g, bt, st, slots, items, ranges);
}
int launch_relax(const Geom& g, const DevState& st, const int* slots, int n, double* out, cudaStream_t s) {
    if (n <= 0) return 0;
    const bool f32 = g.precision == AMR_PREC_MIXED;
    if (g.nx == 8) {
        if (f32)
            launch_k(k_relax<8, float>, n, RelaxThreads<8>::value, sizeof(RelaxSmem<8, float>), s, g, st, slots, out);
        else
            launch_k(k_relax<8, double>, n, RelaxThreads<8>::value, sizeof(RelaxSmem<8, double>), s, g, st, slots,
                     out);
    } else if (g.nx == 12) {
        if (f32)
            launch_k(k_relax<12, float>, n, RelaxThreads<12>::value, sizeof(RelaxSmem<12, float>), s, g, st, slots,
                     out);
        else
            launch_k(k_relax<12, double>, n, RelaxThreads<12>::value, sizeof(RelaxSmem<12, double>), s, g, st, slots,
                     out);
    } else {
        return -1;
    }
    return 0;
}
void launch_coarse_correction(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                              cudaStream_t s) {
    const int half = (g.pnx - 2) / 2;
    if (n <= 0) return;
    const int nt = ((half * half * half + 31) / 32) * 32;
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_coarse_correction<float>, n, nt, 0, s, g, bt, st, slots);
    else
        launch_k(k_coarse_correction<double>, n, nt, 0, s, g, bt, st, slots);
}
void launch_retire(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_retire<float>, n, 256, 0, s, g, st, slots);
    else
        launch_k(k_retire<double>, n, 256, 0, s, g, st, slots);
}
void launch_forces(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                   cudaStream_t s) {
    if (n > 0) launch_k(k_forces, n, 256, 0, s, g, bt, st, slots);
}
void launch_adjust_force(const Geom& g, const DevState& st, const RefluxItem* items, int n, cudaStream_t s) {
    // one thread per coarse face of the item's quadrant: (nx/2)^2 of them
    const int half = (g.pnx - 2) / 2;
    if (n > 0) launch_k(k_adjust_force, n, ((half * half + 31) / 32) * 32, 0, s, g, st, items);
}
void launch_solution_error(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                           double* out, cudaStream_t s) {
    if (n <= 0) return;
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_solution_error<float>, n, 256, 0, s, g, bt, st, slots, out);
    else
        launch_k(k_solution_error<double>, n, 256, 0, s, g, bt, st, slots, out);
}
void launch_phi_time(const Geom& g, const DevState& st, const int* slots, int n, int mode, cudaStream_t s) {
    if (n > 0) launch_k(k_phi_time, n, 256, 0, s, g, st, slots, mode);
}

}  // namespace amr
