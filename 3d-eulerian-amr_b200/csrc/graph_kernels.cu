// Device-resident control flow for the graph-captured step: the relaxation
// sweeps, the L1 error and the CFL step finish with a "last block" that forms
// the reference's recursive sums on the device (same additions in the same
// order as Poisson::vcycle_relax / solution_error / GridNode::max_dt) and sets
// the CUDA-graph WHILE conditions, so no host round trip is needed between
// V-cycles or relaxation passes.  FP64, compiled with --fmad=false.
#include <cuda_runtime.h>

#include "corr.cuh"
#include "euler_state.cuh"
#include "graph.h"
#include "relax_brick.cuh"
#include "launch.cuh"

namespace amr {

// Bottom-up nested sums over levels [0, top).  Values of level `top` are in
// `leaf` (per slot); S(node at m < top) = ((0 + S(c0)) + S(c1)) + ... in
// child order (withown = false), or ((own + S(c0)) + ...) (withown = true:
// own values in `leaf` for every level, `nest` preset to own at level top).  Result for the root is returned to
// thread 0.  Called by one whole block.
__device__ double nested_sum_block(const LevelLists& L, const int* __restrict__ child, const double* leaf,
                                   double* nest, int top, bool withown) {
    for (int m = top - 1; m >= 0; m--) {
        const int* sl = L.slots + L.off[m];
        for (int q = threadIdx.x; q < L.cnt[m]; q += blockDim.x) {
            const int p = sl[q];
            double s = withown ? __ldcg(leaf + p) : 0.0;
            for (int c = 0; c < 8; c++) {
                const int ch = child[8 * p + c];
                if (ch < 0) continue;
                s += (m + 1 == top && !withown) ? __ldcg(leaf + ch) : __ldcg(nest + ch);
            }
            nest[p] = s;
        }
        __threadfence_block();
        __syncthreads();
    }
    return __ldcg(nest + L.slots[L.off[0]]);
}

// Relaxation of one level (Poisson::vcycle_relax, poisson.cpp:88-130) whose
// last block reduces the per-brick residuals as the recursion does and
// decides the relaxation loop of vcycle0 (poisson.cpp:66-70, 74-78):
// mode 0 records resid0 and opens the loop, mode 1 continues it while
// resid / resid0 > ratio.
//
// Ghost zones: in mode 0 they come from the brick's own dphi array (filled
// just before by the face ghost kernel).  In mode 1 the block fills them
// itself -- what Poisson::enforce_dphi_boundaries (poisson.cpp:890-929) would
// copy: a same-level neighbour's first interior layer from the snapshot the
// previous pass published, the parent's value across a coarse-fine face
// (PoissonAMRBound::get_dphi), 0 on a domain face, the mirror on z = 0 -- and
// also stores them into its global ghost cells, so the arrays end the loop
// exactly as the reference leaves them.  Every pass publishes its new first
// interior layers for the next pass.
template <int NX, typename CT>
__device__ __forceinline__ CT ghost_dphi(const Geom& g, const BrickTable& bt, const DevState& st, const CT* snap_rd,
                                         size_t stride, int b, int face, int t1, int t2) {
    constexpr int P = NX + 2;
    const int kind = bt.ftype[6 * b + face];
    const int nbr = bt.fnbr[6 * b + face];
    const CT* D = Corr<CT>::dphi(st);
    if (kind == FACE_SIB) return __ldcg(snap_rd + (size_t)nbr * stride + ((face ^ 1) * NX + (t1 - 1)) * NX + (t2 - 1));
    if (kind == FACE_OUTFLOW) return CT(0);
    const int ax = face >> 1;
    int q[3];
    q[ax] = (face & 1) ? 1 : P - 2;
    q[ax == 0 ? 1 : 0] = t1;
    q[ax == 2 ? 1 : 2] = t2;
    if (kind == FACE_REFLECT) {  // own value mirrored through z = 0, before this pass
        const int kk = q[2] == 1 ? P - 2 : 1;
        return D[(size_t)b * P * P * P + (kk * P + q[1]) * P + q[0]];
    }
    const int v = (face & 1) ? 1 : -1;
    int r[3];
    for (int d = 0; d < 3; d++) {
        const int rel = bt.off[3 * b + d] + (d == ax ? v * (P - 2) : 0) - 2 * bt.off[3 * nbr + d] - (g.bw - 1);
        r[d] = (rel + q[d]) / 2;
    }
    return D[(size_t)nbr * P * P * P + (r[2] * P + r[1]) * P + r[0]];
}

template <int NX, typename CT>
__global__ void __launch_bounds__(NX* NX* NX)
    k_relax_dev(Geom g, BrickTable bt, DevState st, LevelLists L, int level, int mode, double ratio,
                cudaGraphConditionalHandle cond, Control* ctl, double* pres, double* nest, unsigned int* counter,
                CT* snap, size_t stride, size_t snap_half) {
    constexpr int P = NX + 2, P3 = P * P * P, F = NX * NX;
    __shared__ RelaxSmem<NX, CT> sm;
    CT* D = Corr<CT>::dphi(st);
    __shared__ bool last;
    const int b = L.slots[L.off[level] + blockIdx.x];
    const size_t base = (size_t)b * P3;
    const int t = threadIdx.x;
    // snapshot buffers: the previous pass wrote buffer `par`, this one writes par^1
    const int par = mode == 0 ? 0 : ctl->snap_par[level];
    const CT* snap_rd = snap + (size_t)par * snap_half;
    CT* snap_wr = snap + (size_t)(mode == 0 ? 0 : par ^ 1) * snap_half;
    if (mode == 1 && t < 6 * F) {
        const int face = t / F, qq = t % F;
        const int t1 = qq % NX + 1, t2 = qq / NX + 1;
        const CT gv = ghost_dphi<NX, CT>(g, bt, st, snap_rd, stride, b, face, t1, t2);
        const int ax = face >> 1;
        int d[3];
        d[ax] = (face & 1) ? P - 1 : 0;
        d[ax == 0 ? 1 : 0] = t1;
        d[ax == 2 ? 1 : 2] = t2;
        D[base + (d[2] * P + d[1]) * P + d[0]] = gv;
    }
    if (mode == 1) __syncthreads();
    const int c = ((t / (NX * NX) + 1) * P + (t / NX) % NX + 1) * P + t % NX + 1;
    const int ci = t % NX + 1, cj = (t / NX) % NX + 1, ck = t / (NX * NX) + 1;
    CT v;
    const double resid = relax_brick<NX, CT>(sm, D + base, Corr<CT>::dphi1(st) + base, &v);
    D[base + c] = v;
    // publish first interior layers: layer of face f holds the cells adjacent to it
    CT* sw = snap_wr + (size_t)b * stride;
    if (ci == 1) sw[(0 * NX + (cj - 1)) * NX + (ck - 1)] = v;
    if (ci == NX) sw[(1 * NX + (cj - 1)) * NX + (ck - 1)] = v;
    if (cj == 1) sw[(2 * NX + (ci - 1)) * NX + (ck - 1)] = v;
    if (cj == NX) sw[(3 * NX + (ci - 1)) * NX + (ck - 1)] = v;
    if (ck == 1) sw[(4 * NX + (ci - 1)) * NX + (cj - 1)] = v;
    if (ck == NX) sw[(5 * NX + (ci - 1)) * NX + (cj - 1)] = v;
    if (t == 0) pres[b] = resid;
    // last block: reduce and decide
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double r = level == 0 ? __ldcg(pres + b) : nested_sum_block(L, bt.child, pres, nest, level, false);
    if (t == 0) {
        *counter = 0u;
        ctl->relax_calls++;
        ctl->snap_par[level] = mode == 0 ? 0 : par ^ 1;  // the buffer just written
        if (mode == 0) {
            ctl->r0[level] = r;
            ctl->outer[level] = 0;
            cudaGraphSetConditional(cond, 1u);
        } else {
            const int o = ++ctl->outer[level];
            bool again = r / ctl->r0[level] > ratio;
            if (again && o > ctl->max_outer) {
                again = false;
                ctl->status = 1;
            }
            cudaGraphSetConditional(cond, again ? 1u : 0u);
        }
    }
}

// Poisson::solution_error (poisson.cpp:637-669) + the solve loop condition
// (error > tol, bounded by max_cycles).
template <typename CT>
__global__ void k_error_dev(Geom g, BrickTable bt, DevState st, LevelLists L, int nlevels, double tol,
                            cudaGraphConditionalHandle cond, Control* ctl, double* pres, double* nest,
                            unsigned int* counter) {
    CT* D = Corr<CT>::dphi(st);
    const int b = L.all[blockIdx.x];
    const int pnx = g.pnx, nx = pnx - 2, half = nx / 2;
    const double h = bt.h[b];
    const double h3 = h * h * h, hinv = 1.0 / h;
    const size_t base = (size_t)b * g.pnx3;
    __shared__ double red[32];
    __shared__ bool last;
    double sum = 0.0;
    for (int t = threadIdx.x; t < nx * nx * nx; t += blockDim.x) {
        const int i = t % nx + 1, j = (t / nx) % nx + 1, k = t / (nx * nx) + 1;
        const int c = (k * pnx + j) * pnx + i;
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
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        pres[b] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // deepest level: nest = own
    const int* sl = L.slots + L.off[nlevels - 1];
    for (int q = threadIdx.x; q < L.cnt[nlevels - 1]; q += blockDim.x) nest[sl[q]] = __ldcg(pres + sl[q]);
    __syncthreads();
    const double e = nested_sum_block(L, bt.child, pres, nest, nlevels - 1, true);
    if (threadIdx.x == 0) {
        *counter = 0u;
        ctl->err = e;
        ctl->cycles++;
        ctl->cycles_total++;
        bool again = e > tol;
        if (again && ctl->cycles >= ctl->max_cycles) {
            again = false;
            ctl->status = 2;
        }
        cudaGraphSetConditional(cond, again ? 1u : 0u);
    }
}

// Opens a solve loop: cycle counter and status reset, condition 1.
__global__ void k_open_loop(cudaGraphConditionalHandle cond, Control* ctl, int reset_cycles) {
    if (reset_cycles) {
        ctl->cycles = 0;
    }
    cudaGraphSetConditional(cond, 1u);
}

// GridNode::max_dt (grid_node.cpp:163-174) over per-brick steps, then the
// driver's MAXDTINC clamp (hydro_driver.cpp:108-113) against the previous
// step.  One block.
__global__ void k_dt_reduce(BrickTable bt, LevelLists L, int nlevels, const double* __restrict__ per, double* nest,
                            Control* ctl, double maxdtinc) {
    // R(n) = 1 / max(1/own, max_c 1/R(c)); nest holds R
    for (int m = nlevels - 1; m >= 0; m--) {
        const int* sl = L.slots + L.off[m];
        for (int q = threadIdx.x; q < L.cnt[m]; q += blockDim.x) {
            const int p = sl[q];
            double dtinv = 0.0;
            for (int c = 0; c < 8; c++) {
                const int ch = bt.child[8 * p + c];
                if (ch < 0) continue;
                const double cdtinv = 1.0 / __ldcg(nest + ch);
                dtinv = cdtinv > dtinv ? cdtinv : dtinv;
            }
            const double own = 1.0 / __ldcg(per + p);
            dtinv = own > dtinv ? own : dtinv;
            nest[p] = 1.0 / dtinv;
        }
        __threadfence_block();
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double dt = __ldcg(nest + L.slots[L.off[0]]);
        if (ctl->steps > 0) dt = r_min(ctl->last_dt * maxdtinc, dt);
        ctl->dt = dt;
        ctl->last_dt = dt;
        ctl->steps++;
    }
}

// ---------------------------------------------------------------------------
void launch_relax_dev(const Geom& g, const BrickTable& bt, const DevState& st, const LevelLists& L, int level,
                      int mode, double ratio, cudaGraphConditionalHandle cond, Control* ctl, double* pres,
                      double* nest, unsigned int* counter, double* snap, size_t snap_stride, cudaStream_t s) {
    const int n = L.cnt[level];
    if (n <= 0) return;
    // two buffers, each one stride per brick slot of the pool (FP32 entries
    // in the mixed form, in the same allocation)
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_relax_dev<8, float>, n, 512, 0, s, g, bt, st, L, level, mode, ratio, cond, ctl, pres, nest, counter,
                 reinterpret_cast<float*>(snap), snap_stride, snap_stride * (size_t)L.cap);
    else
        launch_k(k_relax_dev<8, double>, n, 512, 0, s, g, bt, st, L, level, mode, ratio, cond, ctl, pres, nest,
                 counter, snap, snap_stride, snap_stride * (size_t)L.cap);
}

void launch_error_dev(const Geom& g, const BrickTable& bt, const DevState& st, const LevelLists& L, int nlevels,
                      double tol, cudaGraphConditionalHandle cond, Control* ctl, double* pres, double* nest,
                      unsigned int* counter, cudaStream_t s) {
    if (g.precision == AMR_PREC_MIXED)
        launch_k(k_error_dev<float>, L.nall, 256, 0, s, g, bt, st, L, nlevels, tol, cond, ctl, pres, nest, counter);
    else
        launch_k(k_error_dev<double>, L.nall, 256, 0, s, g, bt, st, L, nlevels, tol, cond, ctl, pres, nest, counter);
}

void launch_open_loop(cudaGraphConditionalHandle cond, Control* ctl, int reset_cycles, cudaStream_t s) {
    launch_k(k_open_loop, 1, 1, 0, s, cond, ctl, reset_cycles);
}

void launch_dt_reduce(const BrickTable& bt, const LevelLists& L, int nlevels, const double* per, double* nest,
                      Control* ctl, double maxdtinc, cudaStream_t s) {
    launch_k(k_dt_reduce, 1, 1024, 0, s, bt, L, nlevels, per, nest, ctl, maxdtinc);
}

}  // namespace amr
