// Device-resident control flow for the graph-captured step: the relaxation
// sweeps, the L1 error and the CFL step finish with a "last block" that forms
// the reference's recursive sums on the device (same additions in the same
// order as Poisson::vcycle_relax / solution_error / GridNode::max_dt) and sets
// the CUDA-graph WHILE conditions, so no host round trip is needed between
// V-cycles or relaxation passes.  FP64, compiled with --fmad=false.
#include <cuda_runtime.h>

#include "euler_state.cuh"
#include "graph_ops.cuh"
#include "launch.cuh"

namespace amr {

// Byte offset of the level-sum buffers in k_relax_dev's dynamic shared
// memory, and the whole size.
template <int NX, typename CT>
__host__ __device__ constexpr size_t relax_dev_nbuf_offset() {
    return (sizeof(RelaxSmem<NX, CT>) + 15) / 16 * 16;
}
template <int NX, typename CT>
__host__ __device__ constexpr size_t relax_dev_smem() {
    return relax_dev_nbuf_offset<NX, CT>() + 2 * NEST_SMEM * sizeof(double);
}

// Relaxation pass of one level whose last block reduces the per-brick sums
// as the recursion does and decides the relaxation loop of vcycle0
// (poisson.cpp:66-70, 74-78): mode 0 records resid0 and opens the loop,
// mode 1 continues it while resid / resid0 > ratio.
template <int NX, typename CT>
__global__ void __launch_bounds__(RelaxThreads<NX>::value)
    k_relax_dev(Geom g, BrickTable bt, DevState st, LevelLists L, int level, int mode, double ratio,
                cudaGraphConditionalHandle cond, Control* ctl, double* pres, double* nest, unsigned int* counter,
                CT* snap, size_t stride, size_t snap_half) {
    // dynamic shared memory: the staged brick, then the level-sum buffers
    RelaxSmem<NX, CT>& sm = *reinterpret_cast<RelaxSmem<NX, CT>*>(dyn_smem());
    double* nbuf = reinterpret_cast<double*>(dyn_smem() + relax_dev_nbuf_offset<NX, CT>());
    __shared__ bool last;
    const int b = L.slots[L.off[level] + blockIdx.x];
    const int t = threadIdx.x;
    // snapshot buffers: the previous pass wrote buffer `par`, this one writes par^1
    const int par = mode == 0 ? 0 : ctl->snap_par[level];
    const CT* snap_rd = snap + (size_t)par * snap_half;
    CT* snap_wr = snap + (size_t)(mode == 0 ? 0 : par ^ 1) * snap_half;
    op_relax_pass<NX, RelaxThreads<NX>::value, CT>(g, bt, st, b, mode, snap_rd, snap_wr, stride, pres, sm, t,
                                                   BlockSync{});
    // last block: reduce and decide
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double r = level == 0                 ? __ldcg(pres + b)
                     : L.max_cnt <= NEST_SMEM ? nested_sum_smem(L, pres, level, false, nbuf)
                                              : nested_sum_block(L, bt.child, pres, nest, level, false);
    if (t == 0) {
        *counter = 0u;
        ctl->relax_calls++;
        ctl->relax_level[level]++;
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
    __shared__ double nbuf[2 * NEST_SMEM];
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
    double e;
    if (L.max_cnt <= NEST_SMEM) {
        e = nested_sum_smem(L, pres, nlevels - 1, true, nbuf);
    } else {
        // deepest level: nest = own
        const int* sl = L.slots + L.off[nlevels - 1];
        for (int q = threadIdx.x; q < L.cnt[nlevels - 1]; q += blockDim.x) nest[sl[q]] = __ldcg(pres + sl[q]);
        __syncthreads();
        e = nested_sum_block(L, bt.child, pres, nest, nlevels - 1, true);
    }
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
    float* snap32 = reinterpret_cast<float*>(snap);
    const size_t half = snap_stride * (size_t)L.cap;
    const bool f32 = g.precision == AMR_PREC_MIXED;
    if (g.nx == 12) {
        if (f32)
            launch_k(k_relax_dev<12, float>, n, RelaxThreads<12>::value, relax_dev_smem<12, float>(), s, g, bt, st, L,
                     level, mode, ratio, cond, ctl, pres, nest, counter, snap32, snap_stride, half);
        else
            launch_k(k_relax_dev<12, double>, n, RelaxThreads<12>::value, relax_dev_smem<12, double>(), s, g, bt, st,
                     L, level, mode, ratio, cond, ctl, pres, nest, counter, snap, snap_stride, half);
    } else {
        if (f32)
            launch_k(k_relax_dev<8, float>, n, RelaxThreads<8>::value, relax_dev_smem<8, float>(), s, g, bt, st, L,
                     level, mode, ratio, cond, ctl, pres, nest, counter, snap32, snap_stride, half);
        else
            launch_k(k_relax_dev<8, double>, n, RelaxThreads<8>::value, relax_dev_smem<8, double>(), s, g, bt, st, L,
                     level, mode, ratio, cond, ctl, pres, nest, counter, snap, snap_stride, half);
    }
}

int relax_dev_attributes() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, size_t bytes) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    };
    set((const void*)k_relax_dev<8, float>, relax_dev_smem<8, float>());
    set((const void*)k_relax_dev<8, double>, relax_dev_smem<8, double>());
    set((const void*)k_relax_dev<12, float>, relax_dev_smem<12, float>());
    set((const void*)k_relax_dev<12, double>, relax_dev_smem<12, double>());
    return e == cudaSuccess ? 0 : -1;
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
