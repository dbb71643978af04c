// Jacobi sweeps of Poisson::vcycle_relax (poisson.cpp:88-130) on one brick
// staged in shared memory, one thread per interior cell.
//
// Each sweep computes tmp0 = dphi1 + lap(dphi)/6 for every cell from the
// previous sweep's values and adds it; the sweep's sum of tmp0^2 decides the
// loop (ratio to the first sweep's > 0.5, at most 16 sweeps).  The two shared
// buffers alternate so one block barrier per sweep suffices; every thread
// adds the per-warp partial sums itself along the same fixed pairwise tree,
// so all threads take the same loop decision.  (The reference adds the
// squares sequentially; the sums differ in the last bits only.)
#pragma once

namespace amr {

template <int NX, typename CT = double>
struct RelaxSmem {
    static constexpr int P = NX + 2, P3 = P * P * P, NT = NX * NX * NX, NW = NT / 32;
    CT buf[2][P3];
    double red[2][NW];
};

// The sweeps on a brick staged in both buffers (every cell, ghosts
// included): thread t owns interior cell c with dphi1 value d1.  Returns the
// last sweep's sum and leaves the relaxed value of cell c in *out.
template <int NX, typename CT = double>
__device__ __forceinline__ double relax_sweeps(RelaxSmem<NX, CT>& sm, int c, CT d1, CT* out) {
    constexpr int P = RelaxSmem<NX, CT>::P, NW = RelaxSmem<NX, CT>::NW;
    const int t = threadIdx.x;
    double resid0 = 0.0, resid = 0.0;
    int iters = 0, cur = 0;
    do {
        const CT* d = sm.buf[cur];
        const CT div = (d[c + 1] + d[c - 1] + d[c + P] + d[c - P] + d[c + P * P] + d[c - P * P]) - (d[c] * CT(6.0));
        const CT tmp0 = d1 + div * (CT(1.0) / CT(6.0));
        sm.buf[cur ^ 1][c] = d[c] + tmp0;
        double sq = double(tmp0) * double(tmp0);
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if ((t & 31) == 0) sm.red[cur][t >> 5] = sq;
        __syncthreads();
        // pairwise sum of the warp partials (fixed tree, identical in every
        // thread): log2(NW) dependent additions instead of NW
        double r[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) r[w] = sm.red[cur][w];
#pragma unroll
        for (int span = 1; span < NW; span <<= 1)
#pragma unroll
            for (int w = 0; w + span < NW; w += 2 * span) r[w] = r[w] + r[w + span];
        resid = r[0];
        if (iters == 0) resid0 = resid;
        iters++;
        cur ^= 1;
    } while (resid / resid0 > 0.5 && iters < 16);
    *out = sm.buf[cur][c];
    return resid;
}

// Interior cell of thread t in the (NX+2)^3 brick.
template <int NX>
__device__ __forceinline__ int relax_cell(int t) {
    constexpr int P = NX + 2;
    return ((t / (NX * NX) + 1) * P + (t / NX) % NX + 1) * P + t % NX + 1;
}

// Stages the brick (slot base) into both buffers;
// returns the last sweep's sum and leaves the relaxed interior value of this
// thread's cell in *out.  CT is the correction's storage and arithmetic type
// (FP64, or FP32 in the mixed form); the sums of squares are formed in FP64
// either way.
template <int NX, typename CT = double>
__device__ __forceinline__ double relax_brick(RelaxSmem<NX, CT>& sm, const CT* __restrict__ dphi,
                                              const CT* __restrict__ dphi1, CT* out) {
    constexpr int P3 = RelaxSmem<NX, CT>::P3, NT = RelaxSmem<NX, CT>::NT;
    const int t = threadIdx.x;
    for (int q = t; q < P3; q += NT) {
        const CT v = dphi[q];
        sm.buf[0][q] = v;
        sm.buf[1][q] = v;
    }
    const int c = relax_cell<NX>(t);
    const CT d1 = dphi1[c];
    __syncthreads();
    return relax_sweeps<NX, CT>(sm, c, d1, out);
}

// Barrier over `n` threads with id `id` (1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// relax_brick with half the threads: NX^3/2 threads (lt = 0 .. NX^3/2 - 1,
// synchronised by barrier `bar`) each relax cells lt and lt + NX^3/2, so two
// bricks share one block.  Cell c of warp lane l lies in the same 32-cell
// warp group with the same lane as in relax_brick, so the warp partials, their
// pairwise sum and every loop decision are bit for bit those of relax_brick.
// out[0], out[1] receive the two cells' relaxed values.
template <int NX, typename CT = double>
__device__ __forceinline__ double relax_brick_half(RelaxSmem<NX, CT>& sm, const CT* __restrict__ dphi,
                                                   const CT* __restrict__ dphi1, CT* out, int lt, int bar) {
    constexpr int P = RelaxSmem<NX, CT>::P, P3 = RelaxSmem<NX, CT>::P3, NT = RelaxSmem<NX, CT>::NT,
                  NW = RelaxSmem<NX, CT>::NW, HT = NT / 2;
    for (int q = lt; q < P3; q += HT) {
        const CT v = dphi[q];
        sm.buf[0][q] = v;
        sm.buf[1][q] = v;
    }
    int c[2];
    CT d1[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int t = lt + h * HT;
        const int i = t % NX + 1, j = (t / NX) % NX + 1, k = t / (NX * NX) + 1;
        c[h] = (k * P + j) * P + i;
        d1[h] = dphi1[c[h]];
    }
    named_sync(bar, HT);
    double resid0 = 0.0, resid = 0.0;
    int iters = 0, cur = 0;
    do {
        const CT* d = sm.buf[cur];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int cc = c[h];
            const CT div =
                (d[cc + 1] + d[cc - 1] + d[cc + P] + d[cc - P] + d[cc + P * P] + d[cc - P * P]) - (d[cc] * CT(6.0));
            const CT tmp0 = d1[h] + div * (CT(1.0) / CT(6.0));
            sm.buf[cur ^ 1][cc] = d[cc] + tmp0;
            double sq = double(tmp0) * double(tmp0);
            for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
            if ((lt & 31) == 0) sm.red[cur][h * (HT >> 5) + (lt >> 5)] = sq;
        }
        named_sync(bar, HT);
        double r[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) r[w] = sm.red[cur][w];
#pragma unroll
        for (int span = 1; span < NW; span <<= 1)
#pragma unroll
            for (int w = 0; w + span < NW; w += 2 * span) r[w] = r[w] + r[w + span];
        resid = r[0];
        if (iters == 0) resid0 = resid;
        iters++;
        cur ^= 1;
    } while (resid / resid0 > 0.5 && iters < 16);
    out[0] = sm.buf[cur][c[0]];
    out[1] = sm.buf[cur][c[1]];
    return resid;
}

}  // namespace amr
