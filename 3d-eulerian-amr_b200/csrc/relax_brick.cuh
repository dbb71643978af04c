// Jacobi sweeps of Poisson::vcycle_relax (poisson.cpp:88-130) on one brick
// staged in shared memory.
//
// Each sweep computes tmp0 = dphi1 + lap(dphi)/6 for every cell from the
// previous sweep's values and adds it; the sweep's sum of tmp0^2 decides the
// loop (ratio to the first sweep's > 0.5, at most 16 sweeps).  The two shared
// buffers alternate so one barrier per sweep suffices; every thread adds the
// per-warp partial sums itself along the same fixed pairwise tree, so all
// threads take the same loop decision.  (The reference adds the squares
// sequentially; the sums differ in the last bits only.)
//
// Thread layout: TH threads (a multiple of 32 that divides NX^3) relax one
// brick, K = NX^3 / TH cells each; thread lt owns interior cells
// lt + r TH, r < K, counted x fastest.  Cell c's square enters the partial
// of its 32-cell group c / 32 at lane c % 32 whatever TH is, so the warp
// partials, their pairwise sum and every loop decision are the same bit for
// bit for every layout: a whole block of 512 threads on an 8^3 brick, two
// bricks of 256 threads each in one block, 576 threads on a 12^3 brick.
#pragma once

namespace amr {

template <int NX, typename CT = double>
struct RelaxSmem {
    static constexpr int P = NX + 2, P3 = P * P * P, NT = NX * NX * NX, NW = NT / 32;
    CT buf[2][P3];
    double red[2][NW];
};

// Threads of a whole block relaxing one brick of NX^3 interior cells.
template <int NX>
struct RelaxThreads;
template <>
struct RelaxThreads<8> {
    static constexpr int value = 512;  // one cell per thread
};
template <>
struct RelaxThreads<12> {
    static constexpr int value = 576;  // three cells per thread
};

// Barrier over the threads that relax one brick.
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
// Barrier over `n` threads with id `id` (1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
struct NamedSync {
    int id, n;
    __device__ __forceinline__ void operator()() const { named_sync(id, n); }
};

// Dynamic shared memory of a kernel (one declaration for every kernel).
__device__ __forceinline__ unsigned char* dyn_smem() {
    extern __shared__ __align__(16) unsigned char amr_dyn_smem[];
    return amr_dyn_smem;
}

// Interior cell t of the (NX+2)^3 brick.
template <int NX>
__device__ __forceinline__ int relax_cell(int t) {
    constexpr int P = NX + 2;
    return ((t / (NX * NX) + 1) * P + (t / NX) % NX + 1) * P + t % NX + 1;
}

// Sum of the NW warp partials p[0..NW-1] (NW <= 64; every partial is a sum
// of squares, so >= 0) along a fixed pairwise tree, identical in every
// thread: partials 0..31 and 32..63 (0.0 where there is none) are each
// added along the xor butterfly (at span s = 1, 2, 4, 8, 16 partial q takes
// q ^ s), and the two halves' sums added last.  IEEE addition is
// commutative and an absent partner adds +0.0, which leaves a non-negative
// value unchanged, so every lane ends with the tree's sum bit for bit.
// With two halves the first span is taken for both at once: even lanes keep
// the low half's pair sum (q, q ^ 1) and odd lanes the high half's, one
// shuffle carrying the half each lane gives away; spans 2..16 then add
// within the same parity, and one more shuffle at span 1 adds the halves --
// 6 shuffles instead of 10.
template <int NW>
__device__ __forceinline__ double pairwise_sum(const double* p) {
    static_assert(NW <= 64, "at most 64 warp partials");
    const int q = threadIdx.x & 31;
    const double lo = q < NW ? p[q] : 0.0;
    if constexpr (NW <= 32) {
        double v = lo;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        return v;
    } else {
        const double hi = 32 + q < NW ? p[32 + q] : 0.0;
        const bool odd = q & 1;
        double v = (odd ? hi : lo) + __shfl_xor_sync(0xffffffffu, odd ? lo : hi, 1);
#pragma unroll
        for (int s = 2; s < 32; s <<= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        return v + __shfl_xor_sync(0xffffffffu, v, 1);
    }
}

// resid / resid0 > 0.5, the sweep loop's test, without the division.  For
// resid0 >= 2^-1021 (so that 0.5 resid0 is a normal double, exact) the
// correctly rounded quotient exceeds 0.5 exactly when resid > 0.5 resid0:
// rounding is monotonic and 0.5 is a double, so the two can differ only if
// the exact quotient lay in (0.5, 0.5 + 2^-54], which would need
// 0 < resid - 0.5 resid0 <= 2^-54 resid0; but two different doubles differ
// by at least one unit in the last place of the smaller, here of
// 0.5 resid0, which is more than 2^-53 (0.5 resid0) = 2^-54 resid0.  Zero, subnormal, infinite and NaN values
// give the same answer both ways (any resid0 below the bound takes the
// division).
__device__ __forceinline__ bool above_half(double resid, double resid0) {
    return resid0 >= 0x1p-1021 ? resid > 0.5 * resid0 : resid / resid0 > 0.5;
}

// The sweeps on a brick staged in two buffers x, y (x holds every cell,
// ghosts included; y the same ghost faces): thread lt owns the K cells c[r]
// with dphi1 values d1[r]; red holds the per-sweep warp partials
// (2 x NX^3 / 32).  Returns the last sweep's sum and the buffer that holds
// the relaxed brick.
template <int NX, int TH, typename CT, typename Sync>
__device__ __forceinline__ double relax_sweeps_in(CT* x, CT* y, double* red, int lt, const int* c, const CT* d1,
                                                  CT** result, Sync sync, int* sweeps = nullptr) {
    constexpr int P = NX + 2, NW = NX * NX * NX / 32, K = NX * NX * NX / TH, WT = TH / 32;
    static_assert((NX * NX * NX) % TH == 0 && TH % 32 == 0, "relaxation layout");
    double resid0 = 0.0, resid = 0.0;
    int iters = 0, cur = 0;
    do {
        const CT* d = cur ? y : x;
        CT* w_ = cur ? x : y;
        double sq[K];
#pragma unroll
        for (int r = 0; r < K; r++) {
            const int cc = c[r];
            const CT div = (d[cc + 1] + d[cc - 1] + d[cc + P] + d[cc - P] + d[cc + P * P] + d[cc - P * P]) - (d[cc] * CT(6.0));
            const CT tmp0 = d1[r] + div * (CT(1.0) / CT(6.0));
            w_[cc] = d[cc] + tmp0;
            sq[r] = double(tmp0) * double(tmp0);
        }
        // warp partials: cells r and r + 1 of this thread lie in groups
        // r WT + warp and (r + 1) WT + warp, whose butterflies (spans 16, 8,
        // 4, 2, 1) are taken together: at span 16 the lower lanes keep group
        // r's pair sums and the upper ones group r + 1's, one shuffle
        // carrying the value each lane gives away; spans 8..1 stay within a
        // half.  Same pairs, so the same sums, with 5 shuffles instead of 10.
        double* rd = red + cur * NW;
        const int lane = lt & 31, wp = lt >> 5;
#pragma unroll
        for (int r = 0; r + 1 < K; r += 2) {
            const bool up = lane & 16;
            double v = (up ? sq[r + 1] : sq[r]) + __shfl_xor_sync(0xffffffffu, up ? sq[r] : sq[r + 1], 16);
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((lane & 15) == 0) rd[(r + (up ? 1 : 0)) * WT + wp] = v;
        }
        if constexpr (K & 1) {
            double v = sq[K - 1];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) rd[(K - 1) * WT + wp] = v;
        }
        sync();
        resid = pairwise_sum<NW>(rd);
        if (iters == 0) resid0 = resid;
        iters++;
        cur ^= 1;
    } while (above_half(resid, resid0) && iters < 16);
    *result = cur ? y : x;
    if (sweeps) *sweeps = iters;
    return resid;
}

// The same sweeps on a RelaxSmem's two buffers; the relaxed values of this
// thread's cells go to out[r].
template <int NX, int TH, typename CT, typename Sync>
__device__ __forceinline__ double relax_sweeps(RelaxSmem<NX, CT>& sm, int lt, const int* c, const CT* d1, CT* out,
                                               Sync sync) {
    constexpr int K = NX * NX * NX / TH;
    CT* res;
    const double r = relax_sweeps_in<NX, TH, CT>(sm.buf[0], sm.buf[1], &sm.red[0][0], lt, c, d1, &res, sync);
#pragma unroll
    for (int q = 0; q < K; q++) out[q] = res[c[q]];
    return r;
}

// This thread's cells and their dphi1 values.
template <int NX, int TH, typename CT>
__device__ __forceinline__ void relax_cells(int lt, const CT* __restrict__ dphi1, int* c, CT* d1) {
    constexpr int K = NX * NX * NX / TH;
#pragma unroll
    for (int r = 0; r < K; r++) {
        c[r] = relax_cell<NX>(lt + r * TH);
        d1[r] = dphi1[c[r]];
    }
}

// Stages the brick (dphi with ghosts) into both buffers.
template <int NX, int TH, typename CT>
__device__ __forceinline__ void relax_stage(RelaxSmem<NX, CT>& sm, const CT* __restrict__ dphi, int lt) {
    constexpr int P3 = RelaxSmem<NX, CT>::P3;
    for (int q = lt; q < P3; q += TH) {
        const CT v = dphi[q];
        sm.buf[0][q] = v;
        sm.buf[1][q] = v;
    }
}

// Stages the brick and relaxes it: returns the last sweep's sum and leaves
// the relaxed interior values of this thread's cells c[r] in out[r].  CT is
// the correction's storage and arithmetic type (FP64, or FP32 in the mixed
// form); the sums of squares are formed in FP64 either way.
template <int NX, int TH, typename CT, typename Sync>
__device__ __forceinline__ double relax_brick(RelaxSmem<NX, CT>& sm, const CT* __restrict__ dphi,
                                              const CT* __restrict__ dphi1, int lt, int* c, CT* out, Sync sync) {
    constexpr int K = NX * NX * NX / TH;
    relax_stage<NX, TH, CT>(sm, dphi, lt);
    CT d1[K];
    relax_cells<NX, TH, CT>(lt, dphi1, c, d1);
    sync();
    return relax_sweeps<NX, TH, CT>(sm, lt, c, d1, out, sync);
}

}  // namespace amr
