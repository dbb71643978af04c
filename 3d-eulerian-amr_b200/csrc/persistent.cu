// Persistent multigrid solve: the whole V-cycle loop of Poisson::solve (the
// drivers' `while (err > toler) vcycle()`, binary_driver.cpp:296-330) in one
// cooperative launch.  Every dependent step of the reference's sequence --
// restriction of phi level by level, the phi ghost faces / edges / vertices
// of each level, the down sweep (vcycle_down + relax_until(1.0)) and the up
// sweep (coarse correction, relax_until(0.05), retire, ghosts) of each
// level, the forces with their coarse-fine averages, the L1 error -- is a
// phase separated from the next by a grid barrier instead of a kernel
// boundary.  The phases run the same device functions as the
// one-launch-per-step kernels (poisson_ops.cuh, graph_ops.cuh), so the
// result is bitwise that of the plain and graph forms.
//
// Loop decisions (relaxation ratio, L1 error > tol) need the reference's
// nested sums over the per-brick values; every block forms them itself, in
// its own scratch, from the same values, so all blocks take the same
// decision without another barrier.  Per-brick values are double-buffered
// by pass so a block still summing one pass cannot see the next pass's.
//
// The grid barrier spins with a bound: a block that waits longer than the
// control block's wait limit (BARRIER_SPINS polls by default) sets the
// abort word, every block leaves at its next barrier, and the host reports
// AMR_ERR_TIMEOUT.
#include <cuda_runtime.h>

#include "graph_ops.cuh"
#include "launch.cuh"
#include "persistent.h"
#include "poisson_ops.cuh"

namespace amr {

namespace {

constexpr unsigned long long BARRIER_SPINS = 1ull << 22;

__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

// Grid-wide barrier of a cooperative launch; false when the solve aborted.
// The arrival counter only grows: barrier k of the launch completes when it
// reaches k * gridDim.x (target, kept by thread 0), so an arrival is one
// fire-and-forget release add and the wait one acquire load per poll.
// A block whose wait runs out sets the abort word and records status 3
// (AMR_ERR_TIMEOUT) in the control block itself, so the timeout is reported
// whichever block meets it and whatever the other solves of a captured step
// record after it (statuses only grow).
__device__ __forceinline__ void give_up(GridBarrier* bar, int* status) {
    atomicExch(&bar->abort, 1);
    atomicMax(status, 3);
}

__device__ __forceinline__ bool grid_sync(GridBarrier* bar, unsigned& target, unsigned long long limit, int* status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        target += gridDim.x;
        // the release orders the whole block's writes (made before the block
        // barrier above) before the arrival, at GPU scope
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(&bar->count), "r"(1u) : "memory");
        unsigned long long spins = 0;
        for (;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&bar->count) : "memory");
            if ((int)(v - target) >= 0) break;
            if ((spins & 63) == 63 && ld_volatile(&bar->abort)) {
                good = 0;
                break;
            }
            if (++spins > limit) {
                give_up(bar, status);
                good = 0;
                break;
            }
            if (spins > 32) __nanosleep(20);
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Level-sum mailbox.  The publishing block's thread 0 stores sum g, then
// releases lsum_gen = g; readers acquire lsum_gen until it reaches g (the
// generations of a launch are 1, 2, ...; a reader waiting for g never sees
// g + 1, which is published only after a grid barrier the reader has not
// reached yet).  lsum_wait is called by every thread of a block and returns
// the sum in all of them; false when the solve aborted.
__device__ __forceinline__ void lsum_publish(GridBarrier* bar, unsigned g, double r) {
    __stcg(&bar->lsum_val[g & 1], r);
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&bar->lsum_gen), "r"(g) : "memory");
}

__device__ __forceinline__ bool lsum_wait(GridBarrier* bar, unsigned g, double& r, unsigned long long limit,
                                          int* status) {
    __shared__ double s_r;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int good = 1;
        unsigned long long spins = 0;
        for (;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&bar->lsum_gen) : "memory");
            if ((int)(v - g) >= 0) break;
            if ((spins & 63) == 63 && ld_volatile(&bar->abort)) {
                good = 0;
                break;
            }
            if (++spins > limit) {
                give_up(bar, status);
                good = 0;
                break;
            }
            if (spins > 32) __nanosleep(20);
        }
        s_r = good ? __ldcg(&bar->lsum_val[g & 1]) : 0.0;
        s_ok = good;
    }
    __syncthreads();
    r = s_r;
    return s_ok != 0;
}

// Block layout of the solve for bricks of NX^3 interior cells: TPB threads
// per block, NX^3 / TPB cells per thread in the relaxation (every layout
// gives the same results bit for bit).  With 8^3 bricks and 512 threads a
// block relaxes two bricks at once (one per half) on levels with more
// bricks than blocks, so it holds two staged bricks; the other layouts take
// such levels brick by brick.  With 12^3 bricks the FP32 correction's launch
// holds two bricks' buffers, so that levels of up to twice as many bricks as
// worker blocks stay in the shared-memory relaxation loop.  MINB: blocks per
// SM the registers are budgeted for.
template <int NX, int TPB_>
struct SolveLayout {
    static constexpr int TPB = TPB_;
    static constexpr bool HALVES = NX == 8 && TPB == 512;
    static constexpr int NSM = HALVES ? 2 : 1;
    // FP32 corrections of 12^3 bricks: three more brick buffers, for a
    // second brick per block in the shared-memory relaxation loop
    static constexpr bool RES2 = NX == 12;
    static_assert(!RES2 || NSM == 1, "the extra buffers follow the third brick buffer");
    static constexpr int MINB = TPB >= 864 ? 1 : (TPB > 288 ? 2 : (TPB > 256 ? 3 : 4));
    // threads per face in the face-ghost phases
    static constexpr int PF = NX * NX <= TPB / 6 ? NX * NX : TPB / 6;
};

template <int NX, int TPB_, typename CT>
struct Solver {
    using Lay = SolveLayout<NX, TPB_>;
    static constexpr int TPB = Lay::TPB;
    const SolveArgs& a;
    RelaxSmem<NX, CT>* sm;  // Lay::NSM staged bricks
    CT* xbuf;               // a third brick buffer of (NX+2)^3 entries
    double* red;
    double* nbuf;    // 2 * NEST_SMEM doubles of shared memory for the level sums
    double* nest;    // this block's scratch [cap] (level sums of larger trees)
    int relax_par;   // pres buffer of the next relaxation pass
    int status;
    long long relax_calls;
    int max_outer;
    unsigned bar_target = 0;    // thread 0: arrivals that complete the next barrier
    unsigned lsum_gen = 0;      // level sums published so far in this launch
    unsigned pass_seq = 0;      // last pass word used by the shared-memory relaxation loops
    unsigned long long spin_limit = BARRIER_SPINS;  // polls per bounded wait
    unsigned long long t_last;  // block 0: global time at the last barrier exit
    // block 0's phase accounting, in shared memory
    unsigned long long* ph_ns;
    unsigned* ph_n;
    double* ph_bytes;
    unsigned long long* ph_wait;  // [PH_COUNT], then level-sum time and count
    unsigned* lvl_n;              // relaxation passes per level
    unsigned long long* lvl_ns;   // block 0's time in each level's relaxation loops
    unsigned long long* rsplit;   // block 0: the resident loops' time split [4], passes, sweeps
    unsigned mbar = 0;            // shared-memory address of the staging mbarrier (bulk copies)
    unsigned mbar_parity = 0;     // phase parity of its next completion (the same in every thread)

    __device__ static unsigned long long now() {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }

    // barrier closing a phase of class ph
    __device__ bool sync(int ph, int units) {
        const unsigned long long t_arrive = (blockIdx.x == 0 && threadIdx.x == 0) ? now() : 0;
        const bool ok = grid_sync(a.bar, bar_target, spin_limit, &a.ctl->status);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = now();
            ph_wait[ph] += t - t_arrive;
            ph_ns[ph] += t - t_last;
            ph_n[ph]++;
            ph_bytes[ph] += (double)units * phase_bytes(ph);
            t_last = t;
        }
        return ok;
    }

    // Algorithmic HBM bytes of one unit (brick, parent or coarse-fine item)
    // of a phase: the arrays the phase must read and write once, at their
    // storage width (the correction dphi, dphi1 in CT).
    __device__ static double phase_bytes(int ph) {
        constexpr double PNX = NX + 2, H = NX / 2, C = sizeof(CT);
        switch (ph) {
            case PH_SOURCE: return 16 * PNX * PNX * PNX;                                  // rho -> S
            case PH_RESTRICT: return 8 * (8 * PNX * PNX * PNX + 8 * H * H * H);           // 8 children -> parent
            case PH_PHI_FACES: return 16 * 6 * NX * NX;                                   // source cell -> ghost
            case PH_PHI_EDGES: return 16 * 12 * NX;
            case PH_PHI_VERTICES: return 16 * 8;
            case PH_INIT: return 2 * C * PNX * PNX * PNX;                                 // dphi, dphi1 = 0
            case PH_VDOWN: return 8 * (PNX * PNX * PNX + NX * NX * NX) + 2 * C * NX * NX * NX;  // phi, S -> dphi, dphi1
            case PH_DPHI_FACES: return 2 * C * 6 * NX * NX;
            case PH_RELAX_FIRST:
            case PH_RELAX: return C * (PNX * PNX * PNX + 2 * NX * NX * NX + 12 * NX * NX);  // dphi, dphi1 -> dphi, layers
            case PH_CORRECT: return C * (2 * NX * NX * NX + H * H * H);
            case PH_RETIRE: return (16 + C) * NX * NX * NX;                               // phi += dphi
            case PH_FORCES: return 8 * (PNX * PNX * PNX + 3 * (PNX - 1) * (PNX - 1) * (PNX - 1));
            case PH_ADJUST_FORCE: return 8 * 5 * H * H;
            case PH_ERROR: return 8 * (3 * PNX * PNX * PNX + NX * NX * NX) + C * NX * NX * NX;
            default: return 0;
        }
    }

    // this block's share of n items
    template <typename F>
    __device__ void each(int n, F f) {
        for (int q = blockIdx.x; q < n; q += gridDim.x) f(q);
    }

    // one relaxation pass over the n bricks sl[]: one brick per block, or
    // (8^3 bricks) two per block, one per half with two cells per thread,
    // when the level has more bricks than there are blocks; the results are
    // the same either way
    __device__ void relax_pass(const int* sl, int n, int mode, const CT* rd, CT* wr, double* pres) {
        if (!Lay::HALVES || n <= (int)gridDim.x) {
            each(n, [&](int q) {
                op_relax_pass<NX, TPB, CT>(a.g, a.bt, a.st, sl[q], mode, rd, wr, a.stride, pres, sm[0], threadIdx.x,
                                           BlockSync{});
                __syncthreads();
            });
        } else if constexpr (Lay::HALVES) {
            constexpr int HT = TPB / 2;
            const int h = threadIdx.x / HT, lt = threadIdx.x % HT;
            for (int q = 2 * blockIdx.x + h; q < n; q += 2 * gridDim.x) {
                op_relax_pass<NX, HT, CT>(a.g, a.bt, a.st, sl[q], mode, rd, wr, a.stride, pres, sm[h & 1], lt,
                                          NamedSync{1 + h, HT});
                named_sync(1 + h, HT);
            }
        }
    }

    __device__ const int* level(int l) const { return a.L.slots + a.L.off[l]; }

    // enforce_phi_boundaries of one level: faces, then edges (reading the
    // neighbours' face ghosts), then vertices (reading their edge ghosts)
    __device__ bool phi_boundaries(int l) {
        const int* sl = level(l);
        const int n = a.L.cnt[l];
        const int t = threadIdx.x;
        constexpr int PF = Lay::PF;
        each(n, [&](int q) {
            if (t < 6 * PF) op_phi_faces(a.g, a.bt, a.st, a.aux, sl[q], t / PF, t % PF, PF);
        });
        if (!sync(PH_PHI_FACES, n)) return false;
        const int m = a.g.pnx - 2;
        each(n, [&](int q) {
            if (t < 12 * m) op_phi_edge(a.g, a.bt, a.st, a.aux, sl[q], t / m, t % m + 1);
        });
        if (!sync(PH_PHI_EDGES, n)) return false;
        each(n, [&](int q) {
            if (t < 8) op_phi_vertex(a.g, a.bt, a.st, a.aux, sl[q], t);
        });
        return sync(PH_PHI_VERTICES, n);
    }

    // Poisson::vcycle_relax sum over level l (poisson.cpp:107, nested as the
    // recursion adds it) from buffer `buf` of the per-brick sums
    __device__ double level_sum(int l, const double* buf) {
        const unsigned long long t0 = (blockIdx.x == 0 && threadIdx.x == 0) ? now() : 0;
        double r;
        if (l == 0) {
            r = __ldcg(buf + a.L.slots[a.L.off[0]]);
        } else {
            __syncthreads();
            if (a.L.max_cnt <= NEST_SMEM)
                r = nested_sum_smem(a.L, buf, l, false, nbuf);
            else
                r = nested_sum_block(a.L, a.bt.child, buf, nest, l, false);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ph_wait[PH_COUNT] += now() - t0;
            ph_wait[PH_COUNT + 1]++;
        }
        return r;
    }

    __device__ void count_pass(int l) {
        relax_calls++;
        if (blockIdx.x == 0 && threadIdx.x == 0) lvl_n[l]++;
    }

    // the level sum published as generation lsum_gen (block 0 records the
    // time it waits for it)
    __device__ bool wait_sum(double& r) {
        const unsigned long long t0 = (blockIdx.x == 0 && threadIdx.x == 0) ? now() : 0;
        bool ok;
        if constexpr (TAGGED) {
            // the two tagged halves: each carries the generation it belongs
            // to, so a half of an older sum is never taken for this one
            __shared__ double s_r;
            __shared__ int s_ok;
            if (threadIdx.x == 0) {
                CT hi, lo;
                const int good = tagged_get2(a.bar->lsum_tag, lsum_gen, hi, lo);
                s_r = good ? join_halves(hi, lo) : 0.0;
                s_ok = good;
            }
            __syncthreads();
            r = s_r;
            ok = s_ok != 0;
        } else {
            ok = lsum_wait(a.bar, lsum_gen, r, spin_limit, &a.ctl->status);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ph_wait[PH_COUNT] += now() - t0;
            ph_wait[PH_COUNT + 1]++;
        }
        return ok;
    }

    // relax_until (poisson.cpp:66-70, 74-78): ghosts, one pass, then passes
    // with ghosts from the previous pass's snapshot until the level sum has
    // fallen to `ratio` of the first
    __device__ bool relax_until(int l, double ratio) {
        const unsigned long long t0 = (blockIdx.x == 0 && threadIdx.x == 0) ? now() : 0;
        const bool ok = relax_until_(l, ratio);
        if (blockIdx.x == 0 && threadIdx.x == 0) lvl_ns[l] += now() - t0;
        return ok;
    }
    __device__ bool relax_until_(int l, double ratio) {
        const int* sl = level(l);
        const int n = a.L.cnt[l];
        const int t = threadIdx.x;
        CT* snap = reinterpret_cast<CT*>(a.snap);
        constexpr int PF = Lay::PF;
        each(n, [&](int q) {
            if (t < 6 * PF) op_dphi_faces<CT>(a.g, a.bt, a.st, a.aux, sl[q], t / PF, t % PF, PF);
        });
        if (!sync(PH_DPHI_FACES, n)) return false;
        if (n <= (RES2 ? 2 * ((int)gridDim.x - 1) : (int)gridDim.x)) return relax_loop_resident(l, ratio, sl, n, snap);
        int par = 0;
        double* pres = a.pres + (size_t)relax_par * a.L.cap;
        relax_pass(sl, n, 0, snap, snap, pres);
        if (!sync(PH_RELAX_FIRST, n)) return false;
        const double r0 = level_sum(l, pres);
        relax_par ^= 1;
        relax_calls++;
        if (blockIdx.x == 0 && threadIdx.x == 0) lvl_n[l]++;
        int outer = 0;
        for (;;) {
            pres = a.pres + (size_t)relax_par * a.L.cap;
            const CT* rd = snap + (size_t)par * a.snap_half;
            CT* wr = snap + (size_t)(par ^ 1) * a.snap_half;
            relax_pass(sl, n, 1, rd, wr, pres);
            if (!sync(PH_RELAX, n)) return false;
            par ^= 1;
            const double r = level_sum(l, pres);
            relax_par ^= 1;
            relax_calls++;
            if (blockIdx.x == 0 && threadIdx.x == 0) lvl_n[l]++;
            ++outer;
            bool again = r / r0 > ratio;
            if (again && outer > max_outer) {
                again = false;
                status = 1;
            }
            if (!again) break;
        }
        return true;
    }

    // Thread 0 of lanes: waits until the word at p reaches target (acquire);
    // false when the solve aborted or the wait ran out.
    __device__ bool wait_word(const unsigned* p, unsigned target) {
        unsigned long long spins = 0;
        for (;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
            if ((int)(v - target) >= 0) return true;
            if ((spins & 63) == 63 && ld_volatile(&a.bar->abort)) return false;
            if (++spins > spin_limit) {
                give_up(a.bar, &a.ctl->status);
                return false;
            }
            if (spins > 32) __nanosleep(20);
        }
    }

    // Waits (lanes 0-5 of warp 0, one per face) until brick b's same-level
    // neighbours have published pass `seq`; every thread then sees their
    // snapshot layers.
    __device__ bool wait_neighbours(int b, unsigned seq) {
        __shared__ int s_ok;
        if (threadIdx.x < 32) {
            int good = 1;
            const int f = threadIdx.x;
            if (f < 6 && a.bt.ftype[6 * b + f] == FACE_SIB) good = wait_word(a.rpub + a.bt.fnbr[6 * b + f], seq);
            good = __all_sync(0xffffffffu, good);
            if (threadIdx.x == 0) s_ok = good;
        }
        __syncthreads();
        return s_ok != 0;
    }

    // The FP32 correction publishes its face layers as tagged entries (each
    // value with its pass word in one 64-bit store, tagged_put): a neighbour
    // waits on the very values it reads, so a pass needs neither a block
    // barrier nor a release fence before its layers are visible, nor a
    // separate pass word.  The FP64 correction has no room for a tag in a
    // 64-bit store and publishes through the pass words.
    static constexpr bool TAGGED = sizeof(CT) == 4;
    // the launch holds a second brick's three buffers after xbuf, so the
    // shared-memory loop takes levels of up to two bricks per worker block
    static constexpr bool RES2 = Lay::RES2 && TAGGED;
    // snapshot buffer p of tagged entries (their own allocation, zeroed
    // before every launch; pass words start at 1)
    __device__ unsigned long long* tagged_snap(int p) const { return a.tsnap + (size_t)p * a.snap_half; }

    // Publishes the relaxed brick `res` as a pass: its first interior layers
    // to snapshot buffer `wpar`, its sum to pres[b] (tagged: both as tagged
    // entries; untagged: then brick b's pass word is released as `seq`).
    __device__ void resident_publish(int b, const CT* res, const int* c, int wpar, double* pres, double resid,
                                     unsigned seq) {
        constexpr int K = NX * NX * NX / TPB;
        if constexpr (TAGGED) {
            unsigned long long* sw = tagged_snap(wpar) + (size_t)b * a.stride;
            // the layers a same-level neighbour reads (the other faces' ghosts
            // come from the parent, the mirror or the outflow value)
            unsigned sib = 0;
#pragma unroll
            for (int f = 0; f < 6; f++) sib |= a.bt.ftype[6 * b + f] == FACE_SIB ? 1u << f : 0u;
#pragma unroll
            for (int r = 0; r < K; r++)
                relax_layer_put_tagged<NX>(sw, threadIdx.x + r * TPB, float(res[c[r]]), seq, sib);
            if (threadIdx.x == 0) {
                // the FP64 sum as two tagged halves (pres buffer of this pass)
                const int pp = (int)((pres - a.pres) / a.L.cap);
                unsigned long long* w = a.tpres + ((size_t)pp * a.L.cap + b) * 2;
                const unsigned long long bits = (unsigned long long)__double_as_longlong(resid);
                tagged_put(w, __uint_as_float((unsigned)(bits >> 32)), seq);
                tagged_put(w + 1, __uint_as_float((unsigned)bits), seq);
            }
        } else {
            CT* sw = reinterpret_cast<CT*>(a.snap) + (size_t)wpar * a.snap_half + (size_t)b * a.stride;
#pragma unroll
            for (int r = 0; r < K; r++) relax_layer_put<NX, CT>(sw, threadIdx.x + r * TPB, res[c[r]]);
            if (threadIdx.x == 0) pres[b] = resid;
            __syncthreads();
            if (threadIdx.x == 0)
                asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.rpub + b), "r"(seq) : "memory");
        }
    }

    // Two adjacent tagged entries (the halves of an FP64 value): waits until
    // both carry pass word `tag`, loading the two together in every poll.
    __device__ bool tagged_get2(const unsigned long long* p, unsigned tag, CT& hi, CT& lo) {
        unsigned long long spins = 0;
        for (;;) {
            unsigned long long w0, w1;
            asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w0) : "l"(p) : "memory");
            asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w1) : "l"(p + 1) : "memory");
            if ((unsigned)(w0 >> 32) == tag && (unsigned)(w1 >> 32) == tag) {
                hi = CT(__uint_as_float((unsigned)w0));
                lo = CT(__uint_as_float((unsigned)w1));
                return true;
            }
            if ((spins & 63) == 63 && ld_volatile(&a.bar->abort)) return false;
            if (++spins > spin_limit) {
                give_up(a.bar, &a.ctl->status);
                return false;
            }
            if (spins > 8) __nanosleep(20);
        }
    }

    // The FP64 value whose high and low 32 bits were sent as the bit
    // patterns of two tagged FP32 entries.
    __device__ static double join_halves(CT hi, CT lo) {
        const unsigned long long bits = ((unsigned long long)__float_as_uint(float(hi)) << 32) |
                                        __float_as_uint(float(lo));
        return __longlong_as_double((long long)bits);
    }

    // A same-level neighbour's tagged layer value: waits until the entry
    // carries pass word `tag`; false when the solve aborted or the wait ran
    // out.
    __device__ bool tagged_get(const unsigned long long* p, unsigned tag, CT& v) {
        unsigned long long spins = 0;
        for (;;) {
            unsigned long long w;
            asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
            if ((unsigned)(w >> 32) == tag) {
                v = CT(__uint_as_float((unsigned)w));
                return true;
            }
            if ((spins & 63) == 63 && ld_volatile(&a.bar->abort)) return false;
            if (++spins > spin_limit) {
                give_up(a.bar, &a.ctl->status);
                return false;
            }
            if (spins > 8) __nanosleep(20);
        }
    }

    // One pass of brick b from its committed values in `base`, ghost faces
    // from snapshot `rd` (the parent across coarse-fine faces, the mirror of
    // `base` across z = 0, 0 on outflow faces), swept in x and y; nothing is
    // written outside shared memory.  Returns the sum and the buffer with the
    // relaxed brick (x or y).
    __device__ double resident_pass(int b, CT* base, CT* x, CT* y, int rpar, unsigned want, const int* c,
                                    const CT* d1, CT** res, bool& ok) {
        constexpr int K = NX * NX * NX / TPB, F = NX * NX;
#pragma unroll
        for (int r = 0; r < K; r++) x[c[r]] = base[c[r]];
        const CT* rd = reinterpret_cast<const CT*>(a.snap) + (size_t)rpar * a.snap_half;
        int bad = 0;
        for (int q = threadIdx.x; q < 6 * F; q += TPB) {
            int face, t1, t2;
            const int gi = relax_ghost_cell<NX>(q, face, t1, t2);
            CT v;
            if (TAGGED && a.bt.ftype[6 * b + face] == FACE_SIB) {
                const int nbr = a.bt.fnbr[6 * b + face];
                const unsigned long long* p =
                    tagged_snap(rpar) + (size_t)nbr * a.stride + layer_entry<NX>(face ^ 1, t1, t2);
                if (!tagged_get(p, want, v)) {
                    bad = 1;
                    v = CT(0);
                }
            } else {
                v = ghost_dphi<NX, CT>(a.g, a.bt, a.st, rd, a.stride, b, face, t1, t2, base);
            }
            x[gi] = v;
            y[gi] = v;
        }
        ok = !__syncthreads_or(bad);
        if (!ok) return 0.0;
        int sw;
        const double r = relax_sweeps_in<NX, TPB, CT>(x, y, &sm[0].red[0][0], threadIdx.x, c, d1, res, BlockSync{}, &sw);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            rsplit[4]++;
            rsplit[5] += sw;
        }
        return r;
    }

    // Waits (every thread) until the staging mbarrier completes its current
    // phase; false when the wait ran out (the solve is then aborted, and
    // the wait goes on, again bounded, so that no copy is still landing in
    // shared memory when the block leaves).
    __device__ bool wait_staged() {
        unsigned long long spins = 0;
        bool ok = true;
        for (;;) {
            unsigned done;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(mbar), "r"(mbar_parity)
                : "memory");
            if (done) break;
            if (++spins > spin_limit) {
                if (!ok) break;
                ok = false;
                spins = 0;
                if (threadIdx.x == 0) give_up(a.bar, &a.ctl->status);
            }
        }
        mbar_parity ^= 1;
        return ok;
    }

    // Brick b's (NX+2)^3 correction values from dphi into the two sweep
    // buffers x and y: two bulk copies (the TMA engine, from this GPU's own
    // memory, no multicast) issued by one thread and completed on the
    // staging mbarrier, so the other threads load their dphi1 meanwhile.
    // A brick is one contiguous block of P3 values whose size is a multiple
    // of 16 bytes; where an address is not 16-byte aligned (never for the
    // slot pool and the shared buffers, but checked) plain loads stage it.
    // Returns whether bulk copies were issued (then wait_staged follows).
    __device__ bool stage_brick(const CT* D, CT* x, CT* y) {
        constexpr int P3 = (NX + 2) * (NX + 2) * (NX + 2);
        constexpr unsigned BYTES = P3 * sizeof(CT);
        static_assert(BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
        const bool aligned = ((reinterpret_cast<size_t>(D) | reinterpret_cast<size_t>(x) |
                               reinterpret_cast<size_t>(y)) & 15) == 0;
        if (!aligned) {
            for (int q = threadIdx.x; q < P3; q += TPB) {
                const CT v = D[q];
                x[q] = v;
                y[q] = v;
            }
            return false;
        }
        // the buffers' last generic uses are over before the copies start
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned xs = (unsigned)__cvta_generic_to_shared(x);
            const unsigned ys = (unsigned)__cvta_generic_to_shared(y);
            // order this block's generic accesses (and, through the grid
            // barrier before, the other blocks' writes of dphi) before the
            // copies of the async proxy
            asm volatile("fence.proxy.async;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(2 * BYTES)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(xs),
                "l"(D), "r"(BYTES), "r"(mbar)
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(ys),
                "l"(D), "r"(BYTES), "r"(mbar)
                : "memory");
        }
        return true;
    }

    // block 0, thread 0: adds the time since *t to split s and restarts *t
    __device__ void split(int s, unsigned long long& t) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long u = now();
            rsplit[s] += u - t;
            t = u;
        }
    }

    // The server's part of a pass: waits until every brick of the level has
    // published pass word `tag`, forms the level sum of `done` (that pass's
    // sums) and publishes it as generation lsum_gen.  The wait is per brick:
    // pass 1 goes out before the sum of pass 0 is known, so a count of the
    // level's publications could be complete for pass 0 while a slow
    // brick's pass 0 is still missing and a fast one's pass 1 is in.
    __device__ bool serve_sum(int l, const double* done, unsigned tag) {
        if constexpr (TAGGED) {
            // the bricks' tagged sums of this pass: wait on each and take it
            // straight into the shared buffer of the nested sum (or, for a
            // level too large for it, write it back whole to the pres
            // buffer the level sum reads); the sum goes out as two tagged
            // halves, so neither side needs a fence or a flag
            const int* sl = level(l);
            const int n = a.L.cnt[l];
            const int pp = (int)((done - a.pres) / a.L.cap);
            const bool in_smem = a.L.max_cnt <= NEST_SMEM;
            int bad = 0;
            for (int q = threadIdx.x; q < n; q += TPB) {
                const int b = sl[q];
                const unsigned long long* w = a.tpres + ((size_t)pp * a.L.cap + b) * 2;
                CT hi, lo;
                if (!tagged_get2(w, tag, hi, lo)) {
                    bad = 1;
                    continue;
                }
                if (in_smem)
                    nbuf[q] = join_halves(hi, lo);
                else
                    const_cast<double*>(done)[b] = join_halves(hi, lo);
            }
            if (__syncthreads_or(bad)) return false;
            const double r = !in_smem ? level_sum(l, done) : l == 0 ? nbuf[0] : nested_sum_smem_in(a.L, done, l, false, nbuf);
            if (threadIdx.x == 0) {
                const unsigned long long bits = (unsigned long long)__double_as_longlong(r);
                tagged_put(&a.bar->lsum_tag[0], __uint_as_float((unsigned)(bits >> 32)), lsum_gen);
                tagged_put(&a.bar->lsum_tag[1], __uint_as_float((unsigned)bits), lsum_gen);
            }
            // the shared buffer is read again by the next pass's sum
            __syncthreads();
            return true;
        } else {
            // the bricks' pass words (a brick one pass further has put that
            // pass's sum in the other buffer, so `done` is intact)
            const int* sl = level(l);
            const int n = a.L.cnt[l];
            int bad = 0;
            for (int q = threadIdx.x; q < n; q += TPB)
                if (!wait_word(a.rpub + sl[q], tag)) bad = 1;
            if (__syncthreads_or(bad)) return false;
            const double r = level_sum(l, done);
            if (threadIdx.x == 0) lsum_publish(a.bar, lsum_gen, r);
            return true;
        }
    }

    // Brick buffer i (0..2) of the shared-memory loop's brick j (0, 1).
    __device__ CT* resident_buf(int j, int i) const {
        constexpr int P3 = (NX + 2) * (NX + 2) * (NX + 2);
        if (RES2 && j) return xbuf + (size_t)(1 + i) * P3;
        return i == 0 ? sm[0].buf[0] : i == 1 ? sm[0].buf[1] : xbuf;
    }

    // The relaxation loop of a level the blocks can hold in shared memory:
    // one brick per block, the last block (the server) forming the level
    // sums; or, where the level has more bricks than blocks and the launch
    // holds a second set of brick buffers (RES2), two bricks in the first
    // worker blocks and none in the server.  The bricks stay in shared
    // memory for the whole loop.  No grid barrier between passes: a brick
    // waits only for its same-level neighbours' published face layers,
    // computes the next pass from shared memory while the server forms the
    // last pass's nested sum, and publishes it (snapshot layers, sum, pass
    // word) once the sum says the loop goes on -- else the pass is dropped.
    // A block with two bricks takes them one after the other in every pass;
    // a server with a brick (as many bricks as blocks) forms the sum first,
    // then its pass, so its brick trails the others by the sum's latency --
    // a smaller delay than a second brick in one block.  The loop ends with
    // one write of each brick (interior and ghost faces) back to dphi and
    // one grid barrier.  Passes written, their values, the sums and every
    // loop decision are those of the loop in relax_until.
    __device__ bool relax_loop_resident(int l, double ratio, const int* sl, int n, CT* snap) {
        constexpr int NB = RES2 ? 2 : 1;
        constexpr int K = NX * NX * NX / TPB, P3 = (NX + 2) * (NX + 2) * (NX + 2), F = NX * NX;
        const int W = (int)gridDim.x - 1;
        const bool server = (int)blockIdx.x == W;
        // this block's bricks: slot blockIdx.x (the server's too when the
        // level has as many bricks as blocks), and slot blockIdx.x + W in
        // the worker blocks when it has more (-1: none)
        const bool two = n > (int)gridDim.x;
        const int b0 = (int)blockIdx.x < n && !(two && server) ? sl[blockIdx.x] : -1;
        const int b1 = RES2 && two && !server && (int)blockIdx.x + W < n ? sl[blockIdx.x + W] : -1;
        const bool mine = b0 >= 0;
        // three buffers per brick (resident_buf): its committed values (ib0,
        // ib1) and two to sweep in.  The brick loops below are not unrolled;
        // a brick's values are picked by selects so they stay in registers.
        int ib0 = 0, ib1 = 0;
        int c[K];
        CT d1a[K], d1b[K];
        const unsigned seq0 = pass_seq + 1;  // pass word of pass 0
        if (!mine && !server) {
            // a block without a brick has no part in the loop: it goes to
            // the closing barrier (one polled word instead of the loop's
            // published sums) and takes the loop's length from the server,
            // which stores it before it arrives there
            if (!sync(PH_RELAX, 0)) return false;
            const unsigned k = *(volatile const unsigned*)&a.bar->relax_done_k;
            relax_par ^= (1 + k) & 1;
            lsum_gen += 1 + k;
            relax_calls += k + 1;
            pass_seq = seq0 + k;
            return true;
        }
        double* pres = a.pres + (size_t)relax_par * a.L.cap;
#pragma unroll 1
        for (int j = 0; j < NB; j++) {
            const int b = j ? b1 : b0;
            if (b < 0) continue;
            // pass 0: the ghost faces are in dphi (filled by the face phase);
            // the brick is staged by bulk copies while dphi1 is loaded
            const CT* D = Corr<CT>::dphi(a.st) + (size_t)b * P3;
            CT* x = resident_buf(j, 0);
            CT* y = resident_buf(j, 1);
            const bool bulk = stage_brick(D, x, y);
            CT d1[K];
            relax_cells<NX, TPB, CT>(threadIdx.x, Corr<CT>::dphi1(a.st) + (size_t)b * P3, c, d1);
#pragma unroll
            for (int r = 0; r < K; r++) {
                if (j) d1b[r] = d1[r];
                else d1a[r] = d1[r];
            }
            if (bulk && !wait_staged()) return false;
            __syncthreads();
            CT* res;
            const double rs = relax_sweeps_in<NX, TPB, CT>(x, y, &sm[0].red[0][0], threadIdx.x, c, d1, &res,
                                                           BlockSync{});
            const int i = res == x ? 0 : 1;
            if (j) ib1 = i;
            else ib0 = i;
            resident_publish(b, res, c, 0, pres, rs, seq0);
        }
        count_pass(l);
        // One pass of brick j from its committed buffer, the neighbours'
        // layers of pass `want` in snapshot buffer `rpar`: the sum, and in
        // *ri the buffer that holds the result.
        auto pass = [&](int j, int rpar, unsigned want, int* ri, bool& ok) -> double {
            const int b = j ? b1 : b0;
            const int i = j ? ib1 : ib0;
            CT d1[K];
#pragma unroll
            for (int r = 0; r < K; r++) d1[r] = j ? d1b[r] : d1a[r];
            CT* x = resident_buf(j, (i + 1) % 3);
            CT* res;
            const double rs = resident_pass(b, resident_buf(j, i), x, resident_buf(j, (i + 2) % 3), rpar, want, c,
                                            d1, &res, ok);
            *ri = res == x ? (i + 1) % 3 : (i + 2) % 3;
            return rs;
        };
        // pass 1 runs whatever the first sum; that sum is formed meanwhile
        double r0;
        {
            const double* done = pres;
            relax_par ^= 1;
            pres = a.pres + (size_t)relax_par * a.L.cap;
            ++lsum_gen;
            if (server && !serve_sum(l, done, seq0)) return false;
#pragma unroll 1
            for (int j = 0; j < NB; j++) {
                const int b = j ? b1 : b0;
                if (b < 0) continue;
                if (!TAGGED && !wait_neighbours(b, seq0)) return false;
                bool ok;
                int ri;
                const double rs = pass(j, 0, seq0, &ri, ok);
                if (!ok) return false;
                if (j) ib1 = ri;
                else ib0 = ri;
                resident_publish(b, resident_buf(j, ri), c, 1, pres, rs, seq0 + 1);
            }
            if (!wait_sum(r0)) return false;
            count_pass(l);
        }
        int par = 1;         // snapshot buffer written by the last published pass
        unsigned k = 1;      // last published pass
        int outer = 1;
        for (;;) {
            const double* done = pres;
            relax_par ^= 1;
            pres = a.pres + (size_t)relax_par * a.L.cap;
            ++lsum_gen;
            if (server && !serve_sum(l, done, seq0 + k)) return false;
            // this pass of each brick, held until the sum of the last one
            // decides whether it is published
            int ri0 = 0, ri1 = 0;
            double rr0 = 0.0, rr1 = 0.0;
            unsigned long long tt = (blockIdx.x == 0 && threadIdx.x == 0) ? now() : 0;
#pragma unroll 1
            for (int j = 0; j < NB; j++) {
                const int b = j ? b1 : b0;
                if (b < 0) continue;
                if (!TAGGED && !wait_neighbours(b, seq0 + k)) return false;
                split(0, tt);
                bool ok;
                int ri;
                const double rs = pass(j, par, seq0 + k, &ri, ok);
                if (!ok) return false;
                if (j) {
                    ri1 = ri;
                    rr1 = rs;
                } else {
                    ri0 = ri;
                    rr0 = rs;
                }
                split(1, tt);
            }
            double r;
            if (!wait_sum(r)) return false;
            split(2, tt);
            bool again = r / r0 > ratio;
            if (again && outer > max_outer) {
                again = false;
                status = 1;
            }
            if (!again) break;
            if (mine) {
                ib0 = ri0;
                resident_publish(b0, resident_buf(0, ib0), c, par ^ 1, pres, rr0, seq0 + k + 1);
            }
            if (b1 >= 0) {
                ib1 = ri1;
                resident_publish(b1, resident_buf(1, ib1), c, par ^ 1, pres, rr1, seq0 + k + 1);
            }
            split(3, tt);
            par ^= 1;
            ++k;
            count_pass(l);
            ++outer;
        }
#pragma unroll 1
        for (int j = 0; j < NB; j++) {
            const int b = j ? b1 : b0;
            if (b < 0) continue;
            // the committed brick back to dphi: interior and ghost faces
            CT* D = Corr<CT>::dphi(a.st) + (size_t)b * P3;
            const CT* B = resident_buf(j, j ? ib1 : ib0);
#pragma unroll
            for (int r = 0; r < K; r++) D[c[r]] = B[c[r]];
            for (int q = threadIdx.x; q < 6 * F; q += TPB) {
                int face, t1, t2;
                const int gi = relax_ghost_cell<NX>(q, face, t1, t2);
                D[gi] = B[gi];
            }
        }
        if (server && threadIdx.x == 0) a.bar->relax_done_k = k;  // the loop's length for the blocks without a brick
        pass_seq = seq0 + k;
        return sync(PH_RELAX, n * (k + 1));
    }

    // Poisson::vcycle (poisson.cpp:1069-1074) = vcycle0 (poisson.cpp:53-84)
    // without the two dphi ghost fills that nothing reads (see vcycle0 in
    // poisson_host.cpp)
    __device__ bool vcycle() {
        const int t = threadIdx.x;
        const int maxl = a.nlevels - 1;
        each(a.L.nall, [&](int q) { op_set_source(a.g, a.st, a.L.all[q], t, blockDim.x); });
        if (!sync(PH_SOURCE, a.L.nall)) return false;
        for (int l = maxl - 1; l >= 0; l--) {
            const int* pl = a.parents + a.poff[l];
            constexpr int H3 = (NX / 2) * (NX / 2) * (NX / 2);
            each(a.pcnt[l], [&](int q) {
                for (int u = t; u < 8 * H3; u += TPB) op_phi_from_children(a.g, a.bt, a.st, pl[q], u / H3, u % H3);
            });
            if (!sync(PH_RESTRICT, a.pcnt[l])) return false;
        }
        for (int l = 0; l <= maxl; l++)
            if (!phi_boundaries(l)) return false;
        each(a.L.nall, [&](int q) { op_init_vcycle<CT>(a.g, a.st, a.L.all[q], t, blockDim.x); });
        if (!sync(PH_INIT, a.L.nall)) return false;
        // down sweep (levels maxl .. 0), then up sweep (0 .. maxl), as one
        // loop so that the relaxation loop is expanded once
        for (int step = 0; step < 2 * (maxl + 1); step++) {
            const bool down = step <= maxl;
            const int l = down ? maxl - step : step - (maxl + 1);
            const int* sl = level(l);
            if (down) {
                each(a.L.cnt[l], [&](int q) {
                    op_vdown<CT>(a.g, a.bt, a.st, sl[q], a.vitems, a.vranges + 4 * (a.voff[l] + q));
                    __syncthreads();
                });
                if (!sync(PH_VDOWN, a.L.cnt[l])) return false;
            } else if (l > 0) {
                each(a.L.cnt[l], [&](int q) { op_coarse_correction<CT>(a.g, a.bt, a.st, sl[q], t); });
                if (!sync(PH_CORRECT, a.L.cnt[l])) return false;
            }
            if (!relax_until(l, down ? 1.0 : 0.05)) return false;
            if (!down) {
                each(a.L.cnt[l], [&](int q) { op_retire<CT>(a.g, a.st, sl[q], t, blockDim.x); });
                if (!sync(PH_RETIRE, a.L.cnt[l])) return false;
                if (!phi_boundaries(l)) return false;
            }
        }
        return true;
    }

    // compute_forces + adjust_{x,y,z}_force level by level, finest first
    __device__ bool forces() {
        const int t = threadIdx.x;
        each(a.L.nall, [&](int q) { op_forces(a.g, a.bt, a.st, a.L.all[q], t, blockDim.x); });
        if (!sync(PH_FORCES, a.L.nall)) return false;
        for (int l = a.force_levels - 1; l >= 0; l--) {
            const int n = a.foff[l + 1] - a.foff[l];
            if (n <= 0) continue;
            const RefluxItem* it = a.fitems + a.foff[l];
            each(n, [&](int q) { op_adjust_force(a.g, a.st, it[q], t); });
            if (!sync(PH_ADJUST_FORCE, n)) return false;
        }
        return true;
    }

    // Poisson::solution_error (poisson.cpp:637-669), nested over the tree;
    // the per-brick sums with 256 threads, as the error kernels form them
    __device__ bool error(double* err) {
        const int nl = a.nlevels;
        double* perr = a.pres + 2 * (size_t)a.L.cap;
        each(a.L.nall, [&](int q) {
            op_solution_error<CT>(a.g, a.bt, a.st, a.L.all[q], perr, red, 256);
            __syncthreads();
        });
        if (!sync(PH_ERROR, a.L.nall)) return false;
        if (a.L.max_cnt <= NEST_SMEM) {
            *err = nested_sum_smem(a.L, perr, nl - 1, true, nbuf);
            return true;
        }
        // deepest level: nest = own; then own + children level by level
        const int* sl = a.L.slots + a.L.off[nl - 1];
        for (int q = threadIdx.x; q < a.L.cnt[nl - 1]; q += blockDim.x) nest[sl[q]] = __ldcg(perr + sl[q]);
        __syncthreads();
        *err = nested_sum_block(a.L, a.bt.child, perr, nest, nl - 1, true);
        return true;
    }
};

template <int NX, int TPB, typename CT>
__global__ void __launch_bounds__(TPB, SolveLayout<NX, TPB>::MINB) k_solve_persistent(SolveArgs a) {
    // the staged bricks live in dynamic shared memory
    RelaxSmem<NX, CT>* sm = reinterpret_cast<RelaxSmem<NX, CT>*>(dyn_smem());
    __shared__ double red[16];
    __shared__ double nbuf[2 * NEST_SMEM];
    __shared__ double s_err;
    // loop limits are read from the control block (set by the host before
    // every launch; a captured graph keeps its arguments)
    const int max_cycles = *(volatile int*)&a.ctl->max_cycles;
    // the third brick buffer: the second half's staging buffer where the
    // layout has one, else the dynamic shared memory after the staged brick
    CT* xbuf = SolveLayout<NX, TPB>::NSM == 2 ? sm[1].buf[0] : reinterpret_cast<CT*>(sm + 1);
    Solver<NX, TPB, CT> s{a, sm, xbuf, red, nbuf, a.nest + (size_t)blockIdx.x * a.L.cap, 0, 0, 0,
                 *(volatile int*)&a.ctl->max_outer};
    __shared__ unsigned long long s_ph_ns[PH_COUNT];
    __shared__ unsigned s_ph_n[PH_COUNT];
    __shared__ double s_ph_bytes[PH_COUNT];
    __shared__ unsigned long long s_ph_wait[PH_COUNT + 2];
    {
        const int wl = *(volatile int*)&a.ctl->wait_limit;
        if (wl > 0) s.spin_limit = (unsigned long long)wl;
    }
    __shared__ unsigned s_lvl_n[MAX_LEVELS];
    s.lvl_n = s_lvl_n;
    __shared__ unsigned long long s_lvl_ns[MAX_LEVELS];
    s.lvl_ns = s_lvl_ns;
    __shared__ unsigned long long s_rsplit[6];
    s.rsplit = s_rsplit;
    // the mbarrier of the bulk brick copies: one arrival (the issuing
    // thread's, with the bytes it expects) completes a phase
    __shared__ __align__(8) unsigned long long s_mbar;
    s.mbar = (unsigned)__cvta_generic_to_shared(&s_mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s.mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 6) s_rsplit[threadIdx.x] = 0;
    if (threadIdx.x < MAX_LEVELS) {
        s_lvl_n[threadIdx.x] = 0;
        s_lvl_ns[threadIdx.x] = 0;
    }
    s.ph_ns = s_ph_ns;
    s.ph_n = s_ph_n;
    s.ph_bytes = s_ph_bytes;
    s.ph_wait = s_ph_wait;
    if (threadIdx.x < PH_COUNT + 2) s_ph_wait[threadIdx.x] = 0;
    s.t_last = Solver<NX, TPB, CT>::now();
    if (threadIdx.x < PH_COUNT) {
        s_ph_ns[threadIdx.x] = 0;
        s_ph_n[threadIdx.x] = 0;
        s_ph_bytes[threadIdx.x] = 0.0;
    }
    __syncthreads();
    int cycles = 0;
    bool ok = true;
    double err = 0.0;
    for (;;) {
        if (!(ok = s.vcycle())) break;
        if (!(ok = s.forces())) break;
        if (!(ok = s.error(&err))) break;
        if (threadIdx.x == 0) s_err = err;
        __syncthreads();
        err = s_err;
        cycles++;
        if (!(err > a.tol)) break;
        if (cycles >= max_cycles) {
            s.status = 2;
            break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Control* c = a.ctl;
        if (!ok) {
            atomicMax(&c->status, 3);
        } else {
            c->err = err;
            c->cycles = cycles;
            c->cycles_total += cycles;
            c->relax_calls += s.relax_calls;
            if (s.status) atomicMax(&c->status, s.status);
            for (int p = 0; p < PH_COUNT; p++) {
                c->phase_ns[p] += s.ph_ns[p];
                c->phase_n[p] += s.ph_n[p];
                c->phase_bytes[p] += s.ph_bytes[p];
                c->phase_wait_ns[p] += s.ph_wait[p];
            }
            c->level_sum_ns += s.ph_wait[PH_COUNT];
            c->level_sum_n += s.ph_wait[PH_COUNT + 1];
            for (int l = 0; l < MAX_LEVELS; l++) {
                c->relax_level[l] += s.lvl_n[l];
                c->relax_level_ns[l] += s.lvl_ns[l];
            }
            for (int q = 0; q < 4; q++) c->relax_split_ns[q] += s.rsplit[q];
            c->relax_split_passes += s.rsplit[4];
            c->relax_split_sweeps += s.rsplit[5];
        }
    }
}

}  // namespace

template <int NX, int TPB, typename CT>
constexpr size_t solve_smem() {
    using Lay = SolveLayout<NX, TPB>;
    constexpr size_t P3 = (NX + 2) * (NX + 2) * (NX + 2);
    return Lay::NSM * sizeof(RelaxSmem<NX, CT>) + (Lay::NSM == 1 ? sizeof(CT) * P3 : 0) +
           (Lay::RES2 && sizeof(CT) == 4 ? 3 * sizeof(CT) * P3 : 0);
}

namespace {

// The layouts of each brick size, in the order of their layout number.
constexpr int LAYOUTS_8[] = {512, 256};
constexpr int LAYOUTS_12[] = {576, 864, 288};

template <int NX, int TPB, typename CT>
cudaError_t set_attr() {
    return cudaFuncSetAttribute((const void*)k_solve_persistent<NX, TPB, CT>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<NX, TPB, CT>());
}
template <int NX, int TPB, typename CT>
int occupancy() {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_persistent<NX, TPB, CT>, TPB,
                                                      solve_smem<NX, TPB, CT>()) != cudaSuccess)
        return -1;
    return per;
}
template <int NX, int TPB, typename CT>
cudaError_t launch(const SolveArgs& a, int blocks, cudaStream_t s) {
    void* args[] = {const_cast<SolveArgs*>(&a)};
    return cudaLaunchCooperativeKernel((const void*)k_solve_persistent<NX, TPB, CT>, dim3(blocks), dim3(TPB), args,
                                       solve_smem<NX, TPB, CT>(), s);
}

// Calls OP<NX, TPB, CT>::run(args...) for the layout (nx, layout, FP32?);
// returns `bad` for an unknown one.
#define AMR_SOLVE_DISPATCH(nx, layout, f32, bad, CALL)                  \
    do {                                                                \
        if ((nx) == 8) {                                                \
            if ((layout) == 0) return (f32) ? CALL(8, 512, float) : CALL(8, 512, double);   \
            if ((layout) == 1) return (f32) ? CALL(8, 256, float) : CALL(8, 256, double);   \
        } else if ((nx) == 12) {                                        \
            if ((layout) == 0) return (f32) ? CALL(12, 576, float) : CALL(12, 576, double); \
            if ((layout) == 1) return (f32) ? CALL(12, 864, float) : CALL(12, 864, double); \
            if ((layout) == 2) return (f32) ? CALL(12, 288, float) : CALL(12, 288, double); \
        }                                                               \
        return (bad);                                                   \
    } while (0)

#define AMR_OCC(NX, TPB, CT) occupancy<NX, TPB, CT>()
#define AMR_LAUNCH(NX, TPB, CT) launch<NX, TPB, CT>(a, blocks, s)

int occupancy_of(int nx, int layout, bool f32) { AMR_SOLVE_DISPATCH(nx, layout, f32, -1, AMR_OCC); }

}  // namespace

int solve_layouts(int nx) {
    return nx == 8 ? (int)(sizeof(LAYOUTS_8) / sizeof(int)) : nx == 12 ? (int)(sizeof(LAYOUTS_12) / sizeof(int)) : 0;
}

int solve_layout_threads(int nx, int layout) {
    if (layout < 0 || layout >= solve_layouts(nx)) return -1;
    return nx == 8 ? LAYOUTS_8[layout] : LAYOUTS_12[layout];
}

int solve_persistent_attributes() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(set_attr<8, 512, float>());
    chk(set_attr<8, 512, double>());
    chk(set_attr<8, 256, float>());
    chk(set_attr<8, 256, double>());
    chk(set_attr<12, 576, float>());
    chk(set_attr<12, 576, double>());
    chk(set_attr<12, 864, float>());
    chk(set_attr<12, 864, double>());
    chk(set_attr<12, 288, float>());
    chk(set_attr<12, 288, double>());
    return e == cudaSuccess ? 0 : -1;
}

int solve_persistent_blocks(int nx, int precision, int per_sm_cap, int layout) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    int per = occupancy_of(nx, layout, precision == AMR_PREC_MIXED);
    if (per <= 0) return -1;
    if (per_sm_cap > 0 && per_sm_cap < per) per = per_sm_cap;
    return sms * per;
}

cudaError_t launch_solve_persistent(const SolveArgs& a, int blocks, int layout, cudaStream_t s) {
    ++g_launch_tally;
    AMR_SOLVE_DISPATCH(a.g.nx, layout, a.g.precision == AMR_PREC_MIXED, cudaErrorInvalidValue, AMR_LAUNCH);
}

#undef AMR_OCC
#undef AMR_LAUNCH
#undef AMR_SOLVE_DISPATCH

}  // namespace amr
