// Graph-captured step: device-side loop control and its kernels.
#pragma once

#include <cuda_runtime.h>

#include "amr_internal.h"

namespace amr {

constexpr int MAX_LEVELS = 16;

// Per-level brick lists in depth-first order (device pointers + counts).
struct LevelLists {
    const int* slots;  // packed lists
    const int* all;    // all bricks, DFS order
    int nall;
    int cap;           // brick pool capacity (slot range)
    int off[MAX_LEVELS];
    int cnt[MAX_LEVELS];
    // cpos[8 e + c]: position, in the next level's list, of child c of the
    // brick at entry e of the packed level lists (e = off[m] - off[0] + q),
    // or -1
    const int* cpos;
    int max_cnt;  // largest level count
};

// level sums formed in shared memory when every level has at most this
// many bricks
constexpr int NEST_SMEM = 768;

// Loop state shared between graph kernels and the host.
struct Control {
    double r0[MAX_LEVELS];  // first-pass residual of the current relaxation loop per level
    int outer[MAX_LEVELS];  // relaxation passes in the current loop
    double err;             // last L1 error of the solve loop
    double dt, last_dt;     // CFL step of the graph-driven step
    int cycles;             // V-cycles in the current solve
    int max_cycles;
    int max_outer;
    int status;             // 0 ok, 1 relaxation loop cap, 2 V-cycle cap
    long long relax_calls;
    long long cycles_total;  // V-cycles since the context started
    int steps;
    int pad;
    int snap_par[MAX_LEVELS];  // which face-snapshot buffer the next pass reads
    // persistent solve: device time of each phase class (from one barrier's
    // exit to the next, i.e. the slowest block's work plus the barrier), as
    // seen by block 0, and the number of such phases
    unsigned long long phase_ns[16];
    unsigned long long phase_n[16];
    double phase_bytes[16];  // algorithmic HBM bytes of those phases
    // the part of each phase spent at its closing barrier (block 0: from its
    // own arrival, after its share of the work, to the barrier's exit), and
    // the time block 0 spends forming relaxation level sums after a barrier
    unsigned long long phase_wait_ns[16];
    unsigned long long level_sum_ns;
    unsigned long long level_sum_n;
    long long relax_level[MAX_LEVELS];  // relaxation passes per level
    int wait_limit;                     // persistent solve: polls per bounded wait (<= 0: default)
    int pad2;
    // the shared-memory relaxation loops as block 0 sees them: time waiting
    // for the neighbours' passes, computing passes (ghosts and sweeps),
    // waiting for the loop decision, publishing; passes and sweeps counted
    unsigned long long relax_split_ns[4];
    unsigned long long relax_split_passes, relax_split_sweeps;
    // block 0's time in the relaxation loops of each level (from the dphi
    // ghost faces to the loop's closing barrier)
    unsigned long long relax_level_ns[MAX_LEVELS];
};

// phase classes of the persistent solve
enum SolvePhase {
    PH_SOURCE = 0, PH_RESTRICT, PH_PHI_FACES, PH_PHI_EDGES, PH_PHI_VERTICES, PH_INIT, PH_VDOWN, PH_DPHI_FACES,
    PH_RELAX_FIRST, PH_RELAX, PH_CORRECT, PH_RETIRE, PH_FORCES, PH_ADJUST_FORCE, PH_ERROR, PH_COUNT
};

// snap: [2][cap][6][nx][nx] first-interior layers published by every pass
void launch_relax_dev(const Geom& g, const BrickTable& bt, const DevState& st, const LevelLists& L, int level,
                      int mode, double ratio, cudaGraphConditionalHandle cond, Control* ctl, double* pres,
                      double* nest, unsigned int* counter, double* snap, size_t snap_stride, cudaStream_t s);
// raises the dynamic shared-memory limit of the relaxation kernels (call
// outside stream capture)
int relax_dev_attributes();
void launch_error_dev(const Geom& g, const BrickTable& bt, const DevState& st, const LevelLists& L, int nlevels,
                      double tol, cudaGraphConditionalHandle cond, Control* ctl, double* pres, double* nest,
                      unsigned int* counter, cudaStream_t s);
void launch_open_loop(cudaGraphConditionalHandle cond, Control* ctl, int reset_cycles, cudaStream_t s);
void launch_dt_reduce(const BrickTable& bt, const LevelLists& L, int nlevels, const double* per, double* nest,
                      Control* ctl, double maxdtinc, cudaStream_t s);

}  // namespace amr
