// Persistent multigrid solve (persistent.cu): arguments and launch.
#pragma once

#include <cuda_runtime.h>

#include "amr_internal.h"
#include "graph.h"
#include "poisson_ops.cuh"

namespace amr {

// Grid barrier state; zero it before every launch.
struct GridBarrier {
    unsigned int count;  // arrivals since the launch began
    unsigned int pad0;
    int abort;
    int pad;
    // relaxation level sums published by one block: sum g of the launch in
    // lsum_val[g & 1], then lsum_gen = g
    unsigned int lsum_gen;
    unsigned int pad1;
    double lsum_val[2];
    unsigned int pad2;
    // the last pass of the latest shared-memory relaxation loop (stored by
    // the block that forms its sums before the loop's closing barrier)
    unsigned int relax_done_k;
    // the FP32 correction's level sums: the high and low halves of the FP64
    // sum, each tagged with its generation (value and tag in one 64-bit
    // word), on a cache line of their own
    alignas(128) unsigned long long lsum_tag[2];
};

struct SolveArgs {
    Geom g;
    BrickTable bt;
    DevState st;
    LevelLists L;
    PoissonAux aux;
    const int* parents;  // bricks with children, per level: parents + poff[l], pcnt[l]
    int poff[MAX_LEVELS];
    int pcnt[MAX_LEVELS];
    const RefluxItem* fitems;  // coarse-fine items sorted by coarse level (force averages)
    int foff[MAX_LEVELS + 1];
    int force_levels;
    const RefluxItem* vitems;  // items grouped by coarse brick for the down sweep
    const int* vranges;
    int voff[MAX_LEVELS];
    int nlevels;  // levels present
    double tol;
    Control* ctl;  // also holds the loop limits max_cycles, max_outer
    double* pres;  // [3][cap]: two relaxation buffers, one for the L1 error
    double* nest;  // [blocks][cap] per-block nested-sum scratch
    void* snap;    // [2][cap][stride] face snapshots (CT entries)
    unsigned* rpub;  // [cap] last pass a brick published in the shared-memory relaxation loops (zero per launch)
    unsigned long long* tsnap;  // [2][cap][stride] tagged face snapshots of the FP32 correction (zero per launch)
    unsigned long long* tpres;  // [2][cap][2] tagged halves of the per-brick relaxation sums (zero per launch)
    size_t stride;
    size_t snap_half;
    GridBarrier* bar;
};

// Block layouts of the solve kernel for nx^3 bricks (threads per block,
// cells per thread in the relaxation; the same results bit for bit): how
// many there are, and the threads of one (-1 for none).
int solve_layouts(int nx);
int solve_layout_threads(int nx, int layout);
// Blocks of one cooperative launch of a layout on the current device (all
// resident), at most per_sm_cap per SM when per_sm_cap > 0.
int solve_persistent_blocks(int nx, int precision, int per_sm_cap, int layout);
// raises the dynamic shared-memory limit of the solve kernels (call outside
// stream capture)
int solve_persistent_attributes();
cudaError_t launch_solve_persistent(const SolveArgs& a, int blocks, int layout, cudaStream_t s);

}  // namespace amr
