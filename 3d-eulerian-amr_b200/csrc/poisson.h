// Multigrid Poisson solver (poisson/poisson.cpp) on the device brick pool.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "amr_internal.h"

struct amr_ctx;

namespace amr {
// checks the context has self-gravity and allocates the Poisson scratch
// (domain-face tables zeroed, error words) on first use
int poisson_need(amr_ctx* c);
// phi ghosts of one level (faces, edges, vertices) and phi_from_children of
// every level, as the V-cycle runs them (poisson_host.cpp)
int poisson_phi_boundaries(amr_ctx* c, int l);
int poisson_phi_from_children(amr_ctx* c);
// New bricks: zero the Poisson arrays, then phi/phi0 piecewise constant from
// the parent (Poisson::inject_from_parent, poisson.cpp:132-164).
void launch_poisson_new_bricks(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                               cudaStream_t s);
void launch_set_source(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s);
void launch_source_sums(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                        double* msrc, int* allref, cudaStream_t s);
// Walk program of the domain-face potential sum over the DFS-ordered bricks:
// segs[2s], segs[2s+1] = DFS entry range of subtree s; top = the walk above
// the subtrees (entry e >= 0, or subtree s as -s-1).  Device pointers.
struct PhysWalk {
    const int* segs;
    int nseg;
    const int* top;
    int ntop;
};
// Split the DFS-ordered brick levels into subtrees of at most `limit` bricks
// and the walk above them (host).
void build_phys_walk(const int* levels, int n, int limit, std::vector<int>& segs, std::vector<int>& top);
// The context's walk program (device pointers into its walk buffer).
PhysWalk phys_walk(const amr_ctx* c);
// scratch: (subtree, point) partial sums, scratch_cap doubles; points are
// batched so that one batch fits.  Returns -1 when not even one point fits.
int launch_phys_bound(const Geom& g, const BrickTable& bt, const int* bfaces, int nbf, const int* order,
                      const PhysWalk& w, const double* msrc, const int* allref, double* bphi, double* scratch,
                      size_t scratch_cap, cudaStream_t s);
void launch_phi_boundaries(const Geom& g, const BrickTable& bt, const DevState& st, const double* bphi, int* err,
                           const int* slots, int n, cudaStream_t s);
void launch_dphi_boundaries(const Geom& g, const BrickTable& bt, const DevState& st, const double* bphi, int* err,
                            const int* slots, int n, cudaStream_t s);
void launch_phi_from_children(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                              cudaStream_t s);
void launch_init_vcycle(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s);
// vcycle_down of one level (residual / child averages, adjust_{x,y,z}_dphi,
// dphi1 = dphi) in one launch; ranges[4 q + 0..3] = first x, y, z item of
// the brick at list position q in `items` and the end of its items.
void launch_vdown(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                  const RefluxItem* items, const int* ranges, cudaStream_t s);
int launch_relax(const Geom& g, const DevState& st, const int* slots, int n, double* out, cudaStream_t s);
void launch_coarse_correction(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                              cudaStream_t s);
void launch_retire(const Geom& g, const DevState& st, const int* slots, int n, cudaStream_t s);
void launch_forces(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                   cudaStream_t s);
void launch_adjust_force(const Geom& g, const DevState& st, const RefluxItem* items, int n, cudaStream_t s);
void launch_solution_error(const Geom& g, const BrickTable& bt, const DevState& st, const int* slots, int n,
                           double* out, cudaStream_t s);
void launch_phi_time(const Geom& g, const DevState& st, const int* slots, int n, int mode, cudaStream_t s);
}  // namespace amr

void amr_poisson_release(amr_ctx* c);
