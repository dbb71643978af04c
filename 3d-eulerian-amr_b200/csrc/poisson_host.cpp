// Host orchestration of the multigrid Poisson solve (poisson/poisson.cpp
// Poisson::vcycle / vcycle0, the single-star/binary solve() loop) and of the
// self-gravitating RK3 step.  The data-dependent loops (relaxation until a
// residual ratio, V-cycles until the L1 error) read per-brick device
// reductions and combine them with the nesting of the reference's recursion.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <string>
#include <vector>

#include "context.h"
#include "profiler.h"
#include "kernels.h"
#include "poisson.h"

using namespace amr;

#define CUDA_TRY(call)                                                                        \
    do {                                                                                      \
        cudaError_t e__ = (call);                                                             \
        if (e__ != cudaSuccess) {                                                             \
            c->err = std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " + #call; \
            return AMR_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

#define TRY(x)                 \
    do {                       \
        int rc__ = (x);        \
        if (rc__) return rc__; \
    } while (0)

namespace {

int check_launch(amr_ctx* c) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("CUDA launch error: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

int need_gravity(amr_ctx* c) {
    if (!c) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    if (!has_gravity(c)) {
        c->err = "Poisson call on a context created without self-gravity";
        return AMR_ERR_ARG;
    }
    if (!c->d_bphi) {
        const size_t nb = (size_t)c->cap * 6 * c->geom.pnx * c->geom.pnx;
        CUDA_TRY(cudaMalloc(&c->d_bphi, sizeof(double) * nb));
        CUDA_TRY(cudaMemsetAsync(c->d_bphi, 0, sizeof(double) * nb, c->stream));
        CUDA_TRY(cudaMalloc(&c->d_pres, sizeof(double) * c->cap));
        CUDA_TRY(cudaMalloc(&c->d_perr, sizeof(int) * 2));
        CUDA_TRY(cudaMemsetAsync(c->d_perr, 0, sizeof(int) * 2, c->stream));
    }
    return AMR_OK;
}

const int* lvl(amr_ctx* c, int l) { return c->d_slots + c->off_level[l]; }
int nlvl(amr_ctx* c, int l) { return (int)c->level_slots[l].size(); }
const int* all(amr_ctx* c) { return c->d_slots + c->off_all[0]; }
int nall(amr_ctx* c) { return (int)c->all_slots.size(); }

// per-slot device values -> host
int fetch_per_slot(amr_ctx* c, std::vector<double>& v) {
    int maxslot = 0;
    for (int s : c->all_slots) maxslot = std::max(maxslot, s + 1);
    v.assign(maxslot, 0.0);
    CUDA_TRY(cudaMemcpyAsync(v.data(), c->d_pres, sizeof(double) * maxslot, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

// Poisson::vcycle_relax's return value: a node at the target level gives its
// own residual, every coarser node the sum of its children's returns.
double nested_level_sum(const Node* n, int level, const std::vector<double>& per) {
    if (n->level == level) return per[n->slot];
    double r = 0.0;
    for (int q = 0; q < 8; q++)
        if (n->child[q]) r += nested_level_sum(n->child[q], level, per);
    return r;
}

// Poisson::solution_error's return value: own sum, then children's.
double nested_tree_sum(const Node* n, const std::vector<double>& per) {
    double r = per[n->slot];
    for (int q = 0; q < 8; q++)
        if (n->child[q]) r += nested_tree_sum(n->child[q], per);
    return r;
}

int phi_boundaries(amr_ctx* c, int l) {
    {
        ProfScope ps_(c->prof, KC_PHI_BOUND, c->stream, nlvl(c, l));
        launch_phi_boundaries(c->geom, c->bt, c->st, c->d_bphi, c->d_perr, lvl(c, l), nlvl(c, l), c->stream);
    }
    return check_launch(c);
}

int dphi_boundaries(amr_ctx* c, int l) {
    {
        ProfScope ps_(c->prof, KC_DPHI_BOUND, c->stream, nlvl(c, l));
        launch_dphi_boundaries(c->geom, c->bt, c->st, c->d_bphi, c->d_perr, lvl(c, l), nlvl(c, l), c->stream);
    }
    return check_launch(c);
}

int relax(amr_ctx* c, int l, double* resid) {
    int bad;
    {
        ProfScope ps_(c->prof, KC_RELAX, c->stream, nlvl(c, l));
        bad = launch_relax(c->geom, c->st, lvl(c, l), nlvl(c, l), c->d_pres, c->stream);
    }
    if (bad) {
        c->err = "relaxation kernels built for nx == 8 or 12";
        return AMR_ERR_ARG;
    }
    TRY(check_launch(c));
    std::vector<double> per;
    TRY(fetch_per_slot(c, per));
    *resid = nested_level_sum(c->tree.root(), l, per);
    c->relax_calls++;
    if (l < 16) c->relax_level[l]++;
    return AMR_OK;
}

// relax, then relax again with fresh ghosts until the level residual has
// fallen to `ratio` of the first call's (poisson.cpp:66-70, 74-78).
int relax_until(amr_ctx* c, int l, double ratio) {
    double r0, r;
    TRY(dphi_boundaries(c, l));
    TRY(relax(c, l, &r0));
    int outer = 0;
    do {
        TRY(dphi_boundaries(c, l));
        TRY(relax(c, l, &r));
        if (++outer > c->vcycle_max_outer) {
            c->err = "relaxation did not reach its residual ratio";
            return AMR_ERR_NOCONVERGE;
        }
    } while (r / r0 > ratio);
    return AMR_OK;
}

int max_level_present(amr_ctx* c) {
    int m = 0;
    for (Node* n : c->order) m = std::max(m, n->level);
    return m;
}

// Poisson::vcycle0 (poisson.cpp:53-84)
int vcycle0(amr_ctx* c) {
    const int maxlevel = max_level_present(c);
    for (int l = maxlevel - 1; l >= 0; l--)  // phi_from_children: children first
        {
            ProfScope ps_(c->prof, KC_VDOWN, c->stream);
            launch_phi_from_children(c->geom, c->bt, c->st, c->d_slots + c->off_parent[l],
                                     (int)c->parent_slots[l].size(), c->stream);
        }
    TRY(check_launch(c));
    for (int l = 0; l <= maxlevel; l++) TRY(phi_boundaries(c, l));
    {
        ProfScope ps_(c->prof, KC_VDOWN, c->stream);
        launch_init_vcycle(c->geom, c->st, all(c), nall(c), c->stream);
    }
    // The reference fills the dphi ghosts before vcycle_down and before the
    // coarse correction as well; neither reads them and relax_until fills
    // them again first, so those two fills are left out (same results).
    for (int l = maxlevel; l >= 0; l--) {
        {
            ProfScope ps_(c->prof, KC_VDOWN, c->stream, nlvl(c, l));
            launch_vdown(c->geom, c->bt, c->st, lvl(c, l), nlvl(c, l), c->d_vitems,
                         c->d_vranges + 4 * c->off_vrange[l], c->stream);
        }
        TRY(check_launch(c));
        TRY(relax_until(c, l, 1.0));
    }
    for (int l = 0; l <= maxlevel; l++) {
        if (l > 0) {
            ProfScope ps_(c->prof, KC_CORRECT, c->stream);
            launch_coarse_correction(c->geom, c->bt, c->st, lvl(c, l), nlvl(c, l), c->stream);
        }
        TRY(check_launch(c));
        TRY(relax_until(c, l, 0.05));
        {
            ProfScope ps_(c->prof, KC_CORRECT, c->stream);
            launch_retire(c->geom, c->st, lvl(c, l), nlvl(c, l), c->stream);
        }
        TRY(phi_boundaries(c, l));
    }
    return AMR_OK;
}

int compute_forces(amr_ctx* c) {
    {
        ProfScope ps_(c->prof, KC_FORCES, c->stream);
        launch_forces(c->geom, c->bt, c->st, all(c), nall(c), c->stream);
    }
    for (int l = c->tree.prm.max_level; l >= 0; l--) {
        const int n = c->off_reflux[l + 1] - c->off_reflux[l];
        {
            ProfScope ps_(c->prof, KC_FORCES, c->stream);
            launch_adjust_force(c->geom, c->st, c->d_reflux + c->off_reflux[l], n, c->stream);
        }
    }
    return check_launch(c);
}

int solution_error(amr_ctx* c, double* err) {
    {
        ProfScope ps_(c->prof, KC_ERROR, c->stream);
        launch_solution_error(c->geom, c->bt, c->st, all(c), nall(c), c->d_pres, c->stream);
    }
    TRY(check_launch(c));
    std::vector<double> per;
    TRY(fetch_per_slot(c, per));
    *err = nested_tree_sum(c->tree.root(), per);
    return AMR_OK;
}

int check_device_error(amr_ctx* c) {
    int e[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(e, c->d_perr, sizeof(int) * 2, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (e[0]) {
        c->err = "mirror-plane ghost requested at an index the reference aborts on";
        CUDA_TRY(cudaMemsetAsync(c->d_perr, 0, sizeof(int) * 2, c->stream));
        return AMR_ERR_STATE;
    }
    return AMR_OK;
}

}  // namespace

namespace amr {
int poisson_need(amr_ctx* c) { return need_gravity(c); }
int poisson_phi_boundaries(amr_ctx* c, int l) { return phi_boundaries(c, l); }

// Poisson::phi_from_children (poisson.cpp:707-747), children first
int poisson_phi_from_children(amr_ctx* c) {
    const int maxlevel = max_level_present(c);
    for (int l = maxlevel - 1; l >= 0; l--) {
        ProfScope ps_(c->prof, KC_VDOWN, c->stream);
        launch_phi_from_children(c->geom, c->bt, c->st, c->d_slots + c->off_parent[l],
                                 (int)c->parent_slots[l].size(), c->stream);
    }
    return check_launch(c);
}

PhysWalk phys_walk(const amr_ctx* c) {
    return PhysWalk{c->d_pwalk, c->n_pseg, c->d_pwalk + 2 * c->n_pseg, c->n_ptop};
}

void build_phys_walk(const int* levels, int n, int limit, std::vector<int>& segs, std::vector<int>& top) {
    segs.clear();
    top.clear();
    // end[e]: one past the last DFS entry of e's subtree
    std::vector<int> end(n, n), open;
    for (int e = 0; e < n; e++) {
        while (!open.empty() && levels[open.back()] >= levels[e]) {
            end[open.back()] = e;
            open.pop_back();
        }
        open.push_back(e);
    }
    for (int e = 0; e < n;) {
        if (end[e] - e <= limit) {
            top.push_back(-(int)(segs.size() / 2) - 1);
            segs.push_back(e);
            segs.push_back(end[e]);
            e = end[e];
        } else {
            top.push_back(e);
            e++;
        }
    }
}
}  // namespace amr

void amr_poisson_release(amr_ctx* c) {
    if (!c) return;
    void* ptrs[] = {c->d_bphi, c->d_msrc, c->d_allref, c->d_pres, c->d_bfaces, c->d_perr, c->d_own, c->d_pwalk};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

extern "C" {

int amr_upload_poisson(amr_ctx* c, const double* P) {
    TRY(need_gravity(c));
    const int n = nall(c);
    const size_t per = (size_t)n * c->geom.pnx3;
    double* arr[8] = {c->st.phi, c->st.phi0, c->st.dphi, c->st.dphi1, c->st.S, c->st.fx, c->st.fy, c->st.fz};
    TRY(stage_reserve(c, per));
    for (int a = 0; a < 8; a++) {
        CUDA_TRY(cudaMemcpyAsync(c->d_stage, P + a * per, sizeof(double) * per, cudaMemcpyHostToDevice, c->stream));
        launch_scatter(c->d_stage, all(c), n, c->geom.pnx3, arr[a], c->stream);
        TRY(check_launch(c));
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int amr_download_poisson(amr_ctx* c, double* P) {
    TRY(need_gravity(c));
    const int n = nall(c);
    const size_t per = (size_t)n * c->geom.pnx3;
    double* arr[8] = {c->st.phi, c->st.phi0, c->st.dphi, c->st.dphi1, c->st.S, c->st.fx, c->st.fy, c->st.fz};
    TRY(stage_reserve(c, per));
    for (int a = 0; a < 8; a++) {
        launch_gather(arr[a], all(c), n, c->geom.pnx3, c->d_stage, c->stream);
        TRY(check_launch(c));
        CUDA_TRY(cudaMemcpyAsync(P + a * per, c->d_stage, sizeof(double) * per, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    return AMR_OK;
}

int amr_poisson_set_source(amr_ctx* c) {
    TRY(need_gravity(c));
    {
        ProfScope ps_(c->prof, KC_SOURCE, c->stream);
        launch_set_source(c->geom, c->st, all(c), nall(c), c->stream);
    }
    return check_launch(c);
}

// compute_source_sums (with set_source) + compute_physical_boundaries.
int amr_poisson_boundaries(amr_ctx* c) {
    TRY(need_gravity(c));
    TRY(amr_poisson_set_source(c));
    {
        ProfScope ps_(c->prof, KC_SOURCE, c->stream);
        launch_source_sums(c->geom, c->bt, c->st, all(c), nall(c), c->d_msrc, c->d_allref, c->stream);
    }
    {
        ProfScope ps_(c->prof, KC_PHYS_BOUND, c->stream);
        if (launch_phys_bound(c->geom, c->bt, c->d_bfaces, c->n_bfaces, all(c), phys_walk(c), c->d_msrc, c->d_allref,
                              c->d_bphi, c->d_own, c->own_cap, c->stream)) {
            c->err = "domain-face potential scratch too small";
            return AMR_ERR_STATE;
        }
    }
    return check_launch(c);
}

int amr_compute_forces(amr_ctx* c) {
    TRY(need_gravity(c));
    return compute_forces(c);
}

// Poisson::vcycle (poisson.cpp:1069-1074)
int amr_vcycle(amr_ctx* c, double* l1_error) {
    TRY(need_gravity(c));
    TRY(amr_poisson_set_source(c));
    TRY(vcycle0(c));
    TRY(compute_forces(c));
    double e;
    TRY(solution_error(c, &e));
    TRY(check_device_error(c));
    if (l1_error) *l1_error = e;
    return AMR_OK;
}

// The solve() loop of single/driver.h:21-42 and binary_driver.cpp:296-344:
// boundaries, forces, V-cycles until the L1 error <= tol, then restriction
// of the hydro state.
int amr_poisson_solve(amr_ctx* c, double tol, int max_cycles, double* l1_error, int* cycles) {
    TRY(need_gravity(c));
    TRY(amr_poisson_boundaries(c));
    TRY(compute_forces(c));
    double e = 0.0;
    int it = 0;
    do {
        if (it >= max_cycles) {
            c->err = "Poisson solve exceeded max_cycles";
            if (l1_error) *l1_error = e;
            if (cycles) *cycles = it;
            return AMR_ERR_NOCONVERGE;
        }
        TRY(amr_vcycle(c, &e));
        it++;
    } while (e > tol);
    if (l1_error) *l1_error = e;
    if (cycles) *cycles = it;
    if (is_ztwd(c)) TRY(amr_ztwd_pot(c, 0));  // Binary's solve: pot_to_grid (binary_driver.cpp:341)
    return amr_inject_from_children(c);
}

int amr_store_phi(amr_ctx* c) {
    TRY(need_gravity(c));
    {
        ProfScope ps_(c->prof, KC_PHI_TIME, c->stream);
        launch_phi_time(c->geom, c->st, all(c), nall(c), 0, c->stream);
    }
    return check_launch(c);
}

int amr_restore_phi(amr_ctx* c) {
    TRY(need_gravity(c));
    {
        ProfScope ps_(c->prof, KC_PHI_TIME, c->stream);
        launch_phi_time(c->geom, c->st, all(c), nall(c), 1, c->stream);
    }
    return check_launch(c);
}

int amr_restore_half_phi(amr_ctx* c) {
    TRY(need_gravity(c));
    {
        ProfScope ps_(c->prof, KC_PHI_TIME, c->stream);
        launch_phi_time(c->geom, c->st, all(c), nall(c), 2, c->stream);
    }
    return check_launch(c);
}

// Self-gravitating RK3 step: the sub_step/step sequence of
// binary/binary_driver.cpp:346-459 and single/driver.h:83-119 on the Euler
// state (gravity sources inside amr_add_difs).
int amr_grav_step(amr_ctx* c, double dt, double tol, double dynamic_range, int step_index) {
    TRY(need_gravity(c));
    if (!(dt > 0.0)) return AMR_ERR_ARG;
    const int max_cycles = 10000;  // MAX_POISSON_ITER (defs.h:25)
    if (step_index <= 0) {
        TRY(amr_poisson_solve(c, tol, max_cycles, nullptr, nullptr));
        TRY(amr_store_phi(c));
    }
    TRY(amr_store(c));
    const double betas[3] = {1.0, 0.25, 2.0 / 3.0};
    for (int rk = 1; rk <= 3; rk++) {
        TRY(amr_enforce_boundaries(c));
        TRY(amr_compute_fluxes(c));
        TRY(amr_add_difs(c, dt, betas[rk - 1]));
        if (rk == 1)
            TRY(amr_store_phi(c));
        else if (rk == 2)
            TRY(amr_restore_half_phi(c));
        else
            TRY(amr_restore_phi(c));
        TRY(amr_poisson_solve(c, tol, max_cycles, nullptr, nullptr));
    }
    TRY(amr_enforce_boundaries(c));
    if (step_index % 8 == 0) {
        double smax;
        TRY(amr_state_max(c, 0, &smax));
        int changed = 0;
        TRY(amr_check_for_refine(c, smax / dynamic_range, 1, &changed));
        if (changed) {
            TRY(amr_poisson_solve(c, tol / 10.0, max_cycles, nullptr, nullptr));
            TRY(amr_store_phi(c));
        }
    }
    TRY(amr_set_time(c, c->time + dt));
    return AMR_OK;
}

}  // extern "C"
