// ZTWD binary: frame and EOS of the context, potential <-> state
// conversions and the BinaryDriver step sequence (binary/binary_driver.cpp,
// binary/binary.cpp).  The per-call ZTWD kernels are dispatched from the
// ordinary entry points (amr_host.cpp, poisson_host.cpp) when the context's
// physics is AMR_PHYSICS_ZTWD.
#include <cuda_runtime.h>

#include <cstdio>

#include "context.h"
#include "helm_b200.h"
#include "kernels.h"
#include "poisson.h"
#include "ztwd.h"

using namespace amr;

#define TRY(x)                        \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != AMR_OK) return rc_; \
    } while (0)
#define CUDA_TRY(x)                                   \
    do {                                              \
        cudaError_t e_ = (x);                         \
        if (e_ != cudaSuccess) {                      \
            c->err = cudaGetErrorString(e_);          \
            return AMR_ERR_CUDA;                      \
        }                                             \
    } while (0)

namespace amr {

int zt_ready(amr_ctx* c) {
    if (!c) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    if (!is_ztwd(c)) {
        c->err = "ZTWD call on a context created without AMR_PHYSICS_ZTWD";
        return AMR_ERR_ARG;
    }
    if (!c->zt_eos) {
        c->err = "ZTWD context without an EOS: call amr_ztwd_set_eos first";
        return AMR_ERR_STATE;
    }
    return AMR_OK;
}

int zt_check(amr_ctx* c) {
    if (!c->d_zerr) return AMR_OK;
    int e = 0;
    CUDA_TRY(cudaMemcpyAsync(&e, c->d_zerr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (e) {
        static const char* what[] = {"", "state outside the EOS table (helmeos.cpp:216-221)",
                                     "negative c_v (helmeos.cpp:405-409)", "negative c_s^2 (helmeos.cpp:410-415)",
                                     "temperature Newton did not converge (helmeos.cpp:477-480)",
                                     "temperature below the table floor (helmeos.cpp:469-472)"};
        c->err = std::string("ZTWD EOS: ") + (e > 0 && e <= 5 ? what[e] : "unknown status");
        CUDA_TRY(cudaMemsetAsync(c->d_zerr, 0, sizeof(int), c->stream));
        return AMR_ERR_RANGE;
    }
    return AMR_OK;
}

}  // namespace amr

namespace {

const int* all(amr_ctx* c) { return c->d_slots + c->off_all[0]; }
int nall(amr_ctx* c) { return (int)c->all_slots.size(); }

int max_level_present(amr_ctx* c) {
    int m = 0;
    for (Node* n : c->order) m = std::max(m, n->level);
    return m;
}

int check_launch(amr_ctx* c) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

// Binary::pot_from_grid (binary.cpp:857-884): phi of every brick, then the
// phi ghosts of every level (the level-0 call's enforce_phi_boundaries loop)
int pot_from_grid(amr_ctx* c) {
    TRY(poisson_need(c));  // the phi ghost fill reads the domain-face tables
    {
        ProfScope ps_(c->prof, KC_PHI_BOUND, c->stream, (long long)nall(c));
        launch_zt_pot(c->geom, c->bt, c->st, c->zpar, all(c), nall(c), 1, c->stream);
    }
    TRY(check_launch(c));
    const int maxl = max_level_present(c);
    for (int l = 0; l <= maxl; l++) TRY(poisson_phi_boundaries(c, l));
    return AMR_OK;
}

// BinaryDriver::solve (binary_driver.cpp:296-344): the first call rebuilds
// phi from the state and the covered cells from their children
int zt_solve(amr_ctx* c, double tol) {
    if (c->zt_first_solve) {
        TRY(pot_from_grid(c));
        TRY(poisson_phi_from_children(c));
        c->zt_first_solve = 0;
    }
    const int max_cycles = 10000;  // MAX_POISSON_ITER (defs.h:25)
    if (c->cfg.persistent_solve > 0 || c->geom.precision == AMR_PREC_MIXED)
        TRY(amr_graph_solve(c, tol, max_cycles, nullptr, nullptr));
    else
        TRY(amr_poisson_solve(c, tol, max_cycles, nullptr, nullptr));
    return AMR_OK;
}

// BinaryDriver::sub_step (binary_driver.cpp:346-382)
int zt_sub_step(amr_ctx* c, double dt, double beta, int rk, double tol) {
    TRY(amr_enforce_boundaries(c));
    TRY(amr_compute_fluxes(c));
    TRY(amr_add_difs(c, dt, beta));
    if (rk == 1) {
        TRY(amr_store_phi(c));
    } else if (rk == 2) {
        TRY(amr_restore_half_phi(c));
    } else {
        TRY(amr_restore_phi(c));
    }
    return zt_solve(c, tol);
}

}  // namespace

extern "C" {

int amr_ztwd_set_eos(amr_ctx* c, helm_ctx* eos) {
    if (!c || !eos) return AMR_ERR_ARG;
    if (!is_ztwd(c)) {
        c->err = "amr_ztwd_set_eos on a context created without AMR_PHYSICS_ZTWD";
        return AMR_ERR_ARG;
    }
    const HelmTable* H = helm_table_of(eos);
    if (!H || !H->node) {
        c->err = "EOS context has no table";
        return AMR_ERR_ARG;
    }
    c->zpar.H = *H;
    c->zt_eos = true;
    return AMR_OK;
}

int amr_ztwd_set_frame(amr_ctx* c, double omega, double omega0, double fR, double ftheta) {
    if (!c) return AMR_ERR_ARG;
    if (!is_ztwd(c)) {
        c->err = "amr_ztwd_set_frame on a context created without AMR_PHYSICS_ZTWD";
        return AMR_ERR_ARG;
    }
    c->zpar.omega = omega;
    c->zpar.omega0 = omega0;
    c->zpar.fR = fR;
    c->zpar.ftheta = ftheta;
    return AMR_OK;
}

int amr_ztwd_pot(amr_ctx* c, int mode) {
    TRY(zt_ready(c));
    if (mode < 0 || mode > 3) return AMR_ERR_ARG;
    if (mode == 1) return pot_from_grid(c);
    {
        ProfScope ps_(c->prof, KC_OTHER, c->stream, (long long)nall(c));
        launch_zt_pot(c->geom, c->bt, c->st, c->zpar, all(c), nall(c), mode, c->stream);
    }
    return check_launch(c);
}

int amr_ztwd_step(amr_ctx* c, double dt, double tol, double dynamic_range, int step_index, double* dt_used) {
    TRY(zt_ready(c));
    if (!(dt > 0.0)) return AMR_ERR_ARG;
    if (step_index <= 0) {
        TRY(pot_from_grid(c));  // READ_FROM_FILE (binary_defs.h:16): the state carries pot
        TRY(zt_solve(c, tol));
        TRY(amr_store_phi(c));
    }
    TRY(amr_store(c));
    const double maxdtinc = c->cfg.maxdtinc;
    for (;;) {
        TRY(zt_sub_step(c, dt, 1.0, 1, tol));
        TRY(zt_sub_step(c, dt, 0.25, 2, tol));
        TRY(zt_sub_step(c, dt, 2.0 / 3.0, 3, tol));
        double test_dt;
        TRY(amr_max_dt(c, &test_dt));
        if (test_dt < dt / maxdtinc) {
            dt = dt / maxdtinc;
            TRY(amr_restore(c));
            continue;
        }
        break;
    }
    TRY(amr_enforce_boundaries(c));
    if (step_index % 8 == 0) {
        double smax;
        TRY(amr_state_max(c, 0, &smax));
        TRY(amr_ztwd_pot(c, 2));
        int changed = 0;
        TRY(amr_check_for_refine(c, smax / dynamic_range, (step_index % 500) == 0, &changed));
        if (changed) {
            TRY(zt_solve(c, tol / 10.0));
            TRY(amr_store_phi(c));
        }
        TRY(amr_ztwd_pot(c, 3));
    }
    TRY(amr_set_time(c, c->time + dt));
    TRY(zt_check(c));
    if (dt_used) *dt_used = dt;
    return AMR_OK;
}

}  // extern "C"
