// Launch wrappers of the ZTWD binary-state kernels (ztwd_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "amr_internal.h"
#include "helm_internal.h"

namespace amr {

constexpr int ZTWD_NF = 13;  // STATE_NF of the BINARY build (binary/state.h:13-15)

// Frame and EOS of the binary: Binary::Omega / Omega0 (binary.cpp:24-26),
// the centre-of-mass correction force State::fR / ftheta
// (binary_driver.cpp:188-199), State::rho_floor (state_ztwd.cpp:31) and
// State::abar (state_ztwd.cpp:27).
struct ZtwdPar {
    double omega, omega0, fR, ftheta;
    double rho_floor;
    double abar[3];
    HelmTable H;
};

void launch_zt_ghost_fill(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                          const int* slots, int n, cudaStream_t s);
// primitives + fluxes (+ face-averaged normal velocities)
void launch_zt_flux(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                    int n, int* err, cudaStream_t s);
void launch_zt_max_dt(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                      int n, double* dt_out, int* err, cudaStream_t s);
void launch_zt_add_difs(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                        const int* slots, int n, double dt, double beta, int* err, cudaStream_t s);
void launch_zt_inject(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                      const int* slots, int n, int* err, cudaStream_t s);
void launch_zt_prolong(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P,
                       const int* slots, int n, int* err, cudaStream_t s);
// mode 0 pot_to_grid, 1 pot_from_grid, 2 add_pot_et, 3 sub_pot_et
void launch_zt_pot(const Geom& g, const BrickTable& bt, const DevState& st, const ZtwdPar& P, const int* slots,
                   int n, int mode, cudaStream_t s);

}  // namespace amr
