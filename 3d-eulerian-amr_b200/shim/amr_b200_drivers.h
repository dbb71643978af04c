// Reference-side binding of the B200 library: the reference's own drivers
// with their step running through the C ABI (include/amr_b200.h,
// include/helm_b200.h).
//
// This header belongs to the reference's side: a maintainer adds it to the
// reference tree (it includes the reference's headers and builds with its
// defs.h configuration) and links the reference with
//   -I<repo>/include -L<repo>/3d-eulerian-amr_b200/lib -lamr_b200 -lcudart
//
//   GpuHydroDriver   (EULER build)  replaces HydroDriver::step
//                    (euler/hydro_driver.cpp:171-194)
//   GpuBinaryDriver  (BINARY build) replaces BinaryDriver::step
//                    (binary/binary_driver.cpp:384-459)
//
// The tree and every cell (ghost cells included), the time, the root's
// flow-off, the ages, GridNode::refine_alpha and the Binary statics travel
// between the two sides in the reference's own checkpoint format:
// GridNode::write / read (grid/grid_node.cpp:29-57) and Binary::write /
// read (binary/binary.cpp:70-94, 175-203) on the reference side,
// amr_read_checkpoint / amr_write_checkpoint on the library side, which
// read and write that format byte for byte.  So the binding touches no
// private member of the reference (GridNode::age, GridNode::refine_alpha and
// BinaryDriver::root are private).
#pragma once

#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "amr_b200.h"
#include "helm_b200.h"

namespace amr_b200_bind {

[[noreturn]] inline void fail(amr_ctx* ctx, const char* what) {
    fprintf(stderr, "%s failed: %s\n", what, ctx ? amr_last_error(ctx) : "");
    abort();
}

// The reference's tree and state into the library: root->write, then
// amr_read_checkpoint (hdr receives the Binary header, or NULL).
template <class Root>
void upload(amr_ctx* ctx, const Root* root, amr_binary_header* hdr) {
    char path[] = "/tmp/amr_b200_up_XXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) fail(ctx, "mkstemp");
    FILE* fp = fdopen(fd, "wb");
    if (!fp) fail(ctx, "fdopen");
    root->write(fp);
    fclose(fp);
    const int rc = amr_read_checkpoint(ctx, path, hdr);
    unlink(path);
    if (rc != AMR_OK) fail(ctx, "amr_read_checkpoint");
}

// The library's tree and state back into the reference (the octree may have
// changed on the device): amr_write_checkpoint, then the reference's own
// restart path, GridNode::read on a root whose children are gone.
template <class Root>
void download(amr_ctx* ctx, Root* root, const amr_binary_header* hdr) {
    char path[] = "/tmp/amr_b200_down_XXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) fail(ctx, "mkstemp");
    close(fd);
    if (amr_write_checkpoint(ctx, path, hdr, -1.0) != AMR_OK) {
        unlink(path);
        fail(ctx, "amr_write_checkpoint");
    }
    for (int c = 0; c < OCT_NCHILD; c++)
        if (root->get_child(c)) root->destroy_child(c);
    FILE* fp = fopen(path, "rb");
    if (!fp) fail(ctx, "fopen");
    root->read(fp);
    fclose(fp);
    unlink(path);
}

// The library's configuration for the reference's compile-time one.
inline amr_config reference_config(int physics, int nf) {
    amr_config cfg;
    amr_default_config(&cfg);
    cfg.physics = physics;
    cfg.nf = nf;
    cfg.bw = BW;
    cfg.nx = GNX - 2 * BW;
    cfg.grid_dim = GRID_DIM;
    cfg.cfl = GRID_CFL_FACTOR;
    cfg.maxdtinc = MAXDTINC;
    cfg.minmod_theta = MINMOD_THETA;
    cfg.max_refine_level = GridNode::max_refine_level;
#ifdef Z_REFLECT
    cfg.z_reflect = 1;
#else
    cfg.z_reflect = 0;
#endif
#ifdef MIRROR_REFINE_Y
    cfg.mirror_refine_y = 1;
#else
    cfg.mirror_refine_y = 0;
#endif
#ifdef PPM
    cfg.reconstruction = AMR_RECON_PPM;  // Reconstruct::ppm (reconstruct.cpp:92-102)
#else
    cfg.reconstruction = AMR_RECON_MINMOD;
#endif
    return cfg;
}

}  // namespace amr_b200_bind

#ifdef EULER
// HydroDriver whose step (regrid every step, RK3 with the flux correction)
// runs on the device; the reference tree is brought up to date with
// sync_to_reference() before output or any host-side use of the state.
class GpuHydroDriver : public HydroDriver {
    amr_ctx* ctx_ = nullptr;

public:
    explicit GpuHydroDriver(GridNode* r) : HydroDriver(r) {
        const amr_config cfg = amr_b200_bind::reference_config(AMR_PHYSICS_EULER, STATE_NF);
        if (amr_create(&cfg, &ctx_) != AMR_OK) amr_b200_bind::fail(nullptr, "amr_create");
        amr_b200_bind::upload(ctx_, root, nullptr);
    }
    virtual ~GpuHydroDriver() { amr_destroy(ctx_); }
    virtual void step(Real dt, bool = false) {
        if (amr_hydro_step(ctx_, dt, GridNode::min_refine_density) != AMR_OK)
            amr_b200_bind::fail(ctx_, "amr_hydro_step");
        step_cnt++;
        root->set_time(root->get_time() + dt);
    }
    // GridNode::max_dt of the device state
    Real max_dt() const {
        double dt;
        if (amr_max_dt(ctx_, &dt) != AMR_OK) amr_b200_bind::fail(ctx_, "amr_max_dt");
        return dt;
    }
    void sync_to_reference() { amr_b200_bind::download(ctx_, root, nullptr); }
    amr_ctx* context() const { return ctx_; }
};
#endif

#ifdef BINARY
// BinaryDriver whose step (three RK substeps each followed by the multigrid
// solve, the MAXDTINC retry, the regrid every 8 steps) runs on the device.
// The frame (Omega, Omega0, fR, ftheta) is the host's, as in step_to_time
// (binary_driver.cpp:172-215): it is passed in before every step.
class GpuBinaryDriver : public BinaryDriver {
    Binary* root_;  // BinaryDriver::root is private
    amr_ctx* ctx_ = nullptr;
    helm_ctx* eos_ = nullptr;
    amr_binary_header hdr_{};

public:
    // precision / persistent_solve: AMR_PREC_FP64 and 0 (the defaults) step
    // as the reference does, to round-off; AMR_PREC_MIXED_SOLVE and 1 is the
    // benchmark's form (FP32 multigrid correction, each solve one
    // cooperative kernel)
    explicit GpuBinaryDriver(Binary* r, const char* table = "helmholtz.table", int precision = AMR_PREC_FP64,
                             int persistent_solve = 0)
        : BinaryDriver(r), root_(r) {
        amr_config cfg = amr_b200_bind::reference_config(AMR_PHYSICS_ZTWD, STATE_NF);
        cfg.rho_floor = State::rho_floor;
        cfg.precision = precision;
        cfg.persistent_solve = persistent_solve;
        if (amr_create(&cfg, &ctx_) != AMR_OK) amr_b200_bind::fail(nullptr, "amr_create");
        if (helm_create(table, &eos_) != 0) amr_b200_bind::fail(ctx_, "helm_create");
        helm_set_cgs_units(eos_, Binary::Ucm, Binary::Ug, Binary::Us, 1.0);  // Binary::set_units
        if (amr_ztwd_set_eos(ctx_, eos_) != AMR_OK) amr_b200_bind::fail(ctx_, "amr_ztwd_set_eos");
        amr_b200_bind::upload(ctx_, root_, &hdr_);
    }
    virtual ~GpuBinaryDriver() {
        amr_destroy(ctx_);
        helm_destroy(eos_);
    }
    virtual Real step(Real dt, bool = false) {
        amr_ztwd_set_frame(ctx_, Binary::Omega, Binary::Omega0, State::fR, State::ftheta);
        double used = dt;
        if (amr_ztwd_step(ctx_, dt, ELL_TOLER, DYNAMIC_RANGE, step_cnt, &used) != AMR_OK)
            amr_b200_bind::fail(ctx_, "amr_ztwd_step");
        step_cnt++;
        root_->set_time(root_->get_time() + used);
        return used;
    }
    Real max_dt() const {
        double dt;
        if (amr_max_dt(ctx_, &dt) != AMR_OK) amr_b200_bind::fail(ctx_, "amr_max_dt");
        return dt;
    }
    void sync_to_reference() { amr_b200_bind::download(ctx_, root_, &hdr_); }
    amr_ctx* context() const { return ctx_; }
};
#endif
