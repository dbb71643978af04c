// Test-oracle driver for the reference's BINARY/ZTWD build.
//
// Compiled by oracle/build_ref.py together with the reference's own grid/,
// oct_node/, poisson/, binary/ and helmholtz/ sources (BINARY physics, ZTWD
// state, PPM with BW 3).  It is test infrastructure: it sets the binary's
// parameters, builds the octree from the reference's own two-polytrope
// initial data (binary/initialize.cpp), runs the reference's own
// BinaryDriver::step (binary/binary_driver.cpp:346-459) and writes raw
// dumps.  Nothing in the product links or calls it.  Needs helmholtz.table
// in the working directory (read by helmholtz/helmeos.cpp:73-130).
//
// Modes (argv[1]):
//   ztwd <maxlevel> <nsteps> <out.bin>
//       tree + initial state, then <nsteps> BinaryDriver::step calls with dt
//       from GridNode::max_dt and the MAXDTINC clamp; dumps <out.bin>.init
//       (before the first step) and <out.bin> (after the last).
//   time_ztwd <maxlevel> <nsteps>
//       the same, printing wall time per step (JSON) instead of dumping.
//   ztwd_chk <maxlevel> <nsteps> <out.bin> <out.chk>
//       as ztwd, then also the reference's checkpoint of the final state
//       (Binary::write, binary/binary.cpp:70-94).
//   read_chk <in.chk> <out.bin>
//       Binary::read of a checkpoint (binary/binary.cpp:175-203), then a dump.
//
// Binary parameters (a stand-in for the missing SCF model X.start.chk):
// mass ratio q = 0.7, separation a = 0.5, donor radius R2 = 0.17 (its Roche
// lobe radius at this q and a, by Eggleton's formula, is 0.174), donor mass
// from M1 = 2.4e-3, n = 1.5 Lane-Emden profiles as binary/initialize.cpp
// builds them; co-rotating frame with Omega = Omega0 = sqrt(M1 (1+q) / a^3),
// synchronous rotation (lz = rho Omega R^2 after initialize); no centre-of-
// mass correction force (fR = 0) and fixed Omega, i.e. BinaryDriver::step
// without the host-side frame updates of step_to_time.

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>

#define private public
#define protected public
#include "binary/binary.h"
#include "binary/binary_driver.h"
#include "grid/grid_node.h"
#include "poisson/poisson.h"
#undef private
#undef protected

#include "dump.h"

static const double ZT_Q = 0.7, ZT_A = 0.5, ZT_R2 = 0.17, ZT_M1 = 2.4e-3;

static void set_binary_parameters() {
    Binary::q = ZT_Q;
    Binary::a = ZT_A;
    Binary::R2 = ZT_R2;
    Binary::R1 = ZT_R2 * pow(ZT_Q, 1.0 / 3.0);
    Binary::M1 = ZT_M1;
    Binary::n = 1.5;
    Binary::Omega = sqrt(Binary::M1 * (Binary::q + 1.0) / (Binary::a * Binary::a * Binary::a));
    Binary::Omega0 = Binary::Omega;
    State::fR = 0.0;
    State::ftheta = 0.0;
}

extern void initialize(GridNode* g);

// synchronous rotation: inertial angular momentum density rho Omega R^2
static void corotate(GridNode* g) {
    for (int k = 0; k < GNX; k++)
        for (int j = 0; j < GNX; j++)
            for (int i = 0; i < GNX; i++) {
                const _3Vec X = g->X(i, j, k);
                const double R2 = X[0] * X[0] + X[1] * X[1];
                (*g)(i, j, k)[State::lz_index] = (*g)(i, j, k).rho() * Binary::Omega * R2;
            }
}

static void init_binary(GridNode* g) {
    initialize(g);
    corotate(g);
}

static Binary* build_tree(int maxlevel) {
    GridNode::max_refine_level = maxlevel;
    Binary* root = new Binary;
    root->init();
    root->set_time(0.0);
    root->exec_function(init_binary);
    GridNode::min_refine_density = root->state_max().rho() / DYNAMIC_RANGE;
    for (int it = 0; it < maxlevel; it++) {
        root->check_for_refine();
        root->exec_function(init_binary);
    }
    root->inject_from_children();
    root->enforce_boundaries();
    return root;
}

int main(int argc, char* argv[]) {
    if (argc == 4 && std::string(argv[1]) == "read_chk") {
        set_binary_parameters();
        Binary* root = new Binary;
        root->init();
        FILE* fp = fopen(argv[2], "rb");
        if (!fp) {
            perror(argv[2]);
            return 3;
        }
        root->read(fp);
        fclose(fp);
        std::vector<double> extra = {Binary::K1, Binary::Omega, Binary::Omega0, Binary::q, Binary::M1};
        dump(argv[3], root, root, root->get_time(), extra);
        return 0;
    }
    if (argc < 4) {
        fprintf(stderr, "usage: %s ztwd|time_ztwd maxlevel nsteps [out.bin]\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1];
    const int maxlevel = atoi(argv[2]);
    const int nsteps = atoi(argv[3]);
    const bool timing = mode == "time_ztwd";
    const bool chk = mode == "ztwd_chk";
    if (!timing && !((mode == "ztwd" && argc >= 5) || (chk && argc >= 6))) {
        fprintf(stderr, "bad arguments\n");
        return 2;
    }
    set_binary_parameters();
    Binary* root = build_tree(maxlevel);
    std::vector<double> extra;
    // units set by initialize (Binary::set_units from K1): kept for the GPU side
    extra.push_back(Binary::K1);
    extra.push_back(Binary::Ucm);
    extra.push_back(Binary::Ug);
    extra.push_back(Binary::Us);
    extra.push_back(Binary::Omega);
    extra.push_back(Binary::Omega0);
    extra.push_back(GridNode::min_refine_density);
    if (!timing) dump((std::string(argv[4]) + ".init").c_str(), root, root, root->get_time(), extra);
    BinaryDriver driver(root);
    double last = 0.0;
    std::vector<double> dts, secs;
    std::vector<long> zones;
    for (int s = 0; s < nsteps; s++) {
        double dt = root->max_dt();
        if (s > 0) dt = min(last * MAXDTINC, dt);
        zones.push_back((long)root->get_zone_cnt());  // leaf cells the step advances
        const double t0 = omp_get_wtime();
        dt = driver.step(dt);
        secs.push_back(omp_get_wtime() - t0);
        last = dt;
        dts.push_back(dt);
    }
    if (timing) {
        printf("{\"steps\": %d, \"bricks\": %d, \"seconds\": [", nsteps, root->get_node_cnt());
        for (size_t i = 0; i < secs.size(); i++) printf("%s%.6f", i ? ", " : "", secs[i]);
        printf("], \"leaf_cells\": [");
        for (size_t i = 0; i < zones.size(); i++) printf("%s%ld", i ? ", " : "", zones[i]);
        printf("], \"threads\": %d}\n", omp_get_max_threads());
        return 0;
    }
    extra.push_back(double(nsteps));
    for (double d : dts) extra.push_back(d);
    // diagnostics of the final state: Binary::mass_sum of both stars,
    // Binary::sum_lz, GridNode::state_sum of the density, Binary::M1M2data
    for (int frac = 0; frac < 2; frac++) {
        const Vector<Real, 4> m = root->mass_sum(frac);
        for (int q = 0; q < 4; q++) extra.push_back(m[q]);
    }
    extra.push_back(root->sum_lz());
    const Vector<State, 4> ss = root->state_sum();
    for (int q = 0; q < 4; q++) extra.push_back(ss[q][0]);
    // Binary::M1M2data (binary/binary.cpp:718-823): L1 point, lobe marking,
    // the per-star and total integrals
    Binary::binary_integrals_t bi;
    root->M1M2data(&bi);
    const double sc[16] = {bi.m1, bi.m2, bi.mc, bi.js1, bi.js2, bi.jorb, bi.jc, bi.a,
                           bi.q,  bi.total_energy, bi.kinetic, bi.I1, bi.I2, bi.Ic, bi.V1, bi.V2};
    for (double v : sc) extra.push_back(v);
    const _3Vec* vec[4] = {&bi.x1, &bi.xdot1, &bi.x2, &bi.xdot2};
    for (const _3Vec* v : vec)
        for (int q = 0; q < 3; q++) extra.push_back((*v)[q]);
    dump(argv[4], root, root, root->get_time(), extra);
    if (chk) {
        FILE* fp = fopen(argv[5], "wb");
        if (!fp) {
            perror(argv[5]);
            return 3;
        }
        root->write(fp);
        fclose(fp);
    }
    return 0;
}
