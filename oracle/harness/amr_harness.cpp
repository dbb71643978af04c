// Test-oracle driver for the reference AMR code.
//
// This translation unit is compiled together with the reference's own
// grid/, oct_node/, euler/, poisson/ sources (EULER physics selected) by
// oracle/build_ref.py.  It is test infrastructure: it builds octrees, sets
// initial data, runs the reference's own step sequences and writes raw dumps
// that the tests compare the CUDA path against.  Nothing in the product links
// or calls it.
//
// Modes (argv[1]):
//   hydro <ic> <maxlevel> <nsteps> <min_refine_density> <out.bin> [nthreads_hint]
//       Euler step loop of euler/hydro_driver.cpp:171-214 (RK3 + restriction
//       + regrid every step); dt from GridNode::max_dt (grid_node.cpp:163-174)
//       with the MAXDTINC clamp of hydro_driver.cpp:108-113.
//   grav <ic> <maxlevel> <nsteps> <toler> <out.bin>
//       Euler state + self-gravity: Poisson V-cycles (poisson/poisson.cpp)
//       inside the RK3 substep sequence of binary/binary_driver.cpp:296-382,
//       with the gravity coupling of single/single.cpp restated on the
//       Euler state (see GravNode below).
//   poisson <ic> <maxlevel> <ncycles> <out.bin>
//       Builds the tree, then runs `ncycles` V-cycles (Poisson::vcycle,
//       poisson.cpp:1069-1074) and dumps after each.
//   time_hydro / time_grav : same as hydro/grav but prints wall time per
//       step on stdout (JSON) instead of dumping; used as the CPU baseline.
//
// Initial conditions (<ic>): blast, bump, polytrope (defined below).

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include <string>
#include <vector>

// The harness reads the reference's private/protected members (ages,
// refinement flags, Poisson arrays) for the dumps; relax access control for
// the reference headers only.
#define private public
#define protected public
#include "grid/grid_node.h"
#include "poisson/poisson.h"
#include "poisson/poisson_phys_bound.h"
#include "euler/hydro_driver.h"
#include "indexer_2d.h"
extern "C" {
#include "binary/lane_emden.h"
}
#undef private
#undef protected

#ifndef MAXDTINC_H
#define MAXDTINC_H 1.25
#endif

// ---------------------------------------------------------------------------
// initial conditions
// ---------------------------------------------------------------------------
static std::string g_ic = "blast";
static int g_maxlevel = 2;

static const double AMB_P = 1.0e-5;

// blast: rho=1, v=0, p=1e-5; total energy 1.0 spread uniformly over the
// finest-level cells whose centre lies within r < 0.05.
static double blast_energy_density() {
    const double h0 = 2.0 * GRID_DIM / double(GNX - 2 * BW);
    const double h = h0 / double(1 << g_maxlevel);
    const int n = int(0.05 / h) + 2;
    long cnt = 0;
    for (int k = -n; k < n; k++)
        for (int j = -n; j < n; j++)
            for (int i = -n; i < n; i++) {
                const double x = (i + 0.5) * h, y = (j + 0.5) * h, z = (k + 0.5) * h;
                if (sqrt(x * x + y * y + z * z) < 0.05) cnt++;
            }
    return 1.0 / (double(cnt) * h * h * h);
}

// polytrope: n=1.5 Lane-Emden star, central density 1, radius 0.25, centred
// on the origin, ambient floor 1e-10.  K as single/initialize.cpp:16.
static const double POLY_R = 0.25;
static double poly_K() { return pow(POLY_R / 3.65375, 2) * 4.0 * M_PI / (2.5) * pow(1.0, 1.0 / 3.0); }

static double g_blast_e = 0.0;

static void init_cell(GridNode* g, int i, int j, int k) {
    const double gam = State::gamma;
    const double x = g->xc(i), y = g->yc(j), z = g->zc(k);
    double rho = 1.0, vx = 0.0, vy = 0.0, vz = 0.0, p = AMB_P, ei;
    if (g_ic == "blast") {
        ei = p / (gam - 1.0);
        if (sqrt(x * x + y * y + z * z) < 0.05) ei += g_blast_e;
    } else if (g_ic == "bump") {
        const double cx = 0.08, cy = -0.05, cz = 0.06;
        const double r2 = (x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz);
        rho = 1.0 + 9.0 * exp(-r2 / (0.15 * 0.15));
        vx = 0.4;
        vy = 0.25;
        vz = -0.15 + 0.1 * sin(2.0 * M_PI * x);
        p = 0.6;
        ei = p / (gam - 1.0);
    } else if (g_ic == "polytrope") {
        const double K = poly_K();
        const double E1 = sqrt((4.0 * M_PI * pow(1.0, 1.0 - 1.0 / 1.5)) / ((1.5 + 1.0) * K));
        const double h = g->get_dx();
        const int M0 = 2;
        double acc = 0.0;
        for (int k0 = 0; k0 < M0; k0++)
            for (int j0 = 0; j0 < M0; j0++)
                for (int i0 = 0; i0 < M0; i0++) {
                    const double xs = g->xf(i) + (i0 + 0.5) * h / M0;
                    const double ys = g->yf(j) + (j0 + 0.5) * h / M0;
                    const double zs = g->zf(k) + (k0 + 0.5) * h / M0;
                    const double r = sqrt(xs * xs + ys * ys + zs * zs) * E1;
                    if (r < 3.65375) acc += pow(lane_emden(r), 1.5) / double(M0 * M0 * M0);
                }
        rho = acc > 1.0e-10 ? acc : 1.0e-10;
        ei = K * pow(rho, 1.0 + 1.0 / 1.5) / (gam - 1.0);
    } else {
        fprintf(stderr, "unknown ic %s\n", g_ic.c_str());
        exit(2);
    }
    State U = Vector<Real, STATE_NF>(0.0);
    U.set_rho(rho);
    U.set_sx(rho * vx);
    U.set_sy(rho * vy);
    U.set_sz(rho * vz);
    U.set_et(ei + 0.5 * rho * (vx * vx + vy * vy + vz * vz));
    U.set_tau(pow(ei, 1.0 / gam));
    (*g)(i, j, k) = U;
}

// Called by the reference's exec_function (grid_node.cpp:232-241 pattern);
// the reference's euler/initialize.cpp does not compile and is replaced by
// this hook in the oracle build.
void initialize(GridNode* g) {
    for (int k = 0; k < GNX; k++)
        for (int j = 0; j < GNX; j++)
            for (int i = 0; i < GNX; i++) init_cell(g, i, j, k);
}

// ---------------------------------------------------------------------------
// gravity node: the Euler state coupled to the reference Poisson solver.
// compute_phi / compute_source_sums / compute_physical_boundaries restate
// single/single.cpp:207-288 (identical to binary/binary.cpp:938-1019);
// the source terms restate single/single.cpp:49-97 (momentum, no USE_LZ)
// and single/single.cpp:304-383 (ZSTAR energy coupling).
// ---------------------------------------------------------------------------
class GravNode : public Poisson {
public:
    Real src_0[8], src_x[8], src_y[8], src_z[8];
    bool all_refined;
    GravNode() : Poisson() {
        for (int i = 0; i < 8; i++) src_0[i] = src_x[i] = src_y[i] = src_z[i] = 0.0;
        all_refined = false;
    }
    virtual GravNode* new_octnode() const { return new GravNode; }

    virtual Real compute_phi(Real x, Real y, Real z) const {
        Real sum, dx, dy, dz, alpha = 1.0;
#ifdef Z_REFLECT
        alpha *= 2.0;
#endif
        sum = 0.0;
        for (int i = 0; i < 8; i++) {
            dx = x - src_x[i];
            dy = y - src_y[i];
            dz = z - src_z[i];
            if (!all_refined) {
                sum -= alpha * src_0[i] / sqrt(dx * dx + dy * dy + dz * dz);
            } else {
                sum = 0.0;
            }
        }
        for (int i = 0; i < OCT_NCHILD; i++)
            if (get_child(i) != NULL) sum += static_cast<const GravNode*>(get_child(i))->compute_phi(x, y, z);
        return sum;
    }

    void compute_source_sums() {
        if (get_level() == 0) set_source();
        const Indexer2d indexer(1, PNX - 2, 1, PNX - 2);
        const Real h3 = get_dx() * get_dx() * get_dx();
        Real s0[8], sx[8], sy[8], sz[8];
        for (int c = 0; c < 8; c++) s0[c] = sx[c] = sy[c] = sz[c] = 0.0;
        all_refined = true;
        for (int index = 0; index <= indexer.max_index(); index++) {
            const int k = indexer.y(index), j = indexer.x(index);
            for (int i = 1; i < PNX - 1; i++) {
                if (!poisson_zone_is_refined(i, j, k)) {
                    all_refined = false;
                    const int ci = i / (PNX / 2) + ((j / (PNX / 2)) << 1) + ((k / (PNX / 2)) << 2);
                    s0[ci] += S(i, j, k) * h3;
                    sx[ci] += S(i, j, k) * pxc(i) * h3;
                    sy[ci] += S(i, j, k) * pyc(j) * h3;
                    sz[ci] += S(i, j, k) * pzc(k) * h3;
                }
            }
        }
        for (int c = 0; c < 8; c++) {
            if (!all_refined && s0[c] != 0.0) {
                src_x[c] = sx[c] / s0[c];
                src_y[c] = sy[c] / s0[c];
                src_z[c] = sz[c] / s0[c];
                src_0[c] = s0[c] / (4.0 * M_PI);
            } else {
                src_0[c] = 0.0;
                src_x[c] = src_y[c] = src_z[c] = 1.0;
            }
        }
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->compute_source_sums();
    }

    void compute_physical_boundaries(GravNode* root) {
        for (int f = 0; f < OCT_NSIB; f++)
            if (is_phys_bound(f)) static_cast<PoissonPhysBound*>(get_sibling(f))->compute_boundaries(root);
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->compute_physical_boundaries(root);
    }

    // GridNode::sum_*_difs (grid_node.cpp:495-528) followed by the ZSTAR
    // energy coupling of single/single.cpp:304-383: the gravitational work of
    // the face mass flux, 0.5 f(face) * F_rho(face), on both faces of a cell.
    template <int DIR>
    void energy_coupling() {
        const Indexer2d indexer(1, PNX - 2, 1, PNX - 2);
        for (int index = 0; index <= indexer.max_index(); index++) {
            const int k = indexer.y(index), j = indexer.x(index);
            for (int i = 1; i < PNX - 1; i++) {
                const int i0 = i + BW - 1, j0 = j + BW - 1, k0 = k + BW - 1;
                if (DIR == 0) {
                    D(i0, j0, k0)[State::et_index] += 0.5 * fx(i + 0, j, k) * (F(i0 + 0, j0, k0)[State::d_index]);
                    D(i0, j0, k0)[State::et_index] += 0.5 * fx(i + 1, j, k) * (F(i0 + 1, j0, k0)[State::d_index]);
                } else if (DIR == 1) {
                    D(i0, j0, k0)[State::et_index] += 0.5 * fy(i, j + 0, k) * (F(i0, j0 + 0, k0)[State::d_index]);
                    D(i0, j0, k0)[State::et_index] += 0.5 * fy(i, j + 1, k) * (F(i0, j0 + 1, k0)[State::d_index]);
                } else {
                    D(i0, j0, k0)[State::et_index] += 0.5 * fz(i, j, k + 0) * (F(i0, j0, k0 + 0)[State::d_index]);
                    D(i0, j0, k0)[State::et_index] += 0.5 * fz(i, j, k + 1) * (F(i0, j0, k0 + 1)[State::d_index]);
                }
            }
        }
    }
    virtual void sum_x_difs() {
        Grid::sum_x_difs();
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->sum_x_difs();
        energy_coupling<0>();
        if (get_level() == 0) sum_x_flow_off();
    }
    virtual void sum_y_difs() {
        Grid::sum_y_difs();
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->sum_y_difs();
        energy_coupling<1>();
        if (get_level() == 0) sum_y_flow_off();
    }
    virtual void sum_z_difs() {
        Grid::sum_z_difs();
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->sum_z_difs();
        energy_coupling<2>();
        if (get_level() == 0) sum_z_flow_off();
    }

    // single/single.cpp:49-97 without USE_LZ and with ZSTAR: momentum
    // sources from the cell-averaged face forces; then the RK combine.
    void gravity_sources() {
        const Indexer2d indexer(1, PNX - 2, 1, PNX - 2);
        for (int index = 0; index <= indexer.max_index(); index++) {
            const int j = indexer.x(index), k = indexer.y(index);
            for (int i = 1; i < PNX - 1; i++) {
                const int i0 = i + BW - 1, j0 = j + BW - 1, k0 = k + BW - 1;
                Vector<Real, STATE_NF>* Dp = &differential(i0, j0, k0);
                const State s = (*this)(i0, j0, k0);
                const Real fx0 = 0.5 * s.rho() * (fx(i, j, k) + fx(i + 1, j, k));
                const Real fy0 = 0.5 * s.rho() * (fy(i, j, k) + fy(i, j + 1, k));
                const Real fz0 = 0.5 * s.rho() * (fz(i, j, k) + fz(i, j, k + 1));
                (*Dp)[State::sz_index] += fz0;
                (*Dp)[State::sx_index] += fx0;
                (*Dp)[State::sy_index] += fy0;
            }
        }
        for (int c = 0; c < OCT_NCHILD; c++)
            if (get_child(c) != NULL) static_cast<GravNode*>(get_child(c))->gravity_sources();
    }
    virtual void add_difs(Real dt, Real beta) {
        gravity_sources();
        GridNode::add_difs(dt, beta);
    }
};

#include "dump.h"

// ---------------------------------------------------------------------------
// tree construction shared by every mode
// ---------------------------------------------------------------------------
template <class N>
static N* build_tree(double min_refine_density) {
    GridNode::max_refine_level = g_maxlevel;
    GridNode::min_refine_density = min_refine_density;
    g_blast_e = blast_energy_density();
    N* root = new N;
    root->init();
    root->set_time(0.0);
    for (int it = 0; it < g_maxlevel; it++) {
        root->exec_function(initialize);
        root->check_for_refine();
    }
    root->exec_function(initialize);
    // restriction first, then ghost zones, so every ghost slab the step
    // reads is a function of the interior cells alone (the reference's
    // step_to_time does the two in the other order, hydro_driver.cpp:91-92)
    root->inject_from_children();
    root->enforce_boundaries();
    return root;
}

// dt policy for every stepping mode: GridNode::max_dt with the MAXDTINC
// clamp (hydro_driver.cpp:108-113, binary_driver.cpp:116-121) and no
// initial MAXINITDT shrink.
static double next_dt(GridNode* root, int step, double last_dt) {
    double dt = root->max_dt();
    if (step > 0) dt = min(last_dt * MAXDTINC_H, dt);
    return dt;
}

// ---------------------------------------------------------------------------
// gravity driver: binary_driver.cpp:296-382 sequence on GravNode
// ---------------------------------------------------------------------------
struct GravDriver {
    GravNode* root;
    int step_cnt = 0;
    std::vector<double> vcycle_errors;
    int max_cycles = 1000;
    void solve(double tol) {
        root->compute_source_sums();
        root->compute_physical_boundaries(root);
        root->compute_forces();
        double err;
        int iter = 0;
        do {
            if (iter > max_cycles) {
                fprintf(stderr, "too many V-cycles\n");
                exit(4);
            }
            err = root->vcycle();
            vcycle_errors.push_back(err);
            iter++;
        } while (err > tol);
        vcycle_errors.push_back(-double(iter));
        root->inject_from_children();
    }
    void sub_step(double dt, double beta, int rk, double tol) {
        root->enforce_boundaries();
        root->clear_difs();
        root->compute_x_flux();
        root->adjust_x_flux();
        root->sum_x_difs();
        root->compute_y_flux();
        root->adjust_y_flux();
        root->sum_y_difs();
        root->compute_z_flux();
        root->adjust_z_flux();
        root->sum_z_difs();
        root->error_from_parent();
        root->add_difs(dt, beta);
        if (rk == 1) {
            root->store_phi();
        } else if (rk == 2) {
            root->restore_half_phi();
        } else {
            root->restore_phi();
        }
        solve(tol);
    }
    // single/driver.h:83-119 (SingleDriver::step) with DYNAMIC_RANGE from
    // single/single_defs.h:10.
    void step(double dt, double tol) {
        if (step_cnt <= 0) {
            solve(tol);
            root->store_phi();
        }
        root->store();
        sub_step(dt, 1.0, 1, tol);
        sub_step(dt, 0.25, 2, tol);
        sub_step(dt, 2.0 / 3.0, 3, tol);
        root->enforce_boundaries();
        if (step_cnt % 8 == 0) {
            const State smax = root->state_max();
            GridNode::min_refine_density = smax.rho() / 1.0e6;
            if (root->check_for_refine(true)) {
                solve(tol / 10.0);
                root->store_phi();
            }
        }
        step_cnt++;
        root->set_time(root->get_time() + dt);
    }
};

int main(int argc, char* argv[]) {
    if (argc < 2) {
        fprintf(stderr, "usage: see header\n");
        return 2;
    }
    const std::string mode = argv[1];
    if (mode == "hydro" || mode == "time_hydro") {
        if (argc < 7) return 2;
        g_ic = argv[2];
        g_maxlevel = atoi(argv[3]);
        const int nsteps = atoi(argv[4]);
        const double mrd = atof(argv[5]);
        const char* out = argv[6];
        GridNode* root = build_tree<GridNode>(mrd);
        HydroDriver* drv = new HydroDriver(root);
        drv->set_verbosity(0);
        std::vector<double> dts;
        if (mode == "hydro") dump((std::string(out) + ".init").c_str(), root, NULL, root->get_time(), dts);
        double last_dt = 0.0;
        const double t0 = omp_get_wtime();
        for (int s = 0; s < nsteps; s++) {
            const double dt = next_dt(root, s, last_dt);
            last_dt = dt;
            dts.push_back(dt);
            drv->step(dt, false);
        }
        const double t1 = omp_get_wtime();
        if (mode == "hydro") {
            dump(out, root, NULL, root->get_time(), dts);
        } else {
            long leaf = root->get_zone_cnt();
            printf("{\"mode\": \"hydro\", \"steps\": %d, \"seconds\": %.6f, \"leaf_cells\": %ld, \"bricks\": %d, "
                   "\"threads\": %d}\n",
                   nsteps, t1 - t0, leaf, root->get_node_cnt(), omp_get_max_threads());
        }
        return 0;
    }
    if (mode == "grav" || mode == "time_grav") {
        if (argc < 7) return 2;
        g_ic = argv[2];
        g_maxlevel = atoi(argv[3]);
        const int nsteps = atoi(argv[4]);
        const double tol = atof(argv[5]);
        const char* out = argv[6];
        // refinement threshold: state max / DYNAMIC_RANGE as the single-star
        // driver does before every regrid.
        GravNode* root = build_tree<GravNode>(1.0e-6);
        GravDriver drv;
        drv.root = root;
        std::vector<double> extra;
        if (mode == "grav") dump((std::string(out) + ".init").c_str(), root, root, root->get_time(), extra);
        double last_dt = 0.0;
        std::vector<double> dts, step_secs;
        std::vector<int> step_cycles;
        const double t0 = omp_get_wtime();
        for (int s = 0; s < nsteps; s++) {
            const double dt = next_dt(root, s, last_dt);
            last_dt = dt;
            dts.push_back(dt);
            const double ts = omp_get_wtime();
            const size_t nv0 = drv.vcycle_errors.size();
            const long leaf_before = (long)root->get_zone_cnt();
            drv.step(dt, tol);
            step_secs.push_back(omp_get_wtime() - ts);
            int cyc = 0;
            for (size_t q = nv0; q < drv.vcycle_errors.size(); q++)
                if (drv.vcycle_errors[q] >= 0.0) cyc++;
            step_cycles.push_back(cyc);
            if (mode == "time_grav") {
                printf("{\"step\": %d, \"seconds\": %.6f, \"vcycles\": %d, \"bricks\": %d, \"leaf_cells\": %ld}\n", s,
                       step_secs.back(), cyc, root->get_node_cnt(), leaf_before);
                fflush(stdout);
            }
        }
        const double t1 = omp_get_wtime();
        if (mode == "grav") {
            extra.push_back(double(dts.size()));
            extra.insert(extra.end(), dts.begin(), dts.end());
            extra.insert(extra.end(), drv.vcycle_errors.begin(), drv.vcycle_errors.end());
            dump(out, root, root, root->get_time(), extra);
        } else {
            long leaf = root->get_zone_cnt();
            printf("{\"mode\": \"grav\", \"steps\": %d, \"seconds\": %.6f, \"leaf_cells\": %ld, \"bricks\": %d, "
                   "\"threads\": %d, \"vcycles\": %d}\n",
                   nsteps, t1 - t0, leaf, root->get_node_cnt(), omp_get_max_threads(),
                   (int)drv.vcycle_errors.size());
        }
        return 0;
    }
    if (mode == "sample_grav") {
        // Bounded CPU sample of the self-gravitating step: one RK3 hydro step
        // with gravity sources (the substep sequence without its solves) and
        // `nvc` V-cycles, timed separately on the full tree.
        if (argc < 5) return 2;
        g_ic = argv[2];
        g_maxlevel = atoi(argv[3]);
        const int nvc = atoi(argv[4]);
        GravNode* root = build_tree<GravNode>(1.0e-6);
        GravDriver drv;
        drv.root = root;
        root->compute_source_sums();
        root->compute_physical_boundaries(root);
        root->compute_forces();
        root->vcycle();
        const double dt = root->max_dt();
        const double t0 = omp_get_wtime();
        root->store();
        const double betas[3] = {1.0, 0.25, 2.0 / 3.0};
        for (int rk = 0; rk < 3; rk++) {
            root->enforce_boundaries();
            root->clear_difs();
            root->compute_x_flux();
            root->adjust_x_flux();
            root->sum_x_difs();
            root->compute_y_flux();
            root->adjust_y_flux();
            root->sum_y_difs();
            root->compute_z_flux();
            root->adjust_z_flux();
            root->sum_z_difs();
            root->error_from_parent();
            root->add_difs(dt, betas[rk]);
        }
        const double t1 = omp_get_wtime();
        for (int c = 0; c < nvc; c++) root->vcycle();
        const double t2 = omp_get_wtime();
        printf("{\"mode\": \"sample_grav\", \"hydro_rk3_seconds\": %.6f, \"vcycles\": %d, \"vcycle_seconds\": %.6f, "
               "\"leaf_cells\": %ld, \"bricks\": %d, \"threads\": %d}\n",
               t1 - t0, nvc, (t2 - t1) / nvc, (long)root->get_zone_cnt(), root->get_node_cnt(),
               omp_get_max_threads());
        return 0;
    }
    if (mode == "poisson") {
        if (argc < 6) return 2;
        g_ic = argv[2];
        g_maxlevel = atoi(argv[3]);
        const int ncycles = atoi(argv[4]);
        const std::string out = argv[5];
        GravNode* root = build_tree<GravNode>(1.0e-6);
        root->compute_source_sums();
        root->compute_physical_boundaries(root);
        root->compute_forces();
        std::vector<double> errs;
        dump((out + ".init").c_str(), root, root, 0.0, errs);
        for (int c = 0; c < ncycles; c++) {
            errs.push_back(root->vcycle());
            dump((out + "." + std::to_string(c)).c_str(), root, root, 0.0, errs);
        }
        return 0;
    }
    fprintf(stderr, "unknown mode\n");
    return 2;
}
