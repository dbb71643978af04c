/*
 * amr_b200.h -- C ABI of the B200 octree-AMR hydro + gravity step.
 *
 * This is the drop-in boundary for the per-step hot path of
 * STEllAR-GROUP/3d-eulerian-amr.  The reference has no FFI: its operator API
 * is the C++ virtual call surface of the root octree node (GridNode,
 * grid/grid_node.h:46-80; Grid, grid/grid.h:81-97; Poisson,
 * poisson/poisson.h:44-69) driven by HydroDriver / BinaryDriver.  Each entry
 * point below replaces one of those calls on the whole tree (the reference
 * methods recurse from the root; these act on every brick of the tree).
 *
 * Conventions
 *  - Every call returns int status: AMR_OK (0) or a negative AMR_ERR_*; the
 *    reference printf()+abort()s instead (helmholtz/helmeos.cpp:216-221,
 *    binary/binary_driver.cpp:320-324).  amr_last_error() gives the message.
 *  - The library owns all device memory.  Host arrays are plain pointers.
 *  - Bricks are addressed in depth-first pre-order (node, then children
 *    0..7 with ChildIndex = x | y<<1 | z<<2, oct_node/child_index.cpp:13-15),
 *    the order of OctNode::output_tree (oct_node/oct_node.cpp:163-170).
 *  - State arrays are [brick][field][k][j][i], GNX = nx + 2*bw cells per edge
 *    including ghosts, FP64.  Fields (Euler): d, sx, sy, sz, et, tau
 *    (euler/state.cpp:12-17).
 *  - Calls are asynchronous on the context's CUDA stream except those that
 *    return host scalars or host arrays.
 */
#ifndef AMR_B200_H
#define AMR_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AMR_OK 0
#define AMR_ERR_ARG (-1)
#define AMR_ERR_CUDA (-2)
#define AMR_ERR_RANGE (-3)
#define AMR_ERR_NOCONVERGE (-4)
#define AMR_ERR_TIMEOUT (-5)
#define AMR_ERR_STATE (-6)
#define AMR_ERR_CAPACITY (-7)
#define AMR_ERR_NODEVICE (-8)

#define AMR_PHYSICS_EULER 0         /* euler/state.cpp, no gravity */
#define AMR_PHYSICS_EULER_GRAVITY 1 /* Euler state + Poisson self-gravity */
#define AMR_PHYSICS_ZTWD 2          /* BINARY build, ZTWD state (binary/state_ztwd.cpp): 13 fields, Helmholtz
                                       EOS, rotating frame, self-gravity; nf 13, PPM, bw >= 3 */

#define AMR_RECON_MINMOD 0 /* Reconstruct::minmod (reconstruct.cpp:60-71), the EULER build */
#define AMR_RECON_PPM 1    /* Reconstruct::ppm (reconstruct.cpp:22-58), PPM builds; needs bw >= 3 */

#define AMR_PREC_FP64 0  /* plain form: FP64 throughout, reference operation order */
#define AMR_PREC_MIXED 1 /* FP32 KT reconstruction and flux (fluxes accumulated into the FP64 state; the
                            Helmholtz EOS stays FP64) and the FP32 multigrid correction inside FP64
                            defect correction */
#define AMR_PREC_MIXED_SOLVE 2 /* the FP32 multigrid correction only; fluxes in FP64 */

typedef struct amr_ctx amr_ctx;

typedef struct amr_config {
    int bw;               /* BW ghost width (euler/euler_defs.h:28) */
    int nx;               /* interior cells per brick edge, GNX-2*BW (euler_defs.h:30) */
    int nf;               /* STATE_NF (euler/state.h:16) */
    int physics;          /* AMR_PHYSICS_* */
    int precision;        /* AMR_PREC_* */
    int z_reflect;        /* Z_REFLECT: domain z in [0, 2*GRID_DIM], mirror at z=0 */
    int mirror_refine_y;  /* MIRROR_REFINE_Y (euler_defs.h:50) */
    int max_refine_level; /* GridNode::max_refine_level */
    int min_level;        /* MINLEVEL (defs.h:22) */
    int min_grid_life;    /* MIN_GRID_LIFE (defs.h:23) */
    int max_bricks;       /* device brick pool capacity; 0 = host-only context */
    int persistent_solve; /* > 0: the graph forms run each Poisson solve's V-cycle loop as one
                             persistent cooperative kernel (same results bit for bit), with
                             at most this many blocks per SM */
    int reconstruction;   /* AMR_RECON_*: the PPM switch of euler_defs.h:24 (reconstruct.cpp:92-102) */
    double grid_dim;      /* GRID_DIM */
    double origin[3];     /* Grid::origin (grid/grid.h:23) */
    double minmod_theta;  /* MINMOD_THETA (euler_defs.h:21) */
    double cfl;           /* GRID_CFL_FACTOR (euler_defs.h:48) */
    double gamma;         /* State::gamma (euler/state.cpp:9) */
    double rho_floor;     /* State::rho_floor (euler/state.cpp:10) */
    double ei_floor;      /* State::ei_floor (euler/state.cpp:11) */
    double maxdtinc;      /* MAXDTINC (euler_defs.h:47) */
    double grav_g;        /* G_CON (euler/state.h:14) */
} amr_config;

/* Fills the reference's EULER defaults (euler/euler_defs.h, defs.h). */
int amr_default_config(amr_config* cfg);

/* Context: one per tree, one CUDA stream.  cfg->max_bricks == 0 gives a
 * host-only context for octree/refinement logic (every device call then
 * returns AMR_ERR_NODEVICE). */
int amr_create(const amr_config* cfg, amr_ctx** out);
int amr_destroy(amr_ctx* ctx);
const char* amr_last_error(const amr_ctx* ctx);

/* ---- octree (host) ------------------------------------------------------ */
/* GridNode::init (grid/grid_node.cpp:1410-1418): a lone root brick whose six
 * faces are physical boundaries. */
int amr_init_root(amr_ctx* ctx);
/* Rebuild the tree from a depth-first pre-order node list (the order of
 * GridNode::read, grid/grid_node.cpp:45-57): level[n], loc[3n], age[n]. */
int amr_load_tree(amr_ctx* ctx, int n, const int* level, const int* loc, const int* age);
int amr_num_bricks(const amr_ctx* ctx);
/* Tree description in DFS pre-order; any pointer may be NULL. */
int amr_get_tree(const amr_ctx* ctx, int* level, int* loc, int* offset, int* age, int* child_mask,
                 int* refine_mask, double* h);
/* Refinement decision of GridNode::check_for_refine (grid_node.cpp:957-1033)
 * given per-brick octant density flags: flags[8*b+c] != 0 when some interior
 * cell of brick b in octant c has rho > min_refine_density.  Host only;
 * creates/destroys nodes (prolongation of new bricks happens on the device
 * when the context has one).  *changed = use_refine_flags() result. */
int amr_refine_from_flags(amr_ctx* ctx, const unsigned char* flags, int clear, int* changed);
/* Grid::set_time on the whole tree (grid_node.cpp:547-556); t == 0 resets ages. */
int amr_set_time(amr_ctx* ctx, double t);
double amr_get_time(const amr_ctx* ctx);
/* Leaf cells (GridNode::get_zone_cnt, grid_node.cpp:1276-1288). */
long long amr_zone_count(const amr_ctx* ctx);

/* ---- state transfer ------------------------------------------------------ */
int amr_upload_state(amr_ctx* ctx, const double* U);   /* [n][nf][gnx^3] */
int amr_download_state(amr_ctx* ctx, double* U);
/* Poisson arrays phi, phi0, dphi, dphi1, S, fx, fy, fz: [8][n][pnx^3],
 * pnx = nx + 2 (poisson/poisson.h:4). */
int amr_upload_poisson(amr_ctx* ctx, const double* P);
int amr_download_poisson(amr_ctx* ctx, double* P);
/* Root flow-off accumulator FO[nf] (Grid::flow_off, grid/grid.cpp:346). */
int amr_get_flow_off(amr_ctx* ctx, double* fo);
int amr_set_flow_off(amr_ctx* ctx, const double* fo);
int amr_synchronize(amr_ctx* ctx);

/* ---- GridNode call surface (whole tree) --------------------------------- */
int amr_enforce_boundaries(amr_ctx* ctx);          /* grid_node.cpp:59-112 + grid_amr_bound/grid_phys_bound */
int amr_store(amr_ctx* ctx);                       /* grid.cpp:173-186, grid_node.cpp:495-515 */
int amr_restore(amr_ctx* ctx);                     /* grid.cpp:188-199 */
/* compute_{x,y,z}_flux + adjust_{x,y,z}_flux (grid.cpp:215-302,
 * grid_node.cpp:1076-1274). */
int amr_compute_fluxes(amr_ctx* ctx);
/* clear_difs + sum_{x,y,z}_difs (+ flow-off at the root) + add_difs(dt,beta)
 * (grid.cpp:201-213,304-420; grid_node.cpp:337-357,517-551). */
int amr_add_difs(amr_ctx* ctx, double dt, double beta);
int amr_inject_from_children(amr_ctx* ctx);        /* grid_node.cpp:1035-1074 */
int amr_max_dt(amr_ctx* ctx, double* dt);          /* grid.cpp:422-483, grid_node.cpp:163-174 */
/* check_for_refine with the density test on the device. */
int amr_check_for_refine(amr_ctx* ctx, double min_refine_density, int clear, int* changed);
/* GridNode::state_max (grid_node.cpp:1529-1558) for one field. */
int amr_state_max(amr_ctx* ctx, int field, double* vmax);

/* ---- driver sequences ----------------------------------------------------- */
/* HydroDriver::sub_step (euler/hydro_driver.cpp:200-214). */
int amr_sub_step(amr_ctx* ctx, double dt, double beta);
/* amr_sub_step (Euler physics without gravity) as one persistent launch:
 * ghost zones computed where needed, fluxes (FP32 in the mixed form),
 * coarse-fine corrections and the RK combination per brick, finest level
 * first; the result goes to a second state array that then becomes the
 * state.  Interiors are bitwise those of amr_sub_step in the FP64 form; the
 * new state's ghost zones are not filled (amr_enforce_boundaries fills
 * them).  blocks_per_sm > 0 caps the resident blocks per SM (0: as many as
 * fit). */
int amr_fused_sub_step(amr_ctx* ctx, double dt, double beta, int blocks_per_sm);
/* HydroDriver::step (euler/hydro_driver.cpp:171-194): store, RK3 substeps
 * with restriction, boundaries, regrid (min_refine_density), time += dt. */
int amr_hydro_step(amr_ctx* ctx, double dt, double min_refine_density);

/* ---- Poisson (poisson/poisson.h:44-69) ------------------------------------ */
int amr_poisson_set_source(amr_ctx* ctx);                  /* poisson.cpp:950-966 */
int amr_poisson_boundaries(amr_ctx* ctx);                  /* source sums + multipole phys bounds */
int amr_compute_forces(amr_ctx* ctx);                      /* poisson.cpp:223-247 + adjust_*_force */
int amr_vcycle(amr_ctx* ctx, double* l1_error);            /* poisson.cpp:1069-1074 */
int amr_poisson_solve(amr_ctx* ctx, double tol, int max_cycles, double* l1_error, int* cycles);
int amr_store_phi(amr_ctx* ctx);                           /* poisson.cpp:166-181 */
int amr_restore_phi(amr_ctx* ctx);                         /* poisson.cpp:183-198 */
int amr_restore_half_phi(amr_ctx* ctx);                    /* poisson.cpp:200-221 */
/* amr_poisson_boundaries without any device allocation.  No counterpart in
 * the reference: it is for host codes that may not call cudaMalloc once they
 * run (all free device memory handed to their own pool allocator, or a
 * section where an allocation's implicit device synchronisation is not
 * allowed).  Its scratch is a 16 MiB static device array inside this library
 * (held on every GPU that loads the library until exit, shared by all calls:
 * calls that overlap on the GPU race).  It needs the context's Poisson
 * buffers to exist (one earlier ordinary Poisson call, else AMR_ERR_STATE)
 * and rejects trees whose per-point subtree sums exceed the scratch
 * (AMR_ERR_RANGE).  The first call on a device looks up the scratch address;
 * make it before any stream capture.  The context's device must be current. */
int amr_poisson_boundaries_noalloc(amr_ctx* ctx);
/* Self-gravitating RK3 step (binary/binary_driver.cpp:346-459 sequence on the
 * Euler state): per substep hydro + gravity sources, phi time level, solve;
 * regrid every 8 steps at state_max/dynamic_range. */
int amr_grav_step(amr_ctx* ctx, double dt, double tol, double dynamic_range, int step_index);

/* ---- ZTWD binary (AMR_PHYSICS_ZTWD) -----------------------------------------
 * The BINARY build's hydro + gravity with the ZTWD state.  Every entry point
 * above (boundaries, fluxes, add_difs, restriction, CFL step, regrid,
 * Poisson solve) then runs the ZTWD kernels: State::to_prim/to_con,
 * fluxes, eigenvalues, outflow and floor of binary/state_ztwd.cpp with p and
 * c_s from the Helmholtz EOS, Binary::add_difs's gravity and -p div u
 * sources (binary.cpp:205-254), and Binary::pot_to_grid after each solve.
 * Set the EOS and the frame before the first hydro call.  Where the
 * reference aborts inside the EOS (outside the table, Newton failure) the
 * call returns AMR_ERR_RANGE. */
#ifndef HELM_CTX_TYPEDEF
#define HELM_CTX_TYPEDEF
typedef struct helm_ctx helm_ctx;
#endif
/* EOS table and code units (helm_set_cgs_units) of `eos`, which must stay
 * alive while the context uses it; the units are read at this call. */
int amr_ztwd_set_eos(amr_ctx* ctx, helm_ctx* eos);
/* Binary::Omega, Binary::Omega0 (binary.cpp:24-26) and the centre-of-mass
 * correction force State::fR, State::ftheta (binary_driver.cpp:188-199). */
int amr_ztwd_set_frame(amr_ctx* ctx, double omega, double omega0, double fR, double ftheta);
/* binary.cpp:825-936 on every brick: mode 0 Binary::pot_to_grid, 1
 * pot_from_grid (with the phi ghosts of every level), 2 add_pot_et,
 * 3 sub_pot_et. */
int amr_ztwd_pot(amr_ctx* ctx, int mode);
/* BinaryDriver::step (binary_driver.cpp:346-459) without its diagnostics
 * output: on step_index 0 pot_from_grid + the first solve (with
 * phi_from_children) + store_phi; store; three substeps (boundaries, fluxes,
 * Binary::add_difs, phi time level, solve + pot_to_grid + restriction); the
 * MAXDTINC retry (restore and redo with dt / MAXDTINC while the new CFL step
 * is below dt / MAXDTINC); every 8th step the regrid at
 * state_max/dynamic_range between add_pot_et and sub_pot_et, with a solve at
 * tol/10 after a change.  *dt_used gets the step taken.  With
 * amr_config.persistent_solve > 0 (or the mixed precision) each solve runs as
 * amr_graph_solve. */
int amr_ztwd_step(amr_ctx* ctx, double dt, double tol, double dynamic_range, int step_index, double* dt_used);

/* ---- diagnostics (device reductions over the uncovered cells) -------------
 * GridNode::state_sum for one field (grid/grid_node.cpp:1489-1527): out[4] =
 * (sum u h^3, sum u h^3 x, sum u h^3 y, sum u h^3 z).  Binary::mass_sum
 * (binary/binary.cpp:28-68, ZTWD; frac 0 the accretor's density, 1 the
 * donor's): out[4] = (mass, centre of mass x, y, z; z = 0 with Z_REFLECT).
 * Binary::sum_lz (binary.cpp:363-388, ZTWD): the total angular momentum.
 * Per-brick sums in the reference's loop order, added over the tree in its
 * recursion order (results equal the reference's one-thread run). */
int amr_state_sum(amr_ctx* ctx, int field, double* out);
int amr_mass_sum(amr_ctx* ctx, int frac, double* out);
int amr_sum_lz(amr_ctx* ctx, double* out);
/* Binary::M1M2data (binary/binary.cpp:718-823, ZTWD) on the current state,
 * potential (with ghosts) and face forces: the L1 point (find_l1
 * :390-447), the lobe of every cell (mark_lobes :449-492 with the lobe
 * centres of find_phimin :642-690), then out[28] = m1, m2, mc, js1, js2,
 * jorb, jc, a, q, total_energy, kinetic, I1, I2, Ic, V1, V2, x1[3],
 * xdot1[3], x2[3], xdot2[3]; l1[4] (may be NULL) = the L1 point's
 * effective potential, x, y, z.  Searches and sums in the reference's
 * orders. */
int amr_m1m2data(amr_ctx* ctx, double* out, double* l1);

/* ---- checkpoints ------------------------------------------------------------
 * Files in the reference's checkpoint format (X.*.chk): the BINARY build's
 * root header (Binary::write / read, binary/binary.cpp:70-94, 175-203) when
 * hdr is not NULL, then every brick in depth-first pre-order as
 * GridNode::write / Grid::write give it (grid/grid_node.cpp:29-57,
 * grid/grid.cpp:104-146): h, h0, time, offsets and origin, the flow-off
 * vector, the GNX^3 x NF state (ghost cells included, x outermost), the child
 * flags, refine_alpha and the age.  The reader rebuilds the tree, uploads the
 * state and sets the time and the root's flow-off; it checks the offsets and
 * the file length against the context's BW, GNX and NF (AMR_ERR_STATE).
 * The potential is not part of the format (Binary::pot_from_grid rebuilds
 * it from the pot field).  refine_alpha is the value of the reference's
 * static GridNode::refine_alpha written with every brick; a negative value
 * writes the one the last amr_read_checkpoint found (1.0 before any). */
typedef struct amr_binary_header {
    double l1x, h, M1, fill_factor, n, R1, q, a, K1, K2, phi0_1, phi0_2, Omega, phase, Omega0;
    int accretor_type, donor_type;
    unsigned char dummy;
} amr_binary_header;
int amr_write_checkpoint(amr_ctx* ctx, const char* path, const amr_binary_header* hdr, double refine_alpha);
int amr_read_checkpoint(amr_ctx* ctx, const char* path, amr_binary_header* hdr);
/* Headless output in place of the reference's Silo files (GridNode::output,
 * grid/grid_node.cpp:1422-1487): "AMRB200O", int32 {nf, nx, bw, nbricks,
 * has_phi, 0, 0, 0}, double time, then per brick in depth-first pre-order
 * int32 {level, loc[3], offset[3], age, child_mask}, double h, the interior
 * state [nf][nx][nx][nx] and, with self-gravity, the interior potential
 * [nx][nx][nx] (little-endian, no padding).  amr.read_output parses it. */
int amr_write_output(amr_ctx* ctx, const char* path);

/* ---- graph-captured forms --------------------------------------------------
 * The same step and solve with every loop decided on the device: the V-cycle
 * loop and the relaxation loops are CUDA-graph WHILE nodes, the CFL step is
 * reduced on the device, and the captured graph is replayed each step and
 * re-instantiated only when a regrid changes the tree.  Results are those of
 * amr_poisson_solve / amr_grav_step to the last bit. */
int amr_graph_solve(amr_ctx* ctx, double tol, int max_cycles, double* l1_error, int* cycles);
/* dt = GridNode::max_dt clamped to MAXDTINC x the previous step's (no clamp
 * when step_index == 0); *dt_out receives it. */
int amr_graph_grav_step(amr_ctx* ctx, double tol, double dynamic_range, int step_index, double* dt_out);

/* ---- instrumentation ------------------------------------------------------
 * The reference times steps with omp_get_wtime (binary_driver.cpp:115,303);
 * here device time per kernel class comes from CUDA events on the context
 * stream.  Classes 0..19: ghost_fill flux reflux add_difs inject max_dt
 * refine_flags prolong relax vcycle_down phi_boundaries dphi_boundaries
 * forces solution_error source phys_boundary coarse_correction phi_time other
 * fused_substep.
 */
int amr_get_stream(amr_ctx* ctx, void** stream);  /* the context's cudaStream_t */
/* Persistent solve (persistent_solve = 1): device time, count and
 * algorithmic HBM bytes per phase class, summed over the context's
 * persistent solves; n >= 15.  Classes: source restrict phi_faces phi_edges
 * phi_vertices init vcycle_down dphi_faces relax_first relax
 * coarse_correction retire forces adjust_force error.  A phase's time runs
 * from one grid barrier's exit to the next as block 0 sees it (slowest
 * block's work + the barrier). */
int amr_solve_phases(amr_ctx* ctx, double* ms, long long* counts, double* bytes, int n);
/* Duration (CUDA events on the launching stream) of the most recent
 * persistent solve kernel. */
int amr_solve_last_ms(amr_ctx* ctx, float* ms);
/* Total device time (CUDA events around each launch) and number of the
 * persistent solve launches made by amr_graph_solve so far. */
int amr_solve_totals(amr_ctx* ctx, double* ms, long long* count);
/* Relaxation passes (one vcycle_relax call over a level, poisson.cpp:88-130)
 * per level since the context started, in every form of the solve;
 * per_level[0 .. n-1]. */
int amr_relax_passes(amr_ctx* ctx, long long* per_level, int n);
/* Polls each bounded wait of the persistent solve (grid barriers, published
 * level sums) makes before the solve gives up: the waiting block sets the
 * abort word, every block leaves at its next wait, and amr_graph_solve (or
 * the step that called it) returns AMR_ERR_TIMEOUT with the context still
 * usable.  The same limit bounds the fused substep's wait for a finer
 * neighbour's published faces (amr_fused_sub_step then returns
 * AMR_ERR_TIMEOUT; the state is the caller's to restore).  Replaces the
 * reference's unbounded loops; 0 restores the defaults (2^22 polls for the
 * solve, 2^24 for the substep: seconds). */
int amr_set_wait_limit(amr_ctx* ctx, int polls);
/* Block layout of the persistent solve kernel (no reference counterpart:
 * the reference has no kernels): layout 0 .. count-1 of the brick size
 * (8^3: 512 threads, one cell each, two bricks per block on levels with
 * more bricks than blocks; 256 threads, two cells each.  12^3: 576 threads,
 * three cells each; 864, two; 288, six) and the blocks per SM of the launch
 * (0: as many as fit).  Every layout gives the same results bit for bit.
 * The captured graphs are re-captured at their next call.  Needs
 * amr_config.persistent_solve > 0. */
int amr_set_solve_layout(amr_ctx* ctx, int layout, int blocks_per_sm);
/* The persistent solve's shared-memory relaxation loops as its block 0 sees
 * them (that block holds a brick of every level): ms[0..3] = time waiting
 * for the neighbours' passes, computing passes (ghosts and sweeps), waiting
 * for the loop decision, publishing; the passes and Jacobi sweeps it
 * computed.  Accumulated since the context started. */
int amr_solve_relax_split(amr_ctx* ctx, double* ms, long long* passes, long long* sweeps);
/* The persistent solve's block 0 time (ms) in the relaxation loops of each
 * level 0..n-1 (from the level's dphi ghost faces to the loop's closing
 * barrier), accumulated since the context started. */
int amr_solve_relax_level_ms(amr_ctx* ctx, double* ms, int n);
int amr_get_solve_layout(amr_ctx* ctx, int* layout, int* blocks_per_sm, int* threads, int* blocks, int* count);
/* Autotuner of the persistent solve: times a solve to L1 tolerance tol from
 * the context's current potential in every layout with 1, 2 and as many
 * blocks per SM as fit (reps timed solves after an untimed one, the state
 * and the Poisson arrays restored before each: a solve of the ZTWD state
 * also writes its potential field and restricts it), keeps the fastest and
 * leaves the state and the Poisson arrays as they were.  ms[t] (t < ms_cap) receives trial t's mean device
 * time (layout t / 3, blocks per SM 1, 2, all for t % 3; -1 where the trial
 * repeats an earlier launch), *ntrials the number of trials, *best the one
 * kept. */
int amr_autotune_solve(amr_ctx* ctx, double tol, int max_cycles, int reps, double* ms, int ms_cap, int* ntrials,
                       int* best);
/* Of those phase times, the part spent at each phase's closing grid barrier
 * (block 0, from its arrival to the barrier's exit: the slowest block's extra
 * work plus the barrier itself), and the time spent forming the relaxation
 * loops' level sums after their barriers. */
int amr_solve_phase_waits(amr_ctx* ctx, double* wait_ms, int n, double* level_sum_ms, long long* level_sums);
int amr_profile_enable(amr_ctx* ctx, int on);
int amr_profile_reset(amr_ctx* ctx);
int amr_profile_get(amr_ctx* ctx, int cls, double* ms, long long* launches, const char** name);
/* bricks (or correction items) processed by a class's launches */
int amr_profile_units(amr_ctx* ctx, int cls, long long* units);
/* kernels this context has launched so far */
int amr_launch_count(amr_ctx* ctx, long long* kernels);
/* relaxation calls so far, coarse-fine corrections whose depth-first order
 * would matter in the reference (0 under proper nesting), bricks, deepest level */
int amr_stats(amr_ctx* ctx, long long* relax_calls, int* reflux_hazards, int* nbricks, int* max_level);

#ifdef __cplusplus
}
#endif
#endif
