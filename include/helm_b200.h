/* C ABI of the B200 Helmholtz equation of state (helmholtz/helmeos.cpp of
 * STEllAR-GROUP/3d-eulerian-amr), batched.
 *
 * The reference evaluates one point per call on a process-global table that
 * a static constructor reads from ./helmholtz.table (helmeos.cpp:73-130):
 *   helmholtz_eos(eos_t*)                 (p, e, cs, cv, s, dsdt) of (rho, T)
 *   helmholtz_compute_T(eos_t*, bool)     T of (rho, e) or (rho, s) by Newton
 *   helmholtz_set_cgs_units(cm, g, s, K)  code <-> cgs factors
 *   helmholtz_ztwd(p*, e*, zbar, rho)     zero-temperature white dwarf EOS
 * Here a context owns the table on one GPU and every call takes arrays of
 * points: host arrays (the library copies them) or device arrays on a
 * caller's stream.  Where the reference prints and aborts (point outside the
 * table, cv < 0, cs^2 < 0, Newton not converged) the point's status is set
 * instead and the host-array calls return an error code.
 *
 * Status values per point: 0 ok, 1 outside the table (helmeos.cpp:216-221),
 * 2 cv < 0 (:405-409), 3 cs^2 < 0 (:410-415), 4 Newton did not converge in
 * 100 iterations (:477-480), 5 temperature below the table floor (:469-472,
 * :481-484).
 */
#ifndef HELM_B200_H
#define HELM_B200_H

#include "amr_b200.h" /* AMR_OK / AMR_ERR_* codes */

#ifdef __cplusplus
extern "C" {
#endif

#ifndef HELM_CTX_TYPEDEF
#define HELM_CTX_TYPEDEF
typedef struct helm_ctx helm_ctx;
#endif

#define HELM_IMAX 1081 /* densities (log10 ye*rho from -12 to 15), helmeos.cpp:7 */
#define HELM_JMAX 401  /* temperatures (log10 T from 3 to 13), helmeos.cpp:8 */
#define HELM_TMIN 1.0e3

/* read_helm_table (helmeos.cpp:73-130): parse the text table at `path` (9
 * numbers per node, temperature outer, density inner), build the interval
 * tables and upload everything to the current device. */
int helm_create(const char* path, helm_ctx** out);
void helm_destroy(helm_ctx* ctx);
const char* helm_last_error(helm_ctx* ctx);
/* helmholtz_set_cgs_units (helmeos.cpp:132-140). Default: all 1 (cgs). */
int helm_set_cgs_units(helm_ctx* ctx, double cm, double g, double s, double K);

/* helmholtz_eos (helmeos.cpp:164-421) for n points, host arrays.  Any output
 * pointer may be NULL.  Returns AMR_OK, or AMR_ERR_RANGE when some point's
 * status is 1-3 (its outputs are then undefined). */
int helm_eos_batch(helm_ctx* ctx, long long n, const double* rho, const double* T, const double* abar,
                   const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                   int* status);
/* The same on device arrays, asynchronous on `stream` (a cudaStream_t, NULL
 * for the legacy default stream); statuses are left in `status` (required). */
int helm_eos_device(helm_ctx* ctx, long long n, const double* rho, const double* T, const double* abar,
                    const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                    int* status, void* stream);

/* helmholtz_compute_T (helmeos.cpp:436-486) for n points, host arrays:
 * target = e (from_entropy 0) or s (from_entropy 1); T holds the initial
 * guess on entry and the temperature on return.  Outputs p, e, cs, cv, s at
 * that temperature and the Newton iteration count; any may be NULL.  Returns
 * AMR_OK, AMR_ERR_RANGE (status 1-3 or 5) or AMR_ERR_NOCONVERGE (status 4). */
int helm_invert_T_batch(helm_ctx* ctx, long long n, const double* rho, const double* target, const double* abar,
                        const double* zbar, int from_entropy, double* T, double* p, double* e, double* cs,
                        double* cv, double* s, int* iters, int* status);
int helm_invert_T_device(helm_ctx* ctx, long long n, const double* rho, const double* target, const double* abar,
                         const double* zbar, int from_entropy, double* T, double* p, double* e, double* cs,
                         double* cv, double* s, int* iters, int* status, void* stream);

/* helmholtz_ztwd (helmeos.cpp:423-434): zero-temperature white dwarf
 * pressure and energy, host arrays. */
int helm_ztwd_batch(helm_ctx* ctx, long long n, const double* zbar, const double* rho, double* p, double* e);

#ifdef __cplusplus
}
#endif

#endif /* HELM_B200_H */
