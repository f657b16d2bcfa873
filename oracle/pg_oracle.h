/*
 * pg_oracle.h -- CPU restatement of the PEnGUIn hydro step (TEST
 * INFRASTRUCTURE ONLY).
 *
 * This is the checker the CUDA path is compared against.  It restates, in
 * plain C on the host, the reference's per-block algorithm phase by phase:
 * each __syncthreads()-separated phase of a CUDA block becomes a loop over
 * the block's thread indices, the block's shared arrays keep the same
 * aliasing (al/da/a6 over q/dx/tmp1, cs/csfac over umid/pmid, flux over dx),
 * and every arithmetic expression keeps the reference's operation order.
 * Shared arrays start as NaN in every block so that a read of a value the
 * reference never initialised shows up in the results.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library; the product path never does.
 *
 * Parity is pinned against the reference's own CUDA build (oracle/_ref,
 * built from the reference sources by oracle/ref/build_ref.sh and run on a
 * B200): the golden vectors in tests/golden/ were produced by it.  Its host
 * set-up (ghost rings, damping targets) and its planet functions are pinned
 * bit for bit to the reference's own host code, run through
 * oracle/ref/ic_harness.cu and oracle/ref/planet_harness.cu
 * (tests/test_oracle_setup.py, tests/test_planet_reference.py).
 */
#ifndef PG_ORACLE_H
#define PG_ORACLE_H

#include "../include/penguin_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_run orc_run;

/* Load imax*kmax hydr_ring records (dump layout) and build the fixed ghost
 * rings and the axisymmetric profile exactly as the restart path does
 * (main.cu:246-284).                                                        */
orc_run *orc_create(const pg_params *p, const void *rings, size_t bytes);
void     orc_destroy(orc_run *R);
/* Serialise the current rings in the dump layout.                           */
int      orc_save(const orc_run *R, void *rings, size_t bytes);
/* The fixed ghost rings built at creation (lft, rgh, then udr, top when
 * kmax > 1), 14 doubles each: x dx xvol xc z dz zvol zc r p u v w rot_v.
 * count receives the ring count; out may be NULL to query it.              */
int      orc_boundary(const orc_run *R, double *out, size_t n_doubles, int *count);
/* The damping targets (init.cpp:92-183), r p u v w per ring i + imax k.    */
int      orc_targets(const orc_run *R, double *out, size_t n_doubles);

double orc_get_dt(orc_run *R, double dt_old, double frrot);     /* timestep.cu:112 */
void   orc_index_shift(orc_run *R, double dt, double frrot);    /* orbital_advection.cu:45 */
void   orc_sweepx(orc_run *R, double dt, const pg_body *pl, double frrot);  /* ppm.cu:26 */
void   orc_sweepy(orc_run *R, double dt, const pg_body *pl, double frrot);  /* ppm.cu:162 */
void   orc_sweepz(orc_run *R, double dt, const pg_body *pl, double frrot);
void   orc_rotate(orc_run *R);                                   /* ppm.cu:309 */
void   orc_sweep2d(orc_run *R, double dt, const pg_body *pl, double frrot); /* ppm.cu:358 */
void   orc_sweep3d(orc_run *R, double dt, const pg_body *pl, double frrot);
void   orc_damp(orc_run *R, double dt);
double orc_reduce(orc_run *R, const pg_body *pl, double exclude, int mode); /* device_func.cu:169 */

/* Planet (planet.cu:11-93). */
void   orc_init_planet(const pg_params *p, pg_body *pl, double *frrot);
double orc_set_M_p(const pg_params *p, double t);
void   orc_planet_forces(orc_run *R, pg_body *pl, double frrot, double simtime);
void   orc_kick_drift_kick(const pg_params *p, pg_body *pl, double *frrot,
                           double dt, int kick);
double orc_get_ecc(const pg_body *pl, double frrot);
double orc_get_E(const pg_body *pl, double frrot);

/* The restart-path main loop (main.cu:270-441) for nsteps steps with
 * damping inserted after the sweeps.  hist (may be NULL) receives per step:
 * simtime, dt, mass, torque (normalised as main.cu:421).  Returns steps.   */
int orc_run_steps(orc_run *R, int nsteps, int startat, double *hist);

/* Number of OpenMP threads the oracle uses (1 if built without OpenMP). */
int orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
