/*
 * penguin_b200.h -- C ABI of the B200-native PEnGUIn hydro step.
 *
 * One disk run ("pg_run") owns its grid on one GPU: the conserved-variable
 * planes (Sigma, v_r, v_phi) in FP64, stored ring-major in *physical* azimuth
 * order, plus per-ring FARGO bookkeeping (rot_j, inc_j, rot_v, res_v) and the
 * six fixed ghost rings on each radial edge.  Every entry point returns an
 * int status (PG_OK == 0); the text of the last failure is available from
 * pg_last_error().  Nothing here calls exit() or traps on the device.
 *
 * The reference binds these paths as mangled C++ symbols called only from
 * main.cu kernel(); each declaration below names the reference interface it
 * replaces (file:line within fungjeff/penguin_2_0).
 */
#ifndef PENGUIN_B200_H
#define PENGUIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PG_OK                 0
#define PG_ERR_CUDA           1   /* a CUDA runtime call failed                 */
#define PG_ERR_PARAMS         2   /* unsupported or inconsistent parameters     */
#define PG_ERR_NONFINITE      3   /* NaN/Inf or non-positive density detected   */
#define PG_ERR_DT_COLLAPSE    4   /* dt/endtime < 1e-12 (timestep.cu:143)       */
#define PG_ERR_TIMEOUT        5   /* a bounded device wait gave up              */
#define PG_ERR_IO             6   /* dump file missing / short / wrong size     */
#define PG_ERR_STATE          7   /* dump violates an invariant the run keeps   */
#define PG_ERR_NOMEM          8   /* device allocation failed                   */
#define PG_ERR_ARG            9   /* NULL pointer or bad size                   */

/* ---- parameters ---------------------------------------------------------
 * Field names are those of include/variable_types.h:11-20 and
 * include/global.h:16-96 of the reference, turned from compile-time
 * constants into runtime values.  n_pad (6) and arrsize (128, so 116 interior
 * cells per pencil chunk) are fixed: the sweep results depend on that chunk
 * size (the viscosity stencil at chunk edges sees un-remapped neighbours).   */
/* The reference configures itself with macros of these names (global.h:16-26,
 * variable_types.h); a translation unit that includes its headers before this
 * one would otherwise rename the fields.  Each is set aside for the struct
 * and restored after it.  Such a unit sets fields with pg_params_set.      */
#pragma push_macro("ndim")
#undef ndim
#pragma push_macro("flat_flag")
#undef flat_flag
#pragma push_macro("EOS")
#undef EOS
#pragma push_macro("plnt_flag")
#undef plnt_flag
#pragma push_macro("FrRot_flag")
#undef FrRot_flag
#pragma push_macro("kill_flag")
#undef kill_flag
#pragma push_macro("visc_flag")
#undef visc_flag
#pragma push_macro("FARGO_flag")
#undef FARGO_flag
#pragma push_macro("dump_flag")
#undef dump_flag
typedef struct pg_params {
  /* grid (variable_types.h:11-20) */
  int    ndim;            /* 2 (r-phi) or 3 (r-phi-theta)                      */
  int    imax, jmax, kmax;
  /* physics switches (global.h:16-26); flat_flag 1 == "#define flat_flag"   */
  int    flat_flag, bary_flag, EOS, plnt_flag, FrRot_flag, kill_flag;
  int    visc_flag, FARGO_flag, dump_flag;
  /* disk (global.h:32-37) */
  double p_alpha, p_beta, ss_alpha, sc_h, Sigma_0;
  /* planet (global.h:43-46) */
  double M_p, R_p, t_growth, rs_fac;
  /* hydro (global.h:52-69) */
  double gam, courant;
  int    nlft, nrgh, nudr, ntop;
  double endtime, tmovie;
  int    ncycend, nprin;
  /* grid (global.h:76-96) */
  double xmin, xmax, ymin, ymax, zmin, zmax;
  int    ngeomx, ngeomy, ngeomz;
  int    grspx, grspy, grspz;
  double dx_min, dx_max, dy_min, dy_max, dz_min, dz_max;  /* grid.cu lg 4-6 */
  /* run extras that the reference hard-codes elsewhere or lacks */
  uint64_t seed;          /* splitmix64 seed of the initial-condition noise   */
  double noise_amp;       /* multiplicative Sigma noise amplitude (1e-4)      */
  double kill_rin;        /* wave damping for r < kill_rin (0 = none)         */
  double kill_rout;       /* wave damping for r > kill_rout (0 = none)        */
  int    precision;       /* 0 = FP64 throughout; 1 = FP32 planes, FP64
                             geometry, forces, time step and reductions    */
  int    reserved[7];
} pg_params;
#pragma pop_macro("dump_flag")
#pragma pop_macro("FARGO_flag")
#pragma pop_macro("visc_flag")
#pragma pop_macro("kill_flag")
#pragma pop_macro("FrRot_flag")
#pragma pop_macro("plnt_flag")
#pragma pop_macro("EOS")
#pragma pop_macro("flat_flag")
#pragma pop_macro("ndim")

/* Planet state, same fields and order as struct body (variable_types.h:26-37). */
typedef struct pg_body {
  double m, x, y, vx, vy, fx, fy, rs;
} pg_body;

/* Per-step scalars of the fused device-resident loop (main.cu:343-441). */
typedef struct pg_clock {
  double simtime;   /* main.cu:272                                          */
  double timem;     /* time since last dump, main.cu:273                    */
  double dt;        /* dt carried into the next get_dt (old_dt restored)    */
  double dt_used;   /* dt of the last step actually taken                   */
  double frrot;     /* frame rotation FrRot                                 */
  int64_t ncycle;   /* steps taken                                          */
  int    make_pict; /* last step landed on tmovie or endtime                */
  int    done;      /* endtime reached                                      */
  int    status;    /* device status word (PG_OK or PG_ERR_*)               */
  int    pad;
} pg_clock;

typedef struct pg_run pg_run;

/* ---- parameters / host-side set-up -------------------------------------- */

/* Fills *p with the reference defaults of include/global.h:16-96 and
 * include/variable_types.h:11-20 (imax=850, jmax=2000, kmax=1, ...).       */
int pg_default_params(pg_params *p);

/* Fills *p with a named workload: 0 = 2D 256x768 FP64 disk, 1 = 3D
 * 128x1024x32 spherical disk, 2 = 2D 1024x3072 disk.                       */
int pg_config_params(int which, pg_params *p);

/* Checks a parameter set; PG_ERR_PARAMS with a message for combinations
 * that are not implemented (EOS 2, which the reference marks buggy;
 * bary_flag; EOS 1 on FP32 planes, ...) or whose sweep chunking would read
 * already-updated cells (jmax % 116 in 1..5), and sizes above CUDA's grid
 * limit of 65535 blocks in y (imax, and jmax in 3D).  EOS 0 (isothermal)
 * and EOS 1 (isentropic, p = cs2 Sigma^gam / gam) run in 2D and 3D.        */
int pg_check_params(const pg_params *p);

/* Set or read one field by its name ("EOS", "imax", "sc_h", "seed", ...).
 * For callers whose translation unit includes the reference's configuration
 * headers: their flag macros (EOS, ndim, plnt_flag, FrRot_flag, kill_flag,
 * visc_flag, FARGO_flag, dump_flag, flat_flag) make p->EOS unwritable there,
 * while pg_params_set(p, "EOS", EOS) works.  Integer fields take integral
 * values only; an unknown name or a non-integral value for an integer field
 * gives PG_ERR_ARG and leaves the struct as it was.                        */
int pg_params_set(pg_params *p, const char *name, double value);
int pg_params_get(const pg_params *p, const char *name, double *value);

/* Size in bytes of one hydr_ring record of the dump layout
 * (variable_types.h:67-97): 72*jmax + 96; 0 for jmax <= 0.                 */
size_t pg_ring_bytes(int jmax);

/* Writes the seeded initial condition as a reference-layout dump
 * (binary/binary_<label>_00000, main.cu:124 + output.cu:48-55).  Replaces
 * init_grid/init_den/init_speed/init_cells (init.cpp:3-249) with the noise
 * described by p->seed / p->noise_amp.                                    */
int pg_write_ic(const pg_params *p, const char *path);
int pg_build_ic(const pg_params *p, void *rings, size_t bytes);

/* The fixed boundary rings that init_bound (init.cpp:253-543) sets up, on
 * the grid of *p: per ring PG_BOUNDARY_FIELDS doubles x, dx, xvol, xc, z, dz,
 * zvol, zc, Sigma, p, v_r, v_phi, v_theta, rot_v.  Order: the 6 x kmax inner
 * radial rings (ring i + 6 k), the 6 x kmax outer ones, then in 3D the
 * 6 x imax polar layers below the first layer and the 6 x imax above the
 * last (layer k + 6 i; the ones above hold what ntop = 3 fixes).  These are
 * the values the run loads into its ghost rows and polar ghost layers.
 * *count receives the number of rings; out may be null to ask for it.
 * Host only.                                                               */
#define PG_BOUNDARY_FIELDS 14
int pg_boundary_rings(const pg_params *p, double *out, size_t n_doubles, int *count);

/* Run label of create_label() (output.cu:57-88) into buf.                  */
int pg_label(const pg_params *p, char *buf, size_t len);

/* "<dir>/binary_<label>_<NNNNN>": the dump name of main.cu:124 with
 * frame_num() zero padding (global.cu:27-38).                              */
int pg_dump_name(const pg_params *p, const char *dir, int frame, char *buf, size_t len);

/* files/time_<label>.dat rows (main.cu:417-427): simtime, mass, normalised
 * torque, planet x y vx vy fx fy, eccentricity, semi-major axis.  rows holds
 * 11 doubles per row (the pg_history layout); each is written with 16
 * significant digits, space separated, all 11 when p->plnt_flag > 0 and the
 * first two (simtime, mass) without a planet, as the reference does.       */
int pg_write_time_rows(const pg_params *p, const char *path, const double *rows, int nrows,
                       int append);

/* read/para_<label>.dat of write_para_file (output.cu:90-109).              */
int pg_write_para_file(const pg_params *p, const char *path, const char *mainp);

/* ---- run lifetime -------------------------------------------------------- */

/* Replaces the allocation block of main.cu:141-219.  Device memory is owned
 * by the run; the caller owns only the host buffers passed in.            */
int pg_create(const pg_params *p, int device, pg_run **out);
int pg_destroy(pg_run *run);
const char *pg_last_error(const pg_run *run);
int pg_sync(pg_run *run);

/* Restart path: copy_bfile + copy_grid + init_den/init_speed + init_bound
 * (main.cu:246-284, init.cpp:59-90, 253-413).  rings holds imax*kmax records
 * in the dump layout.                                                      */
int pg_load_rings(pg_run *run, const void *rings, size_t bytes);
int pg_load_dump(pg_run *run, const char *path);
/* save_cells (output.cu:48-55) after a device->host copy (main.cu:400).    */
int pg_save_rings(pg_run *run, void *rings, size_t bytes);
int pg_save_dump(pg_run *run, const char *path);

/* ---- the reference's step entry points ----------------------------------- */

/* get_dt (timestep.cu:112-149): CFL rate max over the grid, then
 * min(1.1*dt_old, courant/max).                                           */
int pg_get_dt(pg_run *run, double dt_old, double frrot, double *dt_out);

/* Index_Shift (orbital_advection.cu:45-69): per-ring inc_j, res_v, rot_v.  */
int pg_index_shift(pg_run *run, double dt, double frrot);

/* bundle_sweep2D (ppm.cu:358-386): radial sweep, azimuthal sweep with the
 * FARGO integer shift applied at its store, rotate_rings.  On a 3D run it
 * does what the reference's bundle_sweep2D does on a 3D build: those two
 * sweeps over every polar layer and rotate_rings, without a polar sweep.  */
int pg_sweep2d(pg_run *run, double dt, const pg_body *planet, double frrot);

/* The 3D counterpart the reference calls at main.cu:376 but never defines:
 * radial, azimuthal and polar sweeps, then rotate_rings.                  */
int pg_sweep3d(pg_run *run, double dt, const pg_body *planet, double frrot);

/* One directional sweep: axis 0 = sweepx (ppm.cu:26-160), 1 = sweepy
 * (ppm.cu:162-307) with the FARGO integer shift applied at its store, 2 =
 * the polar sweep of pg_sweep3d.  rot_j is not advanced: call pg_rotate
 * (rotate_rings, ppm.cu:309-322) after the azimuthal sweep when FARGO is on. */
int pg_sweep_axis(pg_run *run, int axis, double dt, const pg_body *planet, double frrot);
int pg_rotate(pg_run *run);

/* Wave damping toward the initial axisymmetric profile for r < kill_rin and
 * r > kill_rout.  The live reference has no damping (global.h:22); this
 * restates the dead kill_wave.cu:19-40 formula on the current layout.      */
int pg_damp(pg_run *run, double dt);

/* GPU_output_reduction (device_func.cu:169-198): mode 0 disk mass,
 * 8 radial force, 9 torque; same per-ring 1024-wide tree order.            */
int pg_reduce(pg_run *run, const pg_body *planet, double exclude, int mode,
              double *out);

/* ---- planet (planet.cu:11-93), host arithmetic ---------------------------
 * The three functions that return a double (no status) return NaN when given
 * a NULL pointer.                                                          */
int pg_init_planet(const pg_params *p, pg_body *planet, double *frrot);
double pg_set_M_p(const pg_params *p, double t);
int pg_planet_forces(pg_run *run, pg_body *planet, double frrot, double simtime);
int pg_kick_drift_kick(const pg_params *p, pg_body *planet, double *frrot,
                       double dt, int kick);
double pg_get_ecc(const pg_body *planet, double frrot);
double pg_get_E(const pg_body *planet, double frrot);

/* ---- fused device-resident loop ------------------------------------------ */

/* Resets the run clock as main.cu:270-330 does for a restart from frame
 * startat: simtime = tmovie*startat, dt = endtime, planet from init_planet. */
int pg_clock_reset(pg_run *run, int startat);
int pg_clock_get(pg_run *run, pg_clock *clk, pg_body *planet);

/* Advances nsteps steps of main.cu:343-441 with dt, FARGO shift, planet
 * kick-drift-kick and the dt clipping to tmovie/endtime all on the device:
 * no host synchronisation inside.  Stops early (without error) after a
 * step that lands on tmovie or endtime, so the caller can dump.  Torque
 * and mass every nprin steps go to a device history read by
 * pg_history().  *taken gets the number of steps done.                    */
int pg_advance(pg_run *run, int nsteps, int *taken);

/* Copies up to max rows of the diagnostics history (simtime, mass, torque
 * normalised as main.cu:421, planet x, y, vx, vy, fx, fy, ecc, a) recorded
 * since the last call; *rows gets the count.                               */
int pg_history(pg_run *run, double *rows, int max, int *rows_out);

/* Same as pg_advance but with the step sequence captured once in a CUDA
 * graph of `chunk` steps and replayed (launch-bound small grids).          */
int pg_advance_graph(pg_run *run, int nsteps, int chunk, int *taken);

/* ---- device buffers (for harnesses that keep data resident) -------------- */
typedef struct pg_device_view {
  void   *sigma, *vr, *vphi;  /* current planes, first interior ring of the
                                 first polar layer, azimuth in physical order */
  int64_t row_stride;         /* elements between rings                      */
  int64_t slab_stride;        /* elements between polar layers (3D)          */
  int    imax, jmax, kmax;
  int    elem_bytes;          /* 8: double planes (precision 0); 4: float
                                 planes (precision 1), where vphi holds
                                 v_phi minus the ring's initial-state v_phi */
  void  *stream;              /* cudaStream_t the run launches on            */
} pg_device_view;
int pg_device_view_get(pg_run *run, pg_device_view *view);

/* Count of kernel launches issued by this run since creation (kernels inside
 * a replayed CUDA graph count once per replay).                             */
int64_t pg_launch_count(const pg_run *run);

/* Kernel timing with CUDA events on the run's stream.  While enabled, every
 * step enqueued by pg_advance / pg_advance_graph records event pairs around
 * its radial (kind 0), azimuthal (1) and polar (2) sweeps and around the
 * whole step (3).  pg_timing_read synchronises, returns per kind the summed
 * milliseconds and the number of timed launches, and clears the record.    */
int pg_timing(pg_run *run, int on);
int pg_timing_read(pg_run *run, double *ms_sum, int64_t *counts, int nkinds);

/* ---- reduction over caller buffers, no device allocation ---------------- */

/* No counterpart in the reference.  Disk mass (mode 0), radial force (8) or
 * torque (9) of one 2D disk, in GPU_output_reduction's summation order, over
 * device arrays the caller owns: sigma[i*row_stride + j] in physical azimuth
 * order, per ring xc, xvol, rot_j, per column yc, yvol; *out is a device
 * double written by the kernel on `stream` (no host copy, no sync).  For
 * callers that must not allocate device memory (a process whose HBM belongs
 * to its own memory pool, a time loop that allocated everything up front and
 * wants no allocation or its implicit synchronisation inside the loop):
 * the entry point calls no cudaMalloc/cudaFree; its scratch is a static
 * __device__ array of PG_NOALLOC_MAX_RINGS doubles that every GPU loading the
 * library keeps until exit.  imax above that limit returns PG_ERR_PARAMS.
 * The first call on a device looks the array up with cudaGetSymbolAddress
 * (make it before any stream capture); calls share the array, so calls that
 * overlap on the GPU race.  Modes 8 and 9 assume a planet (plnt_flag > 0)
 * and, as the reference, test the exclusion radius on the physical azimuth
 * against planet->y without wrapping.  rot_j may be any int (it is reduced
 * modulo jmax).  For imax <= 1024 the result equals the reference's
 * summation order bit for bit; above that the ring partials are summed in
 * 1024-wide blocks, an extension the reference's output_lv3 does not have. */
#define PG_NOALLOC_MAX_RINGS 16384
int pg_reduce_noalloc(const double *sigma, int64_t row_stride, const double *xc,
                      const double *xvol, const int *rot_j, const double *yc,
                      const double *yvol, int imax, int jmax, const pg_body *planet,
                      double exclude, int mode, double p_alpha, double sc_h,
                      double *out, void *stream);

/* ---- post-processing (the reference's read/ tools) on the device ----------
 * Both read the run's current state in physical azimuth order, which is what
 * read/p_init.cpp:108-133 (update_grid) reconstructs from a dump by undoing
 * each ring's rot_j; load a dump with pg_load_dump to process it.
 * pg_post_harmonic: read/p_output.cpp:35-55 (write_har_file) for layer 0,
 *   an[i] = sum_j sin(m yc_j) Sigma_ij, bn[i] = sum_j cos(m yc_j) Sigma_ij,
 *   an, bn host arrays of imax doubles.
 * pg_post_torque: read/transform.cpp:386-420 (get_torque), the disk's torque
 *   on a planet of mass ratio M_p at r = 1, azimuth pi, barycentric frame.
 * Sums run in a different order from the reference's sequential loops, so
 * they agree to rounding.                                                     */
int pg_post_harmonic(pg_run *run, double m, double *an, double *bn);
int pg_post_torque(pg_run *run, double M_p, double *out);

/* ---- batches: many disks stepped together --------------------------------
 * No counterpart in the reference (one disk per process).  A batch steps its
 * member runs together: per step, one launch per phase walks the pencil
 * chunks of every 2D member of a precision group (FP64 or FP32) through a
 * tile queue, and 3D members take their own launches in the same sequence.
 * Each member keeps its own clock, CFL dt, end time and history, exactly as
 * with pg_advance: a member's results do not depend on the other members or
 * on the launch shape.  Members must be created on the batch's device,
 * loaded and clock-reset; while in a batch they are stepped only through
 * it.  pg_batch_advance enqueues nsteps steps of every member (members whose
 * clock has halted idle) in CUDA graphs of `chunk` steps and returns without
 * waiting; pg_batch_sync waits.  pg_batch_status (synchronising) reports per
 * member, in the order added: halted (end time reached, a tmovie dump due, or
 * an error), its status code and its step count.                           */
typedef struct pg_batch pg_batch;
typedef struct pg_batch_member {
  int     halted;
  int     status;              /* PG_OK or the run's failure code           */
  int64_t ncycle;
  double  simtime;
} pg_batch_member;
typedef struct pg_batch_shape {
  int grid_x, grid_y;          /* CTAs of the batched radial / azimuthal
                                  sweeps (0: one CTA per tile)              */
  int minb;                    /* CTAs per SM the sweeps are compiled for:
                                  8 (64 registers) or 4                     */
  int pad;
} pg_batch_shape;
int pg_batch_create(int device, pg_batch **out);
int pg_batch_destroy(pg_batch *b);
const char *pg_batch_last_error(const pg_batch *b);
int pg_batch_add(pg_batch *b, pg_run *run);
int pg_batch_remove(pg_batch *b, pg_run *run);   /* synchronises */
int pg_batch_size(const pg_batch *b);
int pg_batch_advance(pg_batch *b, int nsteps, int chunk);
int pg_batch_sync(pg_batch *b);
int pg_batch_status(pg_batch *b, pg_batch_member *out, int n);
/* launch shape per precision group (0 = FP64, 1 = FP32) */
int pg_batch_set_shape(pg_batch *b, int group, const pg_batch_shape *shape);
int pg_batch_get_shape(const pg_batch *b, int group, pg_batch_shape *shape);
/* Autotuner: times `trial_steps` real steps of the members for each
 * candidate shape of each group and keeps the fastest.  The trial steps
 * advance the members like any others (results do not depend on the shape). */
int pg_batch_tune(pg_batch *b, int trial_steps);
int64_t pg_batch_launch_count(const pg_batch *b);
/* the cudaStream_t the batch launches on (for events around its work) */
void *pg_batch_stream(const pg_batch *b);
/* device memory pg_create allocates for these parameters (admission) */
size_t pg_run_device_bytes(const pg_params *p);

/* ---- serving: continuous batching of arriving disk runs -------------------
 * A server steps every admitted run in one pg_batch.  pg_server_run_trace
 * replays an arrival trace (requests sorted by arrival time, seconds from the
 * call) against the wall clock: requests queue in arrival order; the head is
 * admitted when fewer than max_slots runs are live and its footprint
 * (pg_run_device_bytes) fits in what is left of hbm_budget; each round
 * enqueues `chunk` steps of all live runs, admits arrivals while they run,
 * then retires runs whose clock halted at their end time.  out[i] receives
 * request i's times (arrival, admission, completion), steps and status.
 * With keep_results, each finished run's final dump stays on the host until
 * pg_server_result copies it out (same layout as pg_save_rings).          */
typedef struct pg_server pg_server;
typedef struct pg_completion {
  int64_t id;
  double  arrival_s, admit_s, finish_s;   /* seconds from the start of the trace */
  int64_t steps;
  int64_t cells;
  double  simtime;
  int     status;                         /* PG_OK, or the run's failure code */
  int     pad;
} pg_completion;
int pg_server_create(int device, size_t hbm_budget, int max_slots, int chunk, int keep_results,
                     pg_server **out);
int pg_server_destroy(pg_server *s);
const char *pg_server_last_error(const pg_server *s);
int pg_server_run_trace(pg_server *s, const pg_params *reqs, const double *arrival_s, const int64_t *ids,
                        int n, pg_completion *out);
int pg_server_result(pg_server *s, int64_t id, void *rings, size_t bytes);
int64_t pg_server_rounds(const pg_server *s);
int pg_server_batch(pg_server *s, pg_batch **out);

#ifdef __cplusplus
}
#endif
#endif /* PENGUIN_B200_H */
