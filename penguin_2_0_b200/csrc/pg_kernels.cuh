// pg_kernels.cuh -- device-side data of a run and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pg_ppm.cuh"

namespace pgd {

// Chunking of one pencil direction (ppm.cu:34, 48, 169, 196).
struct Chunking {
  int loop;      // number of 116-cell chunks
  int lim_last;  // lim of the last chunk: n % 116 + 12
  int stuck;     // n % 116 == 0: the reference never updates the last chunk
};

__host__ __device__ inline Chunking make_chunking(int n) {
  Chunking c;
  c.loop = n / REAL + (n % REAL != 0);
  c.lim_last = (n % REAL) + 2 * NPAD;
  c.stuck = (n % REAL == 0);
  return c;
}

// Geometry and per-ring tables, all device pointers.  A "row" counts radial
// rings including the 6 fixed ghost rings on each side (row = i + 6); a
// "ring" index rk = k*nrg + row.
struct Tables {
  int nr, nphi, nk, nrg;
  int occ8;                                     // 128-thread sweeps capped at 64 registers (8 CTAs/SM)
  int zpack;                                    // polar pencils per CTA when nk is one chunk (0: one per CTA)
  int xpack;                                    // radial columns per CTA of the full chunks (1, 2 or 4)
  Chunking cx, cy, cz;
  const double *rx, *rdx, *rxvol, *rxc;         // [nrg]
  const double *radc, *cs2, *nu;                // [nk*nrg]
  const double *gp;                             // [nk*nrg] ghost-ring pressure
  const double *y, *dy, *yvol, *yc;             // [nphi]
  const double *z, *dz, *zvol, *zc;             // [nk + 12]: 6 ghost layers each side
  const double *szc, *czc;                      // [nk + 12]: sin(zc), cos(zc) (k_tables)
  const double *szf, *czf;                      // [nk + 12]: sin(z), cos(z) of the layer faces
  const double *iszc, *iszf, *idz;              // [nk + 12]: 1/sin(zc), 1/sin(z), 1/dz (polar sweep)
  const double *zpar;                           // [5 (nk + 12)]: Eulerian paraset c0..c4 per layer (k_tables)
  const double *nug;                            // [12 nr]: nu of the polar ghost layers (6 below, 6 above) per ring
  const double *val_r, *val_u, *val_v;          // [nk*nrg] damping / FARGO targets
  const double *damp_g, *damp_pw;               // [nk*nrg] zone factor, r^-1.5
  const double *tg;                             // [6*nr*4] theta ghost state (udr): r,p,u,v
  const double *vbg;                            // [nk*nrg] FP32 runs: v_phi background (val.v / ghost v)
  const double *sbg;                            // [nk*nrg] FP32 runs: Sigma background (val.r / ghost r)
  double *res_v, *rot_v;                        // [nk*nrg]
  int *inc_j, *rot_j;                           // [nk*nrg]
};

struct Planes {
  const double *r, *u, *v, *w;
  double *ro, *uo, *vo, *wo;
  const double *p0;   // non-null: pressure of a freshly loaded dump (first sweep only)
};

// FP32 planes: dS = Sigma - S_bg, v_r, dv = v_phi - v_bg, v_theta
struct Planes32 {
  const float *r, *u, *v, *w;
  float *ro, *uo, *vo, *wo;
};

// The device-resident clock of the fused loop (main.cu:270-441).
struct DevClock {
  double simtime, timem, dt, old_dt, dt_step, frrot, frrot_next;
  double endtime, tmovie, courant;
  Body planet;
  long long ncycle, ncycp, ncycend;
  int make_pict, prin, done, halted, status, pad;
  unsigned long long cfl_bits;   // max CFL rate as ordered bits (non-negative)
  int nprin, plnt_flag, frrot_flag, ndim;
  double M_p, t_growth, rs_fac, sc2, R_p, Sigma_0, p_beta;
  double f8, f9;                 // moving planet: disk forces of the step (reductions 8, 9)
  double hist_norm;
  double mass, torque;           // last diagnostics reductions
  double *hist;                  // device history rows (HIST_COLS each)
  int hist_count, hist_cap;
};
constexpr int HIST_COLS = 11;

struct SweepCtl {
  double dt;
  double frrot;
  Body planet;
  DevClock *clk;      // non-null: read dt/planet/frrot from the clock, honour halt
  int fuse;           // sweepy epilogue: damping + CFL + finiteness check
  int shift;          // store at (j + inc_j) mod jmax: the last sweep of a step
  int nocfl;          // with fuse: no CFL rate (a moving planet's FrRot is known only after the step)
};

// Planes a dump is unpacked into / packed from (pg_load_rings, pg_save_rings).
struct DumpPlanes {
  double *r, *u, *v, *w, *p0;    // FP64 run, p0: the dump's pressure
  float *fr, *fu, *fv, *fw;      // FP32 run (residual Sigma and v_phi)
};

// One run of a batch (pg_batch.cu): what its kernels read, in device memory.
struct BatchRun {
  Tables T;
  Phys ph;
  DevClock *clk;
  Planes PX, PY;          // FP64 runs: planes of the radial and of the azimuthal sweep
  Planes32 QX, QY;        // FP32 runs
  const double *p0;       // FP64 run with a freshly loaded dump: its pressure plane,
  long long p0_cycle;     //   read by the radial sweep of the step with ncycle == p0_cycle
  double *ring_part;
  unsigned int *counter;
  double p_alpha;
  int fargo, plnt;
};

// A group of runs walked by one launch: tile t belongs to run r when
// start[r] <= t < start[r + 1].
struct BatchQueue {
  const BatchRun *runs;
  const int *start;       // [nruns + 1] device prefix sums
  int nruns;
  int total;
};

}  // namespace pgd

// launchers (pg_kernels.cu)
namespace pgk {
using namespace pgd;
void tables(const Tables &T, const Phys &ph, int ndim, double kill_rin, double kill_rout, double xmin,
            double xmax, cudaStream_t s);
void sweep_x(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s);
void sweep_y(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s);
void sweep_z(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ntop, cudaStream_t s);
int sweep_launches(const Chunking &ch);
// per-device kernel attributes (dynamic shared memory limits); 0 on success
int setup_device();
int setup_device32();
void cfl_full(const Tables &T, const double *r, const double *u, const double *v, const double *w,
              const double *p0, const Phys &ph, double frrot, int ndim, unsigned long long *out,
              cudaStream_t s);
void index_shift(const Tables &T, double dt, double frrot, int fargo, const DevClock *clk, cudaStream_t s);
void rotate(const Tables &T, const DevClock *clk, cudaStream_t s);
void damp(const Tables &T, double *r, double *u, double *v, double *w, double dt, int ndim, cudaStream_t s);
void reduce(const Tables &T, const double *r, const Body &pl, const DevClock *clk, double exclude,
            int mode, int plnt, double p_alpha, int ndim, double *ring_part, unsigned int *counter,
            double *out, double *hist_row, cudaStream_t s);
void reduce32(const Tables &T, const float *r, const Body &pl, const DevClock *clk, double exclude, int mode,
              int plnt, double p_alpha, int ndim, double *ring_part, unsigned int *counter, double *out,
              cudaStream_t s);
// FP32 sweeps (pg_kernels32.cu)
void sweep_x32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s);
void sweep_y32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s);
void sweep_z32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ntop, cudaStream_t s);
void cfl32(const Tables &T, const Planes32 &cur, const Phys &ph, double frrot, int ndim, int rot_pending,
           unsigned long long *out, int *status, cudaStream_t s);
void damp32(const Tables &T, const Planes32 &cur, double dt, const DevClock *clk, int ndim, cudaStream_t s);
void cfl32_clk(const Tables &T, const Planes32 &cur, const Phys &ph, int ndim, DevClock *clk, cudaStream_t s,
               int rot_pending = 1);
// batched 2D steps over many runs (one launch per phase for all runs)
void batch_prestep(const BatchRun *runs, int nruns, cudaStream_t s);
void batch_poststep(const BatchRun *runs, int nruns, cudaStream_t s);
void batch_record(const BatchRun *runs, int nruns, cudaStream_t s);
void batch_reduce(const BatchQueue &rings, int fp32, int mode, cudaStream_t s);
void batch_sweep_x(const BatchQueue &q, int grid, int minb, cudaStream_t s);
void batch_sweep_x_short(const BatchQueue &q, cudaStream_t s);
void batch_sweep_x32_short(const BatchQueue &q, cudaStream_t s);
void batch_sweep_y(const BatchQueue &q, int grid, int minb, cudaStream_t s);
void batch_sweep_x32(const BatchQueue &q, int grid, int minb, cudaStream_t s);
void batch_sweep_y32(const BatchQueue &q, int grid, int minb, cudaStream_t s);
void damp_clk(const Tables &T, double *r, double *u, double *v, double *w, const DevClock *clk,
              cudaStream_t s);
void cfl_clk(const Tables &T, const double *r, const double *u, const double *v, const double *w,
             const Phys &ph, DevClock *clk, cudaStream_t s);
void prestep(DevClock *clk, const Tables &T, int fargo, cudaStream_t s);
// moving planet (plnt_flag 2): the step's end split around the disk-force reductions
void poststep_drift(DevClock *clk, const Tables &T, cudaStream_t s);
void poststep_kick(DevClock *clk, cudaStream_t s);
void reduce_forces(const Tables &T, const void *r, int fp32, DevClock *clk, double p_alpha, int ndim,
                   double *ring_part, unsigned int *counter, cudaStream_t s);
void cfl_clk_after(const Tables &T, const double *r, const double *u, const double *v, const double *w,
                   const Phys &ph, DevClock *clk, int ndim, cudaStream_t s);
void poststep(DevClock *clk, const Tables &T, cudaStream_t s);
// dump <-> planes: stage holds the dump's field arrays ring by ring ([nr*nk][5][nphi]
// for unpack, whole 72*nphi+96-byte ring records for pack); err bit 1: a density
// that is not finite and positive, bit 2: nonzero w in a 2D dump
void unpack_dump(const Tables &T, const double *stage, const DumpPlanes &D, int ndim, int fp32, int *err,
                 cudaStream_t s);
void fill_ghost_rows(const Tables &T, const double *ghosts, const DumpPlanes &D, int ndim, int fp32,
                     cudaStream_t s);
void pack_dump(const Tables &T, const DumpPlanes &D, const Phys &ph, int ndim, int fp32, int p0_live, unsigned char *out,
               cudaStream_t s);
// post-processing (read/ tools): azimuthal harmonic m per ring of layer 0
// (ab[2i], ab[2i+1]), torque on a planet at r = 1 per ring (ring_out[k*nr+i])
void post_harmonic(const Tables &T, const void *r, int fp32, double m, double *ab, cudaStream_t s);
void post_torque(const Tables &T, const void *r, int fp32, double M_p, double *ring_out, cudaStream_t s);
void record(DevClock *clk, cudaStream_t s);
}  // namespace pgk
