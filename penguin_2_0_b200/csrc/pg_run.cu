// pg_run.cu -- the C ABI of include/penguin_b200.h: one disk run on one GPU.
//
// Device layout of a run (FP64, ring-major, physical azimuth order):
//   planes  r, u (v_r), v (v_phi), w (v_theta, 3D only), two copies (A, B):
//           [nk][nr + 12][nphi], rows 0..5 and nr+6..nr+11 are the fixed
//           ghost rings lft/rgh (init.cpp:253-413), filled at load in both
//           copies and never written by a sweep.  The radial sweep reads A
//           and writes B, the azimuthal sweep reads B and writes A with the
//           FARGO shift applied (so a 2D step ends back in A); the 3D polar
//           sweep reads A and writes B, after which the copies swap roles.
//   p       derived as r*cs2(r_cyl) (the EOS-0 store of ppm.cu:139); the
//           pressure of a freshly loaded dump is kept in a plane `p0` that
//           only the first radial sweep (and the first CFL) reads.
//   tables  per radial row, per ring, per azimuth column, per polar layer.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pg_host.h"
#include "pg_internal.h"
#include "pg_kernels.cuh"

using pgd::NPAD;

struct pg_run {
  pg_params P{};
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int nr = 0, nphi = 0, nk = 0, nrg = 0;
  size_t plane_elems = 0;
  double *planes[2][4] = {{nullptr}};
  float *p32[2][4] = {{nullptr}};      // precision 1: Sigma, v_r, dv_phi, v_theta in FP32
  bool fp32 = false;
  double *vbg = nullptr;   // [nk*nrg] v_phi background of each ring row (FP32 runs)
  double *sbg = nullptr;   // [nk*nrg] Sigma background of each ring row (FP32 runs)
  double *p0 = nullptr;
  bool p0_live = false;
  int cur = 0;
  // tables
  double *tab = nullptr;
  size_t tab_elems = 0;
  int *itab = nullptr;
  pgd::Tables T{};
  pgd::Phys ph{};
  // scratch + clock
  double *ring_part = nullptr;
  unsigned int *counter = nullptr;
  double *dscal = nullptr;
  unsigned long long *cfl = nullptr;
  pgd::DevClock *clk = nullptr;
  double *hist = nullptr;
  int hist_cap = 4096;
  // host side
  bool loaded = false;
  bool clock_ready = false;
  int64_t launches = 0;
  // captured step graphs
  cudaGraphExec_t gexec = nullptr;
  int gsteps = 0;
  int gcur = 0;                    // plane copy current when gexec was captured
  int64_t graph_kernels = 0;       // kernels per replay of gexec
  // early exit of pg_advance*: pinned copies of clk->halted, read a few
  // launches behind the one being queued
  int *h_halt = nullptr;
  cudaEvent_t halt_ev[4] = {};
  // event timing
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_next = 0;
  struct Mark { int kind; size_t a, b; };
  std::vector<Mark> marks;
};

static int ev_pair(pg_run *run, int kind, size_t &a) {
  // reserve two events; record the first now
  while (run->ev_pool.size() < run->ev_next + 2) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return PG_ERR_CUDA;
    run->ev_pool.push_back(e);
  }
  a = run->ev_next;
  run->ev_next += 2;
  if (cudaEventRecord(run->ev_pool[a], run->stream) != cudaSuccess) return PG_ERR_CUDA;
  run->marks.push_back({kind, a, a + 1});
  return PG_OK;
}
static int ev_close(pg_run *run, size_t a) {
  return cudaEventRecord(run->ev_pool[a + 1], run->stream) == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      run->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      return PG_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

static int fail(pg_run *run, int code, const std::string &msg) {
  if (run) run->err = msg;
  // a failed allocation leaves its (non-sticky) error as the runtime's last
  // error; it is reported here, so clear it before a later launch check of
  // any run on this thread reads it as its own
  if (code == PG_ERR_NOMEM) (void)cudaGetLastError();
  return code;
}

static int check_launch(pg_run *run, int n) {
  run->launches += n;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    run->err = std::string("kernel launch: ") + cudaGetErrorString(e);
    return PG_ERR_CUDA;
  }
  return PG_OK;
}

static pgd::Planes32 planes32_fwd(pg_run *run, int src) {
  pgd::Planes32 p;
  p.r = run->p32[src][0]; p.u = run->p32[src][1]; p.v = run->p32[src][2]; p.w = run->p32[src][3];
  p.ro = run->p32[1 - src][0]; p.uo = run->p32[1 - src][1]; p.vo = run->p32[1 - src][2];
  p.wo = run->p32[1 - src][3];
  return p;
}
// the current FP32 planes as both source and target (in-place kernels)
static pgd::Planes32 planes32_cur(pg_run *run) {
  pgd::Planes32 p;
  int c = run->cur;
  p.r = p.ro = run->p32[c][0]; p.u = p.uo = run->p32[c][1]; p.v = p.vo = run->p32[c][2];
  p.w = p.wo = run->p32[c][3];
  return p;
}

static pgd::Planes planes_fwd(pg_run *run, int src, const double *p0) {
  pgd::Planes p;
  p.r = run->planes[src][0]; p.u = run->planes[src][1]; p.v = run->planes[src][2]; p.w = run->planes[src][3];
  p.ro = run->planes[1 - src][0]; p.uo = run->planes[1 - src][1]; p.vo = run->planes[1 - src][2];
  p.wo = run->planes[1 - src][3];
  p.p0 = p0;
  return p;
}

extern "C" {

const char *pg_last_error(const pg_run *run) { return run ? run->err.c_str() : "null run"; }

int64_t pg_launch_count(const pg_run *run) { return run ? run->launches : 0; }

int pg_create(const pg_params *p, int device, pg_run **out) {
  if (!p || !out) return PG_ERR_ARG;
  *out = nullptr;
  std::string why;
  int st = pg::check_params(p, why);
  if (st) {
    std::fprintf(stderr, "pg_create: %s\n", why.c_str());
    return st;
  }
  pg_run *run = new pg_run();
  run->P = *p;
  run->dev = device;
  run->nr = p->imax; run->nphi = p->jmax; run->nk = p->kmax; run->nrg = p->imax + 2 * NPAD;
  auto bail = [&](int code) {
    pg_destroy(run);
    (void)cudaGetLastError();   // reported here: do not leave it for a later launch check
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) { delete run; return PG_ERR_CUDA; }
  if (pgk::setup_device() != 0) return bail(PG_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&run->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(PG_ERR_CUDA);
  run->plane_elems = (size_t)run->nk * run->nrg * run->nphi;
  run->fp32 = (p->precision == 1);
  int nf = (p->ndim == 3) ? 4 : 3;
  for (int b = 0; b < 2; b++)
    for (int f = 0; f < nf; f++) {
      if (run->fp32) {
        if (cudaMalloc(&run->p32[b][f], run->plane_elems * sizeof(float)) != cudaSuccess) return bail(PG_ERR_NOMEM);
      } else {
        if (cudaMalloc(&run->planes[b][f], run->plane_elems * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
      }
    }
  if (!run->fp32 && cudaMalloc(&run->p0, run->plane_elems * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  // double tables
  int nrg = run->nrg, nphi = run->nphi, nk = run->nk, nr = run->nr;
  size_t nring = (size_t)nk * nrg;
  size_t nz = (size_t)nk + 2 * NPAD;
  run->tab_elems = 4 * (size_t)nrg + 10 * nring + 4 * (size_t)nphi + 16 * nz + (size_t)2 * NPAD * nr * 4 +
                   (size_t)2 * NPAD * nr;
  if (cudaMalloc(&run->tab, run->tab_elems * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->itab, 2 * nring * sizeof(int)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  double *t = run->tab;
  pgd::Tables &T = run->T;
  T.nr = nr; T.nphi = nphi; T.nk = nk; T.nrg = nrg;
  {
    // 64-register sweeps (8 CTAs of 128 per SM) by default: ~14% faster on
    // large 2D grids, same arithmetic; PG_SWEEP_OCC=6 keeps ~76 registers
    const char *occ = std::getenv("PG_SWEEP_OCC");
    T.occ8 = (occ && std::atoi(occ) == 6) ? 0 : 1;
    // short chunks packed several per CTA by default: a radial last chunk of
    // at most 64 cells 4 per CTA, an FP64 polar pencil of one chunk 8 per CTA
    // up to 44 cells and 4 above, an FP32 one 4 per CTA (PG_POLAR_PACK=0: one
    // per CTA); same arithmetic per cell either way
    const char *zp = std::getenv("PG_POLAR_PACK");
    T.zpack = (zp && std::atoi(zp) == 0) ? 0 : 4;
    // full radial chunks: 2 adjacent azimuth columns per CTA by default
    // (PG_RADIAL_PACK 1 or 4 for one or four); same arithmetic per cell.
    // Measured on the 128x1024x32 disk: radial 0.727 ms with one column per
    // CTA, 0.660 with two, 0.697 with four
    const char *xp = std::getenv("PG_RADIAL_PACK");
    T.xpack = xp ? std::atoi(xp) : 2;
    if (T.xpack != 2 && T.xpack != 4) T.xpack = 1;
  }
  T.cx = pgd::make_chunking(nr);
  T.cy = pgd::make_chunking(nphi);
  T.cz = pgd::make_chunking(nk);
  T.rx = t; t += nrg; T.rdx = t; t += nrg; T.rxvol = t; t += nrg; T.rxc = t; t += nrg;
  T.radc = t; t += nring; T.cs2 = t; t += nring; T.nu = t; t += nring; T.gp = t; t += nring;
  T.val_r = t; t += nring; T.val_u = t; t += nring; T.val_v = t; t += nring;
  T.damp_g = t; t += nring; T.damp_pw = t; t += nring;
  T.res_v = t; t += nring;
  // rot_v shares the block below (10th ring table)
  T.y = t; t += nphi; T.dy = t; t += nphi; T.yvol = t; t += nphi; T.yc = t; t += nphi;
  T.z = t; t += nz; T.dz = t; t += nz; T.zvol = t; t += nz; T.zc = t; t += nz;
  // szc, czc, szf, czf, iszc, iszf, idz consecutive at stride nz: the polar
  // sweep reads them as lay[0], lay[nz], ... from one pointer per layer
  T.szc = t; t += nz; T.czc = t; t += nz; T.szf = t; t += nz; T.czf = t; t += nz;
  T.iszc = t; t += nz; T.iszf = t; t += nz; T.idz = t; t += nz;
  T.zpar = t; t += 5 * nz;
  T.nug = t; t += (size_t)2 * NPAD * nr;
  T.tg = t; t += (size_t)2 * NPAD * nr * 4;
  if (cudaMalloc(&T.rot_v, nring * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->vbg, nring * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  T.vbg = run->vbg;
  if (cudaMalloc(&run->sbg, nring * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  T.sbg = run->sbg;

  T.inc_j = run->itab; T.rot_j = run->itab + nring;
  // scratch
  if (cudaMalloc(&run->ring_part, (size_t)nr * nk * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->counter, sizeof(unsigned int)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->dscal, 4 * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->cfl, sizeof(unsigned long long)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->clk, sizeof(pgd::DevClock)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMalloc(&run->hist, (size_t)run->hist_cap * pgd::HIST_COLS * sizeof(double)) != cudaSuccess) return bail(PG_ERR_NOMEM);
  if (cudaMemsetAsync(run->counter, 0, sizeof(unsigned int), run->stream) != cudaSuccess) return bail(PG_ERR_CUDA);
  // physics constants
  run->ph.gam = p->gam;
  run->ph.sc2 = p->sc_h * p->sc_h;
  run->ph.vis_nu = p->ss_alpha * p->sc_h * p->sc_h;
  run->ph.p_alpha = p->p_alpha;
  run->ph.p_beta = p->p_beta;
  run->ph.plnt = p->plnt_flag > 0;
  run->ph.flat = p->flat_flag != 0;
  run->ph.visc = p->visc_flag == 1;
  run->ph.eos = p->EOS;
  run->ph.gamfac2 = p->gam + 1.0;
  run->ph.gamfac1 = run->ph.gamfac2 / p->gam / 2.0;
  *out = run;
  return PG_OK;
}

int pg_destroy(pg_run *run) {
  if (!run) return PG_OK;
  cudaSetDevice(run->dev);
  if (run->stream) cudaStreamSynchronize(run->stream);
  if (run->gexec) cudaGraphExecDestroy(run->gexec);
  for (auto e : run->ev_pool) cudaEventDestroy(e);
  for (auto e : run->halt_ev) if (e) cudaEventDestroy(e);
  if (run->h_halt) cudaFreeHost(run->h_halt);
  for (auto &b : run->planes)
    for (auto &f : b) if (f) cudaFree(f);
  for (auto &b : run->p32)
    for (auto &f : b) if (f) cudaFree(f);
  cudaFree(run->vbg);
  cudaFree(run->sbg);
  cudaFree(run->p0);
  cudaFree(run->tab);
  cudaFree(run->itab);
  cudaFree(run->T.rot_v);
  cudaFree(run->ring_part);
  cudaFree(run->counter);
  cudaFree(run->dscal);
  cudaFree(run->cfl);
  cudaFree(run->clk);
  cudaFree(run->hist);
  if (run->stream) cudaStreamDestroy(run->stream);
  delete run;
  return PG_OK;
}

int pg_sync(pg_run *run) {
  if (!run) return PG_ERR_ARG;
  CK(cudaSetDevice(run->dev));
  CK(cudaStreamSynchronize(run->stream));
  return PG_OK;
}

// ---- load / save ----------------------------------------------------------------
int pg_load_rings(pg_run *run, const void *rings, size_t bytes) {
  if (!run || !rings) return PG_ERR_ARG;
  const pg_params &P = run->P;
  size_t rb = pg::ring_bytes(P.jmax);
  if (bytes != rb * (size_t)P.imax * P.kmax)
    return fail(run, PG_ERR_IO, "dump size does not match imax*kmax rings of 72*jmax+96 bytes");
  CK(cudaSetDevice(run->dev));
  const unsigned char *b = (const unsigned char *)rings;
  pg::Geometry g;
  std::string why;
  int st = pg::read_geometry(P, b, g, why);
  if (st) return fail(run, st, why);
  pg::Profile pf{P};
  std::vector<pg::SymDisk> val;
  pg::build_val(pf, g.zxc, g.zzc, val);   // init_den/init_speed on the dump's grid
  const int nr = run->nr, nphi = run->nphi, nk = run->nk, nrg = run->nrg;
  const size_t nring = (size_t)nk * nrg, nz = (size_t)nk + 2 * NPAD;
  // host images of the tables
  std::vector<double> rx(nrg), rdx(nrg), rxvol(nrg), rxc(nrg);
  std::vector<double> gp(nring, 0.0), vr(nring, 0.0), vu(nring, 0.0), vv(nring, 0.0);
  std::vector<double> res_v(nring, 0.0), rot_v(nring, 0.0), vbg(nring, 0.0), sbg(nring, 0.0);
  std::vector<int> inc_j(nring, 0), rot_j(nring, 0);
  std::vector<double> z(nz, 0.0), dz(nz, 0.0), zvol(nz, 0.0), zc(nz, 0.0);
  std::vector<double> tg((size_t)2 * NPAD * nr * 4, 0.0);
  std::vector<pg::GhostRing> lft, rgh, udr, top;
  pg::boundary_rings(pf, g, lft, rgh, udr, top);   // init_bound, init.cpp:253-543
  for (int i = 0; i < NPAD; i++) {
    const pg::GhostRing &L = lft[i], &R = rgh[i];
    rx[i] = L.x; rdx[i] = L.dx; rxvol[i] = L.xvol; rxc[i] = L.xc;
    rx[nr + NPAD + i] = R.x; rdx[nr + NPAD + i] = R.dx; rxvol[nr + NPAD + i] = R.xvol; rxc[nr + NPAD + i] = R.xc;
  }
  for (int i = 0; i < nr; i++) {
    rx[i + NPAD] = g.zxa[i]; rdx[i + NPAD] = g.zdx[i]; rxvol[i + NPAD] = g.xvol[i]; rxc[i + NPAD] = g.zxc[i];
  }
  for (int k = 0; k < nk; k++) {
    for (int i = 0; i < NPAD; i++) {
      size_t a = (size_t)k * nrg + i, c = (size_t)k * nrg + nr + NPAD + i;
      gp[a] = lft[i + NPAD * k].p; rot_v[a] = lft[i + NPAD * k].rot_v; vbg[a] = lft[i + NPAD * k].v; sbg[a] = lft[i + NPAD * k].r;
      gp[c] = rgh[i + NPAD * k].p; rot_v[c] = rgh[i + NPAD * k].rot_v; vbg[c] = rgh[i + NPAD * k].v; sbg[c] = rgh[i + NPAD * k].r;
    }
    for (int i = 0; i < nr; i++) {
      size_t rk = (size_t)k * nrg + i + NPAD;
      pg::RingView rv((unsigned char *)b + rb * (i + (size_t)nr * k), nphi);
      rot_v[rk] = *rv.rot(0); res_v[rk] = *rv.rot(1);
      rot_j[rk] = *rv.rj(0); inc_j[rk] = *rv.rj(1);
      if (rot_j[rk] < 0 || rot_j[rk] >= nphi) return fail(run, PG_ERR_STATE, "rot_j out of range in dump");
      const pg::SymDisk &sv = val[i + (size_t)nr * k];
      vr[rk] = sv.r; vu[rk] = sv.u; vv[rk] = sv.v; vbg[rk] = sv.v; sbg[rk] = sv.r;
    }
  }
  // polar layers: lower ghosts (udr geometry), interior, upper ghosts (top geometry)
  for (int kk = 0; kk < NPAD; kk++) {
    double zl = g.zza[0] - g.zdz[0] * (double)(NPAD - kk), dzl = g.zdz[0];
    z[kk] = zl; dz[kk] = dzl; zc[kk] = zl + 0.5 * dzl; zvol[kk] = pf.vol(zl, dzl, 2);
    double zu = g.zza[nk - 1] + g.zdz[nk - 1] * (double)(kk + 1), dzu = g.zdz[nk - 1];
    size_t q = nk + NPAD + kk;
    z[q] = zu; dz[q] = dzu; zc[q] = zu + 0.5 * dzu; zvol[q] = pf.vol(zu, dzu, 2);
  }
  for (int k = 0; k < nk; k++) {
    z[k + NPAD] = g.zza[k]; dz[k + NPAD] = g.zdz[k]; zvol[k + NPAD] = g.zvol[k]; zc[k + NPAD] = g.zzc[k];
  }
  if (P.ndim == 3) {
    for (int kk = 0; kk < NPAD; kk++)
      for (int i = 0; i < nr; i++) {
        const pg::GhostRing &u = udr[kk + NPAD * i];
        double *q = &tg[((size_t)kk * nr + i) * 4];
        q[0] = u.r; q[1] = u.p; q[2] = u.u; q[3] = u.v;
        const pg::GhostRing &tp = top[kk + NPAD * i];
        q = &tg[((size_t)(NPAD + kk) * nr + i) * 4];
        q[0] = tp.r; q[1] = tp.p; q[2] = tp.u; q[3] = tp.v;
      }
  }
  // ghost rows: phi-uniform r, u, v, p of each fixed radial ghost ring
  std::vector<double> gh((size_t)nk * 2 * NPAD * 4);
  for (int k = 0; k < nk; k++)
    for (int gi = 0; gi < NPAD; gi++) {
      const pg::GhostRing *gs[2] = {&lft[gi + NPAD * k], &rgh[gi + NPAD * k]};
      for (int sd = 0; sd < 2; sd++) {
        double *q = &gh[(((size_t)k * 2 * NPAD) + gi + sd * NPAD) * 4];
        q[0] = gs[sd]->r; q[1] = gs[sd]->u; q[2] = gs[sd]->v; q[3] = gs[sd]->p;
      }
    }
  cudaStream_t s = run->stream;
  pgd::Tables &T = run->T;
  auto up = [&](const double *dst, const std::vector<double> &src) {
    return cudaMemcpyAsync((void *)dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  };
  CK(up(T.rx, rx)); CK(up(T.rdx, rdx)); CK(up(T.rxvol, rxvol)); CK(up(T.rxc, rxc));
  CK(up(T.gp, gp)); CK(up(T.val_r, vr)); CK(up(T.val_u, vu)); CK(up(T.val_v, vv));
  CK(up(T.res_v, res_v)); CK(up(T.rot_v, rot_v)); CK(up(T.vbg, vbg)); CK(up(T.sbg, sbg));
  CK(cudaMemcpyAsync(T.inc_j, inc_j.data(), nring * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(T.rot_j, rot_j.data(), nring * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(up(T.y, g.zya)); CK(up(T.dy, g.zdy)); CK(up(T.yvol, g.yvol)); CK(up(T.yc, g.zyc));
  CK(up(T.z, z)); CK(up(T.dz, dz)); CK(up(T.zvol, zvol)); CK(up(T.zc, zc));
  CK(up(T.tg, tg));
  // the dump's field arrays (the first 40*nphi bytes of each ring record) go
  // to the device as they are and are de-rotated into the planes there
  const size_t pe = run->plane_elems;
  const size_t fbytes = (size_t)40 * nphi;
  double *stage = nullptr, *dgh = nullptr;
  int *derr = nullptr;
  auto release = [&]() { cudaFree(stage); cudaFree(dgh); cudaFree(derr); };
  if (cudaMalloc(&stage, fbytes * nr * nk) != cudaSuccess || cudaMalloc(&dgh, gh.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
    release();
    return fail(run, PG_ERR_NOMEM, "dump staging buffer");
  }
  cudaError_t ce = cudaMemsetAsync(derr, 0, sizeof(int), s);
  if (ce == cudaSuccess) ce = cudaMemcpy2DAsync(stage, fbytes, b, rb, fbytes, (size_t)nr * nk, cudaMemcpyHostToDevice, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(dgh, gh.data(), gh.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  pgd::DumpPlanes D{};
  if (run->fp32) {
    D.fr = run->p32[0][0]; D.fu = run->p32[0][1]; D.fv = run->p32[0][2]; D.fw = run->p32[0][3];
  } else {
    D.r = run->planes[0][0]; D.u = run->planes[0][1]; D.v = run->planes[0][2]; D.w = run->planes[0][3];
    D.p0 = run->p0;
  }
  if (ce == cudaSuccess) {
    pgk::unpack_dump(T, stage, D, P.ndim, run->fp32, derr, s);
    pgk::fill_ghost_rows(T, dgh, D, P.ndim, run->fp32, s);
    ce = cudaGetLastError();
  }
  // the second plane copy starts equal to the first (ghost rows included)
  int nf = (P.ndim == 3) ? 4 : 3;
  for (int f = 0; f < nf && ce == cudaSuccess; f++) {
    if (run->fp32) ce = cudaMemcpyAsync(run->p32[1][f], run->p32[0][f], pe * sizeof(float), cudaMemcpyDeviceToDevice, s);
    else ce = cudaMemcpyAsync(run->planes[1][f], run->planes[0][f], pe * sizeof(double), cudaMemcpyDeviceToDevice, s);
  }
  int herr = 0;
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  release();
  if (ce != cudaSuccess) return fail(run, PG_ERR_CUDA, std::string("dump upload: ") + cudaGetErrorString(ce));
  run->loaded = false;
  if (herr & 1) return fail(run, PG_ERR_STATE, "non-positive density in dump");
  if (herr & 2) return fail(run, PG_ERR_STATE, "2D dump with nonzero w");
  run->launches += 2;
  pgk::tables(T, run->ph, P.ndim, P.kill_rin, P.kill_rout, P.xmin, P.xmax, s);
  if (int e = check_launch(run, 1)) return e;
  CK(cudaStreamSynchronize(s));
  run->cur = 0;
  run->p0_live = !run->fp32;
  run->loaded = true;
  run->clock_ready = false;
  if (run->gexec) { cudaGraphExecDestroy(run->gexec); run->gexec = nullptr; run->gsteps = 0; }
  return PG_OK;
}

int pg_load_dump(pg_run *run, const char *path) {
  if (!run || !path) return PG_ERR_ARG;
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(run, PG_ERR_IO, std::string("cannot open ") + path);
  size_t want = pg::ring_bytes(run->P.jmax) * (size_t)run->P.imax * run->P.kmax;
  std::vector<unsigned char> buf(want);
  size_t got = std::fread(buf.data(), 1, want, f);
  int extra = std::fgetc(f);
  std::fclose(f);
  if (got != want || extra != EOF) return fail(run, PG_ERR_IO, "dump file size does not match the grid");
  return pg_load_rings(run, buf.data(), want);
}

int pg_save_rings(pg_run *run, void *rings, size_t bytes) {
  if (!run || !rings) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  const pg_params &P = run->P;
  size_t rb = pg::ring_bytes(P.jmax);
  if (bytes != rb * (size_t)P.imax * P.kmax) return fail(run, PG_ERR_ARG, "buffer size mismatch");
  CK(cudaSetDevice(run->dev));
  // the whole dump is assembled on the device (fields in storage order,
  // p = Sigma cs2, geometry, rot/inc) and copied back in one transfer
  cudaStream_t s = run->stream;
  unsigned char *stage = nullptr;
  if (cudaMalloc(&stage, bytes) != cudaSuccess) return fail(run, PG_ERR_NOMEM, "dump staging buffer");
  pgd::DumpPlanes D{};
  const int c = run->cur;
  if (run->fp32) {
    D.fr = run->p32[c][0]; D.fu = run->p32[c][1]; D.fv = run->p32[c][2]; D.fw = run->p32[c][3];
  } else {
    D.r = run->planes[c][0]; D.u = run->planes[c][1]; D.v = run->planes[c][2]; D.w = run->planes[c][3];
    D.p0 = run->p0;
  }
  pgk::pack_dump(run->T, D, run->ph, P.ndim, run->fp32, run->p0_live ? 1 : 0, stage, s);
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(rings, stage, bytes, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  cudaFree(stage);
  if (ce != cudaSuccess) return fail(run, PG_ERR_CUDA, std::string("dump download: ") + cudaGetErrorString(ce));
  run->launches += 1;
  return PG_OK;
}

int pg_save_dump(pg_run *run, const char *path) {
  if (!run || !path) return PG_ERR_ARG;
  size_t bytes = pg::ring_bytes(run->P.jmax) * (size_t)run->P.imax * run->P.kmax;
  std::vector<unsigned char> buf(bytes);
  int st = pg_save_rings(run, buf.data(), bytes);
  if (st) return st;
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(run, PG_ERR_IO, std::string("cannot write ") + path);
  size_t w = std::fwrite(buf.data(), 1, bytes, f);
  std::fclose(f);
  return (w == bytes) ? PG_OK : fail(run, PG_ERR_IO, "short write");
}

int pg_device_view_get(pg_run *run, pg_device_view *v) {
  if (!run || !v) return PG_ERR_ARG;
  if (run->fp32) {
    float **fp = run->p32[run->cur];
    v->sigma = fp[0] + (size_t)NPAD * run->nphi;
    v->vr = fp[1] + (size_t)NPAD * run->nphi;
    v->vphi = fp[2] + (size_t)NPAD * run->nphi;
    v->elem_bytes = 4;
  } else {
    v->elem_bytes = 8;
    double **cp = run->planes[run->cur];
    v->sigma = cp[0] + (size_t)NPAD * run->nphi;
    v->vr = cp[1] + (size_t)NPAD * run->nphi;
    v->vphi = cp[2] + (size_t)NPAD * run->nphi;
  }
  v->row_stride = run->nphi;
  v->slab_stride = (int64_t)run->nrg * run->nphi;
  v->imax = run->nr; v->jmax = run->nphi; v->kmax = run->nk;
  v->stream = (void *)run->stream;
  return PG_OK;
}

// ---- the reference's entry points ---------------------------------------------
int pg_get_dt(pg_run *run, double dt_old, double frrot, double *dt_out) {
  if (!run || !dt_out) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  cudaStream_t s = run->stream;
  double **cp = run->planes[run->cur];
  CK(cudaMemsetAsync(run->cfl, 0, sizeof(unsigned long long), s));
  if (run->fp32)
    pgk::cfl32(run->T, planes32_cur(run), run->ph, frrot, run->P.ndim, 0, run->cfl, nullptr, s);
  else
    pgk::cfl_full(run->T, cp[0], cp[1], cp[2], cp[3], run->p0_live ? run->p0 : nullptr, run->ph, frrot,
                  run->P.ndim, run->cfl, s);
  if (int e = check_launch(run, 1)) return e;
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, run->cfl, sizeof(bits), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double rate;
  std::memcpy(&rate, &bits, sizeof(rate));
  double h = run->P.courant / rate;       // dt_lv3 timestep.cu:105
  double dt = 1.1 * dt_old;               // timestep.cu:135-141
  dt = (h < dt) ? h : dt;
  *dt_out = dt;
  if (dt / run->P.endtime < 1.0e-12) return fail(run, PG_ERR_DT_COLLAPSE, "time step too small");
  return PG_OK;
}

int pg_index_shift(pg_run *run, double dt, double frrot) {
  if (!run) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  pgk::index_shift(run->T, dt, frrot, run->P.FARGO_flag, nullptr, run->stream);
  return check_launch(run, 1);
}

static pgd::SweepCtl host_ctl(double dt, const pg_body *pl, double frrot) {
  pgd::SweepCtl c{};
  c.dt = dt;
  c.frrot = frrot;
  c.planet = pgd::Body{pl->m, pl->x, pl->y, pl->vx, pl->vy, pl->fx, pl->fy, pl->rs};
  c.clk = nullptr;
  c.fuse = 0;
  c.shift = 0;
  return c;
}

static int nx(pg_run *run) { return pgk::sweep_launches(run->T.cx); }
static int ny(pg_run *run) { return pgk::sweep_launches(run->T.cy); }
static int nz(pg_run *run) { return pgk::sweep_launches(run->T.cz); }

// On a 3D run this is what the reference's bundle_sweep2D does on a 3D
// build: the radial and azimuthal sweeps of every polar layer (sweepx takes
// the layer from blockIdx.y, ppm.cu:33; sweepy folds it into the ring index,
// ppm.cu:168) and rotate_rings, with no polar sweep.
int pg_sweep2d(pg_run *run, double dt, const pg_body *planet, double frrot) {
  if (!run || !planet) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  pgd::SweepCtl c = host_ctl(dt, planet, frrot);
  cudaStream_t s = run->stream;
  const int nd = run->P.ndim;
  if (run->fp32) {
    pgk::sweep_x32(run->T, planes32_fwd(run, run->cur), run->ph, c, nd, s);
    c.shift = 1;
    pgk::sweep_y32(run->T, planes32_fwd(run, 1 - run->cur), run->ph, c, nd, s);
  } else {
    pgk::sweep_x(run->T, planes_fwd(run, run->cur, run->p0_live ? run->p0 : nullptr), run->ph, c, nd, s);
    c.shift = 1;
    pgk::sweep_y(run->T, planes_fwd(run, 1 - run->cur, nullptr), run->ph, c, nd, s);
  }
  if (run->P.FARGO_flag > 0) pgk::rotate(run->T, nullptr, s);
  run->p0_live = false;
  return check_launch(run, nx(run) + ny(run) + (run->P.FARGO_flag > 0 ? 1 : 0));
}

int pg_sweep3d(pg_run *run, double dt, const pg_body *planet, double frrot) {
  if (!run || !planet) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  if (run->P.ndim != 3) return fail(run, PG_ERR_PARAMS, "pg_sweep3d on a 2D run");
  CK(cudaSetDevice(run->dev));
  pgd::SweepCtl c = host_ctl(dt, planet, frrot);
  cudaStream_t s = run->stream;
  int a = run->cur;
  if (run->fp32) {
    pgk::sweep_x32(run->T, planes32_fwd(run, a), run->ph, c, 3, s);
    pgk::sweep_y32(run->T, planes32_fwd(run, 1 - a), run->ph, c, 3, s);
    c.shift = 1;
    pgk::sweep_z32(run->T, planes32_fwd(run, a), run->ph, c, run->P.ntop, s);
  } else {
    pgk::sweep_x(run->T, planes_fwd(run, a, run->p0_live ? run->p0 : nullptr), run->ph, c, 3, s);
    pgk::sweep_y(run->T, planes_fwd(run, 1 - a, nullptr), run->ph, c, 3, s);
    c.shift = 1;   // the polar sweep is the last one: it applies the FARGO shift
    pgk::sweep_z(run->T, planes_fwd(run, a, nullptr), run->ph, c, run->P.ntop, s);
  }
  if (run->P.FARGO_flag > 0) pgk::rotate(run->T, nullptr, s);
  run->cur = 1 - a;
  run->p0_live = false;
  return check_launch(run, nx(run) + ny(run) + nz(run) + (run->P.FARGO_flag > 0 ? 1 : 0));
}

int pg_sweep_axis(pg_run *run, int axis, double dt, const pg_body *planet, double frrot) {
  if (!run || !planet) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  if (axis < 0 || axis > 2 || (axis == 2 && run->P.ndim != 3)) return fail(run, PG_ERR_ARG, "bad sweep axis");
  CK(cudaSetDevice(run->dev));
  pgd::SweepCtl c = host_ctl(dt, planet, frrot);
  cudaStream_t s = run->stream;
  int a = run->cur;
  // the FARGO shift goes with the last sweep of a step: azimuthal in 2D,
  // polar in 3D.  The dump's p is used only by a leading radial sweep.
  int n = 0;
  if (axis == 0) {
    if (run->fp32) pgk::sweep_x32(run->T, planes32_fwd(run, a), run->ph, c, run->P.ndim, s);
    else pgk::sweep_x(run->T, planes_fwd(run, a, run->p0_live ? run->p0 : nullptr), run->ph, c, run->P.ndim, s);
    n = nx(run);
  } else if (axis == 1) {
    c.shift = run->P.ndim == 2;
    if (run->fp32) pgk::sweep_y32(run->T, planes32_fwd(run, a), run->ph, c, run->P.ndim, s);
    else pgk::sweep_y(run->T, planes_fwd(run, a, nullptr), run->ph, c, run->P.ndim, s);
    n = ny(run);
  } else {
    c.shift = 1;
    if (run->fp32) pgk::sweep_z32(run->T, planes32_fwd(run, a), run->ph, c, run->P.ntop, s);
    else pgk::sweep_z(run->T, planes_fwd(run, a, nullptr), run->ph, c, run->P.ntop, s);
    n = nz(run);
  }
  run->cur = 1 - a;
  run->p0_live = false;
  return check_launch(run, n);
}

int pg_rotate(pg_run *run) {
  if (!run) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  pgk::rotate(run->T, nullptr, run->stream);
  return check_launch(run, 1);
}

int pg_damp(pg_run *run, double dt) {
  if (!run) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  if (run->fp32) {
    pgk::damp32(run->T, planes32_cur(run), dt, nullptr, run->P.ndim, run->stream);
  } else {
    double **cp = run->planes[run->cur];
    pgk::damp(run->T, cp[0], cp[1], cp[2], cp[3], dt, run->P.ndim, run->stream);
  }
  return check_launch(run, 1);
}

int pg_reduce(pg_run *run, const pg_body *planet, double exclude, int mode, double *out) {
  if (!run || !planet || !out) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  if (mode != 0 && mode != 8 && mode != 9) return fail(run, PG_ERR_ARG, "mode must be 0, 8 or 9");
  if (run->P.ndim == 3 && run->nk > 64) return fail(run, PG_ERR_PARAMS, "3D reductions support kmax <= 64");
  CK(cudaSetDevice(run->dev));
  pgd::Body b{planet->m, planet->x, planet->y, planet->vx, planet->vy, planet->fx, planet->fy, planet->rs};
  exclude *= run->P.sc_h;                                 // device_func.cu:171
  if (run->fp32)
    pgk::reduce32(run->T, run->p32[run->cur][0], b, nullptr, exclude, mode, run->P.plnt_flag > 0,
                  run->P.p_alpha, run->P.ndim, run->ring_part, run->counter, run->dscal, run->stream);
  else
    pgk::reduce(run->T, run->planes[run->cur][0], b, nullptr, exclude, mode, run->P.plnt_flag > 0,
                run->P.p_alpha, run->P.ndim, run->ring_part, run->counter, run->dscal, nullptr, run->stream);
  if (int e = check_launch(run, 1)) return e;
  CK(cudaMemcpyAsync(out, run->dscal, sizeof(double), cudaMemcpyDeviceToHost, run->stream));
  CK(cudaStreamSynchronize(run->stream));
  *out = 0.0 + *out;                                       // host sum device_func.cu:195
  return PG_OK;
}

// ---- planet, planet.cu:11-93 (host arithmetic as in the reference) --------------
double pg_set_M_p(const pg_params *p, double t) {
  if (!p) return std::nan("");
  if (t < p->t_growth) return std::fmax(p->M_p * std::sin(pg::kPi * t / (2.0 * p->t_growth)), 0.01 * pg::kEarthMass);
  return p->M_p;
}

int pg_init_planet(const pg_params *p, pg_body *pl, double *frrot) {
  if (!p || !pl || !frrot) return PG_ERR_ARG;
  pg::Profile pf{*p};
  pl->m = pg_set_M_p(p, 0.0);
  pl->x = p->R_p;
  pl->y = pg::kPi;
  pl->vx = 0.0;
  pl->vy = std::pow(pl->x, -1.5);
  *frrot = (p->FrRot_flag == 1) ? pl->vy : 0.0;
  pl->vy -= *frrot;
  pl->rs = p->rs_fac * pf.h(pl->x);
  pl->fx = 0.0; pl->fy = 0.0;
  return PG_OK;
}

int pg_planet_forces(pg_run *run, pg_body *pl, double frrot, double simtime) {
  if (!run || !pl) return PG_ERR_ARG;
  const pg_params &P = run->P;
  pl->m = pg_set_M_p(&P, simtime);
  if (P.plnt_flag == 2) {
    double f8 = 0.0, f9 = 0.0;
    int st = pg_reduce(run, pl, 0.0, 8, &f8);
    if (st) return st;
    pl->fx = P.Sigma_0 * f8 / pl->m - 1.0 / pl->x / pl->x + pl->x * std::pow(pl->vy + frrot, 2);
    st = pg_reduce(run, pl, 0.0, 9, &f9);
    if (st) return st;
    pl->fy = P.Sigma_0 * f9 / pl->m;
  } else {
    pl->fx = -1.0 / pl->x / pl->x + pl->x * std::pow(pl->vy + frrot, 2);
    pl->fy = 0.0;
  }
  return PG_OK;
}

int pg_kick_drift_kick(const pg_params *p, pg_body *pl, double *frrot, double dt, int kick) {
  if (!p || !pl || !frrot) return PG_ERR_ARG;
  if (!kick) {
    pg::Profile pf{*p};
    double old_rad = pl->x;
    pl->x += dt * pl->vx;
    pl->y += dt * pl->vy;
    pl->vy = ((pl->vy + *frrot) * old_rad * old_rad / pl->x / pl->x) - *frrot;
    if (pl->y < 0.0) pl->y += pg::kTwoPi;
    if (pl->y >= pg::kTwoPi) pl->y -= pg::kTwoPi;
    pl->rs = p->rs_fac * pf.h(pl->x);
  } else {
    pl->vx += dt * pl->fx;
    pl->vy += *frrot + dt * pl->fy / pl->x / pl->x;
    *frrot = (p->FrRot_flag == 1) ? pl->vy : 0.0;
    pl->vy -= *frrot;
  }
  return PG_OK;
}

double pg_get_E(const pg_body *p, double frrot) {
  if (!p) return std::nan("");
  double vy = p->vy + frrot;
  return (p->vx * p->vx + vy * vy * p->x * p->x) / 2.0 - 1.0 / p->x;
}

double pg_get_ecc(const pg_body *p, double frrot) {
  if (!p) return std::nan("");
  double vy = p->vy + frrot;
  double L = vy * p->x * p->x;
  return std::sqrt(1.0 + (2.0 * pg_get_E(p, frrot) * L * L));
}

// ---- fused device-resident loop --------------------------------------------------
int pg_clock_reset(pg_run *run, int startat) {
  if (!run) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  const pg_params &P = run->P;
  if (P.ndim == 3 && run->nk > 64) return fail(run, PG_ERR_PARAMS, "3D diagnostics support kmax <= 64");
  CK(cudaSetDevice(run->dev));
  pgd::DevClock c{};
  c.simtime = P.tmovie * (double)startat;                 // main.cu:272
  c.timem = 0.0;
  c.dt = P.endtime;                                       // main.cu:270
  c.endtime = P.endtime; c.tmovie = P.tmovie; c.courant = P.courant;
  pg_body b;
  double fr;
  pg_init_planet(&P, &b, &fr);                            // main.cu:327
  if (int st = pg_planet_forces(run, &b, fr, c.simtime)) return st;  // main.cu:328
  c.planet = pgd::Body{b.m, b.x, b.y, b.vx, b.vy, b.fx, b.fy, b.rs};
  c.frrot = fr; c.frrot_next = fr;
  c.ncycle = 0; c.ncycp = 0; c.ncycend = P.ncycend;
  c.nprin = P.nprin; c.plnt_flag = P.plnt_flag; c.frrot_flag = P.FrRot_flag; c.ndim = P.ndim;
  c.M_p = P.M_p; c.t_growth = P.t_growth; c.rs_fac = P.rs_fac; c.sc2 = P.sc_h * P.sc_h; c.R_p = P.R_p;
  c.Sigma_0 = P.Sigma_0;
  c.p_beta = P.p_beta;
  c.hist_norm = P.M_p * P.M_p * pg::cpow_c(P.R_p, 1.0 - P.p_alpha + (P.p_beta - 1.0)) / (P.sc_h * P.sc_h);
  c.hist = run->hist; c.hist_cap = run->hist_cap; c.hist_count = 0;
  cudaStream_t s = run->stream;
  CK(cudaMemcpyAsync(run->clk, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  // first get_dt's CFL rate (the fused loop takes later ones from sweepy)
  double **cp = run->planes[run->cur];
  if (run->fp32)
    pgk::cfl32(run->T, planes32_cur(run), run->ph, fr, P.ndim, 0, &run->clk->cfl_bits, nullptr, s);
  else
    pgk::cfl_full(run->T, cp[0], cp[1], cp[2], cp[3], run->p0_live ? run->p0 : nullptr, run->ph, fr, P.ndim,
                  &run->clk->cfl_bits, s);
  if (int e = check_launch(run, 1)) return e;
  CK(cudaStreamSynchronize(s));
  run->clock_ready = true;
  return PG_OK;
}

int pg_clock_get(pg_run *run, pg_clock *out, pg_body *planet) {
  if (!run) return PG_ERR_ARG;
  if (!run->clock_ready) return fail(run, PG_ERR_STATE, "clock not reset");
  CK(cudaSetDevice(run->dev));
  pgd::DevClock c;
  CK(cudaMemcpyAsync(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost, run->stream));
  CK(cudaStreamSynchronize(run->stream));
  if (out) {
    out->simtime = c.simtime; out->timem = c.timem; out->dt = c.dt; out->dt_used = c.dt_step;
    out->frrot = c.frrot; out->ncycle = c.ncycle; out->make_pict = c.make_pict; out->done = c.done;
    out->status = c.status; out->pad = c.halted;
  }
  if (planet) {
    planet->m = c.planet.m; planet->x = c.planet.x; planet->y = c.planet.y; planet->vx = c.planet.vx;
    planet->vy = c.planet.vy; planet->fx = c.planet.fx; planet->fy = c.planet.fy; planet->rs = c.planet.rs;
  }
  return PG_OK;
}

// one step of main.cu:343-441 as device work on the run's stream
// One step of the device-resident loop on the FP32 planes: the same launch
// sequence as the FP64 step below, with the float sweeps.
static int enqueue_step32(pg_run *run, pgd::SweepCtl c, int n, size_t e_step) {
  const pg_params &P = run->P;
  cudaStream_t s = run->stream;
  const bool tm = run->timing;
  size_t e_k = 0;
  int a = run->cur;
  if (tm && ev_pair(run, 0, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  pgk::sweep_x32(run->T, planes32_fwd(run, a), run->ph, c, P.ndim, s); n += nx(run);
  if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  const bool moving = P.plnt_flag == 2;
  if (P.ndim == 2) {
    c.fuse = 1;
    c.shift = 1;
    c.nocfl = moving;
    if (tm && ev_pair(run, 1, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    pgk::sweep_y32(run->T, planes32_fwd(run, 1 - a), run->ph, c, 2, s); n += ny(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  } else {
    if (tm && ev_pair(run, 1, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    pgk::sweep_y32(run->T, planes32_fwd(run, 1 - a), run->ph, c, 3, s); n += ny(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    if (tm && ev_pair(run, 2, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    c.shift = 1;
    pgk::sweep_z32(run->T, planes32_fwd(run, a), run->ph, c, P.ntop, s); n += nz(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    run->cur = 1 - a;
    pgk::damp32(run->T, planes32_cur(run), 0.0, run->clk, 3, s); n++;
    if (!moving) { pgk::cfl32_clk(run->T, planes32_cur(run), run->ph, 3, run->clk, s); n++; }
  }
  if (moving) {
    // drift, disk forces on the drifted planet, kick; then the next CFL
    pgk::poststep_drift(run->clk, run->T, s); n++;
    pgk::reduce_forces(run->T, run->p32[run->cur][0], 1, run->clk, P.p_alpha, P.ndim, run->ring_part,
                       run->counter, s); n += 2;
    pgk::poststep_kick(run->clk, s); n++;
    pgk::cfl32_clk(run->T, planes32_cur(run), run->ph, P.ndim, run->clk, s, 0); n++;
  } else {
    pgk::poststep(run->clk, run->T, s); n++;
  }
  pgk::reduce32(run->T, run->p32[run->cur][0], pgd::Body{}, run->clk, 0.0, 0, P.plnt_flag > 0, P.p_alpha, P.ndim,
                run->ring_part, run->counter, &run->clk->mass, s); n++;
  if (P.plnt_flag > 0 && P.ndim == 2) {
    pgk::reduce32(run->T, run->p32[run->cur][0], pgd::Body{}, run->clk, 0.0, 9, 1, P.p_alpha, P.ndim,
                  run->ring_part, run->counter, &run->clk->torque, s); n++;
  }
  pgk::record(run->clk, s); n++;
  if (tm && ev_close(run, e_step)) return fail(run, PG_ERR_CUDA, "event record");
  return check_launch(run, n);
}

static int enqueue_step(pg_run *run, bool first_p0) {
  const pg_params &P = run->P;
  cudaStream_t s = run->stream;
  pgd::SweepCtl c{};
  c.clk = run->clk;
  c.fuse = 0;
  c.shift = 0;
  int a = run->cur;
  int n = 0;
  const bool tm = run->timing;
  size_t e_step = 0, e_k = 0;
  if (tm && ev_pair(run, 3, e_step)) return fail(run, PG_ERR_CUDA, "event record");
  pgk::prestep(run->clk, run->T, P.FARGO_flag, s); n++;
  if (run->fp32) return enqueue_step32(run, c, n, e_step);
  if (tm && ev_pair(run, 0, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  pgk::sweep_x(run->T, planes_fwd(run, a, first_p0 ? run->p0 : nullptr), run->ph, c, P.ndim, s); n += nx(run);
  if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  const bool moving = P.plnt_flag == 2;
  if (P.ndim == 2) {
    c.fuse = 1;
    c.shift = 1;
    c.nocfl = moving;
    if (tm && ev_pair(run, 1, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    pgk::sweep_y(run->T, planes_fwd(run, 1 - a, nullptr), run->ph, c, 2, s); n += ny(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
  } else {
    if (tm && ev_pair(run, 1, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    pgk::sweep_y(run->T, planes_fwd(run, 1 - a, nullptr), run->ph, c, 3, s); n += ny(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    // 3D: the polar sweep applies the FARGO shift; damping and the CFL rate
    // are fused into its store when its chunks are never idle
    if (tm && ev_pair(run, 2, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    c.shift = 1;
    const bool fuse_z = !run->T.cz.stuck;
    c.fuse = fuse_z;
    c.nocfl = moving;
    pgk::sweep_z(run->T, planes_fwd(run, a, nullptr), run->ph, c, P.ntop, s); n += nz(run);
    if (tm && ev_close(run, e_k)) return fail(run, PG_ERR_CUDA, "event record");
    double **cp = run->planes[1 - a];
    if (!fuse_z) {
      pgk::damp_clk(run->T, cp[0], cp[1], cp[2], cp[3], run->clk, s); n++;
      if (!moving) { pgk::cfl_clk(run->T, cp[0], cp[1], cp[2], cp[3], run->ph, run->clk, s); n++; }
    }
    run->cur = 1 - a;
  }
  if (moving) {
    // moving planet (planet.cu:54-93): drift, the disk's forces on the
    // drifted planet (reductions 8 and 9), kick; FrRot is then known and the
    // next get_dt's CFL runs on the stored state
    double **cp = run->planes[run->cur];
    pgk::poststep_drift(run->clk, run->T, s); n++;
    pgk::reduce_forces(run->T, cp[0], 0, run->clk, P.p_alpha, P.ndim, run->ring_part, run->counter, s); n += 2;
    pgk::poststep_kick(run->clk, s); n++;
    pgk::cfl_clk_after(run->T, cp[0], cp[1], cp[2], cp[3], run->ph, run->clk, P.ndim, s); n++;
  } else {
    pgk::poststep(run->clk, run->T, s); n++;
  }
  if (P.plnt_flag > 0 || true) {
    double **cp = run->planes[run->cur];
    pgk::reduce(run->T, cp[0], pgd::Body{}, run->clk, 0.0, 0, P.plnt_flag > 0, P.p_alpha, P.ndim,
                run->ring_part, run->counter, &run->clk->mass, nullptr, s); n++;
    if (P.plnt_flag > 0 && P.ndim == 2) {
      pgk::reduce(run->T, cp[0], pgd::Body{}, run->clk, 0.0, 9, 1, P.p_alpha, P.ndim, run->ring_part,
                  run->counter, &run->clk->torque, nullptr, s); n++;
    }
    pgk::record(run->clk, s); n++;
  }
  if (tm && ev_close(run, e_step)) return fail(run, PG_ERR_CUDA, "event record");
  return check_launch(run, n);
}

// The device clock halts the loop (end time, a tmovie dump, an error); the
// steps queued after that return at once.  HaltProbe bounds that waste: after
// each launch unit (a graph replay, or a group of single steps) it queues a
// copy of clk->halted into pinned memory, and before queueing unit i it reads
// the copy made after unit i-kDepth, so kDepth units stay in flight.
struct HaltProbe {
  static constexpr int kDepth = 4;
  pg_run *run;
  int64_t unit = 0;
  int init() {
    if (run->h_halt) return PG_OK;
    if (cudaHostAlloc(&run->h_halt, kDepth * sizeof(int), cudaHostAllocDefault) != cudaSuccess) return PG_ERR_CUDA;
    for (auto &e : run->halt_ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return PG_ERR_CUDA;
    return PG_OK;
  }
  // true when an earlier unit saw the clock halted
  bool halted_before_next() {
    if (unit < kDepth) return false;
    int slot = (int)(unit % kDepth);
    if (cudaEventSynchronize(run->halt_ev[slot]) != cudaSuccess) return true;   // surfaces in finish_advance
    return run->h_halt[slot] != 0;
  }
  int post() {
    int slot = (int)(unit % kDepth);
    if (cudaMemcpyAsync(&run->h_halt[slot], &run->clk->halted, sizeof(int), cudaMemcpyDeviceToHost,
                        run->stream) != cudaSuccess) return PG_ERR_CUDA;
    if (cudaEventRecord(run->halt_ev[slot], run->stream) != cudaSuccess) return PG_ERR_CUDA;
    unit++;
    return PG_OK;
  }
};

static int finish_advance(pg_run *run, int64_t before, int *taken) {
  pgd::DevClock c;
  CK(cudaMemcpyAsync(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost, run->stream));
  CK(cudaStreamSynchronize(run->stream));
  if (taken) *taken = (int)(c.ncycle - before);
  if (c.status != 0) {
    return fail(run, c.status, c.status == PG_ERR_NONFINITE ? "non-finite or non-positive state"
                                                           : "time step collapsed");
  }
  if (c.halted && !c.done) {
    // landed on tmovie: let the caller dump, then continue
    int zero = 0;
    CK(cudaMemcpyAsync(&run->clk->halted, &zero, sizeof(int), cudaMemcpyHostToDevice, run->stream));
    CK(cudaStreamSynchronize(run->stream));
  }
  return PG_OK;
}

int pg_advance(pg_run *run, int nsteps, int *taken) {
  if (!run) return PG_ERR_ARG;
  if (!run->clock_ready) return fail(run, PG_ERR_STATE, "call pg_clock_reset first");
  CK(cudaSetDevice(run->dev));
  pgd::DevClock c;
  CK(cudaMemcpy(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost));
  int64_t before = c.ncycle;
  HaltProbe hp{run};
  if (int e = hp.init()) return fail(run, e, "halt probe set-up");
  const int group = 16;
  for (int i = 0; i < nsteps; i++) {
    if (i % group == 0 && hp.halted_before_next()) break;
    bool first = run->p0_live;
    if (int e = enqueue_step(run, first)) return e;
    run->p0_live = false;
    if ((i + 1) % group == 0 && hp.post()) return fail(run, PG_ERR_CUDA, "halt probe");
  }
  return finish_advance(run, before, taken);
}

int pg_advance_graph(pg_run *run, int nsteps, int chunk, int *taken) {
  if (!run) return PG_ERR_ARG;
  if (!run->clock_ready) return fail(run, PG_ERR_STATE, "call pg_clock_reset first");
  if (chunk < 1) return fail(run, PG_ERR_ARG, "chunk must be >= 1");
  CK(cudaSetDevice(run->dev));
  if (run->P.ndim == 3 && (chunk & 1)) chunk += 1;   // 3D steps alternate the plane copies
  pgd::DevClock c;
  CK(cudaMemcpy(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost));
  int64_t before = c.ncycle;
  int done = 0;
  if (run->p0_live && nsteps > 0) {
    if (int e = enqueue_step(run, true)) return e;
    run->p0_live = false;
    done = 1;
  }
  if (!run->gexec || run->gsteps != chunk || run->gcur != run->cur) {
    if (run->gexec) { cudaGraphExecDestroy(run->gexec); run->gexec = nullptr; }
    int cur0 = run->cur;
    run->gcur = cur0;   // 3D steps flip the plane copies: the graph is valid for this one
    bool tm = run->timing;
    run->timing = false;
    int64_t l0 = run->launches;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(run->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < chunk; i++) {
      int e = enqueue_step(run, false);
      if (e) { cudaStreamEndCapture(run->stream, &g); run->timing = tm; return e; }
    }
    CK(cudaStreamEndCapture(run->stream, &g));
    run->timing = tm;
    CK(cudaGraphInstantiate(&run->gexec, g, 0));
    cudaGraphDestroy(g);
    run->gsteps = chunk;
    run->graph_kernels = run->launches - l0;
    run->launches = l0;
    run->cur = cur0;
  }
  int64_t per = 0;
  HaltProbe hp{run};
  if (int e = hp.init()) return fail(run, e, "halt probe set-up");
  for (; done + chunk <= nsteps; done += chunk) {
    if (hp.halted_before_next()) { done = nsteps; break; }
    size_t e = 0;
    if (run->timing && ev_pair(run, 3, e)) return fail(run, PG_ERR_CUDA, "event record");
    CK(cudaGraphLaunch(run->gexec, run->stream));
    if (run->timing && ev_close(run, e)) return fail(run, PG_ERR_CUDA, "event record");
    run->launches += run->graph_kernels;
    per++;
    if (hp.post()) return fail(run, PG_ERR_CUDA, "halt probe");
  }
  for (; done < nsteps; done++) {
    if (int e = enqueue_step(run, false)) return e;
  }
  (void)per;
  return finish_advance(run, before, taken);
}

int pg_timing(pg_run *run, int on) {
  if (!run) return PG_ERR_ARG;
  run->timing = on != 0;
  return PG_OK;
}

int pg_timing_read(pg_run *run, double *ms_sum, int64_t *counts, int nkinds) {
  if (!run || !ms_sum || !counts) return PG_ERR_ARG;
  CK(cudaSetDevice(run->dev));
  CK(cudaStreamSynchronize(run->stream));
  for (int k = 0; k < nkinds; k++) { ms_sum[k] = 0.0; counts[k] = 0; }
  for (const auto &m : run->marks) {
    if (m.kind < 0 || m.kind >= nkinds) continue;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, run->ev_pool[m.a], run->ev_pool[m.b]));
    ms_sum[m.kind] += ms;
    counts[m.kind] += 1;
  }
  run->marks.clear();
  run->ev_next = 0;
  return PG_OK;
}

int pg_history(pg_run *run, double *rows, int max, int *rows_out) {
  if (!run || !rows_out) return PG_ERR_ARG;
  if (!run->clock_ready) return fail(run, PG_ERR_STATE, "clock not reset");
  CK(cudaSetDevice(run->dev));
  pgd::DevClock c;
  CK(cudaMemcpyAsync(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost, run->stream));
  CK(cudaStreamSynchronize(run->stream));
  int n = c.hist_count < max ? c.hist_count : max;
  if (n > 0 && rows)
    CK(cudaMemcpy(rows, run->hist, (size_t)n * pgd::HIST_COLS * sizeof(double), cudaMemcpyDeviceToHost));
  int zero = 0;
  CK(cudaMemcpy(&run->clk->hist_count, &zero, sizeof(int), cudaMemcpyHostToDevice));
  *rows_out = n;
  return PG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// post-processing of the current state (read/ tools)
static int post_buffer(pg_run *run, size_t n, double **buf) {
  if (cudaMalloc(buf, n * sizeof(double)) != cudaSuccess) return fail(run, PG_ERR_NOMEM, "post-processing buffer");
  return PG_OK;
}

extern "C" int pg_post_harmonic(pg_run *run, double m, double *an, double *bn) {
  if (!run || !an || !bn) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  double *ab = nullptr;
  if (int e = post_buffer(run, 2 * (size_t)run->nr, &ab)) return e;
  const void *r = run->fp32 ? (const void *)run->p32[run->cur][0] : (const void *)run->planes[run->cur][0];
  pgk::post_harmonic(run->T, r, run->fp32, m, ab, run->stream);
  std::vector<double> h(2 * (size_t)run->nr);
  cudaError_t e1 = cudaGetLastError();
  cudaError_t e2 = cudaMemcpyAsync(h.data(), ab, h.size() * sizeof(double), cudaMemcpyDeviceToHost, run->stream);
  cudaError_t e3 = cudaStreamSynchronize(run->stream);
  cudaFree(ab);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return fail(run, PG_ERR_CUDA, "post_harmonic");
  for (int i = 0; i < run->nr; i++) { an[i] = h[2 * i]; bn[i] = h[2 * i + 1]; }
  return PG_OK;
}

extern "C" int pg_post_torque(pg_run *run, double M_p, double *out) {
  if (!run || !out) return PG_ERR_ARG;
  if (!run->loaded) return fail(run, PG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(run->dev));
  size_t n = (size_t)run->nr * run->nk;
  double *rb = nullptr;
  if (int e = post_buffer(run, n, &rb)) return e;
  const void *r = run->fp32 ? (const void *)run->p32[run->cur][0] : (const void *)run->planes[run->cur][0];
  pgk::post_torque(run->T, r, run->fp32, M_p, rb, run->stream);
  std::vector<double> h(n);
  cudaError_t e1 = cudaGetLastError();
  cudaError_t e2 = cudaMemcpyAsync(h.data(), rb, n * sizeof(double), cudaMemcpyDeviceToHost, run->stream);
  cudaError_t e3 = cudaStreamSynchronize(run->stream);
  cudaFree(rb);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return fail(run, PG_ERR_CUDA, "post_torque");
  double t = 0.0;
  for (size_t q = 0; q < n; q++) t += h[q];
  *out = t;
  return PG_OK;
}

// ---------------------------------------------------------------------------
// device footprint of a run (pg_create's allocations), for admission control
extern "C" size_t pg_run_device_bytes(const pg_params *p) {
  if (!p) return 0;
  auto up = [](size_t b) { return (b + 511) & ~(size_t)511; };
  size_t nr = (size_t)p->imax, nphi = (size_t)p->jmax, nk = (size_t)p->kmax, nrg = nr + 2 * NPAD;
  size_t nring = nk * nrg, nz = nk + 2 * NPAD;
  size_t pe = nring * nphi;
  int nf = (p->ndim == 3) ? 4 : 3;
  size_t es = (p->precision == 1) ? sizeof(float) : sizeof(double);
  size_t b = 2 * (size_t)nf * up(pe * es);
  if (p->precision != 1) b += up(pe * sizeof(double));                         // p0
  b += up((4 * nrg + 10 * nring + 4 * nphi + 16 * nz + 2 * NPAD * nr * 4 + 2 * NPAD * nr) * sizeof(double));
  b += up(2 * nring * sizeof(int)) + 3 * up(nring * sizeof(double));           // itab, rot_v, vbg, sbg
  b += up(nr * nk * sizeof(double)) + up(4) + up(32) + up(8) + up(sizeof(pgd::DevClock));
  b += up((size_t)4096 * pgd::HIST_COLS * sizeof(double));
  return b;
}

namespace pgi {

int run_shape(const pg_run *run, RunShape *o) {
  if (!run || !o) return PG_ERR_ARG;
  o->dev = run->dev;
  o->ndim = run->P.ndim;
  o->fp32 = run->fp32 ? 1 : 0;
  o->loaded = run->loaded ? 1 : 0;
  o->clock_ready = run->clock_ready ? 1 : 0;
  o->p0_live = run->p0_live ? 1 : 0;
  o->moving = run->P.plnt_flag == 2 ? 1 : 0;
  o->eos = run->P.EOS;
  o->nr = run->nr; o->nphi = run->nphi; o->nk = run->nk;
  const pgd::Chunking &cx = run->T.cx;
  const bool short_last = !cx.stuck && cx.lim_last <= 64;
  o->tiles_x = run->nphi * (cx.loop - (short_last ? 1 : 0)) * run->nk;
  o->tiles_xs = short_last ? (run->nphi * run->nk + 3) / 4 : 0;
  o->tiles_y = run->T.cy.loop * run->nr * run->nk;
  return PG_OK;
}

int run_batch_desc(pg_run *run, pgd::BatchRun *d) {
  if (!run || !d) return PG_ERR_ARG;
  if (!run->clock_ready) return fail(run, PG_ERR_STATE, "batch member needs pg_clock_reset first");
  std::memset((void *)d, 0, sizeof(*d));
  d->T = run->T;
  d->ph = run->ph;
  d->clk = run->clk;
  int a = run->cur;
  if (run->fp32) {
    d->QX = planes32_fwd(run, a);
    d->QY = planes32_fwd(run, 1 - a);
  } else {
    d->PX = planes_fwd(run, a, nullptr);
    d->PY = planes_fwd(run, 1 - a, nullptr);
    if (run->p0_live) {
      pgd::DevClock c;
      CK(cudaMemcpy(&c, run->clk, sizeof(c), cudaMemcpyDeviceToHost));
      d->p0 = run->p0;
      d->p0_cycle = c.ncycle;
    }
  }
  d->ring_part = run->ring_part;
  d->counter = run->counter;
  d->p_alpha = run->P.p_alpha;
  d->fargo = run->P.FARGO_flag;
  d->plnt = run->P.plnt_flag > 0;
  return PG_OK;
}

void run_batched(pg_run *run, int64_t launches) {
  run->p0_live = false;
  run->launches += launches;
}

int run_enqueue_on(pg_run *run, cudaStream_t s, int64_t *launches) {
  cudaStream_t own = run->stream;
  int64_t l0 = run->launches;
  run->stream = s;
  int st = enqueue_step(run, run->p0_live);
  run->stream = own;
  run->p0_live = false;
  if (launches) *launches += run->launches - l0;
  return st;
}

pgd::DevClock *run_clock(pg_run *run) { return run->clk; }
int run_cur(const pg_run *run) { return run->cur; }
cudaStream_t run_stream(pg_run *run) { return run->stream; }

}  // namespace pgi
