// pg_host.cpp -- host-side set-up of a disk run: parameters, grid, seeded
// initial condition, dump-record layout, fixed ghost rings and the
// axisymmetric profile.  All of this is host arithmetic in the reference too
// (init.cpp, grid.cu, disk_profile.cu are compiled as host code), so it is
// restated here in C++ with the same operation order; glibc libm on both
// sides gives the same bits.
#include "pg_host.h"

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace pg {

const double kTwoPi = 6.283185307179586476925286766559;
const double kPi = 3.1415926535897932384626433832795;
const double kHalfPi = 1.570796326794896619231321691639751442;
const double kThird = 0.3333333333333333333333333;
const double kEarthMass = 0.000003;
const double kJupiterMass = 0.001;
const double kMMSN = 0.00019126835;

// ---- disk profile (disk_profile.cu) --------------------------------------
// pow with the forms the reference's compiler gives it: its exponents are
// compile-time constants, and pow(x, 0), pow(x, 1), pow(x, -1) and pow(x, 2)
// are folded to 1, x, 1/x and x*x (exact or correctly rounded, where libm's
// pow can differ by an ulp); other exponents stay calls.
double cpow_c(double x, double y) {
  if (y == 0.0) return 1.0;
  if (y == 1.0) return x;
  if (y == -1.0) return 1.0 / x;
  if (y == 2.0) return x * x;
  return std::pow(x, y);
}
double Profile::rho(double r) const {                                           // 9-28
  // the 3D isentropic disk's midplane slope is p_alpha 2/(gam + 1)
  double n = (P.EOS != 0 && P.ndim == 3) ? -P.p_alpha * (2.0 / (P.gam + 1.0)) : -P.p_alpha;
  return cpow_c(r, n);
}
double Profile::cs2(double r) const { return P.sc_h * P.sc_h * cpow_c(r, -P.p_beta); }  // 39-42
double Profile::h(double r) const { return std::sqrt(cs2(r) * r * r * r); }      // 49-52
double Profile::pres(double r) const {                                          // 54-61
  if (P.EOS == 0) return cs2(r) * rho(r);
  return cs2(r) * cpow_c(rho(r), P.gam) / P.gam;
}
double Profile::dP_dr(double r) const {                                          // 63-68
  double p1 = pres(r + 1.27245e-8);
  double p2 = pres(r - 1.27245e-8);
  return (p1 - p2) / 2.5449e-8;
}
double Profile::verfac(double r, double z) const {                               // 70-75
  double c = cs2(r);
  double rr = std::sqrt(r * r + z * z);
  return std::exp((1.0 / rr - 1.0 / r) / c);
}
double Profile::rho(double r, double z) const {                                 // 86-103
  if (P.EOS == 0) return rho(r) * verfac(r, z);
  // isentropic: the polytrope rho^(gam-1) = rho_mid^(gam-1) - (gam-1)/(r cs2)
  // (1 - r/sqrt(r^2 + z^2)), continued above z_0 by a decade per h/6
  const double gm = P.gam - 1.0;
  double h = std::sqrt(cs2(r) * r * r * r);
  double z0 = std::sqrt(2.0 * h * h * cpow_c(r, -P.p_alpha * (2.0 / (P.gam + 1.0)) * gm) / gm);
  if (z < z0) return cpow_c(cpow_c(rho(r), gm) - (gm / (r * cs2(r))) * (1.0 - r / std::sqrt(r * r + z * z)), 1.0 / gm);
  double top = cpow_c(cpow_c(rho(r), gm) - (gm / (r * cs2(r))) * (1.0 - r / std::sqrt(r * r + z0 * z0)), 1.0 / gm);
  return std::pow(10.0, std::log10(top) - 6.0 * (z - z0) / h);
}
double Profile::pres(double r, double z) const {                                // 112-118
  if (P.EOS == 0) return cs2(r) * rho(r, z);
  return cs2(r) * cpow_c(rho(r, z), P.gam) / P.gam;
}
double Profile::dP_s(double r, double pol) const {                               // 128-138
  double dr = 1.27e-7;
  double sp = std::sin(pol), cp = std::cos(pol);
  double r1 = (r + dr) * sp, z1 = (r + dr) * cp;
  double r2 = (r - dr) * sp, z2 = (r - dr) * cp;
  return (pres(r1, z1) - pres(r2, z2)) / (2.0 * dr);
}
double Profile::nu(double r) const {                                             // 149-152
  double vis_nu = P.ss_alpha * P.sc_h * P.sc_h;                                  // global.h:36
  return vis_nu * cpow_c(r, P.p_alpha);
}
double Profile::viscous_vr(double r) const {                                     // 154-160
  if (P.visc_flag == 1) return -1.5 * nu(r) / r;
  return 0.0;
}

// get_vol grid.cu:225-248
double Profile::vol(double xa, double dx, int axis) const {
  double v = 0.0;
  if (axis == 0) {
    if (P.ngeomx == 0) v = dx;
    else if (P.ngeomx == 1) v = dx * (xa + 0.5 * dx);
    else if (P.ngeomx == 2) v = dx * (xa * (xa + dx) + dx * dx * kThird);
  } else if (axis == 1) {
    v = dx;
  } else {
    if (P.ndim == 2) v = 1.0;
    else if (P.ngeomz == 0) v = dx;
    else if (P.ngeomz == 5) v = std::cos(xa) - std::cos(xa + dx);
  }
  return v;
}

// ---- grid generator grid.cu:66-221 -----------------------------------------
// Type 4 (refined toward the centre) takes the radial limits dx_min/dx_max
// and type 6 (refined toward the upper edge) the polar limits dz_min/dz_max
// whichever axis it builds, as the reference's global constants do.
static int make_grid(const pg_params &P, int nz, double lo, double hi, int lg,
                     std::vector<double> &xa, std::vector<double> &xc, std::vector<double> &dx) {
  const double dmin = (lg == 4) ? P.dx_min : P.dz_min;
  const double dmax = (lg == 4) ? P.dx_max : P.dz_max;
  xa.assign(nz, 0.0); xc.assign(nz, 0.0); dx.assign(nz, 0.0);
  if (lg == 0) {
    double f = (hi - lo) / (double)nz;
    for (int n = 0; n < nz; n++) {
      xa[n] = lo + ((double)n) * f;
      dx[n] = f;
      xc[n] = xa[n] + 0.5 * dx[n];
    }
  } else if (lg >= 1 && lg <= 3) {
    double f = (std::log(hi) - std::log(lo)) / (double)nz;
    xa[0] = lo;
    for (int n = 1; n < nz; n++) {
      xa[n] = lo * std::exp(f * ((double)n));
      dx[n - 1] = xa[n] - xa[n - 1];
      xc[n - 1] = xa[n - 1] + 0.5 * dx[n - 1];
    }
    dx[nz - 1] = hi - xa[nz - 1];
    xc[nz - 1] = xa[nz - 1] + 0.5 * dx[nz - 1];
  } else if (lg == 4 || lg == 6) {
    // power-law refinement toward the centre (lg 4) or the upper edge (lg 6)
    if (lg == 4) {
      double xmid = (hi + lo) / 2.0;
      double xp = xmid - lo;
      int N = nz / 2;
      xp -= N * dmin;
      double power = std::log(1.0 - (dmax - dmin) / xp) / std::log(1.0 - 1.0 / N);
      double A = std::pow(xp, 1.0 / power) / (double)N;
      for (int i = 0; i < N; i++) xa[i] = xmid - std::pow((double)(N - i) * A, power) - (double)(N - i) * dmin;
      for (int i = N; i < nz; i++) xa[i] = std::pow((double)(i - N) * A, power) + (double)(i - N) * dmin + xmid;
    } else {
      double xp = hi - lo;
      int N = nz;
      xp -= N * dmin;
      double power = std::log(1.0 - (dmax - dmin) / xp) / std::log(1.0 - 1.0 / N);
      double A = std::pow(xp, 1.0 / power) / (double)N;
      for (int i = 0; i < nz; i++) xa[i] = hi - std::pow((double)(N - i) * A, power) - (double)(N - i) * dmin;
    }
    for (int i = 0; i < nz - 1; i++) { dx[i] = xa[i + 1] - xa[i]; xc[i] = xa[i] + 0.5 * dx[i]; }
    dx[nz - 1] = hi - xa[nz - 1];
    xc[nz - 1] = xa[nz - 1] + 0.5 * dx[nz - 1];
  } else {
    return PG_ERR_PARAMS;  // lg 5 needs the reference's interactive consistency checks
  }
  return PG_OK;
}

// ---- splitmix64 (Steele, Lea & Flood 2014), counter based ------------------
static inline uint64_t splitmix64(uint64_t seed, uint64_t idx) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double ic_uniform(uint64_t seed, uint64_t idx) {
  return (double)(splitmix64(seed, idx) >> 11) * 0x1.0p-53;
}

// ---- axisymmetric profile init_den/init_speed init.cpp:92-183 -------------
void build_val(const Profile &pf, const std::vector<double> &zxc, const std::vector<double> &zzc,
               std::vector<SymDisk> &val) {
  const pg_params &P = pf.P;
  int imax = P.imax, kmax = P.kmax;
  val.assign((size_t)imax * kmax, SymDisk{});
  for (int i = 0; i < imax; i++)
    for (int k = 0; k < kmax; k++) {
      SymDisk &v = val[i + imax * k];
      double r, z;
      if (P.ngeomz == 5) { r = zxc[i] * std::sin(zzc[k]); z = zxc[i] * std::cos(zzc[k]); }
      else { r = zxc[i]; z = zzc[k]; }
      if (P.ndim == 3) { v.r = pf.rho(r, z); v.p = pf.pres(r, z); }
      else { v.r = pf.rho(r); v.p = pf.pres(r); }
    }
  for (int i = 0; i < imax; i++)
    for (int k = 0; k < kmax; k++) {
      SymDisk &v = val[i + imax * k];
      double r, z, vk2, dP;
      if (P.ndim == 2) { r = zxc[i]; z = 0.0; vk2 = 1.0 / r; dP = pf.dP_dr(zxc[i]); }
      else {
        vk2 = 1.0 / zxc[i];
        r = zxc[i] * std::sin(zzc[k]); z = zxc[i] * std::cos(zzc[k]);
        dP = pf.dP_s(zxc[i], zzc[k]);
      }
      (void)z;
      vk2 += zxc[i] * dP / v.r;
      v.v = std::sqrt(vk2);
      v.u = pf.viscous_vr(r);
      v.w = 0.0;
    }
}

// ---- fixed ghost ring init.cpp:259-413 (radial) / 415-539 (theta) ---------
// Records the ring's geometry and its phi-uniform state.  res_v and inc_j
// are zero: the reference never sets them and relies on zeroed pages.
GhostRing make_ghost(const Profile &pf, double x, double dx, double xc, double z, double dz,
                     double zc, int theta_layer) {
  const pg_params &P = pf.P;
  GhostRing g{};
  g.x = x; g.dx = dx; g.xc = xc; g.xvol = pf.vol(x, dx, 0);
  g.z = z; g.dz = dz; g.zc = zc; g.zvol = pf.vol(z, dz, 2);
  double rr = xc, r, zz, rho, Pr, dP, vk;
  if (P.ndim == 2) {
    r = rr; zz = 0.0;
    rho = pf.rho(r); Pr = pf.pres(r); dP = pf.dP_dr(r); vk = 1.0 / r;
  } else if (!theta_layer) {
    r = rr * std::sin(zc); zz = rr * std::cos(zc);
    rho = pf.rho(r, zz); Pr = pf.pres(r, zz); dP = pf.dP_s(rr, zc); vk = 1.0 / rr;
  } else {
    zz = rr * std::cos(zc); r = std::sqrt(rr * rr - zz * zz);
    dP = pf.dP_s(rr, zc);
    rho = pf.rho(r, zz); Pr = pf.pres(r, zz); vk = 1.0 / rr;
  }
  vk += rr * dP / rho;
  vk = std::sqrt(vk);
  g.r = rho; g.p = Pr; g.u = pf.viscous_vr(r); g.v = vk; g.w = 0.0;
  g.rot_v = (P.FARGO_flag == 1) ? vk - 1.0 * xc : 0.0;
  return g;
}

// ---- the fixed boundary rings of init_bound (init.cpp:253-543) ------------
// Radial ghost rings (lft inside, rgh outside; 6 x kmax each, ring i + 6 k)
// continue the grid with the edge cell's width; in 3D the polar layers (udr
// below the first layer, top above the last; 6 x imax each, layer k + 6 i)
// continue it with the edge layer's width.  Each ring carries the disk
// profile's axisymmetric state at its centre.  The reference's lft branch for
// a spherical grid (init.cpp:289-294) forms no density or pressure before
// using them; here every ring takes the profile's values.
void boundary_rings(const Profile &pf, const Geometry &g, std::vector<GhostRing> &lft,
                    std::vector<GhostRing> &rgh, std::vector<GhostRing> &udr, std::vector<GhostRing> &top) {
  const int pad = 6, nr = pf.P.imax, nk = pf.P.kmax;
  lft.assign((size_t)pad * nk, GhostRing{});
  rgh.assign((size_t)pad * nk, GhostRing{});
  for (int i = 0; i < pad; i++)
    for (int k = 0; k < nk; k++) {
      double x = g.zxa[0] - g.zdx[0] * (double)(pad - i), dx = g.zdx[0];
      lft[i + pad * k] = make_ghost(pf, x, dx, x + 0.5 * dx, g.zza[k], g.zdz[k], g.zzc[k], 0);
      x = g.zxa[nr - 1] + g.zdx[nr - 1] * (double)(i + 1);
      dx = g.zdx[nr - 1];
      rgh[i + pad * k] = make_ghost(pf, x, dx, x + 0.5 * dx, g.zza[k], g.zdz[k], g.zzc[k], 0);
    }
  udr.clear();
  top.clear();
  if (pf.P.ndim != 3) return;
  udr.assign((size_t)pad * nr, GhostRing{});
  top.assign((size_t)pad * nr, GhostRing{});
  for (int k = 0; k < pad; k++)
    for (int i = 0; i < nr; i++) {
      double zl = g.zza[0] - g.zdz[0] * (double)(pad - k), dzl = g.zdz[0];
      udr[k + pad * i] = make_ghost(pf, g.zxa[i], g.zdx[i], g.zxc[i], zl, dzl, zl + 0.5 * dzl, 1);
      double zu = g.zza[nk - 1] + g.zdz[nk - 1] * (double)(k + 1), dzu = g.zdz[nk - 1];
      top[k + pad * i] = make_ghost(pf, g.zxa[i], g.zdx[i], g.zxc[i], zu, dzu, zu + 0.5 * dzu, 1);
    }
}

// The grid of a parameter set (init_grid init.cpp:3-57 with get_vol).
int params_geometry(const pg_params &P, Geometry &g) {
  Profile pf{P};
  if (make_grid(P, P.imax, P.xmin, P.xmax, P.grspx, g.zxa, g.zxc, g.zdx) ||
      make_grid(P, P.jmax, P.ymin, P.ymax, P.grspy, g.zya, g.zyc, g.zdy) ||
      make_grid(P, P.kmax, P.zmin, P.zmax, P.grspz, g.zza, g.zzc, g.zdz))
    return PG_ERR_PARAMS;
  g.xvol.resize(P.imax); g.yvol.resize(P.jmax); g.zvol.resize(P.kmax);
  for (int i = 0; i < P.imax; i++) g.xvol[i] = pf.vol(g.zxa[i], g.zdx[i], 0);
  for (int j = 0; j < P.jmax; j++) g.yvol[j] = pf.vol(g.zya[j], g.zdy[j], 1);
  for (int k = 0; k < P.kmax; k++) g.zvol[k] = pf.vol(g.zza[k], g.zdz[k], 2);
  return PG_OK;
}

// ---- dump record layout variable_types.h:67-97 ----------------------------
size_t ring_bytes(int jmax) { return (size_t)72 * jmax + 96; }

RingView::RingView(unsigned char *b, int jmax) : base(b), n(jmax) {}
double *RingView::f(int field) const { return (double *)(base + (size_t)8 * n * field); }
double *RingView::scal(int which) const { return (double *)(base + (size_t)40 * n + 8 * which); }
double *RingView::col(int which) const { return (double *)(base + (size_t)40 * n + 32 + (size_t)8 * n * which); }
double *RingView::zs(int which) const { return (double *)(base + (size_t)72 * n + 32 + 8 * which); }
int *RingView::ik(int which) const { return (int *)(base + (size_t)72 * n + 64 + 4 * which); }
double *RingView::rot(int which) const { return (double *)(base + (size_t)72 * n + 72 + 8 * which); }
int *RingView::rj(int which) const { return (int *)(base + (size_t)72 * n + 88 + 4 * which); }

// ---- parameter sets ---------------------------------------------------------
void default_params(pg_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->ndim = 2; p->imax = 850; p->jmax = 2000; p->kmax = 1;
  p->flat_flag = 1; p->bary_flag = 0; p->EOS = 0; p->plnt_flag = 2; p->FrRot_flag = 1;
  p->kill_flag = 0; p->visc_flag = 1; p->FARGO_flag = 1; p->dump_flag = 1;
  p->p_alpha = 1.5; p->p_beta = 0.5; p->ss_alpha = 0.0001; p->sc_h = 0.05;
  p->Sigma_0 = 1.0 * kMMSN;
  p->M_p = 1.0 * kJupiterMass; p->R_p = 1.0; p->t_growth = 1000.0 * kTwoPi; p->rs_fac = 0.5;
  p->gam = 1.0; p->courant = 0.5;
  p->nlft = 3; p->nrgh = 3; p->nudr = 3; p->ntop = 3;
  p->endtime = 10000.0 * kTwoPi; p->tmovie = 200.0 * kTwoPi;
  p->ncycend = 1000000000; p->nprin = 100;
  p->xmin = 0.2; p->xmax = 3.0; p->ymin = 0.0; p->ymax = kTwoPi;
  p->zmin = kHalfPi - 0.065; p->zmax = kHalfPi;
  p->ngeomx = 1; p->ngeomy = 3; p->ngeomz = 0;
  p->grspx = 1; p->grspy = 0; p->grspz = 0;
  p->dx_min = 0.0012; p->dx_max = 0.002; p->dy_min = 0.0012; p->dy_max = 0.015;
  p->dz_min = 0.0005; p->dz_max = 0.002;
  p->seed = 0; p->noise_amp = 1e-4; p->kill_rin = 0.0; p->kill_rout = 0.0; p->precision = 0;
}

int config_params(int which, pg_params *p) {
  default_params(p);
  // the 2D disk: G=M*=1, h=0.05 with c_s = h r Omega_K (p_beta=1), Sigma ~ 1/r
  p->p_alpha = 1.0; p->p_beta = 1.0; p->ss_alpha = 1e-3; p->sc_h = 0.05;
  p->M_p = 1e-3; p->R_p = 1.0; p->t_growth = 0.0; p->rs_fac = 0.6;
  p->plnt_flag = 1; p->FrRot_flag = 1; p->FARGO_flag = 1; p->visc_flag = 1; p->EOS = 0;
  p->nprin = 100; p->noise_amp = 1e-4; p->seed = 0;
  switch (which) {
    case 0:  // 256 x 768 FP64, 10 orbits, damping r<0.5, r>2.2
      p->imax = 256; p->jmax = 768; p->kmax = 1; p->ndim = 2;
      p->xmin = 0.4; p->xmax = 2.5; p->kill_rin = 0.5; p->kill_rout = 2.2;
      p->endtime = 10.0 * kTwoPi; p->tmovie = p->endtime;
      return PG_OK;
    case 1:  // 3D spherical 128 x 1024 x 32, theta in [pi/2 - 3h, pi/2], 5 orbits
      p->imax = 128; p->jmax = 1024; p->kmax = 32; p->ndim = 3;
      p->ngeomx = 2; p->ngeomy = 4; p->ngeomz = 5;
      p->p_alpha = 1.5; p->p_beta = 1.0; p->M_p = 3e-4;
      p->xmin = 0.5; p->xmax = 2.0; p->zmin = kHalfPi - 0.15; p->zmax = kHalfPi;
      p->nudr = 3; p->ntop = 0;  // fixed upper layers, reflecting midplane
      p->endtime = 5.0 * kTwoPi; p->tmovie = p->endtime;
      return PG_OK;
    case 2:  // 1024 x 3072 FP32 planes, same disk and planet as the 256 x 768 case, 20 orbits
      p->imax = 1024; p->jmax = 3072; p->kmax = 1; p->ndim = 2; p->precision = 1;
      p->xmin = 0.4; p->xmax = 2.5; p->kill_rin = 0.5; p->kill_rout = 2.2;
      p->endtime = 20.0 * kTwoPi; p->tmovie = p->endtime;
      return PG_OK;
    default:
      return PG_ERR_ARG;
  }
}

static int chunk_ok(int n) {
  // pencils are cut in chunks of 116 interior cells (arrsize 128, n_pad 6).
  // A remainder of 1..5 makes the reference's wrap read already-updated
  // cells (ppm.cu:196-241); a single chunk reads r_rg before it is written.
  if (n < 1) return 0;
  int rem = n % 116;
  if (rem >= 1 && rem <= 5) return 0;
  return 1;
}

int check_params(const pg_params *p, std::string &why) {
  if (!p) { why = "null params"; return PG_ERR_ARG; }
  if (p->ndim != 2 && p->ndim != 3) { why = "ndim must be 2 or 3"; return PG_ERR_PARAMS; }
  if (p->imax < 1 || p->jmax < 1 || p->kmax < 1) { why = "grid sizes must be positive"; return PG_ERR_PARAMS; }
  // the azimuthal sweep and the dump kernels launch one block row per ring
  // (grid y), the 3D polar sweep one per azimuthal column: CUDA caps grid y
  // and z at 65535
  if (p->imax > 65535) { why = "imax must be <= 65535 (rings run on CUDA grid y)"; return PG_ERR_PARAMS; }
  if (p->ndim == 3 && (p->jmax > 65535 || p->kmax > 65535)) {
    why = "3D needs jmax, kmax <= 65535 (polar columns run on CUDA grid y)"; return PG_ERR_PARAMS;
  }
  if (p->ndim == 2 && p->kmax != 1) { why = "2D problem needs kmax == 1 (main.cu:130)"; return PG_ERR_PARAMS; }
  if (p->ndim == 3 && p->kmax == 1) { why = "3D problem needs kmax > 1 (main.cu:134)"; return PG_ERR_PARAMS; }
  if (p->EOS == 2) {
    why = "EOS 2 (energy equation) is not implemented: the reference marks it buggy (global.h:18)"; return PG_ERR_PARAMS;
  }
  if (p->EOS != 0 && p->EOS != 1) { why = "EOS must be 0 (isothermal) or 1 (isentropic)"; return PG_ERR_PARAMS; }
  if (!(p->gam >= 1.0)) { why = "gam must be >= 1"; return PG_ERR_PARAMS; }
  if (p->EOS == 1 && p->ndim == 3 && !(p->gam > 1.0)) {
    why = "3D EOS 1 needs gam > 1 (the vertical polytrope divides by gam - 1)"; return PG_ERR_PARAMS;
  }
  if (p->EOS == 1 && p->precision != 0) { why = "the FP32 planes implement EOS 0 only"; return PG_ERR_PARAMS; }
  if (p->bary_flag) { why = "barycentric frame (bary_flag) is not implemented"; return PG_ERR_PARAMS; }
  if (p->kill_flag != 0) { why = "kill_flag is not implemented in the reference; use kill_rin/kill_rout"; return PG_ERR_PARAMS; }
  if (p->plnt_flag < 0 || p->plnt_flag > 2) { why = "plnt_flag must be 0, 1 or 2"; return PG_ERR_PARAMS; }
  if (p->FARGO_flag < 0 || p->FARGO_flag > 2) { why = "FARGO_flag must be 0, 1 or 2"; return PG_ERR_PARAMS; }
  if (p->nlft != 3 || p->nrgh != 3) { why = "only fixed radial boundaries (nlft=nrgh=3) are implemented"; return PG_ERR_PARAMS; }
  if (p->ndim == 2 && !(p->ngeomx == 1 && p->ngeomy == 3)) { why = "2D needs cylindrical geometry (ngeomx=1, ngeomy=3)"; return PG_ERR_PARAMS; }
  if (p->ndim == 3 && !(p->ngeomx == 2 && p->ngeomy == 4 && p->ngeomz == 5)) {
    why = "3D needs spherical geometry (ngeomx=2, ngeomy=4, ngeomz=5)"; return PG_ERR_PARAMS;
  }
  if (p->ndim == 3 && p->kmax < 2 * 3) {
    why = "3D needs kmax >= 6 (the reflecting midplane mirrors 6 layers)"; return PG_ERR_PARAMS;
  }
  if (p->ndim == 3 && !(p->nudr == 3 && (p->ntop == 0 || p->ntop == 3))) {
    why = "3D needs fixed lower theta layers (nudr=3) and a fixed or reflecting top (ntop 3 or 0)"; return PG_ERR_PARAMS;
  }
  if (p->jmax < 122 || !chunk_ok(p->jmax)) {
    why = "jmax must be >= 122 with jmax % 116 not in 1..5 (azimuthal chunk wrap of ppm.cu:191-255)"; return PG_ERR_PARAMS;
  }
  if (p->grspx == 5 || p->grspy == 5 || p->grspz == 5) { why = "grid type 5 is not supported"; return PG_ERR_PARAMS; }
  if (!(p->courant > 0.0) || !(p->endtime > 0.0) || !(p->tmovie > 0.0)) { why = "courant, endtime and tmovie must be positive"; return PG_ERR_PARAMS; }
  if (!(p->xmin > 0.0) || !(p->xmax > p->xmin)) { why = "need 0 < xmin < xmax"; return PG_ERR_PARAMS; }
  if (p->kill_rin > 0.0 && !(p->kill_rin > p->xmin)) { why = "kill_rin must exceed xmin"; return PG_ERR_PARAMS; }
  if (p->kill_rout > 0.0 && !(p->kill_rout < p->xmax)) { why = "kill_rout must be below xmax"; return PG_ERR_PARAMS; }
  if (p->precision != 0 && p->precision != 1) { why = "precision must be 0 (FP64) or 1 (FP32 bulk)"; return PG_ERR_PARAMS; }
  if (p->nprin < 1) { why = "nprin must be >= 1"; return PG_ERR_PARAMS; }
  return PG_OK;
}

// ---- seeded initial condition ------------------------------------------------
// init_grid + init_den + init_speed + init_cells (init.cpp:3-249) with
// Sigma = val.r * (1 + noise_amp*(2U-1)), U = splitmix64(seed, ring*jmax+j),
// v_r = 0, p = Sigma*cs2(r_cyl) or cs2 Sigma^gam/gam (the sweep store of
// ppm.cu:138-143 for EOS 0 / 1), rot_j = 0,
// rot_v = val.v - FrRot*xc (the FARGO_flag 1 value of orbital_advection.cu:22).
int build_ic(const pg_params *p, void *buf, size_t bytes, std::string &why) {
  int st = check_params(p, why);
  if (st) return st;
  const pg_params &P = *p;
  size_t rbytes = ring_bytes(P.jmax);
  if (!buf || bytes != rbytes * (size_t)P.imax * P.kmax) { why = "ring buffer size mismatch"; return PG_ERR_ARG; }
  Profile pf{P};
  std::vector<double> zxa, zxc, zdx, zya, zyc, zdy, zza, zzc, zdz;
  if (make_grid(P, P.imax, P.xmin, P.xmax, P.grspx, zxa, zxc, zdx) ||
      make_grid(P, P.jmax, P.ymin, P.ymax, P.grspy, zya, zyc, zdy) ||
      make_grid(P, P.kmax, P.zmin, P.zmax, P.grspz, zza, zzc, zdz)) {
    why = "unsupported grid type"; return PG_ERR_PARAMS;
  }
  std::vector<SymDisk> val;
  build_val(pf, zxc, zzc, val);
  double frrot = (P.FrRot_flag == 1) ? std::pow(P.R_p, -1.5) : 0.0;  // init_planet planet.cu:42-47
  std::memset(buf, 0, bytes);
  unsigned char *b = (unsigned char *)buf;
  for (int k = 0; k < P.kmax; k++)
    for (int i = 0; i < P.imax; i++) {
      int m = i + P.imax * k;
      RingView rv(b + rbytes * m, P.jmax);
      const SymDisk &v = val[i + P.imax * k];
      double z = zza[k], dz = zdz[k], zc = z + 0.5 * dz;
      double x = zxa[i], dx = zdx[i], xc = x + 0.5 * dx;
      *rv.zs(0) = z; *rv.zs(1) = dz; *rv.zs(3) = zc; *rv.zs(2) = pf.vol(z, dz, 2);
      *rv.scal(0) = x; *rv.scal(1) = dx; *rv.scal(3) = xc; *rv.scal(2) = pf.vol(x, dx, 0);
      *rv.ik(0) = i; *rv.ik(1) = k;
      double rad_cyl = xc;
      if (P.ngeomz == 5) rad_cyl *= std::sin(zc);
      double c2 = pf.cs2(rad_cyl);
      for (int j = 0; j < P.jmax; j++) {
        rv.col(0)[j] = zya[j];
        rv.col(1)[j] = zdy[j];
        rv.col(3)[j] = zya[j] + 0.5 * zdy[j];
        rv.col(2)[j] = pf.vol(zya[j], zdy[j], 1);
        double U = ic_uniform(P.seed, (uint64_t)m * P.jmax + j);
        double sig = v.r * (1.0 + P.noise_amp * (2.0 * U - 1.0));
        rv.f(0)[j] = sig;
        rv.f(1)[j] = (P.EOS == 0) ? sig * c2 : c2 * cpow_c(sig, P.gam) / P.gam;
        rv.f(2)[j] = 0.0;
        rv.f(3)[j] = v.v;
        rv.f(4)[j] = 0.0;
      }
      if (P.FARGO_flag == 1) *rv.rot(0) = v.v - frrot * xc;
      else if (P.FARGO_flag == 2) *rv.rot(0) = (1.0 - frrot) * xc;
      else *rv.rot(0) = 0.0;
      *rv.rot(1) = 0.0;
      *rv.rj(0) = 0; *rv.rj(1) = 0;
    }
  return PG_OK;
}

// create_label output.cu:57-88
static std::string itos(int v) { return std::to_string(v); }
std::string label(const pg_params &P) {
  std::string s = itos(P.imax) + "x" + itos(P.jmax) + "x" + itos(P.kmax) + "_c" + itos((int)std::round(P.sc_h / 0.001));
  if (P.plnt_flag == 2) s += "_pm" + itos((int)std::round(P.M_p / 0.000003)) + "_s" + itos((int)std::round(100.0 * P.rs_fac));
  else if (P.plnt_flag == 1) s += "_p" + itos((int)std::round(P.M_p / 0.000003)) + "_s" + itos((int)std::round(100.0 * P.rs_fac));
  s += "_i" + itos((int)(P.xmin * 100.0)) + "_o" + itos((int)(P.xmax * 100.0));
  if (P.visc_flag == 1) s += "_a" + itos((int)std::round(P.ss_alpha * 10000.0));
  if (P.EOS == 1) {
    s += "_g" + itos((int)std::round(P.gam * 10.0));
  } else {
    if (P.p_alpha + 0.5 * P.p_beta - 1.5 == 1.5) s += "_flatvor";
    if (P.p_beta == 0.0) s += "_iso";
    else s += "_b" + itos((int)(P.p_beta * 10.0));
  }
  if (P.FrRot_flag == 1) s += "_rot";
  if (P.FARGO_flag == 1) s += "_fargo";
  return s;
}

// Geometry read back from dump records: copy_grid init.cpp:59-90.
int read_geometry(const pg_params &P, const unsigned char *b, Geometry &g, std::string &why) {
  size_t rbytes = ring_bytes(P.jmax);
  g.zxa.assign(P.imax, 0.0); g.zxc.assign(P.imax, 0.0); g.zdx.assign(P.imax, 0.0);
  g.zza.assign(P.kmax, 0.0); g.zzc.assign(P.kmax, 0.0); g.zdz.assign(P.kmax, 0.0);
  g.xvol.assign(P.imax, 0.0); g.zvol.assign(P.kmax, 0.0);
  std::vector<char> seen((size_t)P.imax * P.kmax, 0);
  for (int n = 0; n < P.imax * P.kmax; n++) {
    RingView rv((unsigned char *)b + rbytes * n, P.jmax);
    int i = *rv.ik(0), k = *rv.ik(1);
    if (i < 0 || i >= P.imax || k < 0 || k >= P.kmax) { why = "ring index out of range in dump"; return PG_ERR_STATE; }
    if (i + P.imax * k != n) { why = "dump rings are not in ring-major order m = i + imax*k"; return PG_ERR_STATE; }
    seen[n] = 1;
    g.zxa[i] = *rv.scal(0); g.zxc[i] = *rv.scal(3); g.zdx[i] = *rv.scal(1); g.xvol[i] = *rv.scal(2);
    g.zza[k] = *rv.zs(0); g.zzc[k] = *rv.zs(3); g.zdz[k] = *rv.zs(1); g.zvol[k] = *rv.zs(2);
  }
  RingView r0((unsigned char *)b, P.jmax);
  g.zya.assign(r0.col(0), r0.col(0) + P.jmax);
  g.zdy.assign(r0.col(1), r0.col(1) + P.jmax);
  g.yvol.assign(r0.col(2), r0.col(2) + P.jmax);
  g.zyc.assign(r0.col(3), r0.col(3) + P.jmax);
  return PG_OK;
}

}  // namespace pg

// ---- C ABI: parameter helpers -------------------------------------------------
extern "C" {

int pg_default_params(pg_params *p) {
  if (!p) return PG_ERR_ARG;
  pg::default_params(p);
  return PG_OK;
}

int pg_config_params(int which, pg_params *p) {
  if (!p) return PG_ERR_ARG;
  return pg::config_params(which, p);
}

int pg_check_params(const pg_params *p) {
  std::string why;
  return pg::check_params(p, why);
}

size_t pg_ring_bytes(int jmax) { return jmax > 0 ? pg::ring_bytes(jmax) : 0; }

int pg_boundary_rings(const pg_params *p, double *out, size_t n_doubles, int *count) {
  if (!p || !count) return PG_ERR_ARG;
  std::string why;
  int st = pg::check_params(p, why);
  if (st) return st;
  pg::Geometry g;
  if ((st = pg::params_geometry(*p, g))) return st;
  pg::Profile pf{*p};
  std::vector<pg::GhostRing> lft, rgh, udr, top;
  pg::boundary_rings(pf, g, lft, rgh, udr, top);
  const size_t n = lft.size() + rgh.size() + udr.size() + top.size();
  *count = (int)n;
  if (!out) return PG_OK;
  if (n_doubles < n * PG_BOUNDARY_FIELDS) return PG_ERR_ARG;
  double *o = out;
  for (const std::vector<pg::GhostRing> *grp : {&lft, &rgh, &udr, &top})
    for (const pg::GhostRing &r : *grp) {
      const double rec[PG_BOUNDARY_FIELDS] = {r.x, r.dx, r.xvol, r.xc, r.z, r.dz, r.zvol, r.zc,
                                              r.r, r.p, r.u, r.v, r.w, r.rot_v};
      std::memcpy(o, rec, sizeof rec);
      o += PG_BOUNDARY_FIELDS;
    }
  return PG_OK;
}

int pg_build_ic(const pg_params *p, void *rings, size_t bytes) {
  std::string why;
  int st = pg::build_ic(p, rings, bytes, why);
  if (st) std::fprintf(stderr, "pg_build_ic: %s\n", why.c_str());
  return st;
}

int pg_write_ic(const pg_params *p, const char *path) {
  if (!p || !path) return PG_ERR_ARG;
  std::string why;
  int st = pg::check_params(p, why);
  if (st) return st;
  size_t bytes = pg::ring_bytes(p->jmax) * (size_t)p->imax * p->kmax;
  std::vector<unsigned char> buf(bytes);
  st = pg::build_ic(p, buf.data(), bytes, why);
  if (st) return st;
  FILE *f = std::fopen(path, "wb");
  if (!f) return PG_ERR_IO;
  size_t w = std::fwrite(buf.data(), 1, bytes, f);
  std::fclose(f);
  return (w == bytes) ? PG_OK : PG_ERR_IO;
}

int pg_dump_name(const pg_params *p, const char *dir, int frame, char *buf, size_t len) {
  if (!p || !dir || !buf || frame < 0 || frame > 99999) return PG_ERR_ARG;
  char num[8];
  std::snprintf(num, sizeof num, "%05d", frame);
  std::string s = std::string(dir) + "/binary_" + pg::label(*p) + "_" + num;
  if (s.size() + 1 > len) return PG_ERR_ARG;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return PG_OK;
}

int pg_write_time_rows(const pg_params *p, const char *path, const double *rows, int nrows, int append) {
  if (!p || !path || (!rows && nrows > 0) || nrows < 0) return PG_ERR_ARG;
  FILE *f = std::fopen(path, append ? "a" : "w");
  if (!f) return PG_ERR_IO;
  // ofstream with precision(16) prints a double as %.16g; without a planet
  // the row stops after the mass (main.cu:419-425)
  const int ncols = p->plnt_flag > 0 ? 11 : 2;
  for (int r = 0; r < nrows; r++) {
    const double *q = rows + 11 * (size_t)r;
    for (int c = 0; c < ncols; c++) std::fprintf(f, c ? " %.16g" : "%.16g", q[c]);
    std::fputc('\n', f);
  }
  return std::fclose(f) == 0 ? PG_OK : PG_ERR_IO;
}

int pg_write_para_file(const pg_params *p, const char *path, const char *mainp) {
  if (!p || !path || !mainp) return PG_ERR_ARG;
  FILE *f = std::fopen(path, "w");
  if (!f) return PG_ERR_IO;
  // ofstream with precision(16): %.16g
  std::fprintf(f, "%d\n%d\n%d\n%d\n", p->imax, p->jmax, p->kmax, 1);
  std::fprintf(f, "%.16g\n%.16g\n%.16g\n", p->gam, p->sc_h, p->tmovie);
  std::fprintf(f, "%s\n%s\n", mainp, pg::label(*p).c_str());
  std::fprintf(f, "%d\n%d\n%d\n", p->grspx, p->grspy, p->grspz);
  std::fprintf(f, "%.16g %.16g\n%.16g %.16g\n%.16g %.16g\n", p->xmin, p->xmax, p->ymin, p->ymax, p->zmin, p->zmax);
  return std::fclose(f) == 0 ? PG_OK : PG_ERR_IO;
}

int pg_label(const pg_params *p, char *buf, size_t len) {
  if (!p || !buf || len == 0) return PG_ERR_ARG;
  std::string s = pg::label(*p);
  if (s.size() + 1 > len) return PG_ERR_ARG;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return PG_OK;
}

}  // extern "C"

// ---- pg_params by field name ------------------------------------------------
// A translation unit that includes the reference's configuration headers
// cannot name the fields that share a name with its macros (EOS, ndim,
// plnt_flag, ...); it sets them by name instead.
namespace {
struct ParamField {
  const char *name;
  size_t off;
  char kind;   // 'i' int, 'd' double, 'u' uint64
};
#define PGF(n, k) {#n, offsetof(pg_params, n), k}
const ParamField kParamFields[] = {
    PGF(ndim, 'i'), PGF(imax, 'i'), PGF(jmax, 'i'), PGF(kmax, 'i'), PGF(flat_flag, 'i'),
    PGF(bary_flag, 'i'), PGF(EOS, 'i'), PGF(plnt_flag, 'i'), PGF(FrRot_flag, 'i'),
    PGF(kill_flag, 'i'), PGF(visc_flag, 'i'), PGF(FARGO_flag, 'i'), PGF(dump_flag, 'i'),
    PGF(nlft, 'i'), PGF(nrgh, 'i'), PGF(nudr, 'i'), PGF(ntop, 'i'), PGF(ncycend, 'i'),
    PGF(nprin, 'i'), PGF(ngeomx, 'i'), PGF(ngeomy, 'i'), PGF(ngeomz, 'i'), PGF(grspx, 'i'),
    PGF(grspy, 'i'), PGF(grspz, 'i'), PGF(precision, 'i'),
    PGF(p_alpha, 'd'), PGF(p_beta, 'd'), PGF(ss_alpha, 'd'), PGF(sc_h, 'd'), PGF(Sigma_0, 'd'),
    PGF(M_p, 'd'), PGF(R_p, 'd'), PGF(t_growth, 'd'), PGF(rs_fac, 'd'), PGF(gam, 'd'),
    PGF(courant, 'd'), PGF(endtime, 'd'), PGF(tmovie, 'd'), PGF(xmin, 'd'), PGF(xmax, 'd'),
    PGF(ymin, 'd'), PGF(ymax, 'd'), PGF(zmin, 'd'), PGF(zmax, 'd'), PGF(dx_min, 'd'),
    PGF(dx_max, 'd'), PGF(dy_min, 'd'), PGF(dy_max, 'd'), PGF(dz_min, 'd'), PGF(dz_max, 'd'),
    PGF(noise_amp, 'd'), PGF(kill_rin, 'd'), PGF(kill_rout, 'd'),
    PGF(seed, 'u'),
};
#undef PGF

const ParamField *find_field(const char *name) {
  for (const ParamField &f : kParamFields)
    if (std::strcmp(f.name, name) == 0) return &f;
  return nullptr;
}
}  // namespace

extern "C" {

int pg_params_set(pg_params *p, const char *name, double value) {
  if (!p || !name) return PG_ERR_ARG;
  const ParamField *f = find_field(name);
  if (!f) return PG_ERR_ARG;
  unsigned char *base = reinterpret_cast<unsigned char *>(p) + f->off;
  if (f->kind == 'd') {
    std::memcpy(base, &value, sizeof value);
    return PG_OK;
  }
  if (!(value == std::floor(value))) return PG_ERR_ARG;            // integral, not NaN
  if (f->kind == 'i') {
    if (value < -2147483648.0 || value > 2147483647.0) return PG_ERR_ARG;
    int v = (int)value;
    std::memcpy(base, &v, sizeof v);
  } else {
    if (value < 0.0 || value > 9007199254740992.0) return PG_ERR_ARG;   // exact in a double
    uint64_t v = (uint64_t)value;
    std::memcpy(base, &v, sizeof v);
  }
  return PG_OK;
}

int pg_params_get(const pg_params *p, const char *name, double *value) {
  if (!p || !name || !value) return PG_ERR_ARG;
  const ParamField *f = find_field(name);
  if (!f) return PG_ERR_ARG;
  const unsigned char *base = reinterpret_cast<const unsigned char *>(p) + f->off;
  if (f->kind == 'd') {
    std::memcpy(value, base, sizeof(double));
  } else if (f->kind == 'i') {
    int v;
    std::memcpy(&v, base, sizeof v);
    *value = v;
  } else {
    uint64_t v;
    std::memcpy(&v, base, sizeof v);
    *value = (double)v;
  }
  return PG_OK;
}

}  // extern "C"
