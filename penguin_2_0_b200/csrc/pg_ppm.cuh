// pg_ppm.cuh -- device side of one PPM Lagrange-remap pencil chunk.
//
// A chunk is 128 cells along the sweep direction: 116 interior cells plus 6
// ghost cells on each side (n_pad 6, arrsize 128 of variable_types.h:13-16).
// One thread owns one cell; the phases below are separated by CTA barriers
// and read neighbours through shared memory.  Each phase keeps the index
// range and the arithmetic order of the reference routine cited beside it,
// so that the interior results agree with the reference to the last few
// ulps (identical FMA contraction is the aim, not an assumption).
//
// Differences from the reference that do not change results:
//  * chunks of a pencil are independent CTAs reading the pre-sweep state
//    from a separate buffer, instead of one CTA walking the pencil with a
//    6-cell carry (ppm.cu:43-157 carries pre-update values, so the result is
//    the same Jacobi update);
//  * the q remap (remap.cu:123-142) and the q of evolve (evolve.cu:131-135)
//    are skipped: the sweep store overwrites p by the EOS relation
//    (ppm.cu:138-143), so they never reach the stored state;
//  * in 2D the remap of the slot holding w is skipped (w stays exactly 0:
//    the w slot of the radial sweep, the v slot of the azimuthal sweep) and
//    umid *= pmid (evolve.cu:73, used by EOS 2 only) is dropped;
//  * cs2(r) and nu(r) come from per-ring tables computed on the device with
//    the same expressions;
//  * the three parabolas of states and the three or four of remap run side
//    by side, each with its own scratch arrays, where the reference runs
//    them one after another through the same three (al/da/a6 over
//    q/dx/tmp1); every value is the same, the barriers are shared.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pgd {

constexpr int NPAD = 6;
constexpr int ARR = 128;
constexpr int REAL = ARR - 2 * NPAD;   // 116
constexpr int AP = ARR + 2;            // padded shared length (flux[n+1] at n = 127)

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kThird = 0.3333333333333333333333333;
constexpr double kFourthd = 1.3333333333333333333333333;
constexpr double kSmallp = 1.0e-15;
constexpr double kSmallr = 1.0e-15;

struct Body { double m, x, y, vx, vy, fx, fy, rs; };

// Physics constants of the run (global.h), passed by value to kernels.
struct Phys {
  double gam, sc2, vis_nu, p_alpha, p_beta;
  double gamfac1, gamfac2;  // (gam + 1)/gam/2 and gam + 1 (global.h:54-55)
  int plnt;       // plnt_flag > 0
  int flat;       // flat_flag
  int visc;       // visc_flag
  int eos;        // EOS: 0 isothermal, 1 isentropic (global.h:18)
};

// Pressure of a cell from its density by the sweep store's relation
// (ppm.cu:138-143): EOS 0 p = rho cs2, EOS 1 p = cs2 rho^gam / gam.  The
// planes hold no pressure; every reader of p derives it here.  The sweeps
// take EOS as a template argument (the EOS-0 kernels carry no pow); the
// small kernels around them (CFL, dump packing) branch at run time.
template <int EOS>
__device__ __forceinline__ double eos_p(double r, double cs2, const Phys &ph) {
  if (EOS == 0) return r * cs2;
  return cs2 * pow(r, ph.gam) / ph.gam;
}
__device__ __forceinline__ double eos_p_rt(double r, double cs2, const Phys &ph) {
  return ph.eos ? eos_p<1>(r, cs2, ph) : eos_p<0>(r, cs2, ph);
}

// Isentropic Riemann problem (riemann.cu:75-111, the EOS 1 branch): van
// Leer's (1979) Newton iteration for the contact pressure on the Lagrangian
// sound speeds C = sqrt(gam p rho), at most 10 iterations, relative
// tolerance 1e-8; the face velocity is the mean of the two wave fans'.
__device__ __forceinline__ void riemann_isentropic(double pl, double rl, double ul, double pr, double rr,
                                                   double ur, const Phys &ph, double &umid, double &pmid) {
  const double cl = sqrt(ph.gam * pl * rl), cr = sqrt(ph.gam * pr * rr);
  const double vl = 1.0 / rl, vr = 1.0 / rr;
  double pm = pr - pl - cr * (ur - ul);
  pm = pl + pm * cl / (cl + cr);
  pm = fmax(kSmallp, pm);
  double wl = 0.0, wr = 0.0;
  for (int it = 0; it < 10; it++) {
    const double prev = pm;
    wl = cl * sqrt(1.0 + ph.gamfac1 * (pm - pl) / pl);
    wr = cr * sqrt(1.0 + ph.gamfac1 * (pm - pr) / pr);
    double zl = 4.0 * vl * wl * wl, zr = 4.0 * vr * wr * wr;
    zl = -zl * wl / (zl - ph.gamfac2 * (pm - pl));
    zr = zr * wr / (zr - ph.gamfac2 * (pm - pr));
    const double uml = ul - (pm - pl) / wl, umr = ur + (pm - pr) / wr;
    pm = pm + (umr - uml) * (zr * zl) / (zr - zl);
    pm = fmax(kSmallp, pm);
    if (fabs(pm - prev) / pm < 1.0e-8) break;
  }
  umid = 0.5 * ((ul - (pm - pl) / wl) + (ur + (pm - pr) / wr));
  pmid = fmax(kSmallp, pm);
}

struct Par { double c0, c1, c2, c3, c4; };
// paraset coefficients read where they are used from a table (q[0..4]),
// with plain loads that a barrier keeps apart, instead of held in registers
struct ParTab { const double *q; };
template <int I>
__device__ __forceinline__ double par_c(const Par &p) {
  return I == 0 ? p.c0 : I == 1 ? p.c1 : I == 2 ? p.c2 : I == 3 ? p.c3 : p.c4;
}
template <int I>
__device__ __forceinline__ double par_c(const ParTab &p) { return p.q[I]; }

// Shared arrays of one chunk: the sweep kernel's (ppm.cu:38-39) and
// ppmlr's (ppmlr.cu:7-10).  q only serves as parabola storage (al) because
// the q remap is dead in EOS 0 and 1.  s0..s5 are scratch of the parabolas
// that run side by side (three in states, up to four in remap), where the
// reference runs them one after another through q/dx/tmp1.  NT is the CTA
// size: 128 for full chunks, 64 or 32 for a short last chunk (lim <= NT).
template <int NT>
struct ChunkShmData {
  double r[NT + 2], p[NT + 2], u[NT + 2], v[NT + 2], w[NT + 2], xa0[NT + 2], dx0[NT + 2];
  double q[NT + 2], dx[NT + 2], umid[NT + 2], pmid[NT + 2], tmp1[NT + 2];
  double s0[NT + 2], s1[NT + 2], s2[NT + 2], s3[NT + 2], s4[NT + 2], s5[NT + 2];
  // cos(phi - phi_planet) at the start of the step: one value for a radial
  // or polar pencil, whose cells share the azimuth phi (written by cell 0)
  double cf0;
  // sin(phi - phi_planet) at the start of the step (polar pencils, cell 0)
  double sf0;
  // polar pencils (cell 0): 1 / r of the ring, and the planet's reduced
  // mass p.m / (1 + p.m) of its forces
  double irad, plm;
};

// Bytes that bring a per-pencil shared block to TO mod 128.  Kernels that
// pack PACK pencils per CTA (thread t on cell t/PACK of pencil t%PACK) pad to
// 128/PACK: the pencils' pieces of a half-warp's 64-bit access (or a warp's
// 32-bit one) then fall in PACK different bank groups, without conflicts
// (4 pencils: 32 mod 128; 8 pencils: 16 mod 128).
constexpr int shm_pad_to(int size, int to) {
  return ((to - size % 128) + 256) % 128 == 0 ? 128 : ((to - size % 128) + 256) % 128;
}
constexpr int shm_pad_bytes(int size) { return shm_pad_to(size, 32); }

template <int NT, int TO = 32>
struct ChunkShmT : ChunkShmData<NT> {
  char pad_[shm_pad_to((int)sizeof(ChunkShmData<NT>), TO)];
};

// sin and cos of a small angle by their Taylor series (to x^9 and x^8; for
// |x| <= 0.05 the first omitted terms are below 1e-21 relative), else by
// sincos.  The polar sweep's angles move by a fraction of a cell per step,
// so their sines and cosines follow from per-layer or per-pencil values by
// angle addition with these.
__device__ __forceinline__ void sincos_small(double x, double &s, double &c) {
  if (fabs(x) > 0.05) {
    sincos(x, &s, &c);
    return;
  }
  const double x2 = x * x;
  s = x * (1.0 + x2 * (-1.0 / 6.0 + x2 * (1.0 / 120.0 + x2 * (-1.0 / 5040.0 + x2 * (1.0 / 362880.0)))));
  c = 1.0 + x2 * (-0.5 + x2 * (1.0 / 24.0 + x2 * (-1.0 / 720.0 + x2 * (1.0 / 40320.0))));
}

// ---- star + planet gravity, forces.cu:23-182 (non-barycentric frame) ------
// The *_cf forms take cosfac = cos(azi - (p.y + dt p.vy)) from the caller
// (shared by the cells of a pencil at dt = 0); the arithmetic after it is
// the same as in the forms that evaluate it.
__device__ __forceinline__ double planet_cosfac(double azi, const Body &p, double dt) {
  return cos(azi - (p.y + dt * p.vy));
}
// The azimuthal forces' cos and sin of the planet's angle, out of line: one
// copy of their code per kernel instead of one per call site (three per
// cell).  The inlined copies overran the azimuthal sweep's instruction cache
// (73 % hits, 2.3 stall cycles per issue waiting for instructions on the
// 128x1024x32 disk; 81 % and 1.8 out of line, and 2.4 % off the sweep on a
// 2048x6144 disk).  Same calls, same bits.  The radial forces keep cos
// inline: there the call cost more than it saved.
static __device__ __noinline__ double2 pg_cossin(double x) { return make_double2(cos(x), sin(x)); }
__device__ __forceinline__ double grav_rad_cyl_cf(double rad, double cosfac, double z, const Body &p) {
  double plm = p.m;
  double plx = p.x;
  double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p.rs * p.rs);
  return -plm * (rad - plx * cosfac) / (Rp * Rp * Rp) - plm * cosfac / (plx * plx);
}
__device__ __forceinline__ double grav_rad_cyl(double rad, double azi, double z, const Body &p, double dt) {
  return grav_rad_cyl_cf(rad, planet_cosfac(azi, p, dt), z, p);
}
__device__ __forceinline__ double grav_azi_cyl(double rad, double azi, double z, const Body &p, double dt) {
  const double2 cs = pg_cossin(azi - (p.y + dt * p.vy));
  double cosfac = cs.x;
  double sinfac = cs.y;
  double plm = p.m;
  double plx = p.x;
  double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p.rs * p.rs);
  return -plm * plx * sinfac / (Rp * Rp * Rp) + plm * sinfac / plx / plx;
}
__device__ __forceinline__ double grav_rad_sph(double rad, double azi, double pol, const Body &p, double dt) {
  double cosfac = cos(azi - (p.y + dt * p.vy));
  double sinpol = sin(pol);
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return -plm * (rad - plx * cosfac * sinpol) / (Rp * Rp * Rp) - stm / (rad * rad) - plm * sinpol * cosfac / (plx * plx);
}
__device__ __forceinline__ double grav_azi_sph(double rad, double azi, double pol, const Body &p, double dt) {
  double cosfac = cos(azi - (p.y + dt * p.vy));
  double sinfac = sin(azi - (p.y + dt * p.vy));
  double sinpol = sin(pol);
  rad /= sinpol;
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return -plm * plx * sinfac / (Rp * Rp * Rp) + plm * sinpol * sinfac / plx / plx;
}
// the same two forces with sin(pol) formed by the caller (once per cell when
// pol is the cell's fixed polar angle): identical arithmetic otherwise
__device__ __forceinline__ double grav_rad_sph_cf(double rad, double cosfac, double sinpol, const Body &p) {
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return -plm * (rad - plx * cosfac * sinpol) / (Rp * Rp * Rp) - stm / (rad * rad) - plm * sinpol * cosfac / (plx * plx);
}
__device__ __forceinline__ double grav_rad_sph_s(double rad, double azi, double sinpol, const Body &p, double dt) {
  return grav_rad_sph_cf(rad, planet_cosfac(azi, p, dt), sinpol, p);
}
__device__ __forceinline__ double grav_azi_sph_s(double rad, double azi, double sinpol, const Body &p, double dt) {
  const double2 cs = pg_cossin(azi - (p.y + dt * p.vy));
  double cosfac = cs.x;
  double sinfac = cs.y;
  rad /= sinpol;
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return -plm * plx * sinfac / (Rp * Rp * Rp) + plm * sinpol * sinfac / plx / plx;
}
__device__ __forceinline__ double grav_pol_sph_cf(double rad, double cosfac, double sinpol, double cospol,
                                                  const Body &p) {
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  (void)stm;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return plm * plx * cosfac * cospol / (Rp * Rp * Rp) - plm * cosfac * cospol / (sinpol * plx * plx);
}
// grav_pol_sph_cf with the reduced mass p.m / (1 + p.m) formed once by the
// caller (the polar sweep, once per pencil)
__device__ __forceinline__ double grav_pol_sph_plm(double rad, double cosfac, double sinpol, double cospol,
                                                   double plm, const Body &p) {
  double plx = p.x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return plm * plx * cosfac * cospol / (Rp * Rp * Rp) - plm * cosfac * cospol / (sinpol * plx * plx);
}
__device__ __forceinline__ double grav_pol_sph_s(double rad, double azi, double sinpol, double cospol,
                                                 const Body &p, double dt) {
  return grav_pol_sph_cf(rad, planet_cosfac(azi, p, dt), sinpol, cospol, p);
}
__device__ __forceinline__ double grav_pol_sph(double rad, double azi, double pol, const Body &p, double dt) {
  double cosfac = cos(azi - (p.y + dt * p.vy));
  double cospol = cos(pol);
  double sinpol = sin(pol);
  double stm = 1.0 / (1.0 + p.m);
  double plm = p.m * stm;
  double plx = p.x;
  (void)stm;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p.rs * p.rs);
  return plm * plx * cosfac * cospol / (Rp * Rp * Rp) - plm * cosfac * cospol / (sinpol * plx * plx);
}

__device__ __forceinline__ double min3(double A, double B, double C) {   // simple_func.cu:2-14
  if (A < B) { if (C < A) return C; else return A; }
  else       { if (C < B) return C; else return B; }
}
__device__ __forceinline__ double max3(double A, double B, double C) {   // simple_func.cu:16-28
  if (A > B) { if (C > A) return C; else return A; }
  else       { if (C > B) return C; else return B; }
}

// paraset parabola.cu:138-176 (non-uniform PPM interface coefficients)
__device__ __forceinline__ void paraset(int n, int nmin, int nmax, Par &par, const double *dx,
                                        double *a, double *ai, double *b) {
  double dx_n = 0.0, ain = 0.0, bi = 0.0, ci = 0.0, c = 0.0;
  if (n >= nmin && n < nmax - 1) {
    dx_n = dx[n];
    double an = dx_n + dx[n + 1];
    ain = 1.0 / an;
    double bn = an + dx_n;
    bi = 1.0 / bn;
    c = an + dx[n + 1];
    ci = 1.0 / c;
    a[n] = an; ai[n] = ain; b[n] = bn;
  }
  __syncthreads();
  if (n >= nmin + 1 && n < nmax - 2) {
    double d = 1.0 / (a[n - 1] + a[n + 1]);
    par.c0 = dx_n * ain * (1.0 + 2.0 * d * dx[n + 1] * (a[n - 1] * bi - a[n + 1] * ci));
    par.c1 = -d * dx_n * a[n - 1] * bi;
    par.c2 = d * dx[n + 1] * a[n + 1] * ci;
  }
  if (n >= nmin + 1 && n < nmax - 1) {
    double d = dx_n / (a[n - 1] + dx[n + 1]);
    par.c3 = d * b[n - 1] * ain;
    par.c4 = d * c * ai[n - 1];
  }
  __syncthreads();
}

// paraset's coefficients at index L of a width array (the same arithmetic as
// paraset for a cell n = L inside the chunk): c0..c2 need dx[L-1..L+2], c3,
// c4 dx[L-1..L+1].  Used to tabulate the polar sweep's Eulerian
// coefficients once per layer, since every polar pencil has the same widths.
__device__ __forceinline__ void paraset_at(const double *dx, int L, bool full, Par &par) {
  const double dx_n = dx[L];
  const double an = dx_n + dx[L + 1];
  const double ain = 1.0 / an;
  const double bn = an + dx_n;
  const double bi = 1.0 / bn;
  const double c = an + dx[L + 1];
  const double ci = 1.0 / c;
  const double am = dx[L - 1] + dx_n;          // a[n-1]
  const double aim = 1.0 / am;                 // ai[n-1]
  const double bm = am + dx[L - 1];            // b[n-1]
  if (full) {
    const double ap = dx[L + 1] + dx[L + 2];   // a[n+1]
    double d = 1.0 / (am + ap);
    par.c0 = dx_n * ain * (1.0 + 2.0 * d * dx[L + 1] * (am * bi - ap * ci));
    par.c1 = -d * dx_n * am * bi;
    par.c2 = d * dx[L + 1] * ap * ci;
  } else {
    par.c0 = par.c1 = par.c2 = 0.0;
  }
  double d = dx_n / (am + dx[L + 1]);
  par.c3 = d * bm * ain;
  par.c4 = d * c * aim;
}

// parabola parabola.cu:70-133 (CW84 eq 1.5-1.8, 1.10)
__device__ __forceinline__ void parabola(int n, int nmin, int nmax, double flat, const double *val,
                                         double *al, double *da, double *a6, const Par &par) {
  double t1 = 0.0, a = 0.0, ar = 0.0, da_r = 0.0;
  if (n >= nmin + 1 && n < nmax - 1) {
    a = val[n];
    da_r = val[n + 1] - a;
    double da_l = a - val[n - 1];
    t1 = par.c3 * da_r + par.c4 * da_l;
    if (t1 < 0.0) t1 = -min3(-t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
    else          t1 = min3(t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
    if (da_l * da_r < 0.0) t1 = 0.0;
    a6[n] = t1;
  }
  __syncthreads();
  if (n >= nmin + 1 && n < nmax - 2) {
    ar = a + par.c0 * da_r + par.c1 * a6[n + 1] + par.c2 * t1;
    al[n + 1] = ar;
  }
  __syncthreads();
  if (n >= nmin + 2 && n < nmax - 2) {
    double u1 = flat * a;
    double u2 = 1.0 - flat;
    double xr = u1 + u2 * ar;
    double la = u1 + u2 * al[n];
    u1 = xr - la;
    u2 = u1 * u1;
    u1 = u1 * (6.0 * (a - 0.5 * (xr + la)));
    if ((xr - a) * (a - la) <= 0.0) { xr = a; la = a; }
    if (u2 < u1) la = 3.0 * a - 2.0 * xr;
    if (u2 < -u1) xr = 3.0 * a - 2.0 * la;
    da[n] = xr - la;
    a6[n] = 6.0 * (a - 0.5 * (xr + la));
    al[n] = la;
  }
  __syncthreads();
}

// parabola for NF fields at once: the same three phases and, per field, the
// same arithmetic as parabola(), with one barrier per phase for all fields
// instead of one per phase and field.  A field's values and its own a6 are
// reloaded from shared memory after a barrier (same bits) so that only ar
// stays in a register across one.
template <int NF, class PS>
__device__ __forceinline__ void parabola_n(int n, int nmin, int nmax, double flat, const double *const *val,
                                           double *const *al, double *const *da, double *const *a6,
                                           const PS &par) {
  if (n >= nmin + 1 && n < nmax - 1) {
    const double c3 = par_c<3>(par), c4 = par_c<4>(par);
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const double a = val[f][n];
      const double da_r = val[f][n + 1] - a;
      const double da_l = a - val[f][n - 1];
      double t1 = c3 * da_r + c4 * da_l;
      if (t1 < 0.0) t1 = -min3(-t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
      else          t1 = min3(t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
      if (da_l * da_r < 0.0) t1 = 0.0;
      a6[f][n] = t1;
    }
  }
  __syncthreads();
  double ar[NF];
  if (n >= nmin + 1 && n < nmax - 2) {
    const double c0 = par_c<0>(par), c1 = par_c<1>(par), c2 = par_c<2>(par);
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const double a = val[f][n];
      const double da_r = val[f][n + 1] - a;
      const double t1 = a6[f][n];
      ar[f] = a + c0 * da_r + c1 * a6[f][n + 1] + c2 * t1;
      al[f][n + 1] = ar[f];
    }
  }
  __syncthreads();
  if (n >= nmin + 2 && n < nmax - 2) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const double a = val[f][n];
      double u1 = flat * a;
      double u2 = 1.0 - flat;
      double xr = u1 + u2 * ar[f];
      double la = u1 + u2 * al[f][n];
      u1 = xr - la;
      u2 = u1 * u1;
      u1 = u1 * (6.0 * (a - 0.5 * (xr + la)));
      if ((xr - a) * (a - la) <= 0.0) { xr = a; la = a; }
      if (u2 < u1) la = 3.0 * a - 2.0 * xr;
      if (u2 < -u1) xr = 3.0 * a - 2.0 * la;
      da[f][n] = xr - la;
      a6[f][n] = 6.0 * (a - 0.5 * (xr + la));
      al[f][n] = la;
    }
  }
  __syncthreads();
}

// derivs viscosity.cu:2-18
__device__ __forceinline__ void derivs(double &first, double &second, int n, const double *xf, const double *u) {
  double x2 = xf[n] - xf[n - 1];
  double x3 = xf[n + 1] - xf[n - 1];
  double h2 = (u[n] - u[n - 1]) / x2;
  double h3 = (u[n + 1] - u[n - 1]) / x3;
  double A = (h3 - h2) / (x3 - x2);
  double B = (x3 * h2 - x2 * h3) / (x3 - x2);
  second = 2.0 * A;
  first = second * x2 + B;
}

// derivs for several fields of one cell: the face spacings and the three
// divisors depend on the grid only, so they are formed once per cell and the
// divisions become products (within an ulp of derivs)
struct DerivGeom { double x2, x3, i2, i3, i32; };
__device__ __forceinline__ DerivGeom deriv_geom(int n, const double *xf) {
  DerivGeom g;
  g.x2 = xf[n] - xf[n - 1];
  g.x3 = xf[n + 1] - xf[n - 1];
  g.i2 = 1.0 / g.x2;
  g.i3 = 1.0 / g.x3;
  g.i32 = 1.0 / (g.x3 - g.x2);
  return g;
}
__device__ __forceinline__ void derivs_g(double &first, double &second, int n, const DerivGeom &g,
                                         const double *u) {
  double h2 = (u[n] - u[n - 1]) * g.i2;
  double h3 = (u[n + 1] - u[n - 1]) * g.i3;
  double A = (h3 - h2) * g.i32;
  double B = (g.x3 * h2 - g.x2 * h3) * g.i32;
  second = 2.0 * A;
  first = second * g.x2 + B;
}

}  // namespace pgd
