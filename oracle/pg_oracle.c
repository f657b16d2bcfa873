/*
 * pg_oracle.c -- CPU restatement of the PEnGUIn hydro step.  TEST
 * INFRASTRUCTURE: the checker for the CUDA path, never the product.
 *
 * Every function below restates the reference routine cited beside it
 * (paths within fungjeff/penguin_2_0).  A CUDA block of the reference is
 * emulated by `blk`: each __syncthreads()-separated phase is one loop over
 * the block's active thread indices; per-thread registers that live across
 * phases are arrays indexed by thread.  Expressions keep the reference's
 * evaluation order; no FMA contraction happens here (x86-64 baseline ISA), so
 * results differ from the GPU build only by contraction and libm ulps.
 */
#include "pg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NPAD 6
#define ARR 128
#define REAL (ARR - 2 * NPAD)
#define A1 (ARR + 8)

static const double k_twopi = 6.283185307179586476925286766559;
static const double k_pi = 3.1415926535897932384626433832795;
static const double k_third = 0.3333333333333333333333333;
static const double k_fourthd = 1.3333333333333333333333333;
static const double k_smallp = 1.0e-15;
static const double k_smallr = 1.0e-15;
static const double k_earth = 0.000003;

/* ------------------------------------------------------------------------ */
/* data model: hydr_ring (variable_types.h:67-97), SymDisk (58-65)          */

typedef struct {
  double *r, *p, *u, *v, *w;
  double *y, *dy, *yvol, *yc;
  double x, dx, xvol, xc;
  double z, dz, zvol, zc;
  int i, k;
  double rot_v, res_v;
  int rot_j, inc_j;
} oring;

typedef struct { double r, p, u, v, w; } osym;

struct orc_run {
  pg_params P;
  int nr, nphi, nk, nring;
  oring *rings, *lft, *rgh, *udr, *top;
  osym *val;
  double *mem;
};

/* parameters of the current call (the reference's compile-time constants) */
static pg_params G;
static double G_vis_nu;

static void set_globals(const pg_params *p) {
  G = *p;
  G_vis_nu = p->ss_alpha * p->sc_h * p->sc_h;        /* global.h:36 */
}

static double cmin(double a, double b) { return fmin(a, b); }
static double cmax(double a, double b) { return fmax(a, b); }

/* simple_func.cu:2-28 */
static double min3(double A, double B, double C) {
  if (A < B) { if (C < A) return C; else return A; }
  else       { if (C < B) return C; else return B; }
}
static double max3(double A, double B, double C) {
  if (A > B) { if (C > A) return C; else return A; }
  else       { if (C > B) return C; else return B; }
}

/* ------------------------------------------------------------------------ */
/* disk profile (disk_profile.cu)                                           */

/* The profile serves two sides of the reference.  Its set-up (init.cpp: the
 * initial state, the fixed boundary rings, the damping targets) and its planet
 run on the host, where p_alpha, p_beta and gam are compile-time
 * constants and the host compiler turns pow(x, 0|1|-1|2) into 1, x, 1/x, x*x
 * (planet.cu's host functions likewise); hpow restates that folding.  The device kernels (the sweep store's pressure,
 * the damping kernel, the viscosity) call pow as written, so get_cs2 and
 * get_nu keep it. */
static double hpow(double x, double y) {
  if (y == 0.0) return 1.0;
  if (y == 1.0) return x;
  if (y == -1.0) return 1.0 / x;
  if (y == 2.0) return x * x;
  return pow(x, y);
}
static double get_rho1(double r) {                                         /* 9-28 */
  double n = -G.p_alpha;
  if (G.EOS != 0 && G.ndim == 3) n = -G.p_alpha * (2.0 / (G.gam + 1.0));
  return hpow(r, n);
}
static double get_cs2(double r) { return G.sc_h * G.sc_h * pow(r, -G.p_beta); } /* 39-42 */
static double host_cs2(double r) { return G.sc_h * G.sc_h * hpow(r, -G.p_beta); }
static double get_h(double r) { return sqrt(host_cs2(r) * r * r * r); }     /* 49-52 */
static double get_P1(double r) {                                           /* 54-61 */
  if (G.EOS == 0) return host_cs2(r) * get_rho1(r);
  return host_cs2(r) * hpow(get_rho1(r), G.gam) / G.gam;
}
static double get_dP_dr1(double r) {                                       /* 63-68 */
  double p1 = get_P1(r + 1.27245e-8);
  double p2 = get_P1(r - 1.27245e-8);
  return (p1 - p2) / 2.5449e-8;
}
static double get_verfac(double r, double z) {                              /* 70-75 */
  double cs2 = host_cs2(r);
  double rr = sqrt(r * r + z * z);
  return exp((1.0 / rr - 1.0 / r) / cs2);
}
static double get_rho2(double r, double z) {                               /* 86-103 */
  double gamm, h, z_0, base;
  if (G.EOS == 0) return get_rho1(r) * get_verfac(r, z);
  gamm = G.gam - 1.0;
  h = sqrt(host_cs2(r) * r * r * r);
  z_0 = sqrt(2.0 * h * h * hpow(r, -G.p_alpha * (2.0 / (G.gam + 1.0)) * gamm) / gamm);
  if (z < z_0)
    return hpow(hpow(get_rho1(r), gamm) - (gamm / (r * host_cs2(r))) * (1.0 - r / sqrt(r * r + z * z)), 1.0 / gamm);
  base = hpow(hpow(get_rho1(r), gamm) - (gamm / (r * host_cs2(r))) * (1.0 - r / sqrt(r * r + z_0 * z_0)), 1.0 / gamm);
  return pow(10.0, log10(base) - 6.0 * (z - z_0) / h);
}
static double get_P2(double r, double z) {                                 /* 112-118 */
  if (G.EOS == 0) return host_cs2(r) * get_rho2(r, z);
  return host_cs2(r) * hpow(get_rho2(r, z), G.gam) / G.gam;
}
/* the sweep store's pressure (ppm.cu:138-143): EOS 0 r cs2, EOS 1 cs2 r^gam / gam */
static double store_p(double r, double cs2) {
  if (G.EOS == 0) return r * cs2;
  return cs2 * pow(r, G.gam) / G.gam;
}
static double get_dP_s(double r, double pol) {                              /* 128-138 */
  double dr = 1.27e-7;
  double sinpol = sin(pol);
  double cospol = cos(pol);
  double r1 = (r + dr) * sinpol;
  double z1 = (r + dr) * cospol;
  double r2 = (r - dr) * sinpol;
  double z2 = (r - dr) * cospol;
  return (get_P2(r1, z1) - get_P2(r2, z2)) / (2.0 * dr);
}
static double get_nu(double r) { return G_vis_nu * pow(r, G.p_alpha); }    /* 149-152 */
static double get_viscous_vr(double r) {                                   /* 154-160 */
  if (G.visc_flag == 1) return -1.5 * (G_vis_nu * hpow(r, G.p_alpha)) / r;
  return 0.0;
}

/* ------------------------------------------------------------------------ */
/* forces (src/ppm/forces.cu), non-barycentric frame only                   */

typedef struct { double m, x, y, vx, vy, fx, fy, rs; } obody;

static double grav_rad_sph(double rad, double azi, double pol, const obody *p, double dt) { /* 23-50 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double sinpol = sin(pol);
  double stm = 1.0 / (1.0 + p->m);
  double plm = p->m * stm;
  double plx = p->x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p->rs * p->rs);
  return -plm * (rad - plx * cosfac * sinpol) / (Rp * Rp * Rp) - stm / (rad * rad)
         - plm * sinpol * cosfac / (plx * plx);
}
static double grav_azi_sph(double rad, double azi, double pol, const obody *p, double dt) { /* 52-81 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double sinfac = sin(azi - (p->y + dt * p->vy));
  double sinpol = sin(pol);
  rad /= sinpol;
  double stm = 1.0 / (1.0 + p->m);
  double plm = p->m * stm;
  double plx = p->x;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p->rs * p->rs);
  return -plm * plx * sinfac / (Rp * Rp * Rp) + plm * sinpol * sinfac / plx / plx;
}
static double grav_pol_sph(double rad, double azi, double pol, const obody *p, double dt) { /* 83-110 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double cospol = cos(pol);
  double sinpol = sin(pol);
  double stm = 1.0 / (1.0 + p->m);
  double plm = p->m * stm;
  double plx = p->x;
  (void)stm;
  double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol;
  Rp = sqrt(Rp + p->rs * p->rs);
  return plm * plx * cosfac * cospol / (Rp * Rp * Rp) - plm * cosfac * cospol / (sinpol * plx * plx);
}
static double grav_rad_cyl(double rad, double azi, double z, const obody *p, double dt) { /* 112-134 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double plm = p->m;
  double plx = p->x;
  double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p->rs * p->rs);
  return -plm * (rad - plx * cosfac) / (Rp * Rp * Rp) - plm * cosfac / (plx * plx);
}
static double grav_azi_cyl(double rad, double azi, double z, const obody *p, double dt) { /* 136-159 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double sinfac = sin(azi - (p->y + dt * p->vy));
  double plm = p->m;
  double plx = p->x;
  double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p->rs * p->rs);
  return -plm * plx * sinfac / (Rp * Rp * Rp) + plm * sinfac / plx / plx;
}
static double grav_pol_cyl(double rad, double azi, double z, const obody *p, double dt) { /* 161-182 */
  double cosfac = cos(azi - (p->y + dt * p->vy));
  double plm = p->m;
  double plx = p->x;
  double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p->rs * p->rs);
  return -plm * z / (Rp * Rp * Rp);
}

/* get_fx_bound forces.cu:185-224 (face, uses the two neighbouring cells) */
static void get_fx_bound(int n, double dt, double rad, double azi, double pol, double *ftot,
                         const obody *pl, const double *v, const double *w) {
  double grav;
  if (G.ngeomx == 0) { *ftot = 0.0; return; }
  if (G.ngeomx == 1) {
    if (G.plnt_flag > 0) {
      grav = grav_rad_cyl(rad, azi, pol, pl, dt);
      grav += -1.0 / rad / rad;
    } else {
      double dis = sqrt(rad * rad + pol * pol);
      grav = -rad / dis / dis / dis;
    }
    double f = grav;
    f += pow(0.5 * (v[n] + v[n - 1]), 2) / rad / rad / rad;
    *ftot = f;
  } else {
    if (G.plnt_flag > 0) grav = grav_rad_sph(rad, azi, pol, pl, dt);
    else grav = -1.0 / rad / rad;
    double f = grav;
    f += pow(0.5 * (w[n] + w[n - 1]), 2) / rad / rad / rad;
    f += pow(0.5 * (v[n] + v[n - 1]), 2) / rad / pow(rad * sin(pol), 2);
    *ftot = f;
  }
}
/* get_fx forces.cu:226-263 (cell centre) */
static void get_fx(int n, double dt, double rad, double azi, double pol, double *ftot,
                   const obody *pl, const double *v, const double *w) {
  double grav;
  if (G.ngeomx == 0) { *ftot = 0.0; return; }
  if (G.ngeomx == 1) {
    if (G.plnt_flag > 0) {
      grav = grav_rad_cyl(rad, azi, pol, pl, dt);
      grav += -1.0 / rad / rad;
    } else {
      double dis = sqrt(rad * rad + pol * pol);
      grav = -rad / dis / dis / dis;
    }
    double f = grav;
    f += v[n] * v[n] / rad / rad / rad;
    *ftot = f;
  } else {
    if (G.plnt_flag > 0) grav = grav_rad_sph(rad, azi, pol, pl, dt);
    else grav = -1.0 / rad / rad;
    double f = grav;
    f += w[n] * w[n] / rad / rad / rad;
    f += v[n] * v[n] / rad / pow(rad * sin(pol), 2);
    *ftot = f;
  }
}
/* get_fy forces.cu:265-296 */
static void get_fy(double dt, double rad, double azi, double pol, double *ftot, const obody *pl) {
  if (G.ngeomy == 3) *ftot = (G.plnt_flag > 0) ? grav_azi_cyl(rad, azi, pol, pl, dt) : 0.0;
  else if (G.ngeomy == 4) *ftot = (G.plnt_flag > 0) ? grav_azi_sph(rad, azi, pol, pl, dt) : 0.0;
  else *ftot = 0.0;
}
/* get_fz_bound forces.cu:298-334 */
static void get_fz_bound(int n, double dt, double rad, double azi, double pol, double *ftot,
                         const obody *pl, const double *w) {
  double grav;
  if (G.ngeomz == 0) {
    if (G.plnt_flag > 0) grav = grav_pol_cyl(rad, azi, pol, pl, dt);
    else { double dis = sqrt(rad * rad + pol * pol); grav = -pol / dis / dis / dis; }
    *ftot = grav;
  } else {
    grav = (G.plnt_flag > 0) ? grav_pol_sph(rad, azi, pol, pl, dt) : 0.0;
    double rad_cyl = rad * sin(pol);
    double f = grav;
    f += (pow(0.5 * (w[n] + w[n - 1]), 2) * cos(pol)) / rad_cyl / rad_cyl / rad_cyl;
    *ftot = f;
  }
}
/* get_fz forces.cu:336-372 */
static void get_fz(int n, double dt, double rad, double azi, double pol, double *ftot,
                   const obody *pl, const double *w) {
  double grav;
  if (G.ngeomz == 0) {
    if (G.plnt_flag > 0) grav = grav_pol_cyl(rad, azi, pol, pl, dt);
    else { double dis = sqrt(rad * rad + pol * pol); grav = -pol / dis / dis / dis; }
    *ftot = grav;
  } else {
    grav = (G.plnt_flag > 0) ? grav_pol_sph(rad, azi, pol, pl, dt) : 0.0;
    double rad_cyl = rad * sin(pol);
    double f = grav;
    f += (w[n] * w[n] * cos(pol)) / rad_cyl / rad_cyl / rad_cyl;
    *ftot = f;
  }
}

/* ------------------------------------------------------------------------ */
/* one CUDA block of 128 threads                                            */

typedef struct { double c0, c1, c2, c3, c4; } opar;
typedef struct { double rl, pl, ul, rr, pr, ur; } osv;

typedef struct {
  unsigned char act[ARR];
  /* sweep-kernel shared arrays (ppm.cu:38-39, 175-176) */
  double r[A1], p[A1], u[A1], v[A1], w[A1], xa0[A1], dx0[A1];
  /* ppmlr shared arrays (ppmlr.cu:7-10) */
  double q[A1], dx[A1], umid[A1], pmid[A1], tmp1[A1];
  /* per-thread registers */
  double rad[ARR], azi[ARR], pol[ARR], vrot[ARR], dvol0[ARR];
  double flat[ARR], ftot[ARR];
  opar par[ARR];
  osv S[ARR];
  double ps_dxn[ARR], ps_ain[ARR], ps_bi[ARR], ps_ci[ARR], ps_c[ARR];
  double pb_a[ARR], pb_dar[ARR], pb_t1[ARR], pb_ar[ARR];
  double dvol[ARR], xa[ARR], dtdm[ARR], fto1[ARR], fto2[ARR];
  double lvol[ARR], dxf[ARR], dxf2[ARR], fr[ARR], dxn[ARR], dxnm[ARR], mm[ARR], invm[ARR];
  unsigned char delC[ARR];
  double vrho[ARR], vnr[ARR], ddu[ARR], ddv[ARR], ddw[ARR];
  /* carries of the sweep kernels */
  double lt[5][ARR], rg[5][NPAD];
} oblk;

#define FOR_ACT(n) for (int n = 0; n < ARR; n++) if (B->act[n])

static void blk_poison(oblk *B) {
  double nan = NAN;
  double *arrs[] = {B->r, B->p, B->u, B->v, B->w, B->xa0, B->dx0, B->q, B->dx, B->umid, B->pmid, B->tmp1};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++)
    for (int n = 0; n < A1; n++) arrs[a][n] = nan;
  for (int c = 0; c < 5; c++) for (int n = 0; n < NPAD; n++) B->rg[c][n] = nan;
}

/* paraset parabola.cu:138-176 */
static void paraset(oblk *B, int nmin, int nmax, const double *dx, double *a, double *ai, double *b) {
  FOR_ACT(n) {
    B->par[n].c0 = B->par[n].c1 = B->par[n].c2 = B->par[n].c3 = B->par[n].c4 = NAN;
    if (n >= nmin && n < nmax - 1) {
      double dx_n = dx[n];
      double an = dx_n + dx[n + 1];
      double ain = 1.0 / an;
      double bn = an + dx_n;
      double bi = 1.0 / bn;
      double c = an + dx[n + 1];
      double ci = 1.0 / c;
      a[n] = an; ai[n] = ain; b[n] = bn;
      B->ps_dxn[n] = dx_n; B->ps_ain[n] = ain; B->ps_bi[n] = bi; B->ps_ci[n] = ci; B->ps_c[n] = c;
    }
  }
  FOR_ACT(n) {
    double dx_n = B->ps_dxn[n], ain = B->ps_ain[n], bi = B->ps_bi[n], ci = B->ps_ci[n], c = B->ps_c[n];
    if (n >= nmin + 1 && n < nmax - 2) {
      double d = 1.0 / (a[n - 1] + a[n + 1]);
      B->par[n].c0 = dx_n * ain * (1.0 + 2.0 * d * dx[n + 1] * (a[n - 1] * bi - a[n + 1] * ci));
      B->par[n].c1 = -d * dx_n * a[n - 1] * bi;
      B->par[n].c2 = d * dx[n + 1] * a[n + 1] * ci;
    }
    if (n >= nmin + 1 && n < nmax - 1) {
      double d = dx_n / (a[n - 1] + dx[n + 1]);
      B->par[n].c3 = d * b[n - 1] * ain;
      B->par[n].c4 = d * c * ai[n - 1];
    }
  }
}

/* parabola parabola.cu:70-133 (CW84 eq 1.5-1.8, 1.10) */
static void parabola(oblk *B, int nmin, int nmax, const double *flat, const double *val,
                     double *al, double *da, double *a6) {
  FOR_ACT(n) {
    if (n >= nmin + 1 && n < nmax - 1) {
      double a = val[n];
      double da_r = val[n + 1] - a;
      double da_l = a - val[n - 1];
      double t1 = B->par[n].c3 * da_r + B->par[n].c4 * da_l;
      if (t1 < 0.0) t1 = -min3(-t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
      else          t1 = min3(t1, 2.0 * fabs(da_l), 2.0 * fabs(da_r));
      if (da_l * da_r < 0.0) t1 = 0.0;
      a6[n] = t1;
      B->pb_a[n] = a; B->pb_dar[n] = da_r; B->pb_t1[n] = t1;
    }
  }
  FOR_ACT(n) {
    if (n >= nmin + 1 && n < nmax - 2) {
      double a = B->pb_a[n];
      double ar = a + B->par[n].c0 * B->pb_dar[n] + B->par[n].c1 * a6[n + 1] + B->par[n].c2 * B->pb_t1[n];
      al[n + 1] = ar;
      B->pb_ar[n] = ar;
    }
  }
  FOR_ACT(n) {
    if (n >= nmin + 2 && n < nmax - 2) {
      double a = B->pb_a[n];
      double t1 = flat[n] * a;
      double t2 = 1.0 - flat[n];
      double ar = t1 + t2 * B->pb_ar[n];
      double la = t1 + t2 * al[n];
      t1 = ar - la;
      t2 = t1 * t1;
      t1 = t1 * (6.0 * (a - 0.5 * (ar + la)));
      if ((ar - a) * (a - la) <= 0.0) { ar = a; la = a; }
      if (t2 < t1) la = 3.0 * a - 2.0 * ar;
      if (t2 < -t1) ar = 3.0 * a - 2.0 * la;
      da[n] = ar - la;
      a6[n] = 6.0 * (a - 0.5 * (ar + la));
      al[n] = la;
    }
  }
}

/* flatten flatten.cu:7-40 */
static void flatten(oblk *B, int nmax, const double *p, const double *u, double *steep) {
  FOR_ACT(n) {
    int shock = 0;
    steep[n] = 0.0;
    if (n >= 2 && n < nmax - 2) {
      double dp1 = p[n + 1] - p[n - 1];
      double dp2 = p[n + 2] - p[n - 2];
      if (fabs(dp2) < k_smallp) dp2 = k_smallp;
      double ddp = fabs(dp1) / cmin(p[n + 1], p[n - 1]);
      if (ddp > 0.33) shock = 1;
      if (u[n - 1] < u[n + 1]) shock = 0;
      if (shock) {
        ddp = (dp1 / dp2 - 0.75) * 5.0;
        steep[n] = cmax(0.0, ddp);
      }
    }
  }
  FOR_ACT(n) {
    if (n >= 2 && n < nmax - 2) {
      double dp1 = max3(steep[n - 1], steep[n], steep[n + 1]);
      B->flat[n] = cmin(0.5, dp1);
    }
  }
}

/* states states.cu:3-73 */
static void states(oblk *B, int nmax, double hdt, int axis, const obody *pl,
                   double *al, double *da, double *a6, double *cs, double *csfac) {
  paraset(B, 0, nmax, B->dx0, al, da, a6);
  FOR_ACT(n) {
    if (n >= 2 && n < nmax - 1) {
      if (axis == 0)
        get_fx_bound(n, hdt, B->xa0[n], B->azi[n] + hdt * B->vrot[n], B->pol[n], &B->ftot[n], pl, B->v, B->w);
      else if (axis == 1)
        get_fy(hdt, B->rad[n], B->xa0[n] + hdt * B->vrot[n], B->pol[n], &B->ftot[n], pl);
      else
        get_fz_bound(n, hdt, B->rad[n], B->azi[n] + hdt * B->vrot[n], B->xa0[n], &B->ftot[n], pl, B->w);
    }
  }
  FOR_ACT(n) {
    cs[n] = hdt * sqrt(G.gam * B->p[n] / B->r[n]) / B->dx0[n];
    if (axis == 1) cs[n] /= B->rad[n];
    if (axis == 2) { if (G.ngeomz == 5) cs[n] /= B->rad[n]; }
    csfac[n] = 1.0 - k_fourthd * cs[n];
  }
  parabola(B, 0, nmax, B->flat, B->p, al, da, a6);
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double tmp = al[n - 1] + da[n - 1] - cs[n - 1] * (da[n - 1] - csfac[n - 1] * a6[n - 1]);
      B->S[n].pl = cmax(k_smallp, tmp);
      tmp = al[n] + cs[n] * (da[n] + csfac[n] * a6[n]);
      B->S[n].pr = cmax(k_smallp, tmp);
    }
  }
  parabola(B, 0, nmax, B->flat, B->r, al, da, a6);
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double tmp = al[n - 1] + da[n - 1] - cs[n - 1] * (da[n - 1] - csfac[n - 1] * a6[n - 1]);
      B->S[n].rl = cmax(k_smallr, tmp);
      tmp = al[n] + cs[n] * (da[n] + csfac[n] * a6[n]);
      B->S[n].rr = cmax(k_smallr, tmp);
    }
  }
  parabola(B, 0, nmax, B->flat, B->u, al, da, a6);
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double tmp = al[n - 1] + da[n - 1] - cs[n - 1] * (da[n - 1] - csfac[n - 1] * a6[n - 1]);
      B->S[n].ul = tmp + hdt * B->ftot[n];
      tmp = al[n] + cs[n] * (da[n] + csfac[n] * a6[n]);
      B->S[n].ur = tmp + hdt * B->ftot[n];
    }
  }
}

/* riemann riemann.cu:75-111, the EOS 1 branch: van Leer's Newton iteration
 * on the Lagrangian sound speeds (at most 10 passes, tolerance 1e-8) */
static void riemann_newton(double pl, double rl, double ul, double pr, double rr, double ur,
                           double *umid, double *pmid) {
  const double gamfac2 = G.gam + 1.0, gamfac1 = gamfac2 / G.gam / 2.0;
  double cs_l = sqrt(G.gam * pl * rl), cs_r = sqrt(G.gam * pr * rr);
  double pm, t1 = 0.0, t2 = 0.0, en_l, en_r, dum, uml, umr;
  int l;
  rl = 1.0 / rl;
  rr = 1.0 / rr;
  pm = pr - pl - cs_r * (ur - ul);
  pm = pl + pm * cs_l / (cs_l + cs_r);
  pm = cmax(k_smallp, pm);
  for (l = 0; l < 10; l++) {
    dum = pm;
    t1 = 1.0 + gamfac1 * (pm - pl) / pl;
    t2 = 1.0 + gamfac1 * (pm - pr) / pr;
    t1 = cs_l * sqrt(t1);
    t2 = cs_r * sqrt(t2);
    en_l = 4.0 * rl * t1 * t1;
    en_r = 4.0 * rr * t2 * t2;
    en_l = -en_l * t1 / (en_l - gamfac2 * (pm - pl));
    en_r = en_r * t2 / (en_r - gamfac2 * (pm - pr));
    uml = ul - (pm - pl) / t1;
    umr = ur + (pm - pr) / t2;
    pm = pm + (umr - uml) * (en_r * en_l) / (en_r - en_l);
    pm = cmax(k_smallp, pm);
    if (fabs(pm - dum) / pm < 1.0e-8) break;
  }
  uml = ul - (pm - pl) / t1;
  umr = ur + (pm - pr) / t2;
  *umid = 0.5 * (uml + umr);
  *pmid = cmax(k_smallp, pm);
}

/* riemann riemann.cu:3-115: isothermal (EOS 0, 45-53) or isentropic (EOS 1) */
static void riemann(oblk *B, int nmax, double *umid, double *pmid) {
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double pl = B->S[n].pl, rl = B->S[n].rl, ul = B->S[n].ul;
      double pr = B->S[n].pr, rr = B->S[n].rr, ur = B->S[n].ur;
      if (G.EOS == 1) { riemann_newton(pl, rl, ul, pr, rr, ur, &umid[n], &pmid[n]); continue; }
      double t1 = 0.5 * (sqrt(pl / rl) + sqrt(pr / rr));
      double t2 = -0.5 * (ur - ul) / t1;
      double pm = sqrt(pl * pr) * exp(t2);
      umid[n] = ul - t1 * log(pm / pl);
      pmid[n] = cmax(k_smallp, pm);
    }
  }
}

/* evolve evolve.cu:3-166 */
static void evolve(oblk *B, int nmax, double dt, int axis, double FrRot, const obody *pl,
                   double *vfac, double *umid, double *pmid) {
  FOR_ACT(n) vfac[n] = B->xa0[n] + 0.5 * B->dx0[n];
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double delx;
      if (axis == 0) delx = dt * umid[n];
      else if (axis == 1) {
        if (G.ngeomy > 2) delx = dt * (umid[n] / B->rad[n] - B->vrot[n] - FrRot);
        else delx = dt * umid[n];
      } else {
        if (G.ngeomz == 5) delx = dt * umid[n] / B->rad[n];
        else delx = dt * umid[n];
      }
      B->dtdm[n] = dt / (B->r[n] * B->dvol0[n]);
      vfac[n] = B->xa0[n] + delx;
    }
  }
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 3) {
      B->dx[n] = vfac[n + 1] - vfac[n];
      B->xa[n] = vfac[n];
    }
  }
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 3) {
      double xcl = B->xa[n] + 0.5 * B->dx[n];
      if (axis == 0) {
        get_fx(n, 0.0, B->rad[n], B->azi[n], B->pol[n], &B->fto1[n], pl, B->v, B->w);
        get_fx(n, dt, xcl, B->azi[n] + dt * B->vrot[n], B->pol[n], &B->fto2[n], pl, B->v, B->w);
      } else if (axis == 1) {
        get_fy(0.0, B->rad[n], B->azi[n], B->pol[n], &B->fto1[n], pl);
        get_fy(dt, B->rad[n], xcl + dt * B->vrot[n], B->pol[n], &B->fto2[n], pl);
      } else {
        get_fz(n, 0.0, B->rad[n], B->azi[n], B->pol[n], &B->fto1[n], pl, B->w);
        get_fz(n, dt, B->rad[n], B->azi[n] + dt * B->vrot[n], xcl, &B->fto2[n], pl, B->w);
      }
    }
  }
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 2) {
      double xa = B->xa[n], x0 = B->xa0[n], dxn = B->dx[n];
      umid[n] *= pmid[n];
      if (axis == 0) {
        if (G.ngeomx == 0) { B->dvol[n] = dxn; vfac[n] = 1.0; }
        else if (G.ngeomx == 1) { B->dvol[n] = dxn * (xa + 0.5 * dxn); vfac[n] = 0.5 * (xa + x0); }
        else if (G.ngeomx == 2) {
          B->dvol[n] = dxn * (xa * (xa + dxn) + dxn * dxn * k_third);
          vfac[n] = (xa - x0) * (k_third * (xa - x0) + x0) + (x0 * x0);
        }
      } else if (axis == 1) {
        if (G.ngeomy == 0) { B->dvol[n] = dxn; vfac[n] = 1.0; }
        else { B->dvol[n] = dxn * B->rad[n]; vfac[n] = 1.0; }
      } else {
        if (G.ngeomz == 0) { B->dvol[n] = dxn; vfac[n] = 1.0; }
        else if (G.ngeomz == 5) {
          /* cos(a) - cos(b) = 2 sin((a+b)/2) sin((b-a)/2): the value of
           * evolve.cu:119-123 without its cancellation (the polar sweep has
           * no reference driver to match bit for bit) */
          double delx = xa - x0;
          B->dvol[n] = 2.0 * sin(xa + 0.5 * dxn) * sin(0.5 * dxn) * B->rad[n];
          if (delx == 0.0) vfac[n] = sin(xa);
          else vfac[n] = 2.0 * sin(x0 + 0.5 * delx) * sin(0.5 * delx) / delx;
        }
      }
    }
  }
  FOR_ACT(n) {
    if (n >= 3 && n < nmax - 3) {
      B->q[n] = (G.EOS == 0) ? B->p[n] / B->r[n] : B->p[n] / pow(B->r[n], G.gam);   /* evolve.cu:131-135 */
      B->r[n] = cmax(B->r[n] * (B->dvol0[n] / B->dvol[n]), k_smallr);
      double dum = B->u[n];
      double delx = 0.5 * dt * (B->fto1[n] + B->fto2[n]);
      delx += -B->dtdm[n] * (pmid[n + 1] - pmid[n]) * 0.5 * (vfac[n + 1] + vfac[n]);
      B->u[n] = dum + delx;
    }
  }
}

/* get_flux remap.cu:1-10 */
static void get_flux(oblk *B, int nmax, double *flux, const double *al, const double *da,
                     const double *a6, double *out) {
  FOR_ACT(n) {
    if (n >= 6 && n < nmax - 5) {
      if (B->delC[n]) flux[n] = (al[n - 1] + da[n - 1] - B->dxf[n] * (da[n - 1] - B->dxf2[n] * a6[n - 1])) * B->fr[n];
      else            flux[n] = (al[n] - B->dxf[n] * (da[n] + B->dxf2[n] * a6[n])) * B->fr[n];
    }
  }
  FOR_ACT(n) out[n] = flux[n] - flux[n + 1];
}

/* remap remap.cu:14-226 (the q remap sets p, which the sweep store later
 * overwrites by the EOS relation; it is kept here as in the reference) */
static void remap(oblk *B, int nmax, int axis, double *al, double *da, double *a6) {
  double fluxn[ARR];
  paraset(B, 3, nmax - 3, B->dx, al, da, a6);
  FOR_ACT(n) {
    double xa = B->xa[n], x0 = B->xa0[n], lvol = 0.0;
    if (axis == 0) {
      if (G.ngeomx == 0) lvol = xa - x0;
      else if (G.ngeomx == 1) { lvol = xa - x0; lvol *= (x0 + 0.5 * lvol); }
      else if (G.ngeomx == 2) { lvol = xa - x0; lvol *= x0 * xa + k_third * (lvol * lvol); }
    } else if (axis == 1) {
      if (G.ngeomy == 0) lvol = xa - x0;
      else lvol = (xa - x0) * B->rad[n];
    } else {
      if (G.ngeomz == 0) lvol = xa - x0;
      else if (G.ngeomz == 5) {
        double d = xa - x0;   /* remap.cu:53 without cancellation */
        lvol = 2.0 * sin(x0 + 0.5 * d) * sin(0.5 * d) * B->rad[n];
      }
    }
    B->lvol[n] = lvol;
    B->dxf[n] = xa - x0;
    B->delC[n] = (B->dxf[n] >= 0.0);
  }
  parabola(B, 3, nmax - 3, B->flat, B->r, al, da, a6);
  double *flux = B->dx;
  FOR_ACT(n) {
    if (n >= 6 && n < nmax - 5) { B->dxn[n] = B->dx[n]; B->dxnm[n] = B->dx[n - 1]; }
  }
  FOR_ACT(n) {
    if (n >= 6 && n < nmax - 5) {
      if (B->delC[n]) {
        B->dxf[n] = 0.5 * B->dxf[n] / B->dxnm[n];
        B->dxf2[n] = 1.0 - k_fourthd * B->dxf[n];
        B->fr[n] = (al[n - 1] + da[n - 1] - B->dxf[n] * (da[n - 1] - B->dxf2[n] * a6[n - 1])) * B->lvol[n];
      } else {
        B->dxf[n] = 0.5 * B->dxf[n] / B->dxn[n];
        B->dxf2[n] = 1.0 + k_fourthd * B->dxf[n];
        B->fr[n] = (al[n] - B->dxf[n] * (da[n] + B->dxf2[n] * a6[n])) * B->lvol[n];
      }
      flux[n] = B->fr[n];
    }
  }
  FOR_ACT(n) {
    if (n >= 6 && n < nmax - 6) {
      B->mm[n] = B->r[n] * B->dvol[n];
      double lv = (B->mm[n] + B->fr[n] - flux[n + 1]) / B->dvol0[n];
      B->r[n] = cmax(k_smallr, lv);
      B->invm[n] = 1.0 / (B->r[n] * B->dvol0[n]);
    }
  }
  parabola(B, 3, nmax - 3, B->flat, B->u, al, da, a6);
  get_flux(B, nmax, flux, al, da, a6, fluxn);
  FOR_ACT(n) if (n >= 6 && n < nmax - 6) B->u[n] = (B->u[n] * B->mm[n] + fluxn[n]) * B->invm[n];
  parabola(B, 3, nmax - 3, B->flat, B->v, al, da, a6);
  get_flux(B, nmax, flux, al, da, a6, fluxn);
  FOR_ACT(n) if (n >= 6 && n < nmax - 6) B->v[n] = (B->v[n] * B->mm[n] + fluxn[n]) * B->invm[n];
  parabola(B, 3, nmax - 3, B->flat, B->w, al, da, a6);
  get_flux(B, nmax, flux, al, da, a6, fluxn);
  FOR_ACT(n) if (n >= 6 && n < nmax - 6) B->w[n] = (B->w[n] * B->mm[n] + fluxn[n]) * B->invm[n];
  parabola(B, 3, nmax - 3, B->flat, B->q, al, da, a6);
  get_flux(B, nmax, flux, al, da, a6, fluxn);
  FOR_ACT(n) {
    if (n >= 6 && n < nmax - 6) {
      B->q[n] = (B->q[n] * B->mm[n] + fluxn[n]) * B->invm[n];
      B->p[n] = cmax(k_smallp, (G.EOS == 0) ? B->r[n] * B->q[n] : pow(B->r[n], G.gam) * B->q[n]);  /* remap.cu:123-142 */
    }
  }
}

/* ppmlr ppmlr.cu:2-56 */
static void ppmlr(oblk *B, int nmax, double dt, int axis, double FrRot, const obody *pl) {
  FOR_ACT(n) {
    B->q[n] = 0.0; B->dx[n] = 0.0; B->umid[n] = 0.0; B->pmid[n] = 0.0; B->tmp1[n] = 0.0;
    B->flat[n] = 0.0;
  }
  if (G.flat_flag) flatten(B, nmax, B->p, B->u, B->tmp1);
  states(B, nmax, 0.5 * dt, axis, pl, B->q, B->dx, B->tmp1, B->umid, B->pmid);
  riemann(B, nmax, B->umid, B->pmid);
  FOR_ACT(n) { B->dvol[n] = B->dvol0[n]; B->xa[n] = B->xa0[n]; }
  evolve(B, nmax, dt, axis, FrRot, pl, B->tmp1, B->umid, B->pmid);
  remap(B, nmax, axis, B->tmp1, B->umid, B->pmid);
}

/* derivs viscosity.cu:2-18 */
static void derivs(double *first, double *second, int n, const double *xf, const double *u) {
  double x2 = xf[n] - xf[n - 1];
  double x3 = xf[n + 1] - xf[n - 1];
  double h2 = (u[n] - u[n - 1]) / x2;
  double h3 = (u[n + 1] - u[n - 1]) / x3;
  double A = (h3 - h2) / (x3 - x2);
  double Bc = (x3 * h2 - x2 * h3) / (x3 - x2);
  *second = 2.0 * A;
  *first = *second * x2 + Bc;
}

/* device_viscosity_r viscosity.cu:370-421; R per thread */
static void visc_r(oblk *B, int lim, double dt, const double *Rv, const double *x, double *cr,
                   double *u, double *v, double *w, double *nn) {
  FOR_ACT(i) {
    if (i >= 0 && i < lim) {
      double R = Rv[i];
      B->vrho[i] = cr[i];
      B->vnr[i] = get_nu(R) * B->vrho[i];
      nn[i] = B->vnr[i];
      v[i] /= R * R;
    }
  }
  FOR_ACT(i) {
    if (i >= NPAD && i < lim - NPAD) {
      double R = Rv[i], nr = B->vnr[i], rho = B->vrho[i], d1, d2, dn;
      derivs(&dn, &d2, i, x, nn);
      derivs(&d1, &d2, i, x, u);
      double ddu = 2.0 * nr * d2 + 2.0 * dn * d1 + 2.0 * nr * d1 / R - 2.0 * nr * u[i] / R / R;
      B->ddu[i] = u[i] + dt * ddu / rho;
      if (G.ndim > 1) {
        derivs(&d1, &d2, i, x, v);
        double ddv = R * nr * d2 + R * dn * d1 + 3.0 * nr * d1;
        B->ddv[i] = v[i] * R + dt * ddv / rho;
      }
      if (G.ndim == 3) {
        derivs(&d1, &d2, i, x, w);
        double ddw = nr * d2 + dn * d1 + nr * d1 / R;
        B->ddw[i] = w[i] + dt * ddw / rho;
      }
    }
  }
  FOR_ACT(i) {
    if (i >= NPAD && i < lim - NPAD) {
      u[i] = B->ddu[i];
      if (G.ndim > 1) {
        v[i] = B->ddv[i] * Rv[i];
        if (G.ndim == 3) w[i] = B->ddw[i];
      }
    }
  }
}

/* device_viscosity_p viscosity.cu:423-472; R fixed per ring */
static void visc_p(oblk *B, int lim, double dt, double R, const double *x, double *cr,
                   double *u, double *v, double *w, double *nn) {
  FOR_ACT(j) {
    if (j >= 0 && j < lim) {
      B->vrho[j] = cr[j];
      B->vnr[j] = get_nu(R) * B->vrho[j];
      nn[j] = B->vnr[j];
    }
  }
  FOR_ACT(j) {
    if (j >= NPAD && j < lim - NPAD) {
      double nr = B->vnr[j], rho = B->vrho[j], d1, d2, dn;
      derivs(&dn, &d2, j, x, nn);
      derivs(&d1, &d2, j, x, v);
      double ddv = 2.0 * nr * d2 + 2.0 * dn * d1;
      double ddu = 0.0;
      B->ddv[j] = v[j] + dt * ddv / rho;
      if (G.ndim == 3) {
        derivs(&d1, &d2, j, x, w);
        double ddw = nr * d2 + dn * d1;
        B->ddw[j] = w[j] + dt * ddw / rho;
      }
      derivs(&d1, &d2, j, x, u);
      ddu += nr * d2 + dn * d1;
      B->ddu[j] = u[j] + dt * ddu / rho;
    }
  }
  FOR_ACT(j) {
    if (j >= NPAD && j < lim - NPAD) {
      v[j] = B->ddv[j];
      if (G.ndim == 3) w[j] = B->ddw[j];
      u[j] = B->ddu[j];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* the sweep kernels                                                        */

static obody to_obody(const pg_body *b) {
  obody o = {b->m, b->x, b->y, b->vx, b->vy, b->fx, b->fy, b->rs};
  return o;
}

static int wrap1(int j, int n) {
  if (j < 0) j += n;
  if (j >= n) j -= n;
  return j;
}

/* sweepx ppm.cu:26-160: one block per (azimuth column j0, k layer) */
static void sweepx_block(orc_run *R, oblk *B, int j0, int k_ring, double dt, const obody *pl, double FrRot) {
  const int iblk = R->nr, jmax = R->nphi;
  const int loop = (iblk / REAL) + (iblk % REAL != 0);
  oring *cur[ARR];
  int jj[ARR];
  double radc[ARR];
  blk_poison(B);
  for (int l = 0; l < loop; l++) {
    int lim = ARR;
    if (l == loop - 1) lim = (iblk % REAL) + 2 * NPAD;
    for (int i = 0; i < ARR; i++) {
      int i_ring = (i - NPAD) + REAL * l;
      B->act[i] = (i_ring < iblk + NPAD);
      if (!B->act[i]) continue;
      if (i_ring < 0) cur[i] = &R->lft[i_ring + NPAD + NPAD * k_ring];
      else if (i_ring >= iblk) cur[i] = &R->rgh[i_ring - iblk + NPAD * k_ring];
      else cur[i] = &R->rings[i_ring + iblk * k_ring];
    }
    FOR_ACT(i) {
      oring *c = cur[i];
      int j = wrap1(j0 - c->rot_j, jmax);
      jj[i] = j;
      double rad = (G.ngeomx > 0) ? c->xc : 1.0;
      B->rad[i] = rad;
      B->azi[i] = c->yc[j0];
      B->pol[i] = (G.ndim == 3) ? c->zc : 0.0;
      double rad_cyl = rad;
      if (G.ngeomz == 5) rad_cyl *= sin(B->pol[i]);
      radc[i] = rad_cyl;
      B->xa0[i] = c->x;
      B->dx0[i] = c->dx;
      B->dvol0[i] = c->xvol;
      if (l > 0 && i < NPAD) {
        B->r[i] = B->lt[0][i]; B->p[i] = B->lt[1][i]; B->u[i] = B->lt[2][i];
        B->v[i] = B->lt[3][i]; B->w[i] = B->lt[4][i];
      } else {
        B->r[i] = c->r[j]; B->p[i] = c->p[j]; B->u[i] = c->u[j]; B->v[i] = c->v[j]; B->w[i] = c->w[j];
        if (G.ngeomy > 2) B->v[i] *= rad_cyl;
        if (G.ngeomz == 5) B->w[i] *= rad;
      }
    }
    FOR_ACT(i) {
      if (l < loop - 1 && i < NPAD) {
        int s = i + lim - 2 * NPAD;
        B->lt[0][i] = B->r[s]; B->lt[1][i] = B->p[s]; B->lt[2][i] = B->u[s];
        B->lt[3][i] = B->v[s]; B->lt[4][i] = B->w[s];
      }
    }
    FOR_ACT(i) B->vrot[i] = cur[i]->res_v / radc[i];
    ppmlr(B, lim, dt, 0, FrRot, pl);
    if (G.visc_flag == 1) visc_r(B, lim, dt, radc, B->xa0, B->r, B->u, B->v, B->w, B->dx0);
    FOR_ACT(i) {
      if (i >= NPAD && i < lim - NPAD) {
        oring *c = cur[i];
        int j = jj[i];
        c->r[j] = B->r[i];
        c->p[j] = store_p(B->r[i], get_cs2(radc[i]));
        c->u[j] = B->u[i];
        if (G.ngeomy > 2) c->v[j] = B->v[i] / radc[i];
        else c->v[j] = B->v[i];
        if (G.ngeomz == 5) c->w[j] = B->w[i] / B->rad[i];
        else c->w[j] = B->w[i];
      }
    }
  }
}

/* sweepy ppm.cu:162-307: one block per ring */
static void sweepy_block(orc_run *R, oblk *B, int nring, double dt, const obody *pl, double FrRot) {
  const int jmax = R->nphi;
  const int loop = (jmax / REAL) + (jmax % REAL != 0);
  oring *c = &R->rings[nring];
  int jj[ARR];
  blk_poison(B);
  double rad = (G.ngeomx > 0) ? c->xc : 1.0;
  double pol = (G.ndim == 3) ? c->zc : 0.0;
  double rad_cyl = rad;
  if (G.ngeomz == 5) rad_cyl *= sin(pol);
  for (int l = 0; l < loop; l++) {
    int lim = ARR;
    if (l == loop - 1) lim = (jmax % REAL) + 2 * NPAD;
    for (int i = 0; i < ARR; i++) B->act[i] = ((i - NPAD) + REAL * l < jmax + NPAD);
    FOR_ACT(i) {
      int jref = (i - NPAD) + REAL * l;
      int j0 = wrap1(jref, jmax);
      int j = wrap1(j0 - c->rot_j, jmax);
      jj[i] = j;
      B->rad[i] = rad_cyl;
      B->pol[i] = pol;
      B->azi[i] = c->yc[j0];
      B->xa0[i] = c->y[j0];
      B->dx0[i] = c->dy[j0];
      B->dvol0[i] = c->yvol[j0];
      if (jref < 0) { B->xa0[i] -= k_twopi; B->azi[i] -= k_twopi; }
      if (jref >= jmax) { B->xa0[i] += k_twopi; B->azi[i] += k_twopi; }
      if (G.ngeomy > 2) B->dvol0[i] *= rad_cyl;
      if (l > 0 && i < NPAD) {
        B->r[i] = B->lt[0][i]; B->p[i] = B->lt[1][i]; B->u[i] = B->lt[2][i];
        B->v[i] = B->lt[3][i]; B->w[i] = B->lt[4][i];
      } else if (l == loop - 1 && i >= lim - NPAD) {
        int s = i - lim + NPAD;
        B->r[i] = B->rg[0][s]; B->p[i] = B->rg[1][s]; B->u[i] = B->rg[2][s];
        B->v[i] = B->rg[3][s]; B->w[i] = B->rg[4][s];
      } else {
        B->r[i] = c->r[j]; B->p[i] = c->p[j];
        B->u[i] = c->v[j]; B->v[i] = c->w[j]; B->w[i] = c->u[j];
      }
    }
    FOR_ACT(i) {
      if (l == 0 && i >= NPAD && i < 2 * NPAD) {
        int s = i - NPAD;
        B->rg[0][s] = B->r[i]; B->rg[1][s] = B->p[i]; B->rg[2][s] = B->u[i];
        B->rg[3][s] = B->v[i]; B->rg[4][s] = B->w[i];
      }
      if (l < loop - 1 && i < NPAD) {
        int s = i + lim - 2 * NPAD;
        B->lt[0][i] = B->r[s]; B->lt[1][i] = B->p[s]; B->lt[2][i] = B->u[s];
        B->lt[3][i] = B->v[s]; B->lt[4][i] = B->w[s];
      }
    }
    FOR_ACT(i) B->vrot[i] = c->res_v / rad_cyl;
    ppmlr(B, lim, dt, 1, FrRot, pl);
    if (G.visc_flag == 1) {
      FOR_ACT(i) B->xa0[i] *= rad_cyl;
      visc_p(B, lim, dt, rad_cyl, B->xa0, B->r, B->w, B->u, B->v, B->dx0);
    }
    FOR_ACT(i) {
      if (i >= NPAD && i < lim - NPAD) {
        int j = jj[i];
        c->r[j] = B->r[i];
        c->p[j] = store_p(B->r[i], get_cs2(rad_cyl));
        c->u[j] = B->w[i];
        c->v[j] = B->u[i];
        c->w[j] = B->v[i];
      }
    }
  }
}

/* theta sweep (no reference kernel: bundle_sweep3D is called at main.cu:376
 * but never defined).  Modelled on sweepx: one block per (ring i, column j0)
 * walking k, fixed ghost layers udr below k=0 (init.cpp:415-476) and a
 * reflecting midplane above k=kmax-1 (boundary.cu:412-418: mirror, w
 * negated).  Sweep-direction velocity u <- v_theta, v <- v_r, w <- r sin(theta)
 * v_phi, so get_fz's w^2 cos/(r sin)^3 term is the phi centrifugal force.   */
static void sweepz_block(orc_run *R, oblk *B, int i_rad, int j0, double dt, const obody *pl, double FrRot) {
  const int iblk = R->nr, jmax = R->nphi, kmax = R->nk;
  const int loop = (kmax / REAL) + (kmax % REAL != 0);
  oring *cur[ARR];
  int jj[ARR], mir[ARR];
  double radc[ARR];
  blk_poison(B);
  for (int l = 0; l < loop; l++) {
    int lim = ARR;
    if (l == loop - 1) lim = (kmax % REAL) + 2 * NPAD;
    for (int i = 0; i < ARR; i++) {
      int k_ring = (i - NPAD) + REAL * l;
      B->act[i] = (k_ring < kmax + NPAD);
      mir[i] = 0;
      if (!B->act[i]) continue;
      if (k_ring < 0) cur[i] = &R->udr[(k_ring + NPAD) + NPAD * i_rad];
      else if (k_ring >= kmax) {
        if (G.ntop == 0) { cur[i] = &R->rings[i_rad + iblk * (2 * kmax - 1 - k_ring)]; mir[i] = 1; }
        else cur[i] = &R->top[(k_ring - kmax) + NPAD * i_rad];
      } else cur[i] = &R->rings[i_rad + iblk * k_ring];
    }
    FOR_ACT(i) {
      oring *c = cur[i];
      int j = wrap1(j0 - c->rot_j, jmax);
      jj[i] = j;
      int k_ring = (i - NPAD) + REAL * l;
      double rad = c->xc;
      double zc = c->zc, za = c->z, dz = c->dz, zvol = c->zvol;
      if (mir[i]) {
        /* mirror layer: the state of layer 2 kmax - 1 - k, the geometry of
         * the fixed upper ring at this k (init.cpp:485-488) */
        const oring *tg = &R->top[(k_ring - kmax) + NPAD * i_rad];
        za = tg->z; dz = tg->dz; zc = tg->zc; zvol = tg->zvol;
      }
      (void)k_ring;
      B->rad[i] = rad;
      B->azi[i] = c->yc[j0];
      B->pol[i] = zc;
      double rad_cyl = rad * sin(zc);
      radc[i] = rad_cyl;
      B->xa0[i] = za;
      B->dx0[i] = dz;
      B->dvol0[i] = zvol * rad;
      if (l > 0 && i < NPAD) {
        B->r[i] = B->lt[0][i]; B->p[i] = B->lt[1][i]; B->u[i] = B->lt[2][i];
        B->v[i] = B->lt[3][i]; B->w[i] = B->lt[4][i];
      } else {
        double wz = c->w[j];
        if (mir[i]) wz = -wz;
        B->r[i] = c->r[j];
        B->p[i] = c->p[j];
        B->u[i] = wz;
        B->v[i] = c->u[j];
        B->w[i] = c->v[j] * rad_cyl;
      }
    }
    FOR_ACT(i) {
      if (l < loop - 1 && i < NPAD) {
        int s = i + lim - 2 * NPAD;
        B->lt[0][i] = B->r[s]; B->lt[1][i] = B->p[s]; B->lt[2][i] = B->u[s];
        B->lt[3][i] = B->v[s]; B->lt[4][i] = B->w[s];
      }
    }
    FOR_ACT(i) B->vrot[i] = cur[i]->res_v / radc[i];
    ppmlr(B, lim, dt, 2, FrRot, pl);
    if (G.visc_flag == 1) {
      /* arc-length faces; nu*rho scratch in dx0 as the other sweeps do */
      double xs[A1];
      FOR_ACT(i) xs[i] = B->xa0[i] * B->rad[i];
      double Rv[ARR];
      FOR_ACT(i) Rv[i] = radc[i];
      /* z viscosity: sweep velocity (u) gets 2 nu d2 + 2 nu' d1, the others
       * nu d2 + nu' d1 (device_viscosity_p's pattern; viscosity.cu:474-518
       * is the reference's unused z routine) */
      FOR_ACT(i) {
        if (i < lim) {
          B->vrho[i] = B->r[i];
          B->vnr[i] = get_nu(Rv[i]) * B->vrho[i];
          B->dx0[i] = B->vnr[i];
        }
      }
      FOR_ACT(i) {
        if (i >= NPAD && i < lim - NPAD) {
          double nr = B->vnr[i], rho = B->vrho[i], d1, d2, dn;
          derivs(&dn, &d2, i, xs, B->dx0);
          derivs(&d1, &d2, i, xs, B->u);
          B->ddu[i] = B->u[i] + dt * (2.0 * nr * d2 + 2.0 * dn * d1) / rho;
          derivs(&d1, &d2, i, xs, B->v);
          B->ddv[i] = B->v[i] + dt * (nr * d2 + dn * d1) / rho;
        }
      }
      FOR_ACT(i) {
        if (i >= NPAD && i < lim - NPAD) { B->u[i] = B->ddu[i]; B->v[i] = B->ddv[i]; }
      }
    }
    FOR_ACT(i) {
      if (i >= NPAD && i < lim - NPAD) {
        oring *c = cur[i];
        int j = jj[i];
        c->r[j] = B->r[i];
        c->p[j] = store_p(B->r[i], get_cs2(radc[i]));
        c->w[j] = B->u[i];
        c->u[j] = B->v[i];
        c->v[j] = B->w[i] / radc[i];
      }
    }
  }
}

static oblk *blk_alloc(void) { return (oblk *)malloc(sizeof(oblk)); }

void orc_sweepx(orc_run *R, double dt, const pg_body *pl, double frrot) {
  set_globals(&R->P);
  obody o = to_obody(pl);
  int nblk = R->nphi * R->nk;
#pragma omp parallel
  {
    oblk *B = blk_alloc();
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < nblk; b++) sweepx_block(R, B, b % R->nphi, b / R->nphi, dt, &o, frrot);
    free(B);
  }
}

void orc_sweepy(orc_run *R, double dt, const pg_body *pl, double frrot) {
  set_globals(&R->P);
  obody o = to_obody(pl);
#pragma omp parallel
  {
    oblk *B = blk_alloc();
#pragma omp for schedule(dynamic, 2)
    for (int n = 0; n < R->nring; n++) sweepy_block(R, B, n, dt, &o, frrot);
    free(B);
  }
}

void orc_sweepz(orc_run *R, double dt, const pg_body *pl, double frrot) {
  set_globals(&R->P);
  obody o = to_obody(pl);
  int nblk = R->nr * R->nphi;
  /* blocks of one ring i mirror-read layers that other blocks of the same
   * (i, j0) column only write in this block, so columns are independent */
#pragma omp parallel
  {
    oblk *B = blk_alloc();
#pragma omp for schedule(dynamic, 8)
    for (int b = 0; b < nblk; b++) sweepz_block(R, B, b % R->nr, b / R->nr, dt, &o, frrot);
    free(B);
  }
}

/* rotate_rings ppm.cu:309-322 */
void orc_rotate(orc_run *R) {
  for (int n = 0; n < R->nring; n++) {
    int j = R->rings[n].rot_j + R->rings[n].inc_j;
    R->rings[n].rot_j = wrap1(j, R->nphi);
  }
}

/* bundle_sweep2D ppm.cu:358-386 */
void orc_sweep2d(orc_run *R, double dt, const pg_body *pl, double frrot) {
  orc_sweepx(R, dt, pl, frrot);
  orc_sweepy(R, dt, pl, frrot);
  if (R->P.FARGO_flag > 0) orc_rotate(R);
}

void orc_sweep3d(orc_run *R, double dt, const pg_body *pl, double frrot) {
  orc_sweepx(R, dt, pl, frrot);
  orc_sweepy(R, dt, pl, frrot);
  orc_sweepz(R, dt, pl, frrot);
  if (R->P.FARGO_flag > 0) orc_rotate(R);
}

/* Index_Shift orbital_advection.cu:12-43 */
void orc_index_shift(orc_run *R, double dt, double FrRot) {
  set_globals(&R->P);
  for (int n = 0; n < R->nring; n++) {
    oring *c = &R->rings[n];
    double widthy = c->xc * c->dy[0] / dt;
    double rot_v;
    if (G.FARGO_flag == 1) {
      int idx = (int)(c->i + (double)R->nr * c->k);
      rot_v = R->val[idx].v - FrRot * c->xc;
    } else if (G.FARGO_flag == 2) rot_v = (1.0 - FrRot) * c->xc;
    else rot_v = 0.0;
    double jp = c->rot_v / widthy;
    if (jp >= 0.0) { c->inc_j = (int)(jp + 0.5); c->res_v = floor(jp + 0.5) * widthy; }
    else { c->inc_j = (int)(jp - 0.5); c->res_v = floor(jp + 0.5) * widthy; }
    c->rot_v = rot_v;
  }
}

/* dt_lv1 / dt_lv2 / dt_lv3 + get_dt, timestep.cu:12-149.  The block trees
 * of max are order independent, so a running max gives the same value.   */
double orc_get_dt(orc_run *R, double dt, double FrRot) {
  set_globals(&R->P);
  double gmax = 0.0;
  for (int n = 0; n < R->nring; n++) {
    oring *c = &R->rings[n];
    double val = 0.0;
    for (int j = 0; j < R->nphi; j++) {
      double widthz = c->dz, widthy = c->dy[j], widthx = c->dx, rad = c->xc, rad_cyl = rad;
      if (G.ngeomz == 5) rad_cyl *= sin(c->zc);
      if (G.ngeomy > 2) widthy *= rad_cyl;
      if (G.ngeomz > 2) widthz *= rad;
      double cs = sqrt(G.gam * c->p[j] / c->r[j]);
      double t0 = (fabs(c->u[j]) + cs) / widthx;
      double t1 = (fabs(c->v[j] - c->rot_v - FrRot * rad_cyl) + cs) / widthy;
      double rt;
      if (G.ndim == 3) { double t2 = (fabs(c->w[j]) + cs) / widthz; rt = max3(t0, t1, t2); }
      else rt = cmax(t0, t1);
      if (val < rt) val = rt;
    }
    if (gmax < val) gmax = val;
  }
  double hdt = G.courant / gmax;
  dt = 1.1 * dt;
  if (hdt < dt) dt = hdt;
  return dt;
}

/* bin_reduc_sum reduction.cu:123-142 on a 1024 list */
static double tree1024(double *list) {
  for (int len = 1024; len > 1; len /= 2) {
    int half = len / 2;
    for (int n = 0; n < half; n++) list[n] += list[n + half];
  }
  return list[0];
}

/* output_lv1/lv2/lv3 + GPU_output_reduction, device_func.cu:49-198 */
double orc_reduce(orc_run *R, const pg_body *plb, double exclude, int mode) {
  set_globals(&R->P);
  obody pl = to_obody(plb);
  exclude *= G.sc_h;
  int iblk = R->nr, kblk = R->nk, jmax = R->nphi;
  double *d2 = (double *)calloc((size_t)iblk * kblk, sizeof(double));
  double list[1024];
  for (int k = 0; k < kblk; k++)
    for (int i = 0; i < iblk; i++) {
      oring *c = &R->rings[i + iblk * k];
      int loop = jmax / 1024 + (jmax % 1024 != 0);
      double val = 0.0;
      for (int l = 0; l < loop; l++) {
        for (int tt = 0; tt < 1024; tt++) {
          int j = tt + 1024 * l;
          double v = 0.0;
          if (j < jmax) {
            int j0 = wrap1(j + c->rot_j, jmax);
            double rad = c->xc, phi = c->yc[j0];
            if (G.plnt_flag > 0) {
              if (mode == 0) v = c->r[j] * c->xvol * c->yvol[j0] * c->zvol;
              else if (G.ndim == 2 && (mode == 8 || mode == 9)) {
                if ((rad - pl.x) * (rad - pl.x) + rad * rad * (phi - pl.y) * (phi - pl.y) > exclude * exclude) {
                  if (mode == 8) {
                    double t = -grav_rad_cyl(rad, phi, 0.0, &pl, 0.0);
                    t *= (c->r[j] - pow(c->xc, -G.p_alpha)) * c->xvol * c->yvol[j0];
                    v = t;
                  } else {
                    double t = -grav_azi_cyl(rad, phi, 0.0, &pl, 0.0);
                    t *= rad * (c->r[j] - pow(c->xc, -G.p_alpha)) * c->xvol * c->yvol[j0];
                    v = t;
                  }
                }
              }
            } else v = c->r[j] * c->xvol * c->yvol[j0] * c->zvol;
          }
          list[tt] = v;
        }
        val += tree1024(list);
      }
      d2[i + iblk * k] = val;
    }
  double *d1 = d2;
  double *tmp1d = NULL;
  if (G.ndim == 3) {
    /* output_lv2: round_reduc_sum over k (reduction.cu:77-100) */
    tmp1d = (double *)calloc(iblk, sizeof(double));
    double *rl = (double *)malloc(sizeof(double) * kblk);
    for (int i = 0; i < iblk; i++) {
      for (int k = 0; k < kblk; k++) rl[k] = d2[i + iblk * k];
      int len2 = 1; while (len2 < kblk) len2 *= 2;
      while (len2 > 1) {
        int half = len2 / 2;
        for (int n = 0; n < half; n++) if (n + half < kblk) rl[n] += rl[n + half];
        len2 = half;
      }
      tmp1d[i] = rl[0];
    }
    free(rl);
    d1 = tmp1d;
  }
  double out;
  if (iblk <= 1024) {
    for (int i = 0; i < 1024; i++) list[i] = (i < iblk) ? d1[i] : 0.0;
    out = tree1024(list);
  } else {
    out = 0.0;  /* output_lv3 supports iblk <= 1024 only (device_func.cu:158) */
    for (int i = 0; i < iblk; i++) out += d1[i];
  }
  free(d2);
  free(tmp1d);
  return 0.0 + out;
}

/* ------------------------------------------------------------------------ */
/* planet (planet.cu:11-93)                                                 */

static double set_M_p(double t) {                                   /* 28-34 */
  if (t < G.t_growth) return fmax(G.M_p * sin(k_pi * t / (2.0 * G.t_growth)), 0.01 * k_earth);
  return G.M_p;
}

double orc_set_M_p(const pg_params *p, double t) {
  set_globals(p);
  return set_M_p(t);
}

void orc_init_planet(const pg_params *p, pg_body *pl, double *FrRot) { /* 36-52 */
  set_globals(p);
  pl->m = set_M_p(0.0);
  pl->x = G.R_p;
  pl->y = k_pi;
  pl->vx = 0.0;
  pl->vy = pow(pl->x, -1.5);
  if (G.FrRot_flag == 1) *FrRot = pl->vy;
  else *FrRot = 0.0;
  pl->vy -= *FrRot;
  pl->rs = G.rs_fac * get_h(pl->x);
  pl->fx = pl->fy = 0.0;
}

void orc_planet_forces(orc_run *R, pg_body *pl, double FrRot, double simtime) { /* 54-65 */
  set_globals(&R->P);
  pl->m = set_M_p(simtime);
  if (G.plnt_flag == 2) {
    double f8 = orc_reduce(R, pl, 0.0, 8);
    set_globals(&R->P);
    pl->fx = G.Sigma_0 * f8 / pl->m - 1.0 / pl->x / pl->x + pl->x * hpow(pl->vy + FrRot, 2.0);
    double f9 = orc_reduce(R, pl, 0.0, 9);
    set_globals(&R->P);
    pl->fy = G.Sigma_0 * f9 / pl->m;
  } else {
    pl->fx = -1.0 / pl->x / pl->x + pl->x * hpow(pl->vy + FrRot, 2.0);
    pl->fy = 0.0;
  }
}

void orc_kick_drift_kick(const pg_params *p, pg_body *pl, double *FrRot, double dt, int kick) { /* 67-93 */
  set_globals(p);
  if (!kick) {
    double old_rad = pl->x;
    pl->x += dt * pl->vx;
    pl->y += dt * pl->vy;
    pl->vy = ((pl->vy + *FrRot) * old_rad * old_rad / pl->x / pl->x) - *FrRot;
    if (pl->y < 0.0) pl->y += k_twopi;
    if (pl->y >= k_twopi) pl->y -= k_twopi;
    pl->rs = G.rs_fac * get_h(pl->x);
  } else {
    pl->vx += dt * pl->fx;
    pl->vy += *FrRot + dt * pl->fy / pl->x / pl->x;
    if (G.FrRot_flag == 1) *FrRot = pl->vy;
    else *FrRot = 0.0;
    pl->vy -= *FrRot;
  }
}

static double get_L(const pg_body *p, double FrRot) { double vy = p->vy + FrRot; return vy * p->x * p->x; }
double orc_get_E(const pg_body *p, double FrRot) {
  double vy = p->vy + FrRot;
  return (p->vx * p->vx + vy * vy * p->x * p->x) / 2.0 - 1.0 / p->x;
}
double orc_get_ecc(const pg_body *p, double FrRot) {
  return sqrt(1.0 + (2.0 * orc_get_E(p, FrRot) * get_L(p, FrRot) * get_L(p, FrRot)));
}

/* ------------------------------------------------------------------------ */
/* restart set-up: copy_grid + init_den + init_speed + init_bound           */

static void ring_bind(oring *c, double *base, int jmax) {
  c->r = base; c->p = base + jmax; c->u = base + 2 * jmax; c->v = base + 3 * jmax; c->w = base + 4 * jmax;
  c->y = base + 5 * jmax; c->dy = base + 6 * jmax; c->yvol = base + 7 * jmax; c->yc = base + 8 * jmax;
}

static double get_vol(double xa, double dx, int axis) {               /* grid.cu:225-248 */
  double vol = 0.0;
  if (axis == 0) {
    if (G.ngeomx == 0) vol = dx;
    else if (G.ngeomx == 1) vol = dx * (xa + 0.5 * dx);
    else if (G.ngeomx == 2) vol = dx * (xa * (xa + dx) + dx * dx * k_third);
  } else if (axis == 1) vol = dx;
  else {
    if (G.ndim == 2) vol = 1.0;
    else if (G.ngeomz == 0) vol = dx;
    else if (G.ngeomz == 5) vol = cos(xa) - cos(xa + dx);
  }
  return vol;
}

/* one fixed ghost ring (init.cpp:259-413 radial, 415-539 theta) */
static void ghost_fill(oring *g, int jmax, const double *zya, const double *zdy, const double *zyc,
                       double r, double z, double rr, int sph_pol, double zc) {
  double rho, P, dP, vk;
  if (G.ndim == 2) {
    rho = get_rho1(r); P = get_P1(r); dP = get_dP_dr1(r); vk = 1.0 / r;
  } else {
    rho = get_rho2(r, z); P = get_P2(r, z);
    dP = sph_pol ? get_dP_s(rr, zc) : 0.0;
    vk = 1.0 / rr;
  }
  vk += rr * dP / rho;
  vk = sqrt(vk);
  double vr = get_viscous_vr(r);
  for (int j = 0; j < jmax; j++) {
    g->r[j] = rho; g->p[j] = P; g->u[j] = vr; g->v[j] = vk; g->w[j] = 0.0;
    g->y[j] = zya[j]; g->dy[j] = zdy[j]; g->yc[j] = zyc[j]; g->yvol[j] = get_vol(zya[j], zdy[j], 1);
  }
  if (G.FARGO_flag == 1) g->rot_v = vk - 1.0 * g->xc;
  else g->rot_v = 0.0;
  g->rot_j = 0; g->inc_j = 0; g->res_v = 0.0;
}

#define OFF_D(f) ((size_t)(f))
static size_t rb(int jmax) { return (size_t)72 * jmax + 96; }

orc_run *orc_create(const pg_params *p, const void *buf, size_t bytes) {
  set_globals(p);
  int nr = p->imax, nphi = p->jmax, nk = p->kmax;
  int nring = nr * nk;
  if (bytes != rb(nphi) * (size_t)nring) return NULL;
  orc_run *R = (orc_run *)calloc(1, sizeof(orc_run));
  R->P = *p; R->nr = nr; R->nphi = nphi; R->nk = nk; R->nring = nring;
  int nghost = 2 * NPAD * nk + (nk > 1 ? 2 * NPAD * nr : 0);
  size_t per = (size_t)9 * nphi;
  R->mem = (double *)malloc(sizeof(double) * per * (size_t)(nring + nghost));
  R->rings = (oring *)calloc(nring, sizeof(oring));
  R->lft = (oring *)calloc(NPAD * nk, sizeof(oring));
  R->rgh = (oring *)calloc(NPAD * nk, sizeof(oring));
  if (nk > 1) {
    R->udr = (oring *)calloc((size_t)NPAD * nr, sizeof(oring));
    R->top = (oring *)calloc((size_t)NPAD * nr, sizeof(oring));
  }
  double *m = R->mem;
  const unsigned char *src = (const unsigned char *)buf;
  for (int n = 0; n < nring; n++, m += per) {
    oring *c = &R->rings[n];
    const unsigned char *b = src + rb(nphi) * n;
    ring_bind(c, m, nphi);
    memcpy(c->r, b, sizeof(double) * 5 * nphi);
    const unsigned char *t = b + 40 * (size_t)nphi;
    memcpy(&c->x, t, 8); memcpy(&c->dx, t + 8, 8); memcpy(&c->xvol, t + 16, 8); memcpy(&c->xc, t + 24, 8);
    memcpy(c->y, t + 32, sizeof(double) * 4 * nphi);
    t = b + 72 * (size_t)nphi + 32;
    memcpy(&c->z, t, 8); memcpy(&c->dz, t + 8, 8); memcpy(&c->zvol, t + 16, 8); memcpy(&c->zc, t + 24, 8);
    memcpy(&c->i, t + 32, 4); memcpy(&c->k, t + 36, 4);
    memcpy(&c->rot_v, t + 40, 8); memcpy(&c->res_v, t + 48, 8);
    memcpy(&c->rot_j, t + 56, 4); memcpy(&c->inc_j, t + 60, 4);
  }
  /* copy_grid init.cpp:59-90 */
  double *zxa = (double *)malloc(sizeof(double) * nr), *zxc = (double *)malloc(sizeof(double) * nr);
  double *zdx = (double *)malloc(sizeof(double) * nr);
  double *zza = (double *)malloc(sizeof(double) * nk), *zzc = (double *)malloc(sizeof(double) * nk);
  double *zdz = (double *)malloc(sizeof(double) * nk);
  for (int n = 0; n < nring; n++) {
    oring *c = &R->rings[n];
    if (c->i >= 0 && c->i < nr) { zxa[c->i] = c->x; zxc[c->i] = c->xc; zdx[c->i] = c->dx; }
    if (c->k >= 0 && c->k < nk) { zza[c->k] = c->z; zzc[c->k] = c->zc; zdz[c->k] = c->dz; }
  }
  const double *zya = R->rings[0].y, *zyc = R->rings[0].yc, *zdy = R->rings[0].dy;
  /* init_den / init_speed init.cpp:92-183 */
  R->val = (osym *)calloc(nring, sizeof(osym));
  for (int i = 0; i < nr; i++)
    for (int k = 0; k < nk; k++) {
      osym *v = &R->val[i + nr * k];
      double r, z, vk2, dP;
      if (G.ngeomz == 5) { r = zxc[i] * sin(zzc[k]); z = zxc[i] * cos(zzc[k]); }
      else { r = zxc[i]; z = zzc[k]; }
      if (G.ndim == 3) { v->r = get_rho2(r, z); v->p = get_P2(r, z); }
      else { v->r = get_rho1(r); v->p = get_P1(r); }
      if (G.ndim == 2) { r = zxc[i]; z = 0.0; vk2 = 1.0 / r; dP = get_dP_dr1(zxc[i]); }
      else { vk2 = 1.0 / zxc[i]; r = zxc[i] * sin(zzc[k]); z = zxc[i] * cos(zzc[k]); dP = get_dP_s(zxc[i], zzc[k]); }
      vk2 += zxc[i] * dP / v->r;
      v->v = sqrt(vk2);
      v->u = get_viscous_vr(r);
      v->w = 0.0;
    }
  /* init_bound init.cpp:253-413 (radial ghosts; res_v/inc_j zeroed) */
  for (int i = 0; i < NPAD; i++)
    for (int k = 0; k < nk; k++) {
      int ib = i + NPAD * k;
      oring *g = &R->lft[ib];
      ring_bind(g, m, nphi); m += per;
      g->x = zxa[0] - zdx[0] * (double)(NPAD - i);
      g->dx = zdx[0];
      g->xc = g->x + 0.5 * g->dx;
      g->xvol = get_vol(g->x, g->dx, 0);
      g->z = zza[k]; g->dz = zdz[k]; g->zc = zzc[k]; g->zvol = get_vol(zza[k], zdz[k], 2);
      double rr = g->xc, r = rr, z = 0.0;
      if (G.ndim == 3) { r = rr * sin(zzc[k]); z = rr * cos(zzc[k]); }
      ghost_fill(g, nphi, zya, zdy, zyc, r, z, rr, G.ngeomz == 5, zzc[k]);
      g = &R->rgh[ib];
      ring_bind(g, m, nphi); m += per;
      g->x = zxa[nr - 1] + zdx[nr - 1] * (double)(i + 1);
      g->dx = zdx[nr - 1];
      g->xc = g->x + 0.5 * g->dx;
      g->xvol = get_vol(g->x, g->dx, 0);
      g->z = zza[k]; g->dz = zdz[k]; g->zc = zzc[k]; g->zvol = get_vol(zza[k], zdz[k], 2);
      rr = g->xc; r = rr; z = 0.0;
      if (G.ndim == 3) { r = rr * sin(zzc[k]); z = rr * cos(zzc[k]); }
      ghost_fill(g, nphi, zya, zdy, zyc, r, z, rr, G.ngeomz == 5, zzc[k]);
    }
  if (nk > 1) {
    /* theta ghosts below k=0 (init.cpp:415-476); top ones too when fixed */
    for (int kk = 0; kk < NPAD; kk++)
      for (int i = 0; i < nr; i++) {
        int ib = kk + NPAD * i;
        oring *g = &R->udr[ib];
        ring_bind(g, m, nphi); m += per;
        g->z = zza[0] - zdz[0] * (double)(NPAD - kk);
        g->dz = zdz[0]; g->zc = g->z + 0.5 * g->dz; g->zvol = get_vol(g->z, g->dz, 2);
        g->x = zxa[i]; g->dx = zdx[i]; g->xc = zxc[i]; g->xvol = get_vol(zxa[i], zdx[i], 0);
        double rr = zxc[i], z = rr * cos(g->zc), r = sqrt(rr * rr - z * z);
        ghost_fill(g, nphi, zya, zdy, zyc, r, z, rr, 1, g->zc);
        g = &R->top[ib];
        ring_bind(g, m, nphi); m += per;
        g->z = zza[nk - 1] + zdz[nk - 1] * (double)(kk + 1);
        g->dz = zdz[nk - 1]; g->zc = g->z + 0.5 * g->dz; g->zvol = get_vol(g->z, g->dz, 2);
        g->x = zxa[i]; g->dx = zdx[i]; g->xc = zxc[i]; g->xvol = get_vol(zxa[i], zdx[i], 0);
        rr = zxc[i]; z = rr * cos(g->zc); r = sqrt(rr * rr - z * z);
        ghost_fill(g, nphi, zya, zdy, zyc, r, z, rr, 1, g->zc);
      }
  }
  free(zxa); free(zxc); free(zdx); free(zza); free(zzc); free(zdz);
  return R;
}

/* The fixed ghost rings (lft, rgh, then udr, top in 3D), one row of
 * x dx xvol xc z dz zvol zc r p u v w rot_v per ring, in the oracle's own
 * storage order.  count receives the number of rings; out may be NULL.    */
int orc_boundary(const orc_run *R, double *out, size_t n_doubles, int *count) {
  int ng = NPAD * R->nk, nt = (R->nk > 1) ? NPAD * R->nr : 0;
  int n = 2 * ng + 2 * nt;
  *count = n;
  if (!out) return 0;
  if (n_doubles < (size_t)n * 14) return -1;
  const oring *grp[4] = {R->lft, R->rgh, R->udr, R->top};
  int len[4] = {ng, ng, nt, nt};
  double *o = out;
  for (int g = 0; g < 4; g++)
    for (int b = 0; b < len[g]; b++) {
      const oring *c = &grp[g][b];
      double row[14] = {c->x, c->dx, c->xvol, c->xc, c->z, c->dz, c->zvol, c->zc,
                        c->r[0], c->p[0], c->u[0], c->v[0], c->w[0], c->rot_v};
      memcpy(o, row, sizeof row);
      o += 14;
    }
  return 0;
}

/* The axisymmetric profile the damping relaxes toward (r p u v w per
 * ring, ring i + imax k).                                                 */
int orc_targets(const orc_run *R, double *out, size_t n_doubles) {
  size_t n = (size_t)R->nr * R->nk;
  if (n_doubles < n * 5) return -1;
  for (size_t q = 0; q < n; q++) {
    const osym *v = &R->val[q];
    out[5 * q] = v->r; out[5 * q + 1] = v->p; out[5 * q + 2] = v->u;
    out[5 * q + 3] = v->v; out[5 * q + 4] = v->w;
  }
  return 0;
}

void orc_destroy(orc_run *R) {
  if (!R) return;
  free(R->mem); free(R->rings); free(R->lft); free(R->rgh); free(R->udr); free(R->top); free(R->val);
  free(R);
}

int orc_save(const orc_run *R, void *buf, size_t bytes) {
  int nphi = R->nphi;
  if (bytes != rb(nphi) * (size_t)R->nring) return PG_ERR_ARG;
  unsigned char *dst = (unsigned char *)buf;
  memset(dst, 0, bytes);
  for (int n = 0; n < R->nring; n++) {
    const oring *c = &R->rings[n];
    unsigned char *b = dst + rb(nphi) * n;
    memcpy(b, c->r, sizeof(double) * 5 * nphi);
    unsigned char *t = b + 40 * (size_t)nphi;
    memcpy(t, &c->x, 8); memcpy(t + 8, &c->dx, 8); memcpy(t + 16, &c->xvol, 8); memcpy(t + 24, &c->xc, 8);
    memcpy(t + 32, c->y, sizeof(double) * 4 * nphi);
    t = b + 72 * (size_t)nphi + 32;
    memcpy(t, &c->z, 8); memcpy(t + 8, &c->dz, 8); memcpy(t + 16, &c->zvol, 8); memcpy(t + 24, &c->zc, 8);
    memcpy(t + 32, &c->i, 4); memcpy(t + 36, &c->k, 4);
    memcpy(t + 40, &c->rot_v, 8); memcpy(t + 48, &c->res_v, 8);
    memcpy(t + 56, &c->rot_j, 4); memcpy(t + 60, &c->inc_j, 4);
  }
  return PG_OK;
}

/* ------------------------------------------------------------------------ */
/* wave damping: kill_wave.cu:19-40 restated for zones r < kill_rin and
 * r > kill_rout, relaxing toward the axisymmetric profile; p re-derived by
 * the sweep store's relation (Sigma cs2, or cs2 Sigma^gam / gam in EOS 1). */
void orc_damp(orc_run *R, double dt) {
  set_globals(&R->P);
  if (!(G.kill_rin > 0.0) && !(G.kill_rout > 0.0)) return;
  for (int n = 0; n < R->nring; n++) {
    oring *c = &R->rings[n];
    double r = c->xc, f;
    if (G.kill_rin > 0.0 && r < G.kill_rin) f = (G.kill_rin - r) / (G.kill_rin - G.xmin);
    else if (G.kill_rout > 0.0 && r > G.kill_rout) f = (r - G.kill_rout) / (G.xmax - G.kill_rout);
    else continue;
    f *= dt * pow(r, -1.5);
    const osym *v0 = &R->val[c->i + R->nr * c->k];
    double rad_cyl = r;
    if (G.ngeomz == 5) rad_cyl *= sin(c->zc);
    double cs2 = get_cs2(rad_cyl);
    for (int j = 0; j < R->nphi; j++) {
      c->r[j] += f * (v0->r - c->r[j]);
      c->u[j] += f * (v0->u - c->u[j]);
      c->v[j] += f * (v0->v - c->v[j]);
      c->w[j] += f * (-c->w[j]);
      c->p[j] = store_p(c->r[j], cs2);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* restart-path main loop, main.cu:270-441                                  */
int orc_run_steps(orc_run *R, int nsteps, int startat, double *hist) {
  set_globals(&R->P);
  pg_params P = R->P;
  double dt = P.endtime;
  double simtime = P.tmovie * (double)startat, timem = 0.0, old_dt = 0.0;
  int ncycle = 0;
  pg_body pl;
  double FrRot;
  orc_init_planet(&P, &pl, &FrRot);
  orc_planet_forces(R, &pl, FrRot, simtime);
  int make_pict = 0, cont = 1, s;
  for (s = 0; s < nsteps && cont; s++) {
    dt = orc_get_dt(R, dt, FrRot);
    if (ncycle == P.ncycend) cont = 0;
    if (simtime + dt >= P.endtime) { old_dt = dt; dt = P.endtime - simtime; make_pict = 1; cont = 0; }
    if (timem + dt >= P.tmovie) { old_dt = dt; dt = P.tmovie - timem; make_pict = 1; }
    double dt_used = dt;
    orc_index_shift(R, dt, FrRot);
    if (P.plnt_flag > 0) orc_kick_drift_kick(&P, &pl, &FrRot, 0.5 * dt, 1);
    if (P.ndim == 2) orc_sweep2d(R, dt, &pl, FrRot);
    else orc_sweep3d(R, dt, &pl, FrRot);
    orc_damp(R, dt);
    simtime += dt; timem += dt; ncycle++;
    if (P.plnt_flag > 0) {
      orc_kick_drift_kick(&P, &pl, &FrRot, dt, 0);
      orc_planet_forces(R, &pl, FrRot, simtime);
      orc_kick_drift_kick(&P, &pl, &FrRot, 0.5 * dt, 1);
    }
    if (make_pict) { timem = 0.0; make_pict = 0; dt = old_dt; }
    if (hist) {
      double *h = hist + 4 * (size_t)s;
      h[0] = simtime;
      h[1] = dt_used;
      h[2] = orc_reduce(R, &pl, 0.0, 0);
      set_globals(&R->P);
      double norm = P.M_p * P.M_p * hpow(P.R_p, 1.0 - P.p_alpha + (P.p_beta - 1.0)) / (P.sc_h * P.sc_h);
      h[3] = (P.plnt_flag > 0 && P.ndim == 2) ? orc_reduce(R, &pl, 0.0, 9) / norm : 0.0;
    }
    set_globals(&R->P);
  }
  return s;
}

int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
