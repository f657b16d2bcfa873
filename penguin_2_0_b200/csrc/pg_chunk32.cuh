// pg_chunk32.cuh -- the ppmlr chain in FP32 (the run's precision = 1).
//
// Same phases, index ranges and formulas as ppm_chunk (pg_chunk.cuh), with
// these changes that keep FP32 accurate on a Keplerian disk:
//  * Sigma is stored as the residual dS = Sigma - S_bg(ring) from the ring's
//    initial-state density, and the kernels carry Sigma in FP64 per cell
//    (CellIn32::sig): mass m = Sigma dvol and m + f_in - f_out are FP64 with
//    FP32 fluxes, so a per-step change far below Sigma's FP32 spacing (the
//    slow viscous evolution of the disk: ~4e-8 of Sigma per step) is kept
//    instead of being rounded away every step;
//  * azimuthal velocities are residuals dv = v_phi - v_bg(ring): the
//    azimuthal sweep is exactly invariant under a per-ring shift of the
//    velocity (PPM limiters and the isothermal Riemann solver only see
//    differences), and the FARGO residual angular velocity
//    v_bg/r - v_rot - FrRot is an FP64 per-ring constant;
//  * the radial and polar sweeps carry the angular momentum
//    L = r_cyl (v_bg + dv) in FP64 (slot L, its remap uses FP64 masses so
//    that m_new = m + flux_in - flux_out is consistent to rounding); FP32
//    would round L to 6e-8 of v_K, far above the disk's perturbations;
//  * Lagrangian face positions are kept as displacements delx from the
//    Eulerian faces (widths dx = dx0 + delx[n+1] - delx[n]), so FP32 does not
//    lose the small face motions against face coordinates of order 1;
//  * mass moves in FP64: displacements, Lagrangian widths and volumes, the
//    remap's interface coefficients, the density parabola and the swept
//    masses.  In a steady flow (the gas bound to a planet) the same large
//    fluxes cross the same faces every step, and FP32 rounding of them would
//    repeat and add up step after step;
//  * forces, geometry factors and positions are evaluated in FP64 from the
//    FP64 face coordinate of each cell.
#pragma once
#include "pg_chunk.cuh"

namespace pgd {

constexpr float kSmallpF = 1.0e-15f;
constexpr float kSmallrF = 1.0e-15f;
constexpr float kFourthdF = 1.3333333333333333f;

template <int NT>
struct ChunkShm32Data {
  float r[NT + 2], p[NT + 2], u[NT + 2], v[NT + 2], w[NT + 2], dx0[NT + 2];
  float q[NT + 2], dx[NT + 2], umid[NT + 2], pmid[NT + 2], tmp1[NT + 2], dl[NT + 2];
  float s0[NT + 2], s1[NT + 2], s2[NT + 2], s3[NT + 2], s4[NT + 2], s5[NT + 2];   // side-by-side parabolas
  double L[NT + 2], Lal[NT + 2], Lda[NT + 2], La6[NT + 2], Lflux[NT + 2], xa0[NT + 2];
  double Rd[NT + 2], dld[NT + 2];   // FP64 Lagrangian density and face displacements
  double cf0;   // cos(phi - phi_planet) at the start of the step (radial, polar pencils)
};
// padded to TO mod 128 bytes: conflict-free banks for 128 / TO packed
// pencils (32: four, 64: two)
template <int NT, int TO = 32>
struct ChunkShm32 : ChunkShm32Data<NT> {
  char pad_[shm_pad_to((int)sizeof(ChunkShm32Data<NT>), TO)];
};

struct CellIn32 {
  double rad, azi, pol, vrot, dvol0;
  double omres;   // azimuthal sweep: v_bg / r_cyl - v_rot - FrRot (FP64)
  double sig;     // this cell's Sigma in FP64 (S_bg + dS)
  double dx0;     // this cell's Eulerian width in FP64
  double sinpol;  // sin(pol) in 3D (per-layer table)
  double cospol;  // cos(pol) (polar sweep)
  double sinfz;   // sin, cos of the left face angle (polar sweep)
  double cosfz;
};

__device__ __forceinline__ float min3f(float A, float B, float C) {
  if (A < B) { if (C < A) return C; else return A; }
  else       { if (C < B) return C; else return B; }
}
__device__ __forceinline__ float max3f(float A, float B, float C) {
  if (A > B) { if (C > A) return C; else return A; }
  else       { if (C > B) return C; else return B; }
}

struct ParF { float c0, c1, c2, c3, c4; };

__device__ __forceinline__ void paraset32(int n, int nmin, int nmax, ParF &par, const float *dx, float *a,
                                          float *ai, float *b) {
  float dx_n = 0.f, ain = 0.f, bi = 0.f, ci = 0.f, c = 0.f;
  if (n >= nmin && n < nmax - 1) {
    dx_n = dx[n];
    float an = dx_n + dx[n + 1];
    ain = 1.0f / an;
    float bn = an + dx_n;
    bi = 1.0f / bn;
    c = an + dx[n + 1];
    ci = 1.0f / c;
    a[n] = an; ai[n] = ain; b[n] = bn;
  }
  __syncthreads();
  if (n >= nmin + 1 && n < nmax - 2) {
    float d = 1.0f / (a[n - 1] + a[n + 1]);
    par.c0 = dx_n * ain * (1.0f + 2.0f * d * dx[n + 1] * (a[n - 1] * bi - a[n + 1] * ci));
    par.c1 = -d * dx_n * a[n - 1] * bi;
    par.c2 = d * dx[n + 1] * a[n + 1] * ci;
  }
  if (n >= nmin + 1 && n < nmax - 1) {
    float d = dx_n / (a[n - 1] + dx[n + 1]);
    par.c3 = d * b[n - 1] * ain;
    par.c4 = d * c * ai[n - 1];
  }
  __syncthreads();
}

// parabola on values of type T (float, or double for the L slot) with FP32
// coefficients
template <typename T>
__device__ __forceinline__ void parabola32(int n, int nmin, int nmax, float flat, const T *val, T *al, T *da,
                                           T *a6, const ParF &par) {
  T t1 = 0, a = 0, ar = 0, da_r = 0;
  if (n >= nmin + 1 && n < nmax - 1) {
    a = val[n];
    da_r = val[n + 1] - a;
    T da_l = a - val[n - 1];
    t1 = (T)par.c3 * da_r + (T)par.c4 * da_l;
    T two = 2;
    T m1 = two * fabs(da_l), m2 = two * fabs(da_r);
    if (t1 < 0) { T x = -t1; T mn = (x < m1) ? ((m2 < x) ? m2 : x) : ((m2 < m1) ? m2 : m1); t1 = -mn; }
    else        { T x = t1;  T mn = (x < m1) ? ((m2 < x) ? m2 : x) : ((m2 < m1) ? m2 : m1); t1 = mn; }
    if (da_l * da_r < 0) t1 = 0;
    a6[n] = t1;
  }
  __syncthreads();
  if (n >= nmin + 1 && n < nmax - 2) {
    ar = a + (T)par.c0 * da_r + (T)par.c1 * a6[n + 1] + (T)par.c2 * t1;
    al[n + 1] = ar;
  }
  __syncthreads();
  if (n >= nmin + 2 && n < nmax - 2) {
    T f = (T)flat;
    T u1 = f * a;
    T u2 = (T)1 - f;
    T xr = u1 + u2 * ar;
    T la = u1 + u2 * al[n];
    u1 = xr - la;
    u2 = u1 * u1;
    T half = (T)0.5, six = (T)6, three = (T)3, two = (T)2;
    u1 = u1 * (six * (a - half * (xr + la)));
    if ((xr - a) * (a - la) <= 0) { xr = a; la = a; }
    if (u2 < u1) la = three * a - two * xr;
    if (u2 < -u1) xr = three * a - two * la;
    da[n] = xr - la;
    a6[n] = six * (a - half * (xr + la));
    al[n] = la;
  }
  __syncthreads();
}

// parabola32 for NF float fields at once: the same phases and, per field,
// the same arithmetic, one barrier per phase for all fields (see
// parabola_n); a field's value and its own a6 are reloaded after a barrier
template <int NF>
__device__ __forceinline__ void parabola32_n(int n, int nmin, int nmax, float flat, const float *const *val,
                                             float *const *al, float *const *da, float *const *a6,
                                             const ParF &par) {
  if (n >= nmin + 1 && n < nmax - 1) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const float a = val[f][n];
      const float da_r = val[f][n + 1] - a;
      const float da_l = a - val[f][n - 1];
      float t1 = par.c3 * da_r + par.c4 * da_l;
      const float m1 = 2.0f * fabsf(da_l), m2 = 2.0f * fabsf(da_r);
      if (t1 < 0) { float x = -t1; float mn = (x < m1) ? ((m2 < x) ? m2 : x) : ((m2 < m1) ? m2 : m1); t1 = -mn; }
      else        { float x = t1;  float mn = (x < m1) ? ((m2 < x) ? m2 : x) : ((m2 < m1) ? m2 : m1); t1 = mn; }
      if (da_l * da_r < 0) t1 = 0;
      a6[f][n] = t1;
    }
  }
  __syncthreads();
  float ar[NF];
  if (n >= nmin + 1 && n < nmax - 2) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const float a = val[f][n];
      const float da_r = val[f][n + 1] - a;
      const float t1 = a6[f][n];
      ar[f] = a + par.c0 * da_r + par.c1 * a6[f][n + 1] + par.c2 * t1;
      al[f][n + 1] = ar[f];
    }
  }
  __syncthreads();
  if (n >= nmin + 2 && n < nmax - 2) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const float a = val[f][n];
      float u1 = flat * a;
      float u2 = 1.0f - flat;
      float xr = u1 + u2 * ar[f];
      float la = u1 + u2 * al[f][n];
      u1 = xr - la;
      u2 = u1 * u1;
      u1 = u1 * (6.0f * (a - 0.5f * (xr + la)));
      if ((xr - a) * (a - la) <= 0) { xr = a; la = a; }
      if (u2 < u1) la = 3.0f * a - 2.0f * xr;
      if (u2 < -u1) xr = 3.0f * a - 2.0f * la;
      da[f][n] = xr - la;
      a6[f][n] = 6.0f * (a - 0.5f * (xr + la));
      al[f][n] = la;
    }
  }
  __syncthreads();
}

template <int AXIS, bool SPH>
__device__ __forceinline__ double face_force32(int n, double hdt, const CellIn32 &c, double xa0f,
                                               const double *Lv, const float *wv, const Body &pl,
                                               const Phys &ph) {
  // Lv: the FP64 angular-momentum slot (radial: v slot, polar: w slot);
  // wv: the other transverse FP32 slot (radial 3D: w = r v_theta)
  if (AXIS == 0) {
    double rad = xa0f;
    double azi = c.azi + hdt * c.vrot;
    double grav;
    if (!SPH) {
      if (ph.plnt) { grav = grav_rad_cyl(rad, azi, c.pol, pl, hdt); grav += -1.0 / rad / rad; }
      else { double dis = sqrt(rad * rad + c.pol * c.pol); grav = -rad / dis / dis / dis; }
      double vf = 0.5 * (Lv[n] + Lv[n - 1]);
      return grav + vf * vf / rad / rad / rad;
    } else {
      grav = ph.plnt ? grav_rad_sph_s(rad, azi, c.sinpol, pl, hdt) : -1.0 / rad / rad;
      double wf = 0.5 * ((double)wv[n] + (double)wv[n - 1]);
      double vf = 0.5 * (Lv[n] + Lv[n - 1]);
      double rs = rad * c.sinpol;
      return grav + wf * wf / rad / rad / rad + vf * vf / rad / (rs * rs);
    }
  } else if (AXIS == 1) {
    double azi = xa0f + hdt * c.vrot;
    if (!SPH) return ph.plnt ? grav_azi_cyl(c.rad, azi, c.pol, pl, hdt) : 0.0;
    return ph.plnt ? grav_azi_sph_s(c.rad, azi, c.sinpol, pl, hdt) : 0.0;
  } else {
    // the face angle xa0f is the layer's face: sin, cos from the table
    double azi = c.azi + hdt * c.vrot;
    const double sp = c.sinfz, cp = c.cosfz;
    double grav = ph.plnt ? grav_pol_sph_s(c.rad, azi, sp, cp, pl, hdt) : 0.0;
    double rc = c.rad * sp;
    double lf = 0.5 * (Lv[n] + Lv[n - 1]);
    return grav + (lf * lf * cp) / rc / rc / rc;
  }
}

// CF0: cos(azi - p.y) given as cf0 (the dt = 0 force of a radial or polar
// pencil); the polar form takes sin and cos of its angle as sp, cp.
template <int AXIS, bool SPH, bool CF0 = false>
__device__ __forceinline__ double centre_force32(int n, double dt, double rad, double azi, double pol,
                                                 double sinpol, const double *Lv, const float *wv,
                                                 const Body &pl, const Phys &ph, double cf0 = 0.0,
                                                 double sp = 0.0, double cp = 0.0) {
  if (AXIS == 0) {
    double grav;
    if (!SPH) {
      if (ph.plnt) {
        grav = CF0 ? grav_rad_cyl_cf(rad, cf0, pol, pl) : grav_rad_cyl(rad, azi, pol, pl, dt);
        grav += -1.0 / rad / rad;
      }
      else { double dis = sqrt(rad * rad + pol * pol); grav = -rad / dis / dis / dis; }
      return grav + Lv[n] * Lv[n] / rad / rad / rad;
    } else {
      if (ph.plnt) grav = CF0 ? grav_rad_sph_cf(rad, cf0, sinpol, pl) : grav_rad_sph_s(rad, azi, sinpol, pl, dt);
      else grav = -1.0 / rad / rad;
      double w = wv[n];
      double rs = rad * sinpol;
      return grav + w * w / rad / rad / rad + Lv[n] * Lv[n] / rad / (rs * rs);
    }
  } else if (AXIS == 1) {
    if (!SPH) return ph.plnt ? grav_azi_cyl(rad, azi, pol, pl, dt) : 0.0;
    return ph.plnt ? grav_azi_sph_s(rad, azi, sinpol, pl, dt) : 0.0;
  } else {
    (void)pol;
    double grav = 0.0;
    if (ph.plnt) grav = CF0 ? grav_pol_sph_cf(rad, cf0, sp, cp, pl) : grav_pol_sph_s(rad, azi, sp, cp, pl, dt);
    double rc = rad * sp;
    return grav + (Lv[n] * Lv[n] * cp) / rc / rc / rc;
  }
}

// FP32 ppmlr chain; returns this cell's new Sigma in FP64 (cells 6 ..
// nmax-7; the others return c.sig).  Slots: u = sweep velocity (FP32; residual dv_phi in
// the azimuthal sweep); L = FP64 angular momentum (radial: the v slot,
// polar: the w slot); the remaining transverse slot in FP32 (radial 3D: w,
// azimuthal: w = v_r and in 3D v = v_theta, polar: v = v_r).  xa0 holds the
// FP64 face coordinates.
template <int AXIS, bool SPH, bool THREED, int NT>
__device__ __forceinline__ double ppm_chunk32(ChunkShm32Data<NT> &S, int n, int nmax, double dt, double FrRot,
                                            const CellIn32 &c, const Body &pl, const Phys &ph) {
  const bool act = n < nmax;
  const bool hasL = (AXIS != 1);
  float flat = 0.f;
  if (act) { S.q[n] = 0.f; S.dx[n] = 0.f; S.umid[n] = 0.f; S.pmid[n] = 0.f; S.tmp1[n] = 0.f; S.dl[n] = 0.f; }
  __syncthreads();
  if (ph.flat) {
    float *steep = S.tmp1;
    if (act) {
      bool shock = false;
      steep[n] = 0.f;
      if (n >= 2 && n < nmax - 2) {
        float dp1 = S.p[n + 1] - S.p[n - 1];
        float dp2 = S.p[n + 2] - S.p[n - 2];
        if (fabsf(dp2) < kSmallpF) dp2 = kSmallpF;
        float ddp = fabsf(dp1) / fminf(S.p[n + 1], S.p[n - 1]);
        if (ddp > 0.33f) shock = true;
        if (S.u[n - 1] < S.u[n + 1]) shock = false;
        if (shock) {
          ddp = (dp1 / dp2 - 0.75f) * 5.0f;
          steep[n] = fmaxf(0.f, ddp);
        }
      }
    }
    __syncthreads();
    if (n >= 2 && n < nmax - 2) flat = fminf(0.5f, max3f(steep[n - 1], steep[n], steep[n + 1]));
    __syncthreads();
  }
  // ---- states ----
  const double hdt = 0.5 * dt;
  const float hdtf = (float)hdt;
  ParF par;
  paraset32(n, 0, nmax, par, S.dx0, S.q, S.dx, S.tmp1);
  float ftot = 0.f;
  if (n >= 2 && n < nmax - 1) ftot = (float)face_force32<AXIS, SPH>(n, hdt, c, S.xa0[n], S.L, AXIS == 0 ? S.w : S.v, pl, ph);
  __syncthreads();
  if (act) {
    float cs = hdtf * sqrtf(ph.gam * S.p[n] / S.r[n]) / S.dx0[n];
    if (AXIS != 0) cs /= (float)c.rad;
    S.umid[n] = cs;
    S.pmid[n] = 1.0f - kFourthdF * cs;
  }
  // the parabolas of p, rho and u side by side (parabola32_n): al/da/a6 in
  // q/dx/tmp1 (p), s0/s1/s2 (rho), s3/s4/s5 (u)
  float spl = 0.f, spr = 0.f, srl = 0.f, srr = 0.f, sul = 0.f, sur = 0.f;
  const float *cs = S.umid, *csfac = S.pmid;
  float *al = S.q, *da = S.dx, *a6 = S.tmp1;
  {
    const float *val[3] = {S.p, S.r, S.u};
    float *const al3[3] = {S.q, S.s0, S.s3};
    float *const da3[3] = {S.dx, S.s1, S.s4};
    float *const a63[3] = {S.tmp1, S.s2, S.s5};
    parabola32_n<3>(n, 0, nmax, flat, val, al3, da3, a63, par);
    if (n >= 3 && n < nmax - 2) {
      float sl[3], sr[3];
#pragma unroll
      for (int f = 0; f < 3; f++) {
        sl[f] = al3[f][n - 1] + da3[f][n - 1] - cs[n - 1] * (da3[f][n - 1] - csfac[n - 1] * a63[f][n - 1]);
        sr[f] = al3[f][n] + cs[n] * (da3[f][n] + csfac[n] * a63[f][n]);
      }
      spl = fmaxf(kSmallpF, sl[0]);
      spr = fmaxf(kSmallpF, sr[0]);
      srl = fmaxf(kSmallrF, sl[1]);
      srr = fmaxf(kSmallrF, sr[1]);
      sul = sl[2] + hdtf * ftot;
      sur = sr[2] + hdtf * ftot;
    }
  }
  __syncthreads();
  // ---- riemann (isothermal) ----
  if (n >= 3 && n < nmax - 2) {
    float t1 = 0.5f * (sqrtf(spl / srl) + sqrtf(spr / srr));
    float t2 = -0.5f * (sur - sul) / t1;
    float pm = sqrtf(spl * spr) * expf(t2);
    S.umid[n] = sul - t1 * logf(pm / spl);
    S.pmid[n] = fmaxf(kSmallpF, pm);
  }
  __syncthreads();
  // ---- evolve: face displacements delx (dl), widths dx0 + dl[n+1] - dl[n] ----
  float *vfac = S.tmp1;
  const double xa0n = act ? S.xa0[n] : 0.0;
  double dvol = c.dvol0;
  float dtdm = 0.f, fto1 = 0.f, fto2 = 0.f;
  if (n >= 3 && n < nmax - 2) {
    double delx;
    if (AXIS == 0) delx = dt * (double)S.umid[n];
    else if (AXIS == 1) delx = dt * ((double)S.umid[n] / c.rad + c.omres);
    else delx = dt * (double)S.umid[n] / c.rad;
    dtdm = (float)(dt / ((double)S.r[n] * c.dvol0));
    S.dl[n] = (float)delx;
    S.dld[n] = delx;
  }
  __syncthreads();
  double xa = xa0n;
  float dxl = 0.f;
  double dxld = 0.0;
  if (n >= 3 && n < nmax - 3) {
    dxl = S.dx0[n] + (S.dl[n + 1] - S.dl[n]);
    S.dx[n] = dxl;
    dxld = c.dx0 + (S.dld[n + 1] - S.dld[n]);
    xa = xa0n + S.dld[n];
  }
  __syncthreads();
  double sxcl = 0.0;   // polar: sin of the new centre angle, reused by the volume
  if (n >= 3 && n < nmax - 3) {
    double xcl = xa + 0.5 * dxld;
    double a1, a2;
    if (AXIS == 0) {
      a1 = centre_force32<0, SPH, true>(n, 0.0, c.rad, c.azi, c.pol, c.sinpol, S.L, S.w, pl, ph, S.cf0);
      a2 = centre_force32<0, SPH>(n, dt, xcl, c.azi + dt * c.vrot, c.pol, c.sinpol, S.L, S.w, pl, ph);
    } else if (AXIS == 1) {
      a1 = centre_force32<1, SPH>(n, 0.0, c.rad, c.azi, c.pol, c.sinpol, S.L, S.v, pl, ph);
      a2 = centre_force32<1, SPH>(n, dt, c.rad, xcl + dt * c.vrot, c.pol, c.sinpol, S.L, S.v, pl, ph);
    } else {
      a1 = centre_force32<2, SPH, true>(n, 0.0, c.rad, c.azi, c.pol, 0.0, S.L, S.v, pl, ph, S.cf0, c.sinpol,
                                        c.cospol);
      sxcl = sin(xcl);
      a2 = centre_force32<2, SPH>(n, dt, c.rad, c.azi + dt * c.vrot, xcl, 0.0, S.L, S.v, pl, ph, 0.0, sxcl,
                                  cos(xcl));
    }
    fto1 = (float)a1;
    fto2 = (float)a2;
  }
  __syncthreads();
  // polar: the volume factor's two sines, reused by the remap's overlap volume
  double sA = 0.0, sB = 0.0;
  bool haveS = false;
  if (n >= 3 && n < nmax - 2) {
    // as in the reference, the last cell of this range keeps xa = xa0
    // (evolve.cu:36-44 sets xa for n < nmax-3 only)
    double dxn = (n < nmax - 3) ? dxld : (double)S.dx[n];
    double d = (n < nmax - 3) ? S.dld[n] : 0.0;
    if (AXIS == 0) {
      if (!SPH) { dvol = dxn * (xa + 0.5 * dxn); vfac[n] = (float)(xa0n + 0.5 * d); }
      else {
        dvol = dxn * (xa * (xa + dxn) + dxn * dxn * kThird);
        vfac[n] = (float)(d * (kThird * d + xa0n) + (xa0n * xa0n));
      }
    } else if (AXIS == 1) {
      dvol = dxn * c.rad; vfac[n] = 1.0f;
    } else {
      const double sc = (n < nmax - 3) ? sxcl : sin(xa + 0.5 * dxn);
      dvol = 2.0 * sc * sin(0.5 * dxn) * c.rad;
      if (d == 0.0) vfac[n] = (float)sin(xa);
      else {
        sA = sin(xa0n + 0.5 * d);
        sB = sin(0.5 * d);
        haveS = (n < nmax - 3);
        vfac[n] = (float)(2.0 * sA * sB / d);
      }
    }
  }
  __syncthreads();
  double m_d = 0.0;
  if (n >= 3 && n < nmax - 3) {
    double rl = c.sig * (c.dvol0 / dvol);
    m_d = c.sig * c.dvol0;   // Lagrangian mass, FP64
    S.r[n] = fmaxf((float)rl, kSmallrF);
    S.Rd[n] = fmax(rl, (double)kSmallrF);
    float dum = S.u[n];
    float delx = 0.5f * (float)dt * (fto1 + fto2);
    delx += -dtdm * (S.pmid[n + 1] - S.pmid[n]) * 0.5f * (vfac[n + 1] + vfac[n]);
    S.u[n] = dum + delx;
  }
  __syncthreads();
  // ---- remap ----
  al = S.tmp1; da = S.umid; a6 = S.pmid;
  paraset32(n, 3, nmax - 3, par, S.dx, al, da, a6);
  double dd = (n >= 3 && n < nmax - 3) ? S.dld[n] : 0.0;
  double lvol;
  if (AXIS == 0) {
    if (!SPH) lvol = dd * (xa0n + 0.5 * dd);
    else lvol = dd * (xa0n * (xa0n + dd) + kThird * (dd * dd));
  } else if (AXIS == 1) {
    lvol = dd * c.rad;
  } else {
    if (haveS) lvol = 2.0 * sA * sB * c.rad;
    else lvol = 2.0 * sin(xa0n + 0.5 * dd) * sin(0.5 * dd) * c.rad;
  }
  const bool delC = (dd >= 0.0);
  float *flux = S.dx;
  // FP64 mass transport: Lagrangian widths, interface coefficients, density
  // parabola and the swept mass of each face (the L slots are free here)
  double *dxd = S.Lflux;
  if (n >= 3 && n < nmax - 3) dxd[n] = dxld;
  __syncthreads();
  Par pd;
  paraset(n, 3, nmax - 3, pd, dxd, S.Lal, S.Lda, S.La6);
  double dxnn = 0.0, dxnm = 0.0;
  if (n >= 6 && n < nmax - 5) { dxnn = dxd[n]; dxnm = dxd[n - 1]; }
  parabola(n, 3, nmax - 3, (double)flat, S.Rd, S.Lal, S.Lda, S.La6, pd);
  double xd = 0.0, x2d = 0.0, frd = 0.0;
  if (n >= 6 && n < nmax - 5) {
    if (delC) {
      xd = 0.5 * dd / dxnm;
      x2d = 1.0 - kFourthd * xd;
      frd = (S.Lal[n - 1] + S.Lda[n - 1] - xd * (S.Lda[n - 1] - x2d * S.La6[n - 1])) * lvol;
    } else {
      xd = 0.5 * dd / dxnn;
      x2d = 1.0 + kFourthd * xd;
      frd = (S.Lal[n] - xd * (S.Lda[n] + x2d * S.La6[n])) * lvol;
    }
    S.Lflux[n] = frd;
  }
  __syncthreads();
  const float fr = (float)frd, dxf = (float)xd, dxf2 = (float)x2d;
  float mm = 0.f, invm = 0.f;
  double mnew_d = 1.0, sig_new = c.sig;
  if (n >= 6 && n < nmax - 6) {
    mm = S.r[n] * (float)dvol;
    mnew_d = m_d + frd - S.Lflux[n + 1];
    sig_new = fmax((double)kSmallrF, mnew_d / c.dvol0);
    S.r[n] = (float)sig_new;
    invm = 1.0f / (S.r[n] * (float)c.dvol0);
  }
  // the FP32 momentum-like fields side by side (parabola32_n): u, plus w in
  // the radial sweep (3D), w and v in the azimuthal one (v in 3D), v in the
  // polar one; al/da/a6 in tmp1/umid/pmid, s0/s1/s2, s3/s4/s5; the fluxes go
  // to the al arrays once every cell has read its neighbour's parabola
  {
    constexpr int NF = (AXIS == 0) ? (THREED ? 2 : 1) : (AXIS == 1 ? (THREED ? 3 : 2) : 2);
    float *fl[3] = {S.u, S.u, S.u};
    if (AXIS == 0) { fl[1] = S.w; }
    else if (AXIS == 1) { fl[1] = S.w; fl[2] = S.v; }
    else { fl[1] = S.v; }
    float *const al3[3] = {S.tmp1, S.s0, S.s3};
    float *const da3[3] = {S.umid, S.s1, S.s4};
    float *const a63[3] = {S.pmid, S.s2, S.s5};
    parabola32_n<NF>(n, 3, nmax - 3, flat, fl, al3, da3, a63, par);
    float fx[NF];
    if (n >= 6 && n < nmax - 5) {
#pragma unroll
      for (int f = 0; f < NF; f++) {
        if (delC) fx[f] = (al3[f][n - 1] + da3[f][n - 1] - dxf * (da3[f][n - 1] - dxf2 * a63[f][n - 1])) * fr;
        else      fx[f] = (al3[f][n] - dxf * (da3[f][n] + dxf2 * a63[f][n])) * fr;
      }
    }
    __syncthreads();
    if (n >= 6 && n < nmax - 5) {
#pragma unroll
      for (int f = 0; f < NF; f++) al3[f][n] = fx[f];
    }
    __syncthreads();
    if (n >= 6 && n < nmax - 6) {
#pragma unroll
      for (int f = 0; f < NF; f++) fl[f][n] = (fl[f][n] * mm + (fx[f] - al3[f][n + 1])) * invm;
    }
  }
  (void)flux;
  if (hasL) {
    // FP64 angular momentum: L_new = (L m + F_n - F_{n+1}) / (m + f_n - f_{n+1})
    __syncthreads();   // every thread has read the mass flux of face n+1
    parabola(n, 3, nmax - 3, (double)flat, S.L, S.Lal, S.Lda, S.La6, pd);
    if (n >= 6 && n < nmax - 5) {
      if (delC) S.Lflux[n] = (S.Lal[n - 1] + S.Lda[n - 1] - xd * (S.Lda[n - 1] - x2d * S.La6[n - 1])) * frd;
      else      S.Lflux[n] = (S.Lal[n] - xd * (S.Lda[n] + x2d * S.La6[n])) * frd;
    }
    __syncthreads();
    if (n >= 6 && n < nmax - 6) S.L[n] = (S.L[n] * m_d + (S.Lflux[n] - S.Lflux[n + 1])) / mnew_d;
    __syncthreads();
  }
  __syncthreads();
  return sig_new;
}

}  // namespace pgd
