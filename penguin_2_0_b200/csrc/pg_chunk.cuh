// pg_chunk.cuh -- the ppmlr chain (ppmlr.cu:2-56) for one 128-cell chunk,
// specialised per sweep axis at compile time.
//   AXIS 0: radial (cylindrical R, ngeomx 1, or spherical r, ngeomx 2)
//   AXIS 1: azimuthal (ngeomy 3 cylindrical / 4 spherical)
//   AXIS 2: polar angle (ngeomz 5)
// SPH selects the spherical geometry branches (3D), THREED keeps the w
// component alive.
#pragma once
#include "pg_ppm.cuh"

namespace pgd {

// Per-thread inputs of one chunk cell.
struct CellIn {
  double rad;    // ppmlr's rad argument (ring radius; r sin(theta) in sweepy)
  double azi;    // cell-centre azimuth in the physical frame
  double pol;    // polar angle (0 in 2D)
  double vrot;   // res_v / rad_cyl of the cell's ring
  double dvol0;  // Eulerian cell volume along the sweep
  double sinpol; // sin(pol) of the cell (3D radial and azimuthal sweeps)
  // polar sweep: the layer's sin/cos(centre), sin/cos(face) and the
  // reciprocals 1/sin(centre), 1/sin(face), 1/dz read where they are used,
  // from lay[0], lay[nz], ..., lay[6 nz] (the tables szc, czc, szf, czf,
  // iszc, iszf, idz at stride nz; plain loads, which a barrier keeps from
  // being merged: nothing holds them in registers through the chain)
  const double *lay;
  int nz;
  __device__ __forceinline__ double spol() const { return lay[0]; }
  __device__ __forceinline__ double cpol() const { return lay[nz]; }
  __device__ __forceinline__ double sfz() const { return lay[2 * nz]; }
  __device__ __forceinline__ double cfz() const { return lay[3 * nz]; }
  __device__ __forceinline__ double iszc() const { return lay[4 * nz]; }   // 1 / sin(centre)
  __device__ __forceinline__ double iszf() const { return lay[5 * nz]; }   // 1 / sin(face)
  __device__ __forceinline__ double idz() const { return lay[6 * nz]; }    // 1 / dz
};

// x^2 where the reference writes pow(x, 2)
__device__ __forceinline__ double sq(double x) { return x * x; }

template <int AXIS, bool SPH, class SHM>
__device__ __forceinline__ void face_force(int n, double hdt, const CellIn &c, const SHM &S,
                                           const Body &pl, const Phys &ph, double &ftot) {
  if (AXIS == 0) {
    // get_fx_bound forces.cu:185-224 at the left face xa0[n]
    double rad = S.xa0[n];
    double azi = c.azi + hdt * c.vrot;
    // x / r / r / r of forces.cu as x r^-3; products rounded on their own
    // (no fused multiply-add) so that every kernel shape gives the same bits
    const double ir = 1.0 / rad, ir2 = __dmul_rn(ir, ir), ir3 = __dmul_rn(ir2, ir);
    double grav;
    if (!SPH) {
      if (ph.plnt) { grav = grav_rad_cyl(rad, azi, c.pol, pl, hdt); grav += -ir2; }
      else { double dis = sqrt(rad * rad + c.pol * c.pol); grav = -rad / dis / dis / dis; }
      double f = grav;
      f += __dmul_rn(sq(0.5 * (S.v[n] + S.v[n - 1])), ir3);
      ftot = f;
    } else {
      grav = ph.plnt ? grav_rad_sph_s(rad, azi, c.sinpol, pl, hdt) : -ir2;
      double f = grav;
      f += __dmul_rn(sq(0.5 * (S.w[n] + S.w[n - 1])), ir3);
      f += __dmul_rn(sq(0.5 * (S.v[n] + S.v[n - 1])), ir) / sq(rad * c.sinpol);
      ftot = f;
    }
  } else if (AXIS == 1) {
    // get_fy forces.cu:265-296 at xa0[n] + hdt v_rot
    double azi = S.xa0[n] + hdt * c.vrot;
    if (!SPH) ftot = ph.plnt ? grav_azi_cyl(c.rad, azi, c.pol, pl, hdt) : 0.0;
    else ftot = ph.plnt ? grav_azi_sph_s(c.rad, azi, c.sinpol, pl, hdt) : 0.0;
  } else {
    // get_fz_bound forces.cu:298-334 (ngeomz 5) at the face angle xa0[n],
    // whose sin and cos come from the per-layer table; the planet's angle
    // factor cos(azi + hdt v_rot - (p.y + hdt p.vy)) by angle addition from
    // the pencil's start-of-step cos and sin of azi - p.y
    const double sp = c.sfz(), cp = c.cfz();
    double grav = 0.0;
    if (ph.plnt) {
      double sd, cd;
      sincos_small(hdt * (c.vrot - pl.vy), sd, cd);
      grav = grav_pol_sph_plm(c.rad, S.cf0 * cd - S.sf0 * sd, sp, cp, S.plm, pl);
    }
    const double irc = c.iszf() * S.irad;   // 1 / (r sin(face)) from the pencil's and layer's reciprocals
    double f = grav;
    f += __dmul_rn(sq(0.5 * (S.w[n] + S.w[n - 1])) * cp, __dmul_rn(__dmul_rn(irc, irc), irc));
    ftot = f;
  }
}

// get_fx / get_fy / get_fz at a cell centre (forces.cu:226-372).  CF0: the
// planet's cos(azi - p.y) comes in as cf0 (the dt = 0 force of a radial or
// polar pencil, one value per pencil).  The polar form takes sin and cos of
// its angle from the caller (sp, cp).
template <int AXIS, bool SPH, bool CF0 = false, class SHM>
__device__ __forceinline__ double centre_force(int n, double dt, double rad, double azi, double pol,
                                               double sinpol, const SHM &S, const Body &pl, const Phys &ph,
                                               double cf0 = 0.0, double sp = 0.0, double cp = 0.0,
                                               double irc_in = 0.0) {
  if (AXIS == 0) {
    double grav;
    const double ir = 1.0 / rad, ir2 = __dmul_rn(ir, ir), ir3 = __dmul_rn(ir2, ir);
    if (!SPH) {
      if (ph.plnt) {
        grav = CF0 ? grav_rad_cyl_cf(rad, cf0, pol, pl) : grav_rad_cyl(rad, azi, pol, pl, dt);
        grav += -ir2;
      }
      else { double dis = sqrt(rad * rad + pol * pol); grav = -rad / dis / dis / dis; }
      double f = grav;
      f += __dmul_rn(__dmul_rn(S.v[n], S.v[n]), ir3);
      return f;
    } else {
      if (ph.plnt) grav = CF0 ? grav_rad_sph_cf(rad, cf0, sinpol, pl) : grav_rad_sph_s(rad, azi, sinpol, pl, dt);
      else grav = -ir2;
      double f = grav;
      f += __dmul_rn(__dmul_rn(S.w[n], S.w[n]), ir3);
      f += __dmul_rn(__dmul_rn(S.v[n], S.v[n]), ir) / sq(rad * sinpol);
      return f;
    }
  } else if (AXIS == 1) {
    if (!SPH) return ph.plnt ? grav_azi_cyl(rad, azi, pol, pl, dt) : 0.0;
    return ph.plnt ? grav_azi_sph_s(rad, azi, sinpol, pl, dt) : 0.0;
  } else {
    // the polar sweep's form (CF0): the planet's reduced mass and
    // 1 / (r sin) from the caller (irc_in)
    (void)pol;
    double grav = 0.0;
    if (ph.plnt) grav = CF0 ? grav_pol_sph_plm(rad, cf0, sp, cp, S.plm, pl) : grav_pol_sph_s(rad, azi, sp, cp, pl, dt);
    const double irc = CF0 ? irc_in : 1.0 / (rad * sp);
    double f = grav;
    f += __dmul_rn(S.w[n] * S.w[n] * cp, __dmul_rn(__dmul_rn(irc, irc), irc));
    return f;
  }
}

// The ppmlr chain for one chunk.  All threads of the CTA call it (it has
// barriers); cells n >= nmax take no part in any phase.  On return r, u, v
// (and w when THREED) hold the Lagrange-remapped values for 6 <= n < nmax-6.
// The polar sweep (AXIS 2) passes its layers' Eulerian paraset coefficients
// in eul_par (5 per cell of the chunk) and c.lay for its layer tables.
template <int AXIS, bool SPH, bool THREED, int EOS = 0, class SHM>
__device__ __forceinline__ void ppm_chunk(SHM &S, int n, int nmax, double dt, double FrRot,
                                          const CellIn &c, const Body &pl, const Phys &ph,
                                          const double *eul_par = nullptr) {
  const bool act = n < nmax;
  double flat = 0.0;
  if (act) { S.q[n] = 0.0; S.dx[n] = 0.0; S.umid[n] = 0.0; S.pmid[n] = 0.0; S.tmp1[n] = 0.0; }
  __syncthreads();

  // ---- flatten flatten.cu:7-40 (steep in tmp1) ----
  if (ph.flat) {
    double *steep = S.tmp1;
    if (act) {
      bool shock = false;
      steep[n] = 0.0;
      if (n >= 2 && n < nmax - 2) {
        double dp1 = S.p[n + 1] - S.p[n - 1];
        double dp2 = S.p[n + 2] - S.p[n - 2];
        if (fabs(dp2) < kSmallp) dp2 = kSmallp;
        double ddp = fabs(dp1) / fmin(S.p[n + 1], S.p[n - 1]);
        if (ddp > 0.33) shock = true;
        if (S.u[n - 1] < S.u[n + 1]) shock = false;
        if (shock) {
          ddp = (dp1 / dp2 - 0.75) * 5.0;
          steep[n] = fmax(0.0, ddp);
        }
      }
    }
    __syncthreads();
    if (n >= 2 && n < nmax - 2) flat = fmin(0.5, max3(steep[n - 1], steep[n], steep[n + 1]));
    __syncthreads();
  }

  // ---- states states.cu:3-73 ----
  // paraset's temporaries a/ai/b live in q/dx/tmp1; cs = umid, csfac = pmid
  // (ppmlr.cu:30-33).  paraset runs per cell as in the reference:
  // tabulating its Eulerian coefficients in a separate kernel changes their
  // FMA contraction (the last bits), which then shows up at 1e-12 in v_r.
  // The three parabolas of p, rho and u (states.cu:40-64) run side by side
  // (parabola_n), with al/da/a6 in q/dx/tmp1 for p, s0/s1/s2 for rho and
  // s3/s4/s5 for u; each value is the reference's, only the barriers are
  // shared.
  const double hdt = 0.5 * dt;
  Par par;
  // the polar sweep's Eulerian coefficients, one set per layer (k_tables;
  // the polar sweep has no reference kernel whose bits it must follow), are
  // read from the table where the parabolas use them
  constexpr bool eul_tab = (AXIS == 2);
  if (!eul_tab) paraset(n, 0, nmax, par, S.dx0, S.q, S.dx, S.tmp1);
  double ftot = 0.0;
  if (n >= 2 && n < nmax - 1) face_force<AXIS, SPH>(n, hdt, c, S, pl, ph, ftot);
  if (act) {
    double cs;
    if (AXIS == 2) {
      // the polar sweep's dx0 is its layer's dz: 1 / (dz r) from reciprocals
      cs = hdt * sqrt(ph.gam * S.p[n] / S.r[n]) * (c.idz() * S.irad);
    } else {
      cs = hdt * sqrt(ph.gam * S.p[n] / S.r[n]) / S.dx0[n];
      if (AXIS == 1) cs /= c.rad;
    }
    S.umid[n] = cs;
    S.pmid[n] = 1.0 - kFourthd * cs;
  }
  {
    const double *val[3] = {S.p, S.r, S.u};
    double *const al[3] = {S.q, S.s0, S.s3};
    double *const da[3] = {S.dx, S.s1, S.s4};
    double *const a6[3] = {S.tmp1, S.s2, S.s5};
    if (eul_tab) parabola_n<3>(n, 0, nmax, flat, val, al, da, a6, ParTab{eul_par + 5 * n});
    else parabola_n<3>(n, 0, nmax, flat, val, al, da, a6, par);
    const double *cs = S.umid, *csfac = S.pmid;
    double sl[3] = {0.0, 0.0, 0.0}, sr[3] = {0.0, 0.0, 0.0};
    if (n >= 3 && n < nmax - 2) {
#pragma unroll
      for (int f = 0; f < 3; f++) {
        sl[f] = al[f][n - 1] + da[f][n - 1] - cs[n - 1] * (da[f][n - 1] - csfac[n - 1] * a6[f][n - 1]);
        sr[f] = al[f][n] + cs[n] * (da[f][n] + csfac[n] * a6[f][n]);
      }
    }
    // riemann below writes umid/pmid, which hold cs/csfac read above
    __syncthreads();

    // ---- riemann riemann.cu:3-115, isothermal (45-53) or isentropic (75-111) ----
    if (n >= 3 && n < nmax - 2) {
      const double spl = fmax(kSmallp, sl[0]), spr = fmax(kSmallp, sr[0]);
      const double srl = fmax(kSmallr, sl[1]), srr = fmax(kSmallr, sr[1]);
      const double sul = sl[2] + hdt * ftot, sur = sr[2] + hdt * ftot;
      if (EOS == 0) {
        double t1 = 0.5 * (sqrt(spl / srl) + sqrt(spr / srr));
        double t2 = -0.5 * (sur - sul) / t1;
        double pm = sqrt(spl * spr) * exp(t2);
        S.umid[n] = sul - t1 * log(pm / spl);
        S.pmid[n] = fmax(kSmallp, pm);
      } else {
        double um, pm;
        riemann_isentropic(spl, srl, sul, spr, srr, sur, ph, um, pm);
        S.umid[n] = um;
        S.pmid[n] = pm;
      }
    }
  }
  __syncthreads();

  // ---- evolve evolve.cu:3-166 (vfac = tmp1) ----
  // vfac is read only where this chunk sets it below (xa0 + delx, then the
  // geometry factor), so the reference's first fill of it is not needed
  double *vfac = S.tmp1;
  const double xa0n = S.xa0[n];
  double xa = xa0n, dvol = c.dvol0, dtdm = 0.0, fto1 = 0.0, fto2 = 0.0;
  if (n >= 3 && n < nmax - 2) {
    double delx;
    if (AXIS == 0) delx = dt * S.umid[n];
    else if (AXIS == 1) delx = dt * (S.umid[n] / c.rad - c.vrot - FrRot);
    else delx = dt * S.umid[n] / c.rad;
    dtdm = dt / (S.r[n] * c.dvol0);
    vfac[n] = S.xa0[n] + delx;
  }
  __syncthreads();
  if (n >= 3 && n < nmax - 3) {
    S.dx[n] = vfac[n + 1] - vfac[n];
    xa = vfac[n];
  }
  // the centre forces read this cell's own new width only: no barrier
  // polar sweep: sin of the new centre angle, reused by the volume below
  double sxcl = 0.0;
  if (n >= 3 && n < nmax - 3) {
    double xcl = xa + 0.5 * S.dx[n];
    if (AXIS == 0) {
      fto1 = centre_force<0, SPH, true>(n, 0.0, c.rad, c.azi, c.pol, c.sinpol, S, pl, ph, S.cf0);
      fto2 = centre_force<0, SPH>(n, dt, xcl, c.azi + dt * c.vrot, c.pol, c.sinpol, S, pl, ph);
    } else if (AXIS == 1) {
      fto1 = centre_force<1, SPH>(n, 0.0, c.rad, c.azi, c.pol, c.sinpol, S, pl, ph);
      fto2 = centre_force<1, SPH>(n, dt, c.rad, xcl + dt * c.vrot, c.pol, c.sinpol, S, pl, ph);
    } else {
      const double spo = c.spol(), cpo = c.cpol();
      fto1 = centre_force<2, SPH, true>(n, 0.0, c.rad, 0.0, 0.0, 0.0, S, pl, ph, S.cf0, spo, cpo,
                                        c.iszc() * S.irad);
      // sin, cos of the new centre angle from the layer's (xcl moved by a
      // fraction of a cell), and the planet's angle factor at t + dt from
      // the pencil's, by angle addition
      double se, ce, sd, cd;
      sincos_small(xcl - c.pol, se, ce);
      sxcl = spo * ce + cpo * se;
      const double cxcl = cpo * ce - spo * se;
      sincos_small(dt * (c.vrot - pl.vy), sd, cd);
      fto2 = centre_force<2, SPH, true>(n, dt, c.rad, 0.0, xcl, 0.0, S, pl, ph, S.cf0 * cd - S.sf0 * sd, sxcl, cxcl,
                                        1.0 / (c.rad * sxcl));
    }
  }
  __syncthreads();
  // polar sweep: the two sines of the volume factor, reused by the remap's
  // overlap volume (same angles)
  double sA = 0.0, sB = 0.0;
  bool haveS = false;
  if (n >= 3 && n < nmax - 2) {
    double dxn = S.dx[n];
    if (AXIS == 0) {
      if (!SPH) { dvol = dxn * (xa + 0.5 * dxn); vfac[n] = 0.5 * (xa + xa0n); }
      else {
        dvol = dxn * (xa * (xa + dxn) + dxn * dxn * kThird);
        vfac[n] = (xa - xa0n) * (kThird * (xa - xa0n) + xa0n) + (xa0n * xa0n);
      }
    } else if (AXIS == 1) {
      dvol = dxn * c.rad; vfac[n] = 1.0;
    } else {
      // evolve.cu:117-124 with cos(a) - cos(b) written as
      // 2 sin((a+b)/2) sin((b-a)/2): the same value without the
      // cancellation that makes the reference's form depend on libm ulps
      // Sines of angles a fraction of a cell from the face angle xa0 come
      // from its per-layer sin and cos by angle addition (sincos_small).
      double delx = xa - xa0n;
      double sw, cw;
      sincos_small(0.5 * dxn, sw, cw);
      const double sfz = c.sfz(), cfz = c.cfz();
      const double sc = (n < nmax - 3) ? sxcl : sfz * cw + cfz * sw;   // sin(xa0 + dxn / 2)
      dvol = 2.0 * sc * sw * c.rad;
      if (delx == 0.0) vfac[n] = sfz;                                 // sin(xa) = sin(xa0)
      else {
        double sh, ch;
        sincos_small(0.5 * delx, sh, ch);
        sA = sfz * ch + cfz * sh;                                        // sin(xa0 + delx / 2)
        sB = sh;
        haveS = true;
        vfac[n] = 2.0 * sA * sB / delx;
      }
    }
  }
  __syncthreads();
  if (n >= 3 && n < nmax - 3) {
    S.r[n] = fmax(S.r[n] * (c.dvol0 / dvol), kSmallr);
    double dum = S.u[n];
    double delx = 0.5 * dt * (fto1 + fto2);
    delx += -dtdm * (S.pmid[n + 1] - S.pmid[n]) * 0.5 * (vfac[n + 1] + vfac[n]);
    S.u[n] = dum + delx;
  }
  __syncthreads();

  // ---- remap remap.cu:14-226 ----
  // paraset on the Lagrangian widths (temporaries in tmp1/umid/pmid), then
  // the parabolas of rho and of the momentum-like fields (get_flux
  // remap.cu:1-10) side by side: al/da/a6 in p/q/dx0 (rho), umid/pmid/tmp1
  // (u), s0/s1/s2 (v or w) and s3/s4/s5 (w in 3D).  The fluxes, each the
  // reference's expression, go to the al arrays once every cell has read its
  // neighbour's parabola.  2D slots that stay exactly zero are skipped: w in
  // the radial sweep, v (= w) in the azimuthal one, whose w slot carries v_r.
  paraset(n, 3, nmax - 3, par, S.dx, S.tmp1, S.umid, S.pmid);
  double lvol = 0.0;
  if (AXIS == 0) {
    if (!SPH) { lvol = xa - xa0n; lvol *= (xa0n + 0.5 * lvol); }
    else { lvol = xa - xa0n; lvol *= xa0n * xa + kThird * (lvol * lvol); }
  } else if (AXIS == 1) {
    lvol = (xa - xa0n) * c.rad;
  } else {
    // remap.cu:53, cancellation-free form of (cos(xa0) - cos(xa)) * rad
    double d = xa - xa0n;
    if (haveS) lvol = 2.0 * sA * sB * c.rad;
    else {
      double sh, ch;
      sincos_small(0.5 * d, sh, ch);
      lvol = 2.0 * (c.sfz() * ch + c.cfz() * sh) * sh * c.rad;
    }
  }
  double dxf = xa - xa0n;
  const bool delC = (dxf >= 0.0);
  double dxnn = 0.0, dxnm = 0.0;
  if (n >= 6 && n < nmax - 5) { dxnn = S.dx[n]; dxnm = S.dx[n - 1]; }
  constexpr int NF = (THREED ? 4 : 3);
  double *fld[NF];
  fld[0] = S.r;
  fld[1] = S.u;
  if (THREED) { fld[2] = S.v; fld[NF - 1] = S.w; }
  else fld[2] = (AXIS == 1) ? S.w : S.v;
  double *const al[4] = {S.p, S.umid, S.s0, S.s3};
  double *const da[4] = {S.q, S.pmid, S.s1, S.s4};
  double *const a6[4] = {S.dx0, S.tmp1, S.s2, S.s5};
  parabola_n<NF>(n, 3, nmax - 3, flat, fld, al, da, a6, par);
  double fx[NF];
  double dxf2 = 0.0;
  if (n >= 6 && n < nmax - 5) {
    if (delC) {
      dxf = 0.5 * dxf / dxnm;
      dxf2 = 1.0 - kFourthd * dxf;
    } else {
      dxf = 0.5 * dxf / dxnn;
      dxf2 = 1.0 + kFourthd * dxf;
    }
#pragma unroll
    for (int f = 0; f < NF; f++) {
      double t;
      if (delC) t = al[f][n - 1] + da[f][n - 1] - dxf * (da[f][n - 1] - dxf2 * a6[f][n - 1]);
      else      t = al[f][n] - dxf * (da[f][n] + dxf2 * a6[f][n]);
      fx[f] = t * (f == 0 ? lvol : fx[0]);
    }
  }
  __syncthreads();
  if (n >= 6 && n < nmax - 5) {
#pragma unroll
    for (int f = 0; f < NF; f++) al[f][n] = fx[f];
  }
  __syncthreads();
  if (n >= 6 && n < nmax - 6) {
    const double fr = fx[0];
    const double mm = S.r[n] * dvol;
    double lv = (mm + fr - al[0][n + 1]) / c.dvol0;
    S.r[n] = fmax(kSmallr, lv);
    const double invm = 1.0 / (S.r[n] * c.dvol0);
#pragma unroll
    for (int f = 1; f < NF; f++) {
      double fl = fx[f] - al[f][n + 1];
      fld[f][n] = (fld[f][n] * mm + fl) * invm;
    }
  }
  __syncthreads();
}

}  // namespace pgd
