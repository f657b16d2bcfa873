// pg_kernels32.cu -- the FP32 ("precision = 1") sweeps.
//
// State planes in FP32: dS = Sigma - S_bg(ring), v_r, dv = v_phi - v_bg(ring)
// and (3D) v_theta; S_bg, v_bg, geometry, dt, the FARGO offsets, the planet
// and the torque sum stay FP64.  Same grids, chunking and launch shapes as the FP64
// kernels of pg_kernels.cu; the chunk arithmetic is ppm_chunk32.
#include "pg_chunk32.cuh"
#include "pg_kernels.cuh"

namespace pgd {

__device__ __forceinline__ int wrap1f(int j, int n) {
  if (j < 0) j += n;
  if (j >= n) j -= n;
  return j;
}
__device__ __forceinline__ int wrapmf(int j, int n) {
  j %= n;
  return j < 0 ? j + n : j;
}

__device__ __forceinline__ double block_max32(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) {
    double t = __shfl_down_sync(0xffffffffu, v, o);
    v = (t > v || t != t) ? t : v;
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int i = 1; i < nw; i++) v = (red[i] > v || red[i] != red[i]) ? red[i] : v;
  }
  return v;
}

struct StepIn32 {
  double dt, frrot, frrot_next;
  Body pl;
};
__device__ __forceinline__ bool load_step32(const SweepCtl &c, StepIn32 &s) {
  if (c.clk) {
    if (c.clk->halted) return false;
    s.dt = c.clk->dt_step;
    s.frrot = c.clk->frrot;
    s.frrot_next = c.clk->frrot_next;
    s.pl = c.clk->planet;
  } else {
    s.dt = c.dt;
    s.frrot = c.frrot;
    s.frrot_next = c.frrot;
    s.pl = c.planet;
  }
  return true;
}

// three-point derivatives of derivs (viscosity.cu:2-18) written with cell
// widths: xf[n]-xf[n-1] = w[n-1], xf[n+1]-xf[n-1] = w[n-1] + w[n]
template <typename T>
struct DerivGeomW { T x2, x3, i2, i3, i32; };
template <typename T>
__device__ __forceinline__ DerivGeomW<T> deriv_geom_w(int n, const float *w, T scale) {
  DerivGeomW<T> g;
  g.x2 = (T)w[n - 1] * scale;
  g.x3 = g.x2 + (T)w[n] * scale;
  g.i2 = (T)1 / g.x2;
  g.i3 = (T)1 / g.x3;
  g.i32 = (T)1 / (g.x3 - g.x2);
  return g;
}
template <typename T>
__device__ __forceinline__ void derivs_w(T &first, T &second, int n, const DerivGeomW<T> &g, const T *u) {
  T h2 = (u[n] - u[n - 1]) * g.i2;
  T h3 = (u[n + 1] - u[n - 1]) * g.i3;
  T A = (h3 - h2) * g.i32;
  T B = (g.x3 * h2 - g.x2 * h3) * g.i32;
  second = (T)2 * A;
  first = second * g.x2 + B;
}

// ---------------------------------------------------------------------------
// One radial pencil chunk: column j0, chunk l, polar layer k.  The body is
// shared by the per-run kernel and the batched kernels of pg_batch.cu.
template <bool SPH, bool THREED, int NT>
__device__ __forceinline__ void sweep_x32_body(ChunkShm32Data<NT> &S, int n, bool store, const Tables &T,
                                               const Planes32 &P, const Phys &ph, const SweepCtl &ctl,
                                               const StepIn32 &st, int j0, int l, int k) {
  const bool last = (l == T.cx.loop - 1);
  const int nphi = T.nphi, nrg = T.nrg;
  if (last && T.cx.stuck) {
    int i = REAL * l + n;
    if (store && n < REAL && i < T.nr) {
      size_t idx = ((size_t)k * nrg + i + NPAD) * nphi + j0;
      P.ro[idx] = P.r[idx]; P.uo[idx] = P.u[idx]; P.vo[idx] = P.v[idx];
      if (THREED) P.wo[idx] = P.w[idx];
    }
    return;
  }
  const int lim = last ? T.cx.lim_last : ARR;
  const bool act = n < lim;
  const int row = n + REAL * l;
  const int rk = k * nrg + row;
  const size_t idx = (size_t)rk * nphi + j0;
  CellIn32 c{1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0};
  double rad_cyl = 1.0, vbg = 0.0, sbg = 0.0;
  if (act) {
    c.rad = T.rxc[row];
    rad_cyl = T.radc[rk];
    vbg = T.vbg[rk];
    sbg = T.sbg[rk];
    c.azi = T.yc[j0];
    c.pol = THREED ? T.zc[k + NPAD] : 0.0;
    c.sinpol = THREED ? T.szc[k + NPAD] : 0.0;
    c.dvol0 = T.rxvol[row];
    // the pencil's planet angle factor at the start of the step, once
    if (n == 0) S.cf0 = ph.plnt ? planet_cosfac(c.azi, st.pl, 0.0) : 0.0;
    c.vrot = T.res_v[rk] / rad_cyl;
    S.xa0[n] = T.rx[row];
    S.dx0[n] = (float)T.rdx[row];
    c.dx0 = T.rdx[row];
    c.sig = sbg + (double)P.r[idx];
    float r = (float)c.sig;
    S.r[n] = r;
    S.u[n] = P.u[idx];
    S.L[n] = rad_cyl * (vbg + (double)P.v[idx]);
    if (THREED) S.w[n] = (float)((double)P.w[idx] * c.rad);
    else S.w[n] = 0.f;
    bool ghost = (row < NPAD) || (row >= T.nr + NPAD);
    S.p[n] = ghost ? (float)T.gp[rk] : r * (float)T.cs2[rk];
  }
  __syncthreads();
  const double sig = ppm_chunk32<0, SPH, THREED, NT>(S, n, lim, st.dt, st.frrot, c, st.pl, ph);
  if (ph.visc) {
    // device_viscosity_r viscosity.cu:370-421: u in FP32, Omega = L/R^2 in FP64
    const double R = rad_cyl;
    float rho = 0.f, nr = 0.f, ddu = 0.f, ddw = 0.f;
    double ddv = 0.0;
    float *nn = S.q;
    double *om = S.Lal;
    if (act) {
      rho = S.r[n];
      nr = (float)T.nu[rk] * rho;
      nn[n] = nr;
      om[n] = S.L[n] / (R * R);
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      float d1, d2, dn;
      const DerivGeomW<float> gf = deriv_geom_w<float>(n, S.dx0, 1.0f);
      const DerivGeomW<double> gd = deriv_geom_w<double>(n, S.dx0, 1.0);
      const float Rf = (float)R;
      derivs_w<float>(dn, d2, n, gf, nn);
      derivs_w<float>(d1, d2, n, gf, S.u);
      float t = 2.0f * nr * d2 + 2.0f * dn * d1 + 2.0f * nr * d1 / Rf - 2.0f * nr * S.u[n] / Rf / Rf;
      ddu = S.u[n] + (float)st.dt * t / rho;
      double e1, e2;
      derivs_w<double>(e1, e2, n, gd, om);
      double tv = R * (double)nr * e2 + R * (double)dn * e1 + 3.0 * (double)nr * e1;
      ddv = om[n] * R + st.dt * tv / (double)rho;
      if (THREED) {
        derivs_w<float>(d1, d2, n, gf, S.w);
        t = nr * d2 + dn * d1 + nr * d1 / Rf;
        ddw = S.w[n] + (float)st.dt * t / rho;
      }
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      S.u[n] = ddu;
      S.L[n] = ddv * R;
      if (THREED) S.w[n] = ddw;
    }
  }
  if (store && n >= NPAD && n < lim - NPAD) {
    P.ro[idx] = (float)(sig - sbg);
    P.uo[idx] = S.u[n];
    P.vo[idx] = (float)(S.L[n] / rad_cyl - vbg);
    if (THREED) P.wo[idx] = (float)((double)S.w[n] / c.rad);
  }
}

template <bool SPH, bool THREED, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k32_sweep_x(Tables T, Planes32 P, Phys ph, SweepCtl ctl, int l0) {
  __shared__ ChunkShm32<NT> S;
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  sweep_x32_body<SPH, THREED, NT>(S, threadIdx.x, true, T, P, ph, ctl, st, blockIdx.x, blockIdx.y + l0,
                                  blockIdx.z);
}

// Full radial chunks (and a last chunk of more than 64 cells, in the same
// launch) of PACK adjacent columns per CTA, thread t on cell t / PACK of
// column t % PACK, as k_sweep_x_cols: a warp's loads and stores of one ring
// cover PACK adjacent floats.  The pencils' shared blocks are padded to
// 128 / PACK mod 128 bytes.
template <int PACK>
using Px32Shm = ChunkShm32<ARR, 128 / PACK>;
template <int PACK>
constexpr int px32_shm_bytes() { return PACK * (int)sizeof(Px32Shm<PACK>); }
template <bool SPH, bool THREED, int PACK, int MINB>
__global__ void __launch_bounds__(ARR * PACK, MINB) k32_sweep_x_cols(Tables T, Planes32 P, Phys ph, SweepCtl ctl) {
  extern __shared__ __align__(16) unsigned char px32_shm[];
  Px32Shm<PACK> *S = reinterpret_cast<Px32Shm<PACK> *>(px32_shm);
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  const int p = threadIdx.x % PACK, n = threadIdx.x / PACK;
  int col = blockIdx.x * PACK + p;
  const bool store = col < T.nphi;
  if (!store) col = T.nphi - 1;
  sweep_x32_body<SPH, THREED, ARR>(S[p], n, store, T, P, ph, ctl, st, col, blockIdx.y, blockIdx.z);
}

// short last chunks of radial pencils packed 4 columns per CTA (see
// k_sweep_x_packed)
constexpr int PX32_LIM = 64;
template <bool SPH, bool THREED, int MINB>
__global__ void __launch_bounds__(4 * PX32_LIM, MINB) k32_sweep_x_packed(Tables T, Planes32 P, Phys ph,
                                                                         SweepCtl ctl) {
  __shared__ ChunkShm32<PX32_LIM> S[4];
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  const int p = threadIdx.x & 3, n = threadIdx.x >> 2;
  const int npen = T.nphi * T.nk;
  int col = blockIdx.x * 4 + p;
  const bool store = col < npen;
  if (!store) col = npen - 1;
  sweep_x32_body<SPH, THREED, PX32_LIM>(S[p], n, store, T, P, ph, ctl, st, col % T.nphi, T.cx.loop - 1,
                                        col / T.nphi);
}

// ---------------------------------------------------------------------------
// One azimuthal chunk: chunk l of ring i in polar layer k; FARGO shift at
// the store and, with ctl.fuse, damping and the CFL rate in the epilogue.
template <bool SPH, bool THREED, int NT>
__device__ __forceinline__ void sweep_y32_body(ChunkShm32<NT> &S, double *red, const Tables &T,
                                               const Planes32 &P, const Phys &ph, const SweepCtl &ctl,
                                               const StepIn32 &st, int l, int i, int k) {
  const int n = threadIdx.x;
  const int nphi = T.nphi, nrg = T.nrg;
  const int row = i + NPAD;
  const int rk = k * nrg + row;
  const size_t base = (size_t)rk * nphi;
  const int inc = ctl.shift ? T.inc_j[rk] : 0;
  const bool last = (l == T.cy.loop - 1);
  const double rad = T.rxc[row];
  const double rad_cyl = T.radc[rk];
  const double vbg = T.vbg[rk];
  const double sbg = T.sbg[rk];
  double rate = 0.0;
  bool bad = false;
  float dampf = 0.f;
  double dampd = 0.0;
  bool do_damp = false;
  if (ctl.fuse) {
    double g = T.damp_g[rk];
    if (g > 0.0) { do_damp = true; dampd = g * (st.dt * T.damp_pw[rk]); dampf = (float)dampd; }
  }
  // CFL frame offset of this ring: v - rot_v - FrRot r = dv + (v_bg - rot_v - FrRot r)
  const double voff = vbg - T.rot_v[rk] - st.frrot_next * rad_cyl;
  auto finish = [&](int jo, double sig, float u, float dv, float w) {
    if (ctl.fuse) {
      if (do_damp) {
        // damp the stored (rounded) state, as the separate damping kernel does
        sig = sbg + (double)(float)(sig - sbg);
        sig += dampd * (T.val_r[rk] - sig);
        u += dampf * ((float)T.val_u[rk] - u);
        dv += dampf * (-dv);
        if (THREED) w += dampf * (-w);
      }
      double p = sig * T.cs2[rk];
      double cs = sqrt(ph.gam * p / sig);
      int js = wrapmf(jo - (T.rot_j[rk] + inc), nphi);
      double widthy = T.dy[js] * rad_cyl;
      double t0 = (fabs((double)u) + cs) / T.rdx[row];
      double t1 = (fabs((double)dv + voff) + cs) / widthy;
      double rt;
      if (THREED) {
        double t2 = (fabs((double)w) + cs) / (T.dz[k + NPAD] * rad);
        rt = max3(t0, t1, t2);
      } else {
        rt = fmax(t0, t1);
      }
      rate = (rt > rate || rt != rt) ? rt : rate;
      if (!(sig > 0.0) || !isfinite(sig) || !isfinite(u) || !isfinite(dv)) bad = true;
    }
    size_t o = base + jo;
    P.ro[o] = (float)(sig - sbg); P.uo[o] = u; P.vo[o] = dv;
    if (THREED) P.wo[o] = w;
  };
  if (last && T.cy.stuck) {
    int j = REAL * l + n;
    if (n < REAL && j < nphi) {
      size_t s = base + j;
      finish(wrapmf(j + inc, nphi), sbg + (double)P.r[s], P.u[s], P.v[s], THREED ? P.w[s] : 0.f);
    }
  } else {
    const int lim = last ? T.cy.lim_last : ARR;
    const bool act = n < lim;
    const int jref = n - NPAD + REAL * l;
    const int j0 = wrap1f(jref, nphi);
    CellIn32 c;
    c.rad = rad_cyl;
    c.pol = THREED ? T.zc[k + NPAD] : 0.0;
    c.sinpol = THREED ? T.szc[k + NPAD] : 0.0;
    c.vrot = T.res_v[rk] / rad_cyl;
    c.omres = vbg / rad_cyl - c.vrot - st.frrot;
    c.azi = 0.0; c.dvol0 = 1.0; c.sig = 1.0; c.dx0 = 0.0;
    if (act) {
      size_t s = base + j0;
      double azi = T.yc[j0];
      double xa0 = T.y[j0];
      double dvol0 = T.yvol[j0];
      if (jref < 0) { xa0 -= kTwoPi; azi -= kTwoPi; }
      if (jref >= nphi) { xa0 += kTwoPi; azi += kTwoPi; }
      dvol0 *= rad_cyl;
      c.azi = azi;
      c.dvol0 = dvol0;
      S.xa0[n] = xa0;
      S.dx0[n] = (float)T.dy[j0];
      c.dx0 = T.dy[j0];
      c.sig = sbg + (double)P.r[s];
      float r = (float)c.sig;
      S.r[n] = r;
      S.p[n] = r * (float)T.cs2[rk];
      S.u[n] = P.v[s];
      S.v[n] = THREED ? P.w[s] : 0.f;
      S.w[n] = P.u[s];
    }
    __syncthreads();
    const double sig = ppm_chunk32<1, SPH, THREED, NT>(S, n, lim, st.dt, st.frrot, c, st.pl, ph);
    if (ph.visc) {
      // device_viscosity_p viscosity.cu:423-472 on x = r_cyl phi (widths dx0 r_cyl)
      const float R = (float)rad_cyl;
      float rho = 0.f, nr = 0.f, ddu = 0.f, ddv = 0.f, ddw = 0.f;
      float *nn = S.q;
      if (act) {
        rho = S.r[n];
        nr = (float)T.nu[rk] * rho;
        nn[n] = nr;
      }
      __syncthreads();
      if (n >= NPAD && n < lim - NPAD) {
        float d1, d2, dn;
        const DerivGeomW<float> gf = deriv_geom_w<float>(n, S.dx0, R);
        derivs_w<float>(dn, d2, n, gf, nn);
        derivs_w<float>(d1, d2, n, gf, S.u);
        float t = 2.0f * nr * d2 + 2.0f * dn * d1;
        float tu = 0.0f;
        ddv = S.u[n] + (float)st.dt * t / rho;
        if (THREED) {
          derivs_w<float>(d1, d2, n, gf, S.v);
          t = nr * d2 + dn * d1;
          ddw = S.v[n] + (float)st.dt * t / rho;
        }
        derivs_w<float>(d1, d2, n, gf, S.w);
        tu += nr * d2 + dn * d1;
        ddu = S.w[n] + (float)st.dt * tu / rho;
      }
      __syncthreads();
      if (n >= NPAD && n < lim - NPAD) {
        S.u[n] = ddv;
        if (THREED) S.v[n] = ddw;
        S.w[n] = ddu;
      }
    }
    if (n >= NPAD && n < lim - NPAD) finish(wrapmf(j0 + inc, nphi), sig, S.w[n], S.u[n], THREED ? S.v[n] : 0.f);
  }
  if (ctl.fuse) {
    __syncthreads();
    double m = block_max32(rate, red);
    int anybad = __syncthreads_or(bad);
    if (n == 0) {
      if (!ctl.nocfl && (m > 0.0 || m != m))
        atomicMax(&ctl.clk->cfl_bits, (unsigned long long)__double_as_longlong(m));
      if (anybad) atomicExch(&ctl.clk->status, 3);
    }
  }
}

template <bool SPH, bool THREED, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k32_sweep_y(Tables T, Planes32 P, Phys ph, SweepCtl ctl, int l0) {
  __shared__ ChunkShm32<NT> S;
  __shared__ double red[NT / 32];
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  sweep_y32_body<SPH, THREED, NT>(S, red, T, P, ph, ctl, st, blockIdx.x + l0, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// One polar pencil chunk (ring i, column j0, chunk l), cell n of it; with
// `store` false the pencil is computed and not stored.
template <int NT>
__device__ __forceinline__ void sweep_z32_body(ChunkShm32Data<NT> &S, int n, bool store, const Tables &T,
                                               const Planes32 &P, const Phys &ph, const SweepCtl &ctl,
                                               const StepIn32 &st, int ntop, int i, int j0, int l) {
  const int nphi = T.nphi, nrg = T.nrg, nk = T.nk;
  const int row = i + NPAD;
  const bool last = (l == T.cz.loop - 1);
  if (last && T.cz.stuck) {
    int k = REAL * l + n;
    if (store && n < REAL && k < nk) {
      size_t idx = ((size_t)k * nrg + row) * nphi + j0;
      int inc = ctl.shift ? T.inc_j[k * nrg + row] : 0;
      size_t o = ((size_t)k * nrg + row) * nphi + wrapmf(j0 + inc, nphi);
      P.ro[o] = P.r[idx]; P.uo[o] = P.u[idx]; P.vo[o] = P.v[idx]; P.wo[o] = P.w[idx];
    }
    return;
  }
  const int lim = last ? T.cz.lim_last : ARR;
  const bool act = n < lim;
  const int kr = n - NPAD + REAL * l;
  const double rad = T.rxc[row];
  CellIn32 c{rad, T.yc[j0], 0.0, 0.0, 1.0, 0.0, 1.0};
  // the pencil's planet angle factor at the start of the step, once
  if (n == 0) S.cf0 = ph.plnt ? planet_cosfac(c.azi, st.pl, 0.0) : 0.0;
  double rad_cyl = 1.0, vbg = 0.0, sbg = 0.0;
  if (act) {
    double za, dz, zc, zvol, L;
    float r, p, u, w;
    int kz = kr + NPAD;
    za = T.z[kz]; dz = T.dz[kz]; zc = T.zc[kz]; zvol = T.zvol[kz];
    // sin, cos of the layer's centre and face angles from the tables
    c.sinpol = T.szc[kz]; c.cospol = T.czc[kz]; c.sinfz = T.szf[kz]; c.cosfz = T.czf[kz];
    rad_cyl = rad * c.sinpol;
    if (kr < 0) {
      const double *g = T.tg + ((size_t)kz * T.nr + i) * 4;
      c.sig = g[0];
      r = (float)g[0]; p = (float)g[1]; u = (float)g[2]; w = 0.f;
      L = g[3] * rad_cyl;
      c.vrot = 0.0;
    } else if (kr >= nk) {
      if (ntop == 0) {
        int km = 2 * nk - 1 - kr;
        int rkm = km * nrg + row;
        size_t s = (size_t)rkm * nphi + j0;
        c.sig = T.sbg[rkm] + (double)P.r[s];
        r = (float)c.sig; p = r * (float)T.cs2[rkm]; u = P.u[s]; w = -P.w[s];
        L = (T.vbg[rkm] + (double)P.v[s]) * rad_cyl;
        c.vrot = T.res_v[rkm] / T.radc[rkm];
      } else {
        const double *g = T.tg + ((size_t)(NPAD + (kr - nk)) * T.nr + i) * 4;
        c.sig = g[0];
        r = (float)g[0]; p = (float)g[1]; u = (float)g[2]; w = 0.f;
        L = g[3] * rad_cyl;
        c.vrot = 0.0;
      }
    } else {
      int rkk = kr * nrg + row;
      size_t idx = (size_t)rkk * nphi + j0;
      rad_cyl = T.radc[rkk];
      vbg = T.vbg[rkk];
      sbg = T.sbg[rkk];
      c.sig = sbg + (double)P.r[idx];
      r = (float)c.sig; p = r * (float)T.cs2[rkk]; u = P.u[idx]; w = P.w[idx];
      L = (vbg + (double)P.v[idx]) * rad_cyl;
      c.vrot = T.res_v[rkk] / rad_cyl;
    }
    c.pol = zc;
    c.dvol0 = zvol * rad;
    S.xa0[n] = za;
    S.dx0[n] = (float)dz;
    c.dx0 = dz;
    S.r[n] = r; S.p[n] = p;
    S.u[n] = w;        // v_theta
    S.v[n] = u;        // v_r
    S.L[n] = L;        // r sin(theta) v_phi, FP64
    S.w[n] = 0.f;
  }
  __syncthreads();
  const double sig = ppm_chunk32<2, true, true, NT>(S, n, lim, st.dt, st.frrot, c, st.pl, ph);
  if (ph.visc) {
    float rho = 0.f, nr = 0.f, ddu = 0.f, ddv = 0.f;
    float *nn = S.q;
    const float R = (float)rad;
    if (act) {
      rho = S.r[n];
      double nu = (kr >= 0 && kr < nk) ? T.nu[kr * nrg + row]
                                        : T.nug[(kr < 0 ? kr + NPAD : kr - nk + NPAD) * T.nr + i];
      nr = (float)nu * rho;
      nn[n] = nr;
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      float d1, d2, dn;
      const DerivGeomW<float> gf = deriv_geom_w<float>(n, S.dx0, R);
      derivs_w<float>(dn, d2, n, gf, nn);
      derivs_w<float>(d1, d2, n, gf, S.u);
      ddu = S.u[n] + (float)st.dt * (2.0f * nr * d2 + 2.0f * dn * d1) / rho;
      derivs_w<float>(d1, d2, n, gf, S.v);
      ddv = S.v[n] + (float)st.dt * (nr * d2 + dn * d1) / rho;
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) { S.u[n] = ddu; S.v[n] = ddv; }
  }
  if (store && n >= NPAD && n < lim - NPAD) {
    int rkk = kr * nrg + row;
    int inc = ctl.shift ? T.inc_j[rkk] : 0;
    size_t o = (size_t)rkk * nphi + wrapmf(j0 + inc, nphi);
    P.ro[o] = (float)(sig - sbg);
    P.wo[o] = S.u[n];
    P.uo[o] = S.v[n];
    P.vo[o] = (float)(S.L[n] / rad_cyl - vbg);
  }
}

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k32_sweep_z(Tables T, Planes32 P, Phys ph, SweepCtl ctl, int ntop,
                                                        int l0) {
  __shared__ ChunkShm32<NT> S;
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  sweep_z32_body<NT>(S, threadIdx.x, true, T, P, ph, ctl, st, ntop, blockIdx.x, blockIdx.y, blockIdx.z + l0);
}

// single-chunk polar pencils packed 4 per CTA (the FP64 kernel
// k_sweep_z_packed packs 8 of up to 44 cells)
constexpr int PZ32_LIM = 56;
template <int PACK, int MINB>
__global__ void __launch_bounds__(PACK * PZ32_LIM, MINB) k32_sweep_z_packed(Tables T, Planes32 P, Phys ph,
                                                                            SweepCtl ctl, int ntop) {
  __shared__ ChunkShm32<PZ32_LIM> S[PACK];
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  const int p = threadIdx.x % PACK, n = threadIdx.x / PACK;
  const int npen = T.nr * T.nphi;
  int col = blockIdx.x * PACK + p;
  const bool store = col < npen;
  if (!store) col = npen - 1;
  sweep_z32_body<PZ32_LIM>(S[p], n, store, T, P, ph, ctl, st, ntop, col / T.nphi, col % T.nphi, 0);
}

// Pencils of at most 44 cells (kmax 32) eight per CTA, as the FP64 packed
// polar kernel: 352 threads = 11 whole warps (four pencils of 44 cells fill
// 5.5 warps of a 6-warp CTA), 3 CTAs per SM, shared blocks sized for 44
// cells and padded to 16 mod 128 bytes (dynamic: 8 of them take 50 KB).
constexpr int PZ32_8_THREADS = 352;
constexpr int PZ32_8_LIM = PZ32_8_THREADS / 8;
using Pz32Shm8 = ChunkShm32<PZ32_8_LIM, 16>;
constexpr int pz32_shm8_bytes() { return 8 * (int)sizeof(Pz32Shm8); }
__global__ void __launch_bounds__(PZ32_8_THREADS, 3) k32_sweep_z_packed8(Tables T, Planes32 P, Phys ph, SweepCtl ctl,
                                                                         int ntop) {
  extern __shared__ __align__(16) unsigned char pz32_shm[];
  Pz32Shm8 *S = reinterpret_cast<Pz32Shm8 *>(pz32_shm);
  StepIn32 st;
  if (!load_step32(ctl, st)) return;
  const int p = threadIdx.x % 8, n = threadIdx.x / 8;
  const int npen = T.nr * T.nphi;
  int col = blockIdx.x * 8 + p;
  const bool store = col < npen;
  if (!store) col = npen - 1;
  sweep_z32_body<PZ32_8_LIM>(S[p], n, store, T, P, ph, ctl, st, ntop, col / T.nphi, col % T.nphi, 0);
}

// ---------------------------------------------------------------------------
__global__ void k32_cfl(Tables T, const float *R, const float *U, const float *V, const float *W, Phys ph,
                        double frrot, int ndim, int rot_pending, unsigned long long *out, int *status,
                        DevClock *clk) {
  __shared__ double red[32];
  if (clk) {
    // device-resident loop: after the step's last sweep, with this step's shift pending
    if (clk->halted) return;
    frrot = clk->frrot_next;
    out = &clk->cfl_bits;
    status = &clk->status;
  }
  int i = blockIdx.x, k = blockIdx.y;
  int row = i + NPAD, rk = k * T.nrg + row;
  size_t base = (size_t)rk * T.nphi;
  double rad = T.rxc[row], rad_cyl = T.radc[rk];
  double voff = T.vbg[rk] - T.rot_v[rk] - frrot * rad_cyl;
  int rotn = T.rot_j[rk] + (rot_pending ? T.inc_j[rk] : 0);
  double rate = 0.0;
  bool bad = false;
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    int js = wrapmf(j - rotn, T.nphi);
    double r = T.sbg[rk] + (double)R[base + j];
    double p = r * T.cs2[rk];
    double cs = sqrt(ph.gam * p / r);
    double t0 = (fabs((double)U[base + j]) + cs) / T.rdx[row];
    double t1 = (fabs((double)V[base + j] + voff) + cs) / (T.dy[js] * rad_cyl);
    double rt;
    if (ndim == 3) {
      double t2 = (fabs((double)W[base + j]) + cs) / (T.dz[k + NPAD] * rad);
      rt = max3(t0, t1, t2);
    } else {
      rt = fmax(t0, t1);
    }
    rate = (rt > rate || rt != rt) ? rt : rate;
    if (!(r > 0.0) || !isfinite(r) || !isfinite(U[base + j]) || !isfinite(V[base + j])) bad = true;
  }
  double m = block_max32(rate, red);
  int anybad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    if (m > 0.0 || m != m) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    if (anybad && status) atomicExch(status, 3);
  }
}

__global__ void k32_damp(Tables T, float *R, float *U, float *V, float *W, double dt, const DevClock *clk,
                         int ndim) {
  if (clk) {
    if (clk->halted) return;
    dt = clk->dt_step;
  }
  int i = blockIdx.x, k = blockIdx.y;
  int rk = k * T.nrg + i + NPAD;
  double g = T.damp_g[rk];
  if (!(g > 0.0)) return;
  double fd = g * (dt * T.damp_pw[rk]);
  float f = (float)fd;
  size_t base = (size_t)rk * T.nphi;
  double sbg = T.sbg[rk], vr = T.val_r[rk];
  float vu = (float)T.val_u[rk];
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    double sig = sbg + (double)R[base + j];
    sig += fd * (vr - sig);
    R[base + j] = (float)(sig - sbg);
    U[base + j] += f * (vu - U[base + j]);
    V[base + j] += f * (-V[base + j]);
    if (ndim == 3) W[base + j] += f * (-W[base + j]);
  }
}

// ---------------------------------------------------------------------------
// Batched FP32 sweeps: tiles of every run of a group in one launch (see the
// FP64 batched kernels in pg_kernels.cu for the tile queue).
__device__ __forceinline__ int batch_find32(const BatchQueue &q, int t) {
  int lo = 0, hi = q.nruns;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (q.start[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) kb32_sweep_x(BatchQueue q) {
  __shared__ ChunkShm32<128> S;
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find32(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    StepIn32 st;
    if (load_step32(ctl, st)) {
      const int lt = t - q.start[r], nphi = b.T.nphi;
      sweep_x32_body<false, false, 128>(S, threadIdx.x, true, b.T, b.QX, b.ph, ctl, st, lt % nphi, lt / nphi, 0);
    }
    __syncthreads();
  }
}

// radial last chunks of at most 64 cells, 4 columns per tile (see kb_sweep_x_short)
__global__ void __launch_bounds__(256, 4) kb32_sweep_x_short(BatchQueue q) {
  __shared__ ChunkShm32<64> S[4];
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find32(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    StepIn32 st;
    if (load_step32(ctl, st)) {
      const int p = threadIdx.x & 3, n = threadIdx.x >> 2, nphi = b.T.nphi;
      int col = 4 * (t - q.start[r]) + p;
      const bool store = col < nphi;
      if (!store) col = nphi - 1;
      sweep_x32_body<false, false, 64>(S[p], n, store, b.T, b.QX, b.ph, ctl, st, col, b.T.cx.loop - 1, 0);
    }
    __syncthreads();
  }
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) kb32_sweep_y(BatchQueue q) {
  __shared__ ChunkShm32<128> S;
  __shared__ double red[4];
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find32(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    ctl.fuse = 1;
    ctl.shift = 1;
    StepIn32 st;
    if (load_step32(ctl, st)) {
      const int lt = t - q.start[r], loop = b.T.cy.loop;
      sweep_y32_body<false, false, 128>(S, red, b.T, b.QY, b.ph, ctl, st, lt % loop, lt / loop, 0);
    }
    __syncthreads();
  }
}

}  // namespace pgd

namespace pgk {
using namespace pgd;

static inline int cta_for32(int lim) { return lim <= 32 ? 32 : (lim <= 64 ? 64 : 128); }

// 128-thread FP32 sweeps: the radial kernel at 4 CTAs per SM (80 registers;
// at 64 it spills and runs slower), the azimuthal one at 8 (64 registers, no
// spills in 2D: 6-9 % faster than at 80)
#define PG32_X(SPHV, TD, NTV, grid, l0)                                                          \
  do {                                                                                           \
    if ((NTV) == 128) k32_sweep_x<SPHV, TD, 128, 4><<<grid, 128, 0, s>>>(T, P, ph, c, l0);       \
    else if ((NTV) == 64) k32_sweep_x<SPHV, TD, 64, 1><<<grid, 64, 0, s>>>(T, P, ph, c, l0);     \
    else k32_sweep_x<SPHV, TD, 32, 1><<<grid, 32, 0, s>>>(T, P, ph, c, l0);                      \
  } while (0)
#define PG32_Y(SPHV, TD, NTV, grid, l0)                                                          \
  do {                                                                                           \
    if ((NTV) == 128) k32_sweep_y<SPHV, TD, 128, 8><<<grid, 128, 0, s>>>(T, P, ph, c, l0);       \
    else if ((NTV) == 64) k32_sweep_y<SPHV, TD, 64, 1><<<grid, 64, 0, s>>>(T, P, ph, c, l0);     \
    else k32_sweep_y<SPHV, TD, 32, 1><<<grid, 32, 0, s>>>(T, P, ph, c, l0);                      \
  } while (0)

// A last chunk of more than 64 cells runs in the full chunks' launch (the
// bodies give chunk loop-1 its lim_last), as in the FP64 sweeps.
void sweep_x32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  const Chunking &ch = T.cx;
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  const bool merge = !ch.stuck && full > 0 && ch.lim_last > 64;
  if (merge) full = ch.loop;
  if (full > 0) {
    if (!ch.stuck && T.xpack == 2) {
      // two adjacent columns per 256-thread CTA (a stuck last chunk keeps
      // the one-column kernel)
      dim3 grid((T.nphi + 1) / 2, full, T.nk);
      if (ndim == 3) k32_sweep_x_cols<true, true, 2, 3><<<grid, 2 * ARR, px32_shm_bytes<2>(), s>>>(T, P, ph, c);
      else k32_sweep_x_cols<false, false, 2, 3><<<grid, 2 * ARR, px32_shm_bytes<2>(), s>>>(T, P, ph, c);
    } else {
      dim3 grid(T.nphi, full, T.nk);
      if (ndim == 3) PG32_X(true, true, 128, grid, 0);
      else PG32_X(false, false, 128, grid, 0);
    }
  }
  if (!ch.stuck && !merge) {
    if (T.zpack && ch.lim_last <= PX32_LIM) {
      int npen = T.nphi * T.nk, blocks = (npen + 3) / 4, nt = 4 * ch.lim_last;
      if (ndim == 3) k32_sweep_x_packed<true, true, 4><<<blocks, nt, 0, s>>>(T, P, ph, c);
      else k32_sweep_x_packed<false, false, 4><<<blocks, nt, 0, s>>>(T, P, ph, c);
      return;
    }
    dim3 grid(T.nphi, 1, T.nk);
    int nt = cta_for32(ch.lim_last), l0 = ch.loop - 1;
    if (ndim == 3) PG32_X(true, true, nt, grid, l0);
    else PG32_X(false, false, nt, grid, l0);
  }
}

void sweep_y32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  const Chunking &ch = T.cy;
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  const bool merge = !ch.stuck && full > 0 && ch.lim_last > 64;
  if (merge) full = ch.loop;
  if (full > 0) {
    dim3 grid(full, T.nr, T.nk);
    if (ndim == 3) PG32_Y(true, true, 128, grid, 0);
    else PG32_Y(false, false, 128, grid, 0);
  }
  if (!ch.stuck && !merge) {
    dim3 grid(1, T.nr, T.nk);
    int nt = cta_for32(ch.lim_last), l0 = ch.loop - 1;
    if (ndim == 3) PG32_Y(true, true, nt, grid, l0);
    else PG32_Y(false, false, nt, grid, l0);
  }
}

// the 8-pencil FP32 polar kernel's shared blocks exceed the 48 KiB default
int setup_device32() {
  return cudaFuncSetAttribute(k32_sweep_z_packed8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              pz32_shm8_bytes()) == cudaSuccess ? 0 : 1;
}

void sweep_z32(const Tables &T, const Planes32 &P, const Phys &ph, const SweepCtl &c, int ntop, cudaStream_t s) {
  const Chunking &ch = T.cz;
  if (T.zpack && ch.loop == 1 && !ch.stuck && ch.lim_last <= PZ32_LIM) {
    int npen = T.nr * T.nphi;
    if (8 * ch.lim_last <= PZ32_8_THREADS)
      k32_sweep_z_packed8<<<(npen + 7) / 8, 8 * ch.lim_last, pz32_shm8_bytes(), s>>>(T, P, ph, c, ntop);
    else
      k32_sweep_z_packed<4, 5><<<(npen + 3) / 4, 4 * ch.lim_last, 0, s>>>(T, P, ph, c, ntop);
    return;
  }
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  const bool merge = !ch.stuck && full > 0 && ch.lim_last > 64;
  if (merge) full = ch.loop;
  if (full > 0) {
    dim3 grid(T.nr, T.nphi, full);
    k32_sweep_z<128, 4><<<grid, 128, 0, s>>>(T, P, ph, c, ntop, 0);
  }
  if (!ch.stuck && !merge) {
    dim3 grid(T.nr, T.nphi, 1);
    int nt = cta_for32(ch.lim_last), l0 = ch.loop - 1;
    if (nt == 32) k32_sweep_z<32, 1><<<grid, 32, 0, s>>>(T, P, ph, c, ntop, l0);
    else if (nt == 64) k32_sweep_z<64, 1><<<grid, 64, 0, s>>>(T, P, ph, c, ntop, l0);
    else k32_sweep_z<128, 4><<<grid, 128, 0, s>>>(T, P, ph, c, ntop, l0);
  }
}

void cfl32(const Tables &T, const Planes32 &cur, const Phys &ph, double frrot, int ndim, int rot_pending,
           unsigned long long *out, int *status, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k32_cfl<<<grid, 256, 0, s>>>(T, cur.r, cur.u, cur.v, cur.w, ph, frrot, ndim, rot_pending, out, status, nullptr);
}

void cfl32_clk(const Tables &T, const Planes32 &cur, const Phys &ph, int ndim, DevClock *clk, cudaStream_t s,
               int rot_pending) {
  dim3 grid(T.nr, T.nk);
  k32_cfl<<<grid, 256, 0, s>>>(T, cur.r, cur.u, cur.v, cur.w, ph, 0.0, ndim, rot_pending, nullptr, nullptr, clk);
}

void damp32(const Tables &T, const Planes32 &cur, double dt, const DevClock *clk, int ndim, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k32_damp<<<grid, 256, 0, s>>>(T, cur.ro, cur.uo, cur.vo, cur.wo, dt, clk, ndim);
}


void batch_sweep_x32(const BatchQueue &q, int grid, int minb, cudaStream_t s) {
  if (q.total <= 0) return;
  int g = (grid > 0 && grid < q.total) ? grid : q.total;
  if (minb >= 8) kb32_sweep_x<8><<<g, 128, 0, s>>>(q);
  else kb32_sweep_x<4><<<g, 128, 0, s>>>(q);
}
void batch_sweep_x32_short(const BatchQueue &q, cudaStream_t s) {
  if (q.total > 0) kb32_sweep_x_short<<<q.total, 256, 0, s>>>(q);
}
void batch_sweep_y32(const BatchQueue &q, int grid, int minb, cudaStream_t s) {
  if (q.total <= 0) return;
  int g = (grid > 0 && grid < q.total) ? grid : q.total;
  if (minb >= 8) kb32_sweep_y<8><<<g, 128, 0, s>>>(q);
  else kb32_sweep_y<4><<<g, 128, 0, s>>>(q);
}

}  // namespace pgk
