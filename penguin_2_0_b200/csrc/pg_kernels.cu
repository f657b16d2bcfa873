// pg_kernels.cu -- sm_100a kernels of the hydro step.
//
//   k_sweep_x   radial sweep (ppm.cu:26-160), one CTA per (phi column, chunk, k)
//   k_sweep_y   azimuthal sweep (ppm.cu:162-307), one CTA per (chunk, ring);
//               the FARGO integer shift (rotate_rings, ppm.cu:309-322) is
//               applied at its store; optional fused epilogue: wave damping,
//               CFL rate max (dt_lv1, timestep.cu:12-73) and a finiteness
//               check into the run's status word
//   k_sweep_z   polar sweep (3D), one CTA per (ring i, phi column, chunk)
//   k_cfl       standalone CFL rate max
//   k_index     Index_Shift (orbital_advection.cu:12-43)
//   k_reduce    output_lv1/lv2/lv3 (device_func.cu:49-167) in the same tree
//               order, finished by the last CTA
//   k_prestep / k_poststep  the scalar part of main.cu:343-441 on device
#include "pg_chunk.cuh"
#include "pg_kernels.cuh"

namespace pgd {

__device__ __forceinline__ int wrap1(int j, int n) {
  if (j < 0) j += n;
  if (j >= n) j -= n;
  return j;
}
__device__ __forceinline__ int wrapm(int j, int n) {
  j %= n;
  return j < 0 ? j + n : j;
}

// ordered encoding of a non-negative double (NaN sorts above +inf)
__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ double block_max(double v, double *red) {
  // reduce within the CTA; only thread 0's result is meaningful
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

// The step's dt, planet and frame rotation: either the launch arguments or
// the device clock of the fused loop.
struct StepIn {
  double dt, frrot, frrot_next;
  Body pl;
};
__device__ __forceinline__ bool load_step(const SweepCtl &c, StepIn &s) {
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

// ---------------------------------------------------------------------------
// radial sweep
// One radial pencil chunk: column j0, chunk l, polar layer k.  The body is
// shared by the per-run kernel and the batched kernels of pg_batch.cu.
template <bool SPH, bool THREED, int NT, int EOS = 0>
__device__ __forceinline__ void sweep_x_body(ChunkShmData<NT> &S, int n, bool store, const Tables &T, const Planes &P,
                                             const Phys &ph, const SweepCtl &ctl, const StepIn &st, int j0, int l,
                                             int k) {
  const bool last = (l == T.cx.loop - 1);
  const int nphi = T.nphi, nrg = T.nrg;
  if (last && T.cx.stuck) {
    // ppm.cu:48 gives this chunk lim = 12: its rings keep their values
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
  const int row = n + REAL * l;              // ghost-inclusive radial row
  const int rk = k * nrg + row;
  const size_t idx = (size_t)rk * nphi + j0;
  CellIn c;
  double rad_cyl = 1.0;
  if (act) {
    c.rad = T.rxc[row];
    rad_cyl = T.radc[rk];
    c.azi = T.yc[j0];
    c.pol = THREED ? T.zc[k + NPAD] : 0.0;
    c.sinpol = THREED ? T.szc[k + NPAD] : 0.0;
    c.dvol0 = T.rxvol[row];
    // the pencil's planet angle factor at the start of the step, once
    if (n == 0) S.cf0 = ph.plnt ? planet_cosfac(c.azi, st.pl, 0.0) : 0.0;
    c.vrot = T.res_v[rk] / rad_cyl;
    S.xa0[n] = T.rx[row];
    S.dx0[n] = T.rdx[row];
    double r = P.r[idx];
    S.r[n] = r;
    S.u[n] = P.u[idx];
    S.v[n] = P.v[idx] * rad_cyl;
    if (THREED) S.w[n] = P.w[idx] * c.rad;
    else S.w[n] = 0.0;
    bool ghost = (row < NPAD) || (row >= T.nr + NPAD);
    S.p[n] = ghost ? T.gp[rk] : (P.p0 ? P.p0[idx] : eos_p<EOS>(r, T.cs2[rk], ph));
  } else {
    c.rad = 1.0; c.azi = 0.0; c.pol = 0.0; c.dvol0 = 1.0; c.vrot = 0.0; c.sinpol = 0.0;
  }
  __syncthreads();
  ppm_chunk<0, SPH, THREED, EOS>(S, n, lim, st.dt, st.frrot, c, st.pl, ph);
  // device_viscosity_r viscosity.cu:370-421 (nu*rho scratch in dx0)
  if (ph.visc) {
    const double R = rad_cyl;
    double rho = 0.0, nr = 0.0, ddu = 0.0, ddv = 0.0, ddw = 0.0;
    if (act) {
      rho = S.r[n];
      nr = T.nu[rk] * rho;
      S.dx0[n] = nr;
      S.v[n] /= R * R;
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      double d1, d2, dn;
      const DerivGeom g = deriv_geom(n, S.xa0);
      const double iR = 1.0 / R, dtr = st.dt / rho;
      derivs_g(dn, d2, n, g, S.dx0);
      derivs_g(d1, d2, n, g, S.u);
      double t = 2.0 * nr * d2 + 2.0 * dn * d1 + 2.0 * nr * d1 * iR - 2.0 * nr * S.u[n] * iR * iR;
      ddu = S.u[n] + t * dtr;
      derivs_g(d1, d2, n, g, S.v);
      t = R * nr * d2 + R * dn * d1 + 3.0 * nr * d1;
      ddv = S.v[n] * R + t * dtr;
      if (THREED) {
        derivs_g(d1, d2, n, g, S.w);
        t = nr * d2 + dn * d1 + nr * d1 * iR;
        ddw = S.w[n] + t * dtr;
      }
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      S.u[n] = ddu;
      S.v[n] = ddv * R;
      if (THREED) S.w[n] = ddw;
    }
  }
  if (store && n >= NPAD && n < lim - NPAD) {
    P.ro[idx] = S.r[n];
    P.uo[idx] = S.u[n];
    P.vo[idx] = S.v[n] / rad_cyl;
    if (THREED) P.wo[idx] = S.w[n] / c.rad;
  }
}

template <bool SPH, bool THREED, int NT, int MINB, int EOS = 0>
__global__ void __launch_bounds__(NT, MINB) k_sweep_x(Tables T, Planes P, Phys ph, SweepCtl ctl, int l0) {
  __shared__ ChunkShmT<NT> S;
  StepIn st;
  if (!load_step(ctl, st)) return;
  sweep_x_body<SPH, THREED, NT, EOS>(S, threadIdx.x, true, T, P, ph, ctl, st, blockIdx.x, blockIdx.y + l0, blockIdx.z);
}

// The short last chunk of radial pencils (lim <= 64 cells): 4 adjacent
// columns share a CTA of 4 * lim threads, thread t on cell t / 4 of column
// t % 4 (a warp's loads of one ring cover 4 adjacent doubles), instead of one
// column per 32/64-thread CTA with idle lanes.  Columns past the last one
// repeat it without storing.
// A last chunk of at most 32 cells (the 128-ring disk's is 12 + 12) takes
// shared blocks sized for 32: 4.9 KB per pencil instead of 9.5, so about
// twice as many CTAs fit on an SM.
constexpr int PX_LIM = 64;
template <bool SPH, bool THREED, int MINB, int LIM = PX_LIM>
__global__ void __launch_bounds__(4 * LIM, MINB) k_sweep_x_packed(Tables T, Planes P, Phys ph, SweepCtl ctl) {
  __shared__ ChunkShmT<LIM> S[4];
  StepIn st;
  if (!load_step(ctl, st)) return;
  const int p = threadIdx.x & 3, n = threadIdx.x >> 2;
  const int npen = T.nphi * T.nk;
  int col = blockIdx.x * 4 + p;
  const bool store = col < npen;
  if (!store) col = npen - 1;
  sweep_x_body<SPH, THREED, LIM>(S[p], n, store, T, P, ph, ctl, st, col % T.nphi, T.cx.loop - 1, col / T.nphi);
}

// Full radial chunks (and a last chunk of more than 64 cells, in the same
// launch) of PACK adjacent columns per CTA (128 * PACK threads,
// thread t on cell t / PACK of column t % PACK): a warp's loads and stores of
// one ring cover PACK adjacent doubles, where one column per CTA touches a
// separate 32-byte sector per cell.  Columns past the last one repeat it
// without storing.  The pencils' shared blocks are dynamic (4 of them exceed
// the 48 KiB a kernel may declare statically) and padded to 128 / PACK mod
// 128 bytes, so the pencils' accesses fall in different banks.
template <int PACK>
using PxShm = ChunkShmT<ARR, 128 / PACK>;
template <int PACK>
constexpr int px_shm_bytes() { return PACK * (int)sizeof(PxShm<PACK>); }
template <bool SPH, bool THREED, int PACK, int MINB>
__global__ void __launch_bounds__(ARR * PACK, MINB) k_sweep_x_cols(Tables T, Planes P, Phys ph, SweepCtl ctl) {
  extern __shared__ __align__(16) unsigned char px_shm[];
  PxShm<PACK> *S = reinterpret_cast<PxShm<PACK> *>(px_shm);
  StepIn st;
  if (!load_step(ctl, st)) return;
  const int p = threadIdx.x % PACK, n = threadIdx.x / PACK;
  int col = blockIdx.x * PACK + p;
  const bool store = col < T.nphi;
  if (!store) col = T.nphi - 1;
  sweep_x_body<SPH, THREED, ARR>(S[p], n, store, T, P, ph, ctl, st, col, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// azimuthal sweep with the FARGO shift at the store and the fused epilogue
// One azimuthal chunk: chunk l of ring i in polar layer k; FARGO shift at
// the store and, with ctl.fuse, damping and the CFL rate in the epilogue.
template <bool SPH, bool THREED, int NT, int EOS = 0>
__device__ __forceinline__ void sweep_y_body(ChunkShmT<NT> &S, double *red, const Tables &T, const Planes &P,
                                             const Phys &ph, const SweepCtl &ctl, const StepIn &st, int l, int i,
                                             int k) {
  const int n = threadIdx.x;
  const int nphi = T.nphi, nrg = T.nrg;
  const int row = i + NPAD;
  const int rk = k * nrg + row;
  const size_t base = (size_t)rk * nphi;
  const int inc = ctl.shift ? T.inc_j[rk] : 0;
  const bool last = (l == T.cy.loop - 1);
  const double rad = T.rxc[row];
  const double rad_cyl = T.radc[rk];
  double rate = 0.0;
  bool bad = false;
  double dampf = 0.0;
  bool do_damp = false;
  if (ctl.fuse) {
    double g = T.damp_g[rk];
    if (g > 0.0) { do_damp = true; dampf = g * (st.dt * T.damp_pw[rk]); }
  }
  // stores one finished cell at physical column jo (post-shift)
  auto finish = [&](int jo, double r, double u, double v, double w) {
    if (ctl.fuse) {
      if (do_damp) {
        r += dampf * (T.val_r[rk] - r);
        u += dampf * (T.val_u[rk] - u);
        v += dampf * (T.val_v[rk] - v);
        if (THREED) w += dampf * (-w);
      }
      // dt_lv1 timestep.cu:36-57 on the stored state (p by the EOS relation)
      double p = eos_p<EOS>(r, T.cs2[rk], ph);
      double cs = sqrt(ph.gam * p / r);
      int js = wrapm(jo - (T.rot_j[rk] + inc), nphi);
      double widthy = T.dy[js] * rad_cyl;
      double t0 = (fabs(u) + cs) / T.rdx[row];
      double t1 = (fabs(v - T.rot_v[rk] - st.frrot_next * rad_cyl) + cs) / widthy;
      double rt;
      if (THREED) {
        double t2 = (fabs(w) + cs) / (T.dz[k + NPAD] * rad);
        rt = max3(t0, t1, t2);
      } else {
        rt = fmax(t0, t1);
      }
      rate = (rt > rate || rt != rt) ? rt : rate;
      if (!(r > 0.0) || !isfinite(r) || !isfinite(u) || !isfinite(v)) bad = true;
    }
    size_t o = base + jo;
    P.ro[o] = r; P.uo[o] = u; P.vo[o] = v;
    if (THREED) P.wo[o] = w;
  };
  // the cell this thread stores, if any: finish() is called once below, so
  // the fused epilogue appears once in the kernel's code
  int jo_st = -1;
  double st_r = 0.0, st_u = 0.0, st_v = 0.0, st_w = 0.0;
  if (last && T.cy.stuck) {
    // ppm.cu:196 gives this chunk lim = 12: its cells keep their values and
    // only move with the ring's rotation
    int j = REAL * l + n;
    if (n < REAL && j < nphi) {
      size_t s = base + j;
      jo_st = wrapm(j + inc, nphi);
      st_r = P.r[s]; st_u = P.u[s]; st_v = P.v[s]; st_w = THREED ? P.w[s] : 0.0;
    }
  } else {
    const int lim = last ? T.cy.lim_last : ARR;
    const bool act = n < lim;
    const int jref = n - NPAD + REAL * l;
    const int j0 = wrap1(jref, nphi);
    CellIn c;
    c.rad = rad_cyl;
    c.pol = THREED ? T.zc[k + NPAD] : 0.0;
    c.sinpol = THREED ? T.szc[k + NPAD] : 0.0;
    c.vrot = T.res_v[rk] / rad_cyl;
    c.azi = 0.0; c.dvol0 = 1.0;
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
      S.dx0[n] = T.dy[j0];
      double r = P.r[s];
      S.r[n] = r;
      S.p[n] = eos_p<EOS>(r, T.cs2[rk], ph);
      S.u[n] = P.v[s];
      S.v[n] = THREED ? P.w[s] : 0.0;
      S.w[n] = P.u[s];
    }
    __syncthreads();
    ppm_chunk<1, SPH, THREED, EOS>(S, n, lim, st.dt, st.frrot, c, st.pl, ph);
    // device_viscosity_p viscosity.cu:423-472 with x = r_cyl * phi_face,
    // u -> w slot (v_r), v -> u slot (v_phi), w -> v slot (v_theta)
    if (ph.visc) {
      const double R = rad_cyl;
      double rho = 0.0, nr = 0.0, ddu = 0.0, ddv = 0.0, ddw = 0.0;
      if (act) {
        S.xa0[n] *= R;
        rho = S.r[n];
        nr = T.nu[rk] * rho;
        S.dx0[n] = nr;
      }
      __syncthreads();
      if (n >= NPAD && n < lim - NPAD) {
        double d1, d2, dn;
        const DerivGeom g = deriv_geom(n, S.xa0);
        const double dtr = st.dt / rho;
        derivs_g(dn, d2, n, g, S.dx0);
        derivs_g(d1, d2, n, g, S.u);
        double t = 2.0 * nr * d2 + 2.0 * dn * d1;
        double tu = 0.0;
        ddv = S.u[n] + t * dtr;
        if (THREED) {
          derivs_g(d1, d2, n, g, S.v);
          t = nr * d2 + dn * d1;
          ddw = S.v[n] + t * dtr;
        }
        derivs_g(d1, d2, n, g, S.w);
        tu += nr * d2 + dn * d1;
        ddu = S.w[n] + tu * dtr;
      }
      __syncthreads();
      if (n >= NPAD && n < lim - NPAD) {
        S.u[n] = ddv;
        if (THREED) S.v[n] = ddw;
        S.w[n] = ddu;
      }
    }
    if (n >= NPAD && n < lim - NPAD) {
      jo_st = wrapm(j0 + inc, nphi);
      st_r = S.r[n]; st_u = S.w[n]; st_v = S.u[n]; st_w = THREED ? S.v[n] : 0.0;
    }
  }
  if (jo_st >= 0) finish(jo_st, st_r, st_u, st_v, st_w);
  if (ctl.fuse) {
    __syncthreads();
    double m = block_max(rate, red);
    int anybad = __syncthreads_or(bad);
    if (n == 0) {
      if (!ctl.nocfl && (m > 0.0 || m != m)) atomicMax(&ctl.clk->cfl_bits, dbits(m));
      if (anybad) atomicExch(&ctl.clk->status, 3);
    }
  }
}

template <bool SPH, bool THREED, int NT, int MINB, int EOS = 0>
__global__ void __launch_bounds__(NT, MINB) k_sweep_y(Tables T, Planes P, Phys ph, SweepCtl ctl, int l0) {
  __shared__ ChunkShmT<NT> S;
  __shared__ double red[NT / 32];
  StepIn st;
  if (!load_step(ctl, st)) return;
  sweep_y_body<SPH, THREED, NT, EOS>(S, red, T, P, ph, ctl, st, blockIdx.x + l0, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// polar-angle sweep (3D, ngeomz 5): no reference kernel exists
// (bundle_sweep3D is called at main.cu:376 and never defined).  Modelled on
// the radial sweep: pencils along k for one (i, phi column), fixed lower
// layers (init.cpp:415-476) and a reflecting midplane (boundary.cu:412-418,
// mirror with v_theta negated) or fixed upper layers.  Slots: u <- v_theta,
// v <- v_r, w <- r sin(theta) v_phi (so get_fz's w^2 cos/(r sin)^3 is the
// centrifugal term); viscosity follows device_viscosity_p's pattern on the
// arc length r*theta.
//
// One pencil chunk: ring i, column j0, chunk l; n is this thread's cell in
// the chunk and `store` false computes without storing (padding pencils of
// the packed kernel).
template <int NT, int EOS = 0>
__device__ __forceinline__ void sweep_z_body(ChunkShmData<NT> &S, int n, bool store, const Tables &T, const Planes &P,
                                             const Phys &ph, const SweepCtl &ctl, const StepIn &st, int ntop,
                                             int i, int j0, int l) {
  const int nphi = T.nphi, nrg = T.nrg, nk = T.nk;
  const int row = i + NPAD;
  const bool last = (l == T.cz.loop - 1);
  // with ctl.fuse (a 3D step whose polar chunks are never idle) the store
  // also damps and takes the next get_dt's CFL rate, as the separate damping
  // and CFL kernels would on the stored state (k_damp_clk, k_cfl_clk)
  __shared__ unsigned long long s_rate;
  __shared__ int s_bad;
  if (ctl.fuse && threadIdx.x == 0) { s_rate = 0ull; s_bad = 0; }
  if (last && T.cz.stuck) {
    int k = REAL * l + n;
    if (store && n < REAL && k < nk) {
      size_t idx = ((size_t)k * nrg + row) * nphi + j0;
      int inc = ctl.shift ? T.inc_j[k * nrg + row] : 0;
      size_t o = ((size_t)k * nrg + row) * nphi + wrapm(j0 + inc, nphi);
      P.ro[o] = P.r[idx]; P.uo[o] = P.u[idx]; P.vo[o] = P.v[idx]; P.wo[o] = P.w[idx];
    }
    return;
  }
  const int lim = last ? T.cz.lim_last : ARR;
  const bool act = n < lim;
  const int kr = n - NPAD + REAL * l;   // layer, -6 .. nk+5
  const double rad = T.rxc[row];
  CellIn c;
  c.rad = rad;
  c.azi = T.yc[j0];
  c.pol = 0.0; c.vrot = 0.0; c.dvol0 = 1.0; c.sinpol = 0.0;
  c.lay = T.szc; c.nz = nk + 2 * NPAD;
  // the pencil's planet angle factor at the start of the step, and its
  // sine (the polar chain's angle additions), once
  if (n == 0) {
    S.cf0 = ph.plnt ? planet_cosfac(c.azi, st.pl, 0.0) : 0.0;
    S.sf0 = ph.plnt ? sin(c.azi - (st.pl.y + 0.0 * st.pl.vy)) : 0.0;
    S.irad = 1.0 / rad;
    const double stm = 1.0 / (1.0 + st.pl.m);
    S.plm = st.pl.m * stm;
  }
  double rad_cyl = 1.0;
  size_t idx = 0;
  if (act) {
    double za, dz, zc, zvol;
    double r, p, u, v, w;
    if (kr < 0) {
      // fixed lower layer udr[kk + 6 i] (phi uniform, never rotated)
      int kk = kr + NPAD;
      za = T.z[kk]; dz = T.dz[kk]; zc = T.zc[kk]; zvol = T.zvol[kk];
      const double *g = T.tg + ((size_t)kk * T.nr + i) * 4;
      r = g[0]; p = g[1]; u = g[2]; v = g[3]; w = 0.0;
      rad_cyl = rad * T.szc[kk];
      c.vrot = 0.0;
    } else if (kr >= nk) {
      int km = 2 * nk - 1 - kr;          // mirror layer
      int kz = kr + NPAD;                // ghost geometry slot
      za = T.z[kz]; dz = T.dz[kz]; zc = T.zc[kz]; zvol = T.zvol[kz];
      rad_cyl = rad * T.szc[kz];
      if (ntop == 0) {
        int rkm = km * nrg + row;
        size_t s = (size_t)rkm * nphi + j0;
        r = P.r[s]; p = eos_p<EOS>(r, T.cs2[rkm], ph); u = P.u[s]; v = P.v[s]; w = -P.w[s];
        c.vrot = T.res_v[rkm] / T.radc[rkm];
      } else {
        const double *g = T.tg + ((size_t)(NPAD + (kr - nk)) * T.nr + i) * 4;
        r = g[0]; p = g[1]; u = g[2]; v = g[3]; w = 0.0;
        c.vrot = 0.0;
      }
    } else {
      int kz = kr + NPAD;
      int rkk = kr * nrg + row;
      za = T.z[kz]; dz = T.dz[kz]; zc = T.zc[kz]; zvol = T.zvol[kz];
      rad_cyl = T.radc[rkk];
      idx = (size_t)rkk * nphi + j0;
      r = P.r[idx]; p = eos_p<EOS>(r, T.cs2[rkk], ph); u = P.u[idx]; v = P.v[idx]; w = P.w[idx];
      c.vrot = T.res_v[rkk] / rad_cyl;
    }
    c.pol = zc;
    c.lay = T.szc + (kr + NPAD);      // sin, cos of the layer's centre angle
    c.nz = nk + 2 * NPAD;             // and of its left face angle
    c.dvol0 = zvol * rad;
    S.xa0[n] = za;
    S.dx0[n] = dz;
    S.r[n] = r; S.p[n] = p;
    S.u[n] = w;                 // v_theta
    S.v[n] = u;                 // v_r
    S.w[n] = v * rad_cyl;       // angular momentum about the axis
  }
  __syncthreads();
  ppm_chunk<2, true, true, EOS>(S, n, lim, st.dt, st.frrot, c, st.pl, ph, T.zpar + 5 * REAL * l);
  if (ph.visc) {
    double rho = 0.0, nr = 0.0, ddu = 0.0, ddv = 0.0;
    if (act) {
      S.xa0[n] *= rad;
      rho = S.r[n];
      // nu at this layer's r sin(theta): the table for interior layers, the
      // same expression (get_nu disk_profile.cu:149-152) for ghost layers
      double nu = (kr >= 0 && kr < nk) ? T.nu[kr * nrg + row]
                                        : T.nug[(kr < 0 ? kr + NPAD : kr - nk + NPAD) * T.nr + i];
      nr = nu * rho;
      S.dx0[n] = nr;
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) {
      double d1, d2, dn;
      const DerivGeom g = deriv_geom(n, S.xa0);
      const double dtr = st.dt / rho;
      derivs_g(dn, d2, n, g, S.dx0);
      derivs_g(d1, d2, n, g, S.u);
      ddu = S.u[n] + (2.0 * nr * d2 + 2.0 * dn * d1) * dtr;
      derivs_g(d1, d2, n, g, S.v);
      ddv = S.v[n] + (nr * d2 + dn * d1) * dtr;
    }
    __syncthreads();
    if (n >= NPAD && n < lim - NPAD) { S.u[n] = ddu; S.v[n] = ddv; }
  }
  if (store && n >= NPAD && n < lim - NPAD) {
    // the polar sweep is the last of a 3D step: the FARGO integer shift of
    // each layer (rotate_rings, ppm.cu:309-322) is applied at this store
    const int rkk = kr * nrg + row;
    int inc = ctl.shift ? T.inc_j[rkk] : 0;
    const int jo = wrapm(j0 + inc, nphi);
    size_t o = (size_t)rkk * nphi + jo;
    // an interior cell's rad_cyl is radc (read again here rather than held
    // through the chain)
    double r = S.r[n], vr = S.v[n], vp = S.w[n] / T.radc[rkk], vt = S.u[n];
    if (ctl.fuse) {
      const double g = T.damp_g[rkk];
      if (g > 0.0) {
        const double f = g * (st.dt * T.damp_pw[rkk]);
        r += f * (T.val_r[rkk] - r);
        vr += f * (T.val_u[rkk] - vr);
        vp += f * (T.val_v[rkk] - vp);
        vt += f * (-vt);
      }
      if (!ctl.nocfl) {
        const double rad_c = T.radc[rkk];
        const int js = wrapm(jo - (T.rot_j[rkk] + inc), nphi);
        double p = eos_p<EOS>(r, T.cs2[rkk], ph);
        double cs = sqrt(ph.gam * p / r);
        double t0 = (fabs(vr) + cs) / T.rdx[row];
        double t1 = (fabs(vp - T.rot_v[rkk] - st.frrot_next * rad_c) + cs) / (T.dy[js] * rad_c);
        double t2 = (fabs(vt) + cs) / (T.dz[kr + NPAD] * rad);
        double rt = max3(t0, t1, t2);
        if (rt > 0.0 || rt != rt) atomicMax(&s_rate, dbits(rt));
      }
      if (!(r > 0.0) || !isfinite(r) || !isfinite(vr) || !isfinite(vp)) s_bad = 1;
    }
    P.ro[o] = r;
    P.wo[o] = vt;
    P.uo[o] = vr;
    P.vo[o] = vp;
  }
  if (ctl.fuse) {
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_rate) atomicMax(&ctl.clk->cfl_bits, s_rate);
      if (s_bad) atomicExch(&ctl.clk->status, 3);
    }
  }
}

template <int NT, int MINB, int EOS = 0>
__global__ void __launch_bounds__(NT, MINB) k_sweep_z(Tables T, Planes P, Phys ph, SweepCtl ctl, int ntop, int l0) {
  __shared__ ChunkShmT<NT> S;
  StepIn st;
  if (!load_step(ctl, st)) return;
  sweep_z_body<NT, EOS>(S, threadIdx.x, true, T, P, ph, ctl, st, ntop, blockIdx.x, blockIdx.y, blockIdx.z + l0);
}

// Polar sweep of single-chunk pencils (nk <= PZ_LIM - 12, the usual 3D
// disk): PACK pencils of lim = nk + 12 cells share a CTA of PACK * lim
// threads instead of one pencil per CTA of 32/64 threads with idle lanes.
// Measured on the 128x1024x32 disk (pencils of 44 cells): 4 pencils per CTA
// at 5 CTAs/SM (56 registers) took the polar sweep from 1.85 to 1.30 ms, and
// with the later arithmetic savings it ran at 1.04 ms; 8 pencils per CTA, 352
// threads = 11 whole warps where 4 pencils leave half of a sixth warp idle,
// at 3 CTAs/SM (56 registers, 33 resident warps against 30) take it to
// 0.93 ms.  Pencils longer than 44 cells keep 4 per CTA.  An earlier 8-pencil
// form at 2 CTAs/SM, before the bank padding, ran at 1.63 ms.
// The 8-pencil kernel's shared blocks are sized for 44 cells (LIMZ; 52 KB
// per CTA instead of 67), which leaves L1 room for the spill slots of its
// 56-register threads; with the layer tables and paraset coefficients read
// where they are used instead of held through the chain (4x fewer local
// loads, 1.0 M per launch) that took the polar sweep from 0.781 to 0.707 ms.
// Thread t works on cell t / PACK of pencil t % PACK,
// and the PACK pencils of a CTA are consecutive azimuth columns of a ring,
// so a warp's loads of one layer cover PACK adjacent doubles.  Pencils past
// the last column repeat the last one without storing.
constexpr int PZ_LIM = 56;
constexpr int PZ8_THREADS = 352;   // 8 pencils of up to 44 cells, 3 CTAs per SM
constexpr int PZ8_LIM = PZ8_THREADS / 8;
template <int PACK, int LIMZ = PZ_LIM>
using PzShm = ChunkShmT<LIMZ, 128 / PACK>;
template <int PACK, int LIMZ = PZ_LIM>
constexpr int pz_shm_bytes() { return PACK * (int)sizeof(PzShm<PACK, LIMZ>); }
template <int PACK, int MINB, int MAXT = PACK * PZ_LIM, int LIMZ = PZ_LIM>
__global__ void __launch_bounds__(MAXT, MINB) k_sweep_z_packed(Tables T, Planes P, Phys ph, SweepCtl ctl, int ntop) {
  // the PACK pencils' shared blocks, dynamic: 8 of them (52 KB) exceed the
  // 48 KiB a kernel may declare statically
  extern __shared__ __align__(16) unsigned char pz_shm[];
  PzShm<PACK, LIMZ> *S = reinterpret_cast<PzShm<PACK, LIMZ> *>(pz_shm);
  StepIn st;
  if (!load_step(ctl, st)) return;
  const int p = threadIdx.x % PACK, n = threadIdx.x / PACK;
  const int npen = T.nr * T.nphi;
  int col = blockIdx.x * PACK + p;
  const bool store = col < npen;
  if (!store) col = npen - 1;
  sweep_z_body<LIMZ>(S[p], n, store, T, P, ph, ctl, st, ntop, col / T.nphi, col % T.nphi, 0);
}

// ---------------------------------------------------------------------------
// tables: cs2, nu and the damping factors per ring, on the device so that
// they carry the same bits as the reference's inline get_cs2/get_nu calls
__global__ void k_tables(Tables T, Phys ph, int ndim, double kill_rin, double kill_rout,
                         double xmin, double xmax) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n = T.nk * T.nrg;
  const int nz = T.nk + 2 * NPAD;
  if (t < nz) {
    // sin, cos of every polar layer's centre and face angles (ghost layers
    // included), and the reciprocals the polar sweep multiplies by where its
    // divisions by r sin(theta) and r dz would otherwise repeat per cell
    const_cast<double *>(T.szc)[t] = sin(T.zc[t]);
    const_cast<double *>(T.czc)[t] = cos(T.zc[t]);
    const_cast<double *>(T.szf)[t] = sin(T.z[t]);
    const_cast<double *>(T.czf)[t] = cos(T.z[t]);
    const_cast<double *>(T.iszc)[t] = 1.0 / sin(T.zc[t]);
    const_cast<double *>(T.iszf)[t] = 1.0 / sin(T.z[t]);
    const_cast<double *>(T.idz)[t] = 1.0 / T.dz[t];
    // the polar sweep's Eulerian paraset coefficients: every polar pencil
    // has the layers' widths dz, so they are one set per layer (c0..c2 where
    // dz[t + 2] exists, c3 and c4 where dz[t + 1] does)
    Par par{0.0, 0.0, 0.0, 0.0, 0.0};
    if (t >= 1 && t + 1 < nz) paraset_at(T.dz, t, t + 2 < nz, par);
    double *zp = const_cast<double *>(T.zpar) + 5 * t;
    zp[0] = par.c0; zp[1] = par.c1; zp[2] = par.c2; zp[3] = par.c3; zp[4] = par.c4;
  }
  if (ndim == 3 && t < 2 * NPAD * T.nr) {
    // nu at r sin(theta) of the 12 polar ghost layers of ring i (slot g:
    // layer g - 6 below the grid, or layer nk + g - 6 above it), the
    // expression the polar viscosity uses for them (get_nu
    // disk_profile.cu:149-152)
    const int i = t % T.nr, g = t / T.nr;
    const int kz = (g < NPAD) ? g : T.nk + g;          // ghost layer + NPAD
    const double rcg = T.rxc[i + NPAD] * sin(T.zc[kz]);    // T.szc[kz], which this launch writes
    const_cast<double *>(T.nug)[t] = ph.vis_nu * pow(rcg, ph.p_alpha);
  }
  if (t >= n) return;
  int k = t / T.nrg, row = t % T.nrg;
  double rad = T.rxc[row];
  double rc = rad;
  if (ndim == 3) rc *= sin(T.zc[k + NPAD]);
  double *radc = const_cast<double *>(T.radc);
  double *cs2 = const_cast<double *>(T.cs2);
  double *nu = const_cast<double *>(T.nu);
  double *dg = const_cast<double *>(T.damp_g);
  double *dp = const_cast<double *>(T.damp_pw);
  radc[t] = rc;
  cs2[t] = ph.sc2 * pow(rc, -ph.p_beta);          // get_cs2 disk_profile.cu:39-42
  nu[t] = ph.vis_nu * pow(rc, ph.p_alpha);        // get_nu disk_profile.cu:149-152
  double g = 0.0;
  bool interior = row >= NPAD && row < T.nr + NPAD;
  if (interior) {
    double r = rad;
    if (kill_rin > 0.0 && r < kill_rin) g = (kill_rin - r) / (kill_rin - xmin);
    else if (kill_rout > 0.0 && r > kill_rout) g = (r - kill_rout) / (xmax - kill_rout);
  }
  dg[t] = g;
  dp[t] = pow(rad, -1.5);
}

// standalone CFL rate (dt_lv1 timestep.cu:12-73), one CTA per ring
__global__ void k_cfl(Tables T, const double *R, const double *U, const double *V, const double *W,
                      const double *P0, Phys ph, double frrot, int ndim, unsigned long long *out) {
  __shared__ double red[32];
  int i = blockIdx.x, k = blockIdx.y;
  int row = i + NPAD, rk = k * T.nrg + row;
  size_t base = (size_t)rk * T.nphi;
  double rad = T.rxc[row], rad_cyl = T.radc[rk];
  double rate = 0.0;
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    // physical column j holds storage index js = j - rot_j
    int js = wrapm(j - T.rot_j[rk], T.nphi);
    double r = R[base + j];
    double p = P0 ? P0[base + j] : eos_p_rt(r, T.cs2[rk], ph);
    double cs = sqrt(ph.gam * p / r);
    double t0 = (fabs(U[base + j]) + cs) / T.rdx[row];
    double t1 = (fabs(V[base + j] - T.rot_v[rk] - frrot * rad_cyl) + cs) / (T.dy[js] * rad_cyl);
    double rt;
    if (ndim == 3) {
      double t2 = (fabs(W[base + j]) + cs) / (T.dz[k + NPAD] * rad);
      rt = max3(t0, t1, t2);
    } else {
      rt = fmax(t0, t1);
    }
    rate = (rt > rate || rt != rt) ? rt : rate;
  }
  double m = block_max(rate, red);
  if (threadIdx.x == 0 && (m > 0.0 || m != m)) atomicMax(out, dbits(m));
}

// Index_Shift orbital_advection.cu:12-43 for every interior ring
__device__ __forceinline__ void index_shift_ring(const Tables &T, int t, double dt, double FrRot, int fargo) {
  int k = t / T.nr, i = t % T.nr;
  int row = i + NPAD, rk = k * T.nrg + row;
  double xc = T.rxc[row];
  double widthy = xc * T.dy[0] / dt;
  double rot_v;
  if (fargo == 1) rot_v = T.val_v[rk] - FrRot * xc;
  else if (fargo == 2) rot_v = (1.0 - FrRot) * xc;
  else rot_v = 0.0;
  double jp = T.rot_v[rk] / widthy;
  if (jp >= 0.0) { T.inc_j[rk] = (int)(jp + 0.5); T.res_v[rk] = floor(jp + 0.5) * widthy; }
  else { T.inc_j[rk] = (int)(jp - 0.5); T.res_v[rk] = floor(jp + 0.5) * widthy; }
  T.rot_v[rk] = rot_v;
}

__global__ void k_index(Tables T, double dt, double frrot, int fargo, const DevClock *clk) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (clk) {
    if (clk->halted) return;
    dt = clk->dt_step;
    frrot = clk->frrot_next;  // unused path; the fused loop shifts in k_prestep
  }
  if (t >= T.nr * T.nk) return;
  index_shift_ring(T, t, dt, frrot, fargo);
}

// rotate_rings ppm.cu:309-322
__global__ void k_rotate(Tables T, const DevClock *clk) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (clk && clk->halted) return;
  if (t >= T.nr * T.nk) return;
  int k = t / T.nr, i = t % T.nr;
  int rk = k * T.nrg + i + NPAD;
  int j = T.rot_j[rk] + T.inc_j[rk];
  T.rot_j[rk] = wrap1(j, T.nphi);
}

// standalone damping (same rule as the fused sweepy epilogue)
__global__ void k_damp(Tables T, double *R, double *U, double *V, double *W, double dt, int ndim) {
  int i = blockIdx.x, k = blockIdx.y;
  int rk = k * T.nrg + i + NPAD;
  double g = T.damp_g[rk];
  if (!(g > 0.0)) return;
  double f = g * (dt * T.damp_pw[rk]);
  size_t base = (size_t)rk * T.nphi;
  double vr = T.val_r[rk], vu = T.val_u[rk], vv = T.val_v[rk];
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    R[base + j] += f * (vr - R[base + j]);
    U[base + j] += f * (vu - U[base + j]);
    V[base + j] += f * (vv - V[base + j]);
    if (ndim == 3) W[base + j] += f * (-W[base + j]);
  }
}

// damping with the step's dt from the clock (3D fused loop)
__global__ void k_damp_clk(Tables T, double *R, double *U, double *V, double *W, const DevClock *clk) {
  if (clk->halted) return;
  int i = blockIdx.x, k = blockIdx.y;
  int rk = k * T.nrg + i + NPAD;
  double g = T.damp_g[rk];
  if (!(g > 0.0)) return;
  double f = g * (clk->dt_step * T.damp_pw[rk]);
  size_t base = (size_t)rk * T.nphi;
  double vr = T.val_r[rk], vu = T.val_u[rk], vv = T.val_v[rk];
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    R[base + j] += f * (vr - R[base + j]);
    U[base + j] += f * (vu - U[base + j]);
    V[base + j] += f * (vv - V[base + j]);
    W[base + j] += f * (-W[base + j]);
  }
}

// CFL rate for the next step (3D fused loop): rot_j has not been rotated yet
__global__ void k_cfl_clk(Tables T, const double *R, const double *U, const double *V, const double *W,
                          Phys ph, DevClock *clk, int ndim, int rot_pending) {
  __shared__ double red[32];
  if (clk->halted) return;
  int i = blockIdx.x, k = blockIdx.y;
  int row = i + NPAD, rk = k * T.nrg + row;
  size_t base = (size_t)rk * T.nphi;
  double rad = T.rxc[row], rad_cyl = T.radc[rk];
  double frrot = clk->frrot_next;
  int rotn = T.rot_j[rk] + (rot_pending ? T.inc_j[rk] : 0);
  double rate = 0.0;
  bool bad = false;
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    int js = wrapm(j - rotn, T.nphi);
    double r = R[base + j];
    double p = eos_p_rt(r, T.cs2[rk], ph);
    double cs = sqrt(ph.gam * p / r);
    double t0 = (fabs(U[base + j]) + cs) / T.rdx[row];
    double t1 = (fabs(V[base + j] - T.rot_v[rk] - frrot * rad_cyl) + cs) / (T.dy[js] * rad_cyl);
    double rt;
    if (ndim == 3) {
      double t2 = (fabs(W[base + j]) + cs) / (T.dz[k + NPAD] * rad);
      rt = max3(t0, t1, t2);
    } else {
      rt = fmax(t0, t1);
    }
    rate = (rt > rate || rt != rt) ? rt : rate;
    if (!(r > 0.0) || !isfinite(r) || !isfinite(U[base + j]) || !isfinite(V[base + j])) bad = true;
  }
  double m = block_max(rate, red);
  int anybad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    if (m > 0.0 || m != m) atomicMax(&clk->cfl_bits, dbits(m));
    if (anybad) atomicExch(&clk->status, 3);
  }
}

// ---------------------------------------------------------------------------
// output_lv1 (per ring, 1024 threads, storage order, bin_reduc_sum per 1024
// cells, running sum across chunks), output_lv2 (3D: round_reduc_sum over
// k) and output_lv3 (bin_reduc_sum over <=1024 rings) of device_func.cu.
// The last CTA to finish does lv2/lv3, so one launch gives the final value.
__device__ __forceinline__ double tree1024(double *list) {
  for (int len = 1024; len > 1; len >>= 1) {
    int half = len >> 1;
    if ((int)threadIdx.x < half) list[threadIdx.x] += list[threadIdx.x + half];
    __syncthreads();
  }
  return list[0];
}

// Rings t0, t0 + tstep, ... (t = i + nr * k: ring i of polar layer k), each
// summed on its own as one CTA of the reference sums it; the last of the
// run's nblocks CTAs to finish adds up the run's partial sums.
template <typename RT>
__device__ __forceinline__ void reduce_body(const Tables &T, const RT *R, Body pl, const DevClock *clk,
                                            double exclude, int mode, int plnt, double p_alpha, int ndim,
                                            double *ring_part, unsigned int *counter, double *out,
                                            double *hist_row, int t0, int tstep, unsigned nblocks,
                                            bool every_step = false) {
  __shared__ double list[1024];
  __shared__ bool is_last;
  if (clk) {
    if (!every_step && !clk->prin) return;
    if (every_step && clk->halted) return;
    pl = clk->planet;
  }
  const int tt = threadIdx.x;
  for (int rt = t0; rt < T.nr * T.nk; rt += tstep) {
    const int i = rt % T.nr, k = rt / T.nr;
    const int row = i + NPAD, rk = k * T.nrg + row;
    const int nphi = T.nphi;
    const size_t base = (size_t)rk * nphi;
    const int rot = T.rot_j[rk];
    const double rad = T.rxc[row], xvol = T.rxvol[row];
    const double zvol = (ndim == 3) ? T.zvol[k + NPAD] : 1.0;
    // FP32 planes hold Sigma - S_bg(ring)
    const double r_off = (sizeof(RT) == 4) ? T.sbg[rk] : 0.0;
    const int loop = nphi / 1024 + (nphi % 1024 != 0);
    double val = 0.0;
    for (int l = 0; l < loop; l++) {
      int j = tt + 1024 * l;   // storage index
      double v = 0.0;
      if (j < nphi) {
        int j0 = wrap1(j + rot, nphi);
        double phi = T.yc[j0];
        double r = r_off + (double)R[base + j0];
        if (plnt) {
          if (mode == 0) v = r * xvol * T.yvol[j0] * zvol;
          else if (ndim == 2 && (mode == 8 || mode == 9)) {
            if ((rad - pl.x) * (rad - pl.x) + rad * rad * (phi - pl.y) * (phi - pl.y) > exclude * exclude) {
              if (mode == 8) {
                double t = -grav_rad_cyl(rad, phi, 0.0, pl, 0.0);
                t *= (r - pow(rad, -p_alpha)) * xvol * T.yvol[j0];
                v = t;
              } else {
                double t = -grav_azi_cyl(rad, phi, 0.0, pl, 0.0);
                t *= rad * (r - pow(rad, -p_alpha)) * xvol * T.yvol[j0];
                v = t;
              }
            }
          }
        } else {
          v = r * xvol * T.yvol[j0] * zvol;
        }
      }
      list[tt] = v;
      __syncthreads();
      double s = tree1024(list);
      if (tt == 0) val += s;
      __syncthreads();
    }
    if (tt == 0) ring_part[i + T.nr * k] = val;
  }
  if (tt == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    is_last = (prev == nblocks - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // lv2 (3D): round_reduc_sum over k per ring i, reduction.cu:77-100
  const volatile double *part = ring_part;
  int nr = T.nr, nk = T.nk;
  // lv3: rings in chunks of 1024 (the reference supports iblk <= 1024)
  double total = 0.0;
  for (int base_i = 0; base_i < nr; base_i += 1024) {
    int ii = base_i + tt;
    double v = 0.0;
    if (ii < nr) {
      if (ndim == 3) {
        // pairwise tree over k with the reference's half-point order
        double acc[64];
        int kk = nk < 64 ? nk : 64;
        for (int q = 0; q < kk; q++) acc[q] = part[ii + nr * q];
        int len2 = 1;
        while (len2 < nk) len2 *= 2;
        while (len2 > 1) {
          int half = len2 / 2;
          for (int q = 0; q < half; q++) if (q + half < kk) acc[q] += acc[q + half];
          len2 = half;
        }
        v = acc[0];
      } else {
        v = part[ii];
      }
    }
    list[tt] = v;
    __syncthreads();
    double s = tree1024(list);
    if (tt == 0) total += s;
    __syncthreads();
  }
  if (tt == 0) {
    double res = 0.0 + total;
    if (out) *out = res;
    (void)hist_row;
    *counter = 0u;
  }
}

// ---------------------------------------------------------------------------
// Mass sums of runs with many rings: one warp per ring (RW rings per CTA).
// Lane L holds list[L + 32 m], m = 0..31, of a 1024-cell block, its 32 loads
// issued together; tree1024's levels 512..32 pair values inside a lane and
// levels 16..1 across lanes by shuffle.  Every addition has the same two
// operands as in tree1024, and __dadd_rn keeps the cell's product from being
// fused into the first one, so the sums are bitwise those of reduce_body.
// Used where cells are cheap (mass) and rings plentiful; the force sums and
// small runs keep reduce_body's one cell per thread.
constexpr int RW = 4;
__device__ __forceinline__ double warp_tree1024(double (&v)[32]) {
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
#pragma unroll
    for (int m = 0; m < h; m++) v[m] = __dadd_rn(v[m], v[m + h]);
  }
  double x = v[0];
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    const double y = __shfl_down_sync(0xffffffffu, x, d);
    if (lane < d) x = __dadd_rn(x, y);
  }
  return x;   // lane 0: the block's sum
}

template <typename RT>
__global__ void __launch_bounds__(32 * RW) k_reduce_mass_w(Tables T, const RT *R, const DevClock *clk, int ndim,
                                                           double *ring_part, unsigned int *counter, double *out) {
  __shared__ double list[1024];
  __shared__ bool is_last;
  if (clk && !clk->prin) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nr = T.nr, nk = T.nk, nphi = T.nphi;
  for (int rt = blockIdx.x * RW + w; rt < nr * nk; rt += gridDim.x * RW) {
    const int i = rt % nr, k = rt / nr;
    const int row = i + NPAD, rk = k * T.nrg + row;
    const size_t base = (size_t)rk * nphi;
    const int rot = T.rot_j[rk];
    const double xvol = T.rxvol[row];
    const double zvol = (ndim == 3) ? T.zvol[k + NPAD] : 1.0;
    // FP32 planes hold Sigma - S_bg(ring)
    const double r_off = (sizeof(RT) == 4) ? T.sbg[rk] : 0.0;
    const int loop = nphi / 1024 + (nphi % 1024 != 0);
    double val = 0.0;
    for (int l = 0; l < loop; l++) {
      double v[32];
#pragma unroll
      for (int m = 0; m < 32; m++) {
        const int j = lane + 32 * m + 1024 * l;   // storage index
        double x = 0.0;
        if (j < nphi) {
          const int j0 = wrap1(j + rot, nphi);
          const double r = r_off + (double)R[base + j0];
          x = r * xvol * T.yvol[j0] * zvol;
        }
        v[m] = x;
      }
      const double sum = warp_tree1024(v);
      if (lane == 0) val += sum;
    }
    if (lane == 0) ring_part[i + nr * k] = val;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // lv2 (3D: round_reduc_sum over k per ring, reduction.cu:77-100), then lv3
  // over the rings in blocks of 1024, as reduce_body
  const volatile double *part = ring_part;
  double total = 0.0;
  for (int base_i = 0; base_i < nr; base_i += 1024) {
    for (int q4 = threadIdx.x; q4 < 1024; q4 += 32 * RW) {
      const int ii = base_i + q4;
      double v = 0.0;
      if (ii < nr) {
        if (ndim == 3) {
          double acc[64];
          int kk = nk < 64 ? nk : 64;
          for (int q = 0; q < kk; q++) acc[q] = part[ii + nr * q];
          int len2 = 1;
          while (len2 < nk) len2 *= 2;
          while (len2 > 1) {
            int half = len2 / 2;
            for (int q = 0; q < half; q++) if (q + half < kk) acc[q] += acc[q + half];
            len2 = half;
          }
          v = acc[0];
        } else {
          v = part[ii];
        }
      }
      list[q4] = v;
    }
    __syncthreads();
    if (w == 0) {
      double v[32];
#pragma unroll
      for (int m = 0; m < 32; m++) v[m] = list[lane + 32 * m];
      const double sum = warp_tree1024(v);
      if (lane == 0) total += sum;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double res = 0.0 + total;
    if (out) *out = res;
    *counter = 0u;
  }
}

template <typename RT>
__global__ void __launch_bounds__(1024) k_reduce(Tables T, const RT *R, Body pl, const DevClock *clk,
                                                 double exclude, int mode, int plnt, double p_alpha,
                                                 int ndim, double *ring_part, unsigned int *counter,
                                                 double *out, double *hist_row) {
  reduce_body<RT>(T, R, pl, clk, exclude, mode, plnt, p_alpha, ndim, ring_part, counter, out, hist_row,
                  blockIdx.x, gridDim.x, gridDim.x);
}

// moving planet: the disk's radial (mode 8) and azimuthal (mode 9) force
// sums on the drifted planet, every step, into the clock
template <typename RT>
__global__ void __launch_bounds__(1024) k_reduce_forces(Tables T, const RT *R, DevClock *clk, int mode,
                                                        double p_alpha, int ndim, double *ring_part,
                                                        unsigned int *counter) {
  reduce_body<RT>(T, R, Body{}, clk, 0.0, mode, 1, p_alpha, ndim, ring_part, counter,
                  mode == 8 ? &clk->f8 : &clk->f9, nullptr, blockIdx.x, gridDim.x, gridDim.x, true);
}

// append a diagnostics row when this step prints (main.cu:414-428)
__device__ __forceinline__ void record_body(DevClock *clk) {
  DevClock &c = *clk;
  if (!c.prin) return;
  if (c.hist && c.hist_count < c.hist_cap) {
    double *h = c.hist + (size_t)HIST_COLS * c.hist_count;
    Body &p = c.planet;
    double vy = p.vy + c.frrot;
    double L = vy * p.x * p.x;                                        // get_L planet.cu:11-15
    double E = (p.vx * p.vx + vy * vy * p.x * p.x) / 2.0 - 1.0 / p.x; // get_E planet.cu:17-21
    h[0] = c.simtime;
    h[1] = c.mass;
    h[2] = c.torque / c.hist_norm;
    h[3] = p.x; h[4] = p.y; h[5] = p.vx; h[6] = p.vy; h[7] = p.fx; h[8] = p.fy;
    h[9] = sqrt(1.0 + (2.0 * E * L * L));
    h[10] = -1.0 / (2.0 * E);
    c.hist_count += 1;
  }
  c.prin = 0;
}

__global__ void k_record(DevClock *clk) { record_body(clk); }

// ---------------------------------------------------------------------------
// planet (planet.cu:28-93), device copies of the host arithmetic
__device__ double d_set_M_p(const DevClock &c, double t) {
  if (t < c.t_growth) return fmax(c.M_p * sin(3.1415926535897932384626433832795 * t / (2.0 * c.t_growth)), 0.01 * 0.000003);
  return c.M_p;
}
__device__ void d_kick(Body &pl, double &FrRot, double dt, int frflag) {
  pl.vx += dt * pl.fx;
  pl.vy += FrRot + dt * pl.fy / pl.x / pl.x;
  FrRot = (frflag == 1) ? pl.vy : 0.0;
  pl.vy -= FrRot;
}
// The planet's arithmetic is host code in the reference (planet.cu), whose
// compiler folds pow with the constant exponents 0, 1, -1 and 2 into 1, x,
// 1/x and x*x; the device copies below use the same forms (other exponents
// stay pow calls), and round products that feed a sum on their own, as the
// host does.
__device__ __forceinline__ double pow_host_form(double x, double y) {
  if (y == 0.0) return 1.0;
  if (y == 1.0) return x;
  if (y == -1.0) return 1.0 / x;
  if (y == 2.0) return __dmul_rn(x, x);
  return pow(x, y);
}
__device__ void d_drift(Body &pl, double FrRot, double dt, const DevClock &c) {
  double old_rad = pl.x;
  pl.x += dt * pl.vx;
  pl.y += dt * pl.vy;
  pl.vy = ((pl.vy + FrRot) * old_rad * old_rad / pl.x / pl.x) - FrRot;
  if (pl.y < 0.0) pl.y += 6.283185307179586476925286766559;
  if (pl.y >= 6.283185307179586476925286766559) pl.y -= 6.283185307179586476925286766559;
  // rs = rs_fac*get_h(x), get_h = sqrt(cs2(x) x^3); cs2 = sc2 * x^-p_beta is
  // evaluated on the host for the fixed-orbit case and never changes there
  (void)c;
}
// moving planet: the drift moves x, and the softening follows it as
// kick_drift_kick does on the host, rs = rs_fac h(x), h = sqrt(cs2(x) x^3)
// with cs2 = sc_h^2 x^-p_beta (disk_profile.cu:39-52)
__device__ void d_drift_moving(Body &pl, double FrRot, double dt, const DevClock &c) {
  d_drift(pl, FrRot, dt, c);
  pl.rs = c.rs_fac * sqrt(c.sc2 * pow_host_form(pl.x, -c.p_beta) * pl.x * pl.x * pl.x);
}
__device__ void d_forces_fixed(Body &pl, double FrRot) {
  pl.fx = -1.0 / pl.x / pl.x + __dmul_rn(pl.x, pow_host_form(pl.vy + FrRot, 2.0));
  pl.fy = 0.0;
}

// get_dt host part + dt clipping + Index_Shift + half kick (main.cu:345-370)
__device__ __forceinline__ void prestep_body(DevClock *clk, const Tables &T, int fargo) {
  __shared__ double s_dt, s_frrot;
  __shared__ int s_run;
  if (threadIdx.x == 0) {
    DevClock &c = *clk;
    int run = !(c.halted || c.done);
    if (run && c.status != 0) { c.halted = 1; run = 0; }
    if (run) {
      double rate = __longlong_as_double((long long)c.cfl_bits);
      double hdt = c.courant / rate;               // dt_lv3 timestep.cu:105
      double dt = 1.1 * c.dt;                      // timestep.cu:135-141
      dt = (hdt < dt) ? hdt : dt;
      if (dt / c.endtime < 1.0e-12 || !(dt > 0.0)) { c.status = 4; c.halted = 1; run = 0; }
      else {
        c.prin = 0;
        if (c.ncycle == c.ncycend) { c.prin = 1; c.done = 1; }
        if (c.simtime + dt >= c.endtime) {
          c.old_dt = dt; dt = c.endtime - c.simtime; c.prin = 1; c.make_pict = 1; c.done = 1;
        }
        if (c.timem + dt >= c.tmovie) { c.old_dt = dt; dt = c.tmovie - c.timem; c.make_pict = 1; }
        c.dt = dt;
        c.dt_step = dt;
        s_dt = dt;
        s_frrot = c.frrot;   // Index_Shift sees FrRot before the kick
        // kick_drift_kick(planet, FrRot, ..., 0.5*dt, true) main.cu:370
        if (c.plnt_flag > 0) d_kick(c.planet, c.frrot, 0.5 * dt, c.frrot_flag);
        // FrRot at the next get_dt, for the fused CFL: replay drift, forces
        // and kick on copies (fixed planet: forces are analytic)
        Body b = c.planet;
        double fr = c.frrot;
        if (c.plnt_flag > 0) {
          d_drift(b, fr, dt, c);
          d_forces_fixed(b, fr);
          d_kick(b, fr, 0.5 * dt, c.frrot_flag);
        }
        c.frrot_next = fr;
        c.cfl_bits = 0ull;
      }
    }
    s_run = run;
  }
  __syncthreads();
  if (!s_run) return;
  for (int t = threadIdx.x; t < T.nr * T.nk; t += blockDim.x) index_shift_ring(T, t, s_dt, s_frrot, fargo);
}

__global__ void k_prestep(DevClock *clk, Tables T, int fargo) { prestep_body(clk, T, fargo); }

// simtime/drift/forces/kick/dump bookkeeping (main.cu:378-412)
// phase 0: the whole end of a step; with a moving planet phase 1 (rotation,
// time, drift, mass) and phase 2 (forces from the disk reductions f8, f9
// made between the two, kick, bookkeeping; planet.cu:54-93, main.cu:378-412)
__device__ __forceinline__ void poststep_body(DevClock *clk, const Tables &T, int phase = 0) {
  int t = threadIdx.x;
  DevClock &c = *clk;
  int halted = c.halted;
  __syncthreads();
  if (halted) return;
  // rotate_rings ppm.cu:309-322
  for (int q = t; phase != 2 && q < T.nr * T.nk; q += blockDim.x) {
    int k = q / T.nr, i = q % T.nr;
    int rk = k * T.nrg + i + NPAD;
    T.rot_j[rk] = wrap1(T.rot_j[rk] + T.inc_j[rk], T.nphi);
  }
  if (t != 0) return;
  double dt = c.dt_step;
  if (phase != 2) {
    c.simtime += dt;
    c.timem += dt;
    c.ncycle += 1;
    c.ncycp += 1;
  }
  if (phase == 0) {
    if (c.plnt_flag > 0) {
      d_drift(c.planet, c.frrot, dt, c);
      c.planet.m = d_set_M_p(c, c.simtime);
      d_forces_fixed(c.planet, c.frrot);
      d_kick(c.planet, c.frrot, 0.5 * dt, c.frrot_flag);
    }
  } else if (phase == 1) {
    d_drift_moving(c.planet, c.frrot, dt, c);
    c.planet.m = d_set_M_p(c, c.simtime);
    return;
  } else {
    // planet_forces planet.cu:58-59 with the disk sums of this state
    Body &p = c.planet;
    p.fx = c.Sigma_0 * c.f8 / p.m - 1.0 / p.x / p.x + __dmul_rn(p.x, pow_host_form(p.vy + c.frrot, 2.0));
    p.fy = c.Sigma_0 * c.f9 / p.m;
    d_kick(p, c.frrot, 0.5 * dt, c.frrot_flag);
    c.frrot_next = c.frrot;      // the CFL of the next get_dt runs after this kernel
  }
  if (c.ncycp == c.nprin) { c.ncycp = 0; c.prin = 1; }
  if (c.make_pict) {
    c.timem = 0.0;
    c.make_pict = 0;
    c.dt = c.old_dt;
    c.halted = 1;   // the host dumps before continuing
  }
  if (c.done) c.halted = 1;
}

__global__ void k_poststep(DevClock *clk, Tables T) { poststep_body(clk, T); }
__global__ void k_poststep_drift(DevClock *clk, Tables T) { poststep_body(clk, T, 1); }
__global__ void k_poststep_kick(DevClock *clk, Tables T) { poststep_body(clk, T, 2); }

// ---------------------------------------------------------------------------
// Dump <-> planes.  The dump holds each ring's field arrays in storage order
// (j_store = j_phys - rot_j, init.cpp:241, output.cu:48-55); the planes hold
// physical order.  Thread (j, ring i, layer k) moves one cell.
__global__ void k_unpack_dump(Tables T, const double *stage, DumpPlanes D, int ndim, int fp32, int *err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y, k = blockIdx.z;
  const int nphi = T.nphi;
  if (j >= nphi) return;
  const int rk = k * T.nrg + i + NPAD;
  int jp = j + T.rot_j[rk];
  if (jp >= nphi) jp -= nphi;
  const double *f = stage + ((size_t)i + (size_t)T.nr * k) * 5 * nphi;
  const double r = f[j], p = f[nphi + j], u = f[2 * nphi + j], v = f[3 * nphi + j], w = f[4 * nphi + j];
  if (!(r > 0.0) || !isfinite(r)) atomicOr(err, 1);
  if (ndim == 2 && w != 0.0) atomicOr(err, 2);
  const size_t o = (size_t)rk * nphi + jp;
  if (fp32) {
    D.fr[o] = (float)(r - T.sbg[rk]);
    D.fu[o] = (float)u;
    D.fv[o] = (float)(v - T.vbg[rk]);
    if (ndim == 3) D.fw[o] = (float)w;
  } else {
    D.r[o] = r; D.u[o] = u; D.v[o] = v; D.p0[o] = p;
    if (ndim == 3) D.w[o] = w;
  }
}

// the fixed radial ghost rings (init_bound, init.cpp:253-413): phi-uniform
// r, u, v, p per ghost row, w = 0
__global__ void k_fill_ghost_rows(Tables T, const double *ghosts, DumpPlanes D, int ndim, int fp32) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, gi = blockIdx.y, k = blockIdx.z;
  if (j >= T.nphi) return;
  const int row = gi < NPAD ? gi : T.nr + gi;
  const int rk = k * T.nrg + row;
  const double *g = ghosts + ((size_t)k * 2 * NPAD + gi) * 4;
  const size_t o = (size_t)rk * T.nphi + j;
  if (fp32) {
    D.fr[o] = (float)(g[0] - T.sbg[rk]);
    D.fu[o] = (float)g[1];
    D.fv[o] = (float)(g[2] - T.vbg[rk]);
    if (ndim == 3) D.fw[o] = 0.f;
  } else {
    D.r[o] = g[0]; D.u[o] = g[1]; D.v[o] = g[2]; D.p0[o] = g[3];
    if (ndim == 3) D.w[o] = 0.0;
  }
}

// whole ring records (72*nphi + 96 bytes) in the dump layout
__global__ void k_pack_dump(Tables T, DumpPlanes D, Phys ph, int ndim, int fp32, int p0_live, unsigned char *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y, k = blockIdx.z;
  const int nphi = T.nphi, row = i + NPAD, rk = k * T.nrg + row, kz = k + NPAD;
  if (j >= nphi) return;
  unsigned char *base = out + ((size_t)i + (size_t)T.nr * k) * ((size_t)72 * nphi + 96);
  int jp = j + T.rot_j[rk];
  if (jp >= nphi) jp -= nphi;
  const size_t o = (size_t)rk * nphi + jp;
  double *f = (double *)base;
  double r, u, v, w;
  if (fp32) {
    r = T.sbg[rk] + (double)D.fr[o];
    u = D.fu[o];
    v = T.vbg[rk] + (double)D.fv[o];
    w = (ndim == 3) ? (double)D.fw[o] : 0.0;
  } else {
    r = D.r[o]; u = D.u[o]; v = D.v[o];
    w = (ndim == 3) ? D.w[o] : 0.0;
  }
  f[j] = r;
  f[nphi + j] = p0_live ? D.p0[o] : eos_p_rt(r, T.cs2[rk], ph);   // the store's p, ppm.cu:138-143
  f[2 * nphi + j] = u;
  f[3 * nphi + j] = v;
  f[4 * nphi + j] = w;
  double *col = (double *)(base + (size_t)40 * nphi + 32);
  col[j] = T.y[j]; col[nphi + j] = T.dy[j]; col[2 * nphi + j] = T.yvol[j]; col[3 * nphi + j] = T.yc[j];
  if (j == 0) {
    double *sc = (double *)(base + (size_t)40 * nphi);
    sc[0] = T.rx[row]; sc[1] = T.rdx[row]; sc[2] = T.rxvol[row]; sc[3] = T.rxc[row];
    double *zs = (double *)(base + (size_t)72 * nphi + 32);
    zs[0] = T.z[kz]; zs[1] = T.dz[kz]; zs[2] = T.zvol[kz]; zs[3] = T.zc[kz];
    int *ik = (int *)(base + (size_t)72 * nphi + 64);
    ik[0] = i; ik[1] = k;
    double *rot = (double *)(base + (size_t)72 * nphi + 72);
    rot[0] = T.rot_v[rk]; rot[1] = T.res_v[rk];
    int *rj = (int *)(base + (size_t)72 * nphi + 88);
    rj[0] = T.rot_j[rk]; rj[1] = T.inc_j[rk];
  }
}

// ---------------------------------------------------------------------------
// Post-processing of a state (the reference's read/ tools, on the device).
// Both work on the physical-order planes, which is what read/p_init.cpp:108-133
// (update_grid) builds from a dump by undoing each ring's rot_j.
__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
  return t;
}

// write_har_file, read/p_output.cpp:35-55: per ring of layer 0,
// a = sum_j sin(m yc_j) Sigma_j and b = sum_j cos(m yc_j) Sigma_j
template <typename RT>
__global__ void k_post_harmonic(Tables T, const RT *R, double m, double *ab) {
  __shared__ double red[32];
  const int i = blockIdx.x, rk = i + NPAD;
  const size_t base = (size_t)rk * T.nphi;
  const double off = (sizeof(RT) == 4) ? T.sbg[rk] : 0.0;   // FP32 planes hold Sigma - S_bg
  double a = 0.0, b = 0.0;
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    double sig = off + (double)R[base + j];
    a += sin(m * T.yc[j]) * sig;
    b += cos(m * T.yc[j]) * sig;
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) { ab[2 * i] = a; ab[2 * i + 1] = b; }
}

// get_torque, read/transform.cpp:386-420: torque of the disk on a planet of
// mass ratio M_p at r = 1, azimuth pi, in the barycentric frame (star at
// distance M_p/(1+M_p) opposite), softening 3e-6 in Rp^2; one sum per ring
template <typename RT>
__global__ void k_post_torque(Tables T, const RT *R, double M_p, double *ring_out) {
  __shared__ double red[32];
  const int i = blockIdx.x, k = blockIdx.y;
  const int row = i + NPAD, rk = k * T.nrg + row, kz = k + NPAD;
  const size_t base = (size_t)rk * T.nphi;
  const double off = (sizeof(RT) == 4) ? T.sbg[rk] : 0.0;
  const double stm = 1.0 / (1.0 + M_p), plm = M_p * stm, plx = 1.0 * stm, stx = 1.0 * plm;
  const double rad = T.rxc[row], z = T.zc[kz], dxz = T.rdx[row] * T.dz[kz];
  double t = 0.0;
  for (int j = threadIdx.x; j < T.nphi; j += blockDim.x) {
    double azi = T.yc[j];
    double cosfac = cos(azi - 3.1415926535897932384626433832795);
    double sinfac = sin(azi - 3.1415926535897932384626433832795);
    double Rp = rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z;
    Rp = sqrt(Rp + 0.000003);
    double Rs = sqrt(rad * rad + stx * stx + 2.0 * stx * rad * cosfac + z * z);
    double rho = off + (double)R[base + j];
    t += rho * (plm * plx * sinfac / (Rp * Rp * Rp) - stm * stx * sinfac / (Rs * Rs * Rs)) * rad * T.dy[j] * dxz;
  }
  t = block_sum(t, red);
  if (threadIdx.x == 0) ring_out[k * T.nr + i] = t;
}

// ---------------------------------------------------------------------------
// Batched 2D steps: one launch per phase walks the tiles of every run of a
// group.  A tile is one pencil chunk (sweeps) or one ring (reductions); the
// run of tile t is found by bisection in the queue's prefix sums.  Each
// tile runs the same body as the per-run kernels, so a run's results do not
// depend on the batch it is in or on the launch shape.
__device__ __forceinline__ int batch_find(const BatchQueue &q, int t) {
  int lo = 0, hi = q.nruns;   // q.start[lo] <= t < q.start[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (q.start[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void kb_prestep(const BatchRun *runs) {
  const BatchRun &b = runs[blockIdx.x];
  prestep_body(b.clk, b.T, b.fargo);
}
__global__ void kb_poststep(const BatchRun *runs) {
  const BatchRun &b = runs[blockIdx.x];
  poststep_body(b.clk, b.T);
}
__global__ void kb_record(const BatchRun *runs) { record_body(runs[blockIdx.x].clk); }

template <typename RT>
__global__ void __launch_bounds__(1024) kb_reduce(BatchQueue q, int mode) {
  const int r = batch_find(q, blockIdx.x);
  const BatchRun &b = q.runs[r];
  if (mode == 9 && !b.plnt) return;
  const RT *R;
  if constexpr (sizeof(RT) == 4) R = (const RT *)b.QX.r;   // a 2D step ends in its first planes
  else R = (const RT *)b.PX.r;
  double *out = (mode == 0) ? &b.clk->mass : &b.clk->torque;
  reduce_body<RT>(b.T, R, Body{}, b.clk, 0.0, mode, mode == 9 ? 1 : b.plnt, b.p_alpha, 2, b.ring_part, b.counter,
                  out, nullptr, blockIdx.x - q.start[r], b.T.nr, (unsigned)b.T.nr);
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) kb_sweep_x(BatchQueue q) {
  __shared__ ChunkShmT<128> S;
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    StepIn st;
    if (load_step(ctl, st)) {
      const int lt = t - q.start[r], nphi = b.T.nphi;
      Planes P = b.PX;
      P.p0 = (b.p0 && b.clk->ncycle == b.p0_cycle) ? b.p0 : nullptr;
      sweep_x_body<false, false, 128>(S, threadIdx.x, true, b.T, P, b.ph, ctl, st, lt % nphi, lt / nphi, 0);
    }
    __syncthreads();
  }
}

// radial last chunks of at most 64 cells: tile t of a member covers columns
// 4t .. 4t+3, thread i on cell i / 4 of column 4t + i % 4 (threads past the
// chunk's lim idle; columns past the last one repeat it without storing)
__global__ void __launch_bounds__(256, 4) kb_sweep_x_short(BatchQueue q) {
  __shared__ ChunkShmT<64> S[4];
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    StepIn st;
    if (load_step(ctl, st)) {
      const int p = threadIdx.x & 3, n = threadIdx.x >> 2, nphi = b.T.nphi;
      int col = 4 * (t - q.start[r]) + p;
      const bool store = col < nphi;
      if (!store) col = nphi - 1;
      Planes P = b.PX;
      P.p0 = (b.p0 && b.clk->ncycle == b.p0_cycle) ? b.p0 : nullptr;
      sweep_x_body<false, false, 64>(S[p], n, store, b.T, P, b.ph, ctl, st, col, b.T.cx.loop - 1, 0);
    }
    __syncthreads();
  }
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) kb_sweep_y(BatchQueue q) {
  __shared__ ChunkShmT<128> S;
  __shared__ double red[4];
  for (int t = blockIdx.x; t < q.total; t += gridDim.x) {
    const int r = batch_find(q, t);
    const BatchRun &b = q.runs[r];
    SweepCtl ctl{};
    ctl.clk = b.clk;
    ctl.fuse = 1;
    ctl.shift = 1;
    StepIn st;
    if (load_step(ctl, st)) {
      const int lt = t - q.start[r], loop = b.T.cy.loop;
      sweep_y_body<false, false, 128>(S, red, b.T, b.PY, b.ph, ctl, st, lt % loop, lt / loop, 0);
    }
    __syncthreads();
  }
}

}  // namespace pgd

// ---------------------------------------------------------------------------
namespace pgk {
using namespace pgd;

// CTA size for a chunk of `lim` active cells
static inline int cta_for(int lim) { return lim <= 32 ? 32 : (lim <= 64 ? 64 : 128); }

// Occupancy variant of the 128-thread sweeps: MINB 1 lets the compiler keep
// ~76 registers (6 CTAs per SM), MINB 8 caps them at 64 (8 CTAs per SM, a
// few spilled values).  Chosen per run (pg_run's tuning, PG_SWEEP_OCC).
// Isentropic runs (EOS 1) use the MINB 1 kernels and no pencil packing.
template <bool SPHV, bool TD, int EOS>
static void launch_x(int nt, int occ8, dim3 grid, int l0, const Tables &T, const Planes &P, const Phys &ph,
                     const SweepCtl &c, cudaStream_t s) {
  if constexpr (EOS == 0) {
    // 2D radial chunks: 7 CTAs per SM (72 registers, no spills) run 3 % faster
    // than 8 (64, spilling); the 3D radial kernel spills at 72 as well and
    // keeps 8
    if (nt == 128 && occ8) { k_sweep_x<SPHV, TD, 128, SPHV ? 8 : 7><<<grid, 128, 0, s>>>(T, P, ph, c, l0); return; }
  }
  if (nt == 128) k_sweep_x<SPHV, TD, 128, 1, EOS><<<grid, 128, 0, s>>>(T, P, ph, c, l0);
  else if (nt == 64) k_sweep_x<SPHV, TD, 64, 1, EOS><<<grid, 64, 0, s>>>(T, P, ph, c, l0);
  else k_sweep_x<SPHV, TD, 32, 1, EOS><<<grid, 32, 0, s>>>(T, P, ph, c, l0);
}
template <bool SPHV, bool TD, int EOS>
static void launch_y(int nt, int occ8, dim3 grid, int l0, const Tables &T, const Planes &P, const Phys &ph,
                     const SweepCtl &c, cudaStream_t s) {
  if constexpr (EOS == 0) {
    if (nt == 128 && occ8) { k_sweep_y<SPHV, TD, 128, 8><<<grid, 128, 0, s>>>(T, P, ph, c, l0); return; }
  }
  if (nt == 128) k_sweep_y<SPHV, TD, 128, 1, EOS><<<grid, 128, 0, s>>>(T, P, ph, c, l0);
  else if (nt == 64) k_sweep_y<SPHV, TD, 64, 1, EOS><<<grid, 64, 0, s>>>(T, P, ph, c, l0);
  else k_sweep_y<SPHV, TD, 32, 1, EOS><<<grid, 32, 0, s>>>(T, P, ph, c, l0);
}
template <int EOS>
static void launch_z(int nt, int occ8, dim3 grid, int l0, int ntop, const Tables &T, const Planes &P,
                     const Phys &ph, const SweepCtl &c, cudaStream_t s) {
  if constexpr (EOS == 0) {
    if (nt == 128 && occ8) { k_sweep_z<128, 8><<<grid, 128, 0, s>>>(T, P, ph, c, ntop, l0); return; }
  }
  if (nt == 128) k_sweep_z<128, 1, EOS><<<grid, 128, 0, s>>>(T, P, ph, c, ntop, l0);
  else if (nt == 64) k_sweep_z<64, 1, EOS><<<grid, 64, 0, s>>>(T, P, ph, c, ntop, l0);
  else k_sweep_z<32, 1, EOS><<<grid, 32, 0, s>>>(T, P, ph, c, ntop, l0);
}

template <int EOS>
static void sweep_x_t(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  const Chunking &ch = T.cx;
  const int occ8 = T.occ8;
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  // a last chunk of more than 64 cells runs in the full chunks' launch (the
  // body gives chunk loop-1 its lim_last), whose tail it fills
  const bool merge = !ch.stuck && full > 0 && ch.lim_last > 64;
  if (merge) full = ch.loop;
  if (full > 0) {
    bool done = false;
    if constexpr (EOS == 0) {
      // a stuck last chunk (imax % 116 == 0) keeps the one-column kernel
      const int xp = (ch.stuck || !occ8) ? 1 : T.xpack;
      if (xp == 2 || xp == 4) {
        dim3 grid((T.nphi + xp - 1) / xp, full, T.nk);
        if (xp == 2) {
          if (ndim == 3) k_sweep_x_cols<true, true, 2, 4><<<grid, 2 * ARR, px_shm_bytes<2>(), s>>>(T, P, ph, c);
          else k_sweep_x_cols<false, false, 2, 4><<<grid, 2 * ARR, px_shm_bytes<2>(), s>>>(T, P, ph, c);
        } else {
          if (ndim == 3) k_sweep_x_cols<true, true, 4, 2><<<grid, 4 * ARR, px_shm_bytes<4>(), s>>>(T, P, ph, c);
          else k_sweep_x_cols<false, false, 4, 2><<<grid, 4 * ARR, px_shm_bytes<4>(), s>>>(T, P, ph, c);
        }
        done = true;
      }
    }
    if (!done) {
      dim3 grid(T.nphi, full, T.nk);
      if (ndim == 3) launch_x<true, true, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
      else launch_x<false, false, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
    }
  }
  if (!ch.stuck && !merge) {
    if constexpr (EOS == 0) {
      if (T.zpack && ch.lim_last <= PX_LIM) {
        int npen = T.nphi * T.nk, blocks = (npen + 3) / 4, nt = 4 * ch.lim_last;
        if (ch.lim_last <= 32) {
          if (ndim == 3) k_sweep_x_packed<true, true, 8, 32><<<blocks, nt, 0, s>>>(T, P, ph, c);
          else k_sweep_x_packed<false, false, 8, 32><<<blocks, nt, 0, s>>>(T, P, ph, c);
        } else {
          if (ndim == 3) k_sweep_x_packed<true, true, 4><<<blocks, nt, 0, s>>>(T, P, ph, c);
          else k_sweep_x_packed<false, false, 4><<<blocks, nt, 0, s>>>(T, P, ph, c);
        }
        return;
      }
    }
    dim3 grid(T.nphi, 1, T.nk);
    int nt = cta_for(ch.lim_last);
    int l0 = ch.loop - 1;
    if (ndim == 3) launch_x<true, true, EOS>(nt, occ8, grid, l0, T, P, ph, c, s);
    else launch_x<false, false, EOS>(nt, occ8, grid, l0, T, P, ph, c, s);
  }
}
void sweep_x(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  if (ph.eos) sweep_x_t<1>(T, P, ph, c, ndim, s);
  else sweep_x_t<0>(T, P, ph, c, ndim, s);
}

template <int EOS>
static void sweep_y_t(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  const Chunking &ch = T.cy;
  const int occ8 = T.occ8;
  if (!ch.stuck && cta_for(ch.lim_last) == 128) {
    // a last chunk of more than 64 cells takes the full chunks' 128-thread
    // CTAs: one launch for all of them (the body gives chunk loop-1 its
    // lim_last), whose CTAs fill the tail of the full chunks' last wave
    dim3 grid(ch.loop, T.nr, T.nk);
    if (ndim == 3) launch_y<true, true, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
    else launch_y<false, false, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
    return;
  }
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  if (full > 0) {
    dim3 grid(full, T.nr, T.nk);
    if (ndim == 3) launch_y<true, true, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
    else launch_y<false, false, EOS>(128, occ8, grid, 0, T, P, ph, c, s);
  }
  if (!ch.stuck) {
    dim3 grid(1, T.nr, T.nk);
    int nt = cta_for(ch.lim_last);
    int l0 = ch.loop - 1;
    if (ndim == 3) launch_y<true, true, EOS>(nt, occ8, grid, l0, T, P, ph, c, s);
    else launch_y<false, false, EOS>(nt, occ8, grid, l0, T, P, ph, c, s);
  }
}
void sweep_y(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ndim, cudaStream_t s) {
  if (ph.eos) sweep_y_t<1>(T, P, ph, c, ndim, s);
  else sweep_y_t<0>(T, P, ph, c, ndim, s);
}

template <int EOS>
static void sweep_z_t(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ntop, cudaStream_t s) {
  const Chunking &ch = T.cz;
  if constexpr (EOS == 0) {
    if (T.zpack && ch.loop == 1 && !ch.stuck && ch.lim_last <= PZ_LIM) {
      int npen = T.nr * T.nphi;
      if (8 * ch.lim_last <= PZ8_THREADS)    // whole warps: 8 pencils of 44 cells (kmax 32) are 11
        k_sweep_z_packed<8, 3, PZ8_THREADS, PZ8_LIM>
            <<<(npen + 7) / 8, 8 * ch.lim_last, pz_shm_bytes<8, PZ8_LIM>(), s>>>(T, P, ph, c, ntop);
      else
        k_sweep_z_packed<4, 5><<<(npen + 3) / 4, 4 * ch.lim_last, pz_shm_bytes<4>(), s>>>(T, P, ph, c, ntop);
      return;
    }
  }
  int full = ch.stuck ? ch.loop : ch.loop - 1;
  const bool merge = !ch.stuck && full > 0 && ch.lim_last > 64;   // as in sweep_x_t
  if (merge) full = ch.loop;
  if (full > 0) {
    dim3 grid(T.nr, T.nphi, full);
    launch_z<EOS>(128, T.occ8, grid, 0, ntop, T, P, ph, c, s);
  }
  if (!ch.stuck && !merge) {
    dim3 grid(T.nr, T.nphi, 1);
    launch_z<EOS>(cta_for(ch.lim_last), T.occ8, grid, ch.loop - 1, ntop, T, P, ph, c, s);
  }
}
void sweep_z(const Tables &T, const Planes &P, const Phys &ph, const SweepCtl &c, int ntop, cudaStream_t s) {
  if (ph.eos) sweep_z_t<1>(T, P, ph, c, ntop, s);
  else sweep_z_t<0>(T, P, ph, c, ntop, s);
}

// kernels launched by one sweep_* call: every sweep runs a last chunk of
// more than 64 cells in the full chunks' launch, a shorter one in a launch
// of its own
int sweep_launches(const Chunking &ch) { return (ch.stuck || ch.loop == 1 || ch.lim_last > 64) ? 1 : 2; }

// Per-device kernel attributes, set with the device current before the first
// launch (pg_create): the packed polar kernels and the column-packed radial
// kernels take their shared blocks as dynamic shared memory, above the
// 48 KiB default limit.
int setup_device() {
  // 8 polar pencils of up to 44 cells: 52 KB of shared blocks per CTA.  No
  // carveout preference: the driver's choice leaves L1 room for the spill
  // slots of 3 CTAs (polar sweep 0.707 ms on the 128x1024x32 disk, against
  // 0.715 at a 72 % carveout and 0.728 at 100 %)
  cudaError_t e = cudaFuncSetAttribute(k_sweep_z_packed<8, 3, PZ8_THREADS, PZ8_LIM>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, pz_shm_bytes<8, PZ8_LIM>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_z_packed<4, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             pz_shm_bytes<4>());
  // the column-packed radial kernels: 2 columns (37 KB) or 4 (75 KB) per CTA
  const void *cols2[2] = {(const void *)k_sweep_x_cols<true, true, 2, 4>, (const void *)k_sweep_x_cols<false, false, 2, 4>};
  const void *cols4[2] = {(const void *)k_sweep_x_cols<true, true, 4, 2>, (const void *)k_sweep_x_cols<false, false, 4, 2>};
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaFuncSetAttribute(cols2[i], cudaFuncAttributeMaxDynamicSharedMemorySize, px_shm_bytes<2>());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(cols4[i], cudaFuncAttributeMaxDynamicSharedMemorySize, px_shm_bytes<4>());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(cols4[i], cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
  if (e != cudaSuccess) return 1;
  return setup_device32();
}

void cfl_full(const Tables &T, const double *r, const double *u, const double *v, const double *w,
              const double *p0, const Phys &ph, double frrot, int ndim, unsigned long long *out,
              cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k_cfl<<<grid, 256, 0, s>>>(T, r, u, v, w, p0, ph, frrot, ndim, out);
}

void index_shift(const Tables &T, double dt, double frrot, int fargo, const DevClock *clk, cudaStream_t s) {
  int n = T.nr * T.nk;
  k_index<<<(n + 127) / 128, 128, 0, s>>>(T, dt, frrot, fargo, clk);
}

void rotate(const Tables &T, const DevClock *clk, cudaStream_t s) {
  int n = T.nr * T.nk;
  k_rotate<<<(n + 127) / 128, 128, 0, s>>>(T, clk);
}

void damp(const Tables &T, double *r, double *u, double *v, double *w, double dt, int ndim, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k_damp<<<grid, 256, 0, s>>>(T, r, u, v, w, dt, ndim);
}

void damp_clk(const Tables &T, double *r, double *u, double *v, double *w, const DevClock *clk,
              cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k_damp_clk<<<grid, 256, 0, s>>>(T, r, u, v, w, clk);
}

void cfl_clk(const Tables &T, const double *r, const double *u, const double *v, const double *w,
             const Phys &ph, DevClock *clk, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k_cfl_clk<<<grid, 256, 0, s>>>(T, r, u, v, w, ph, clk, 3, 1);
}

// The ring sums run on two 1024-thread CTAs per SM, each taking every
// grid-th ring: most steps print nothing and every CTA returns at once, so
// a grid of one CTA per ring would only pay for starting them.
static int reduce_grid(const Tables &T) {
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const int rings = T.nr * T.nk;
  return rings < 2 * nsm ? rings : 2 * nsm;
}

// The mass sums of a run with at least 1024 rings go one warp per ring
// (k_reduce_mass_w): on the 128x1024x32 disk 4096 rings in one wave of
// warps instead of 14 rings in turn per 1024-thread CTA.
static bool mass_warp(const Tables &T) { return T.nr * T.nk >= 1024; }
static int mass_grid(const Tables &T) { return (T.nr * T.nk + RW - 1) / RW; }

void reduce(const Tables &T, const double *r, const Body &pl, const DevClock *clk, double exclude,
            int mode, int plnt, double p_alpha, int ndim, double *ring_part, unsigned int *counter,
            double *out, double *hist_row, cudaStream_t s) {
  if ((mode == 0 || !plnt) && mass_warp(T)) {
    k_reduce_mass_w<double><<<mass_grid(T), 32 * RW, 0, s>>>(T, r, clk, ndim, ring_part, counter, out);
    return;
  }
  k_reduce<double><<<reduce_grid(T), 1024, 0, s>>>(T, r, pl, clk, exclude, mode, plnt, p_alpha, ndim, ring_part, counter,
                                         out, hist_row);
}

void reduce32(const Tables &T, const float *r, const Body &pl, const DevClock *clk, double exclude, int mode,
              int plnt, double p_alpha, int ndim, double *ring_part, unsigned int *counter, double *out,
              cudaStream_t s) {
  if ((mode == 0 || !plnt) && mass_warp(T)) {
    k_reduce_mass_w<float><<<mass_grid(T), 32 * RW, 0, s>>>(T, r, clk, ndim, ring_part, counter, out);
    return;
  }
  k_reduce<float><<<reduce_grid(T), 1024, 0, s>>>(T, r, pl, clk, exclude, mode, plnt, p_alpha, ndim, ring_part, counter,
                                        out, nullptr);
}

void prestep(DevClock *clk, const Tables &T, int fargo, cudaStream_t s) {
  k_prestep<<<1, 256, 0, s>>>(clk, T, fargo);
}

void poststep_drift(DevClock *clk, const Tables &T, cudaStream_t s) {
  k_poststep_drift<<<1, 256, 0, s>>>(clk, T);
}
void poststep_kick(DevClock *clk, cudaStream_t s) {
  Tables T{};
  k_poststep_kick<<<1, 1, 0, s>>>(clk, T);
}
void reduce_forces(const Tables &T, const void *r, int fp32, DevClock *clk, double p_alpha, int ndim,
                   double *ring_part, unsigned int *counter, cudaStream_t s) {
  const int grid = reduce_grid(T);
  for (int mode : {8, 9}) {
    if (fp32)
      k_reduce_forces<float><<<grid, 1024, 0, s>>>(T, (const float *)r, clk, mode, p_alpha, ndim, ring_part, counter);
    else
      k_reduce_forces<double><<<grid, 1024, 0, s>>>(T, (const double *)r, clk, mode, p_alpha, ndim, ring_part, counter);
  }
}
void cfl_clk_after(const Tables &T, const double *r, const double *u, const double *v, const double *w,
                   const Phys &ph, DevClock *clk, int ndim, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  k_cfl_clk<<<grid, 256, 0, s>>>(T, r, u, v, w, ph, clk, ndim, 0);
}

void post_harmonic(const Tables &T, const void *r, int fp32, double m, double *ab, cudaStream_t s) {
  if (fp32) k_post_harmonic<float><<<T.nr, 256, 0, s>>>(T, (const float *)r, m, ab);
  else k_post_harmonic<double><<<T.nr, 256, 0, s>>>(T, (const double *)r, m, ab);
}
void post_torque(const Tables &T, const void *r, int fp32, double M_p, double *ring_out, cudaStream_t s) {
  dim3 grid(T.nr, T.nk);
  if (fp32) k_post_torque<float><<<grid, 256, 0, s>>>(T, (const float *)r, M_p, ring_out);
  else k_post_torque<double><<<grid, 256, 0, s>>>(T, (const double *)r, M_p, ring_out);
}

void unpack_dump(const Tables &T, const double *stage, const DumpPlanes &D, int ndim, int fp32, int *err,
                 cudaStream_t s) {
  dim3 grid((T.nphi + 255) / 256, T.nr, T.nk);
  k_unpack_dump<<<grid, 256, 0, s>>>(T, stage, D, ndim, fp32, err);
}
void fill_ghost_rows(const Tables &T, const double *ghosts, const DumpPlanes &D, int ndim, int fp32,
                     cudaStream_t s) {
  dim3 grid((T.nphi + 255) / 256, 2 * NPAD, T.nk);
  k_fill_ghost_rows<<<grid, 256, 0, s>>>(T, ghosts, D, ndim, fp32);
}
void pack_dump(const Tables &T, const DumpPlanes &D, const Phys &ph, int ndim, int fp32, int p0_live, unsigned char *out,
               cudaStream_t s) {
  dim3 grid((T.nphi + 255) / 256, T.nr, T.nk);
  k_pack_dump<<<grid, 256, 0, s>>>(T, D, ph, ndim, fp32, p0_live, out);
}

void poststep(DevClock *clk, const Tables &T, cudaStream_t s) {
  k_poststep<<<1, 256, 0, s>>>(clk, T);
}

void record(DevClock *clk, cudaStream_t s) {
  k_record<<<1, 1, 0, s>>>(clk);
}

void tables(const Tables &T, const Phys &ph, int ndim, double kill_rin, double kill_rout, double xmin,
            double xmax, cudaStream_t s) {
  int n = T.nk * T.nrg;
  if (2 * NPAD * T.nr > n) n = 2 * NPAD * T.nr;         // the polar ghost-layer nu table
  if (T.nk + 2 * NPAD > n) n = T.nk + 2 * NPAD;
  k_tables<<<(n + 127) / 128, 128, 0, s>>>(T, ph, ndim, kill_rin, kill_rout, xmin, xmax);
}


void batch_prestep(const BatchRun *runs, int nruns, cudaStream_t s) {
  if (nruns > 0) kb_prestep<<<nruns, 256, 0, s>>>(runs);
}
void batch_poststep(const BatchRun *runs, int nruns, cudaStream_t s) {
  if (nruns > 0) kb_poststep<<<nruns, 256, 0, s>>>(runs);
}
void batch_record(const BatchRun *runs, int nruns, cudaStream_t s) {
  if (nruns > 0) kb_record<<<nruns, 1, 0, s>>>(runs);
}
void batch_reduce(const BatchQueue &rings, int fp32, int mode, cudaStream_t s) {
  if (rings.total <= 0) return;
  if (fp32) kb_reduce<float><<<rings.total, 1024, 0, s>>>(rings, mode);
  else kb_reduce<double><<<rings.total, 1024, 0, s>>>(rings, mode);
}
void batch_sweep_x(const BatchQueue &q, int grid, int minb, cudaStream_t s) {
  if (q.total <= 0) return;
  int g = (grid > 0 && grid < q.total) ? grid : q.total;
  if (minb >= 8) kb_sweep_x<8><<<g, 128, 0, s>>>(q);
  else kb_sweep_x<4><<<g, 128, 0, s>>>(q);
}
void batch_sweep_x_short(const BatchQueue &q, cudaStream_t s) {
  if (q.total > 0) kb_sweep_x_short<<<q.total, 256, 0, s>>>(q);
}
void batch_sweep_y(const BatchQueue &q, int grid, int minb, cudaStream_t s) {
  if (q.total <= 0) return;
  int g = (grid > 0 && grid < q.total) ? grid : q.total;
  if (minb >= 8) kb_sweep_y<8><<<g, 128, 0, s>>>(q);
  else kb_sweep_y<4><<<g, 128, 0, s>>>(q);
}

}  // namespace pgk
