// pg_noalloc.cu -- a disk-mass / force / torque reduction that allocates no
// device memory.
//
// Who needs it: callers that hold their own device buffers and must not
// allocate.  Examples: a serving process that has handed all of its HBM to
// its own memory pool (a cudaMalloc there fails or steals from the pool), or
// a driver loop (such as the reference's main.cu with its own GPU_plan
// buffers) that allocates once at start-up and wants no allocation, nor the
// implicit device synchronisation cudaMalloc/cudaFree may bring, inside its
// time loop.  pg_reduce needs a pg_run, whose creation allocates; this entry
// point works on plain device pointers the caller owns.
//
// Scratch: the per-ring partial sums and the completion counter live in
// file-scope __device__ arrays of fixed size, PG_NOALLOC_MAX_RINGS rings
// (16384 doubles = 128 KiB, plus one counter).  Every GPU that loads this
// library keeps that memory until the process exits.  All calls share it:
// calls whose kernels overlap on the GPU (different streams, no ordering
// between them) race on it and give wrong results; calls on one stream, or
// otherwise ordered, are safe.  The counter is cleared by every call before
// its kernel runs; the partial sums are fully rewritten by each call.
//
// Set-up: the first call on each device looks up the device address of the
// scratch arrays with cudaGetSymbolAddress, with that device current, and
// caches it.  Make that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "../../include/penguin_b200.h"
#include "pg_ppm.cuh"

namespace {

static __device__ __align__(256) double g_ring_part[PG_NOALLOC_MAX_RINGS];
static __device__ __align__(256) unsigned int g_done[1];

// per device: the scratch symbols' addresses, looked up once.  ready is set
// with release order after part and done, so a thread that sees it set (acquire)
// also sees the pointers; the mutex keeps two first calls from looking up at once.
struct Scratch {
  std::atomic<bool> ready;
  double *part;
  unsigned int *done;
};
static Scratch g_scratch[64];
static std::mutex g_setup_mu;

__device__ __forceinline__ double tree1024(double *list) {
  for (int len = 1024; len > 1; len >>= 1) {
    int half = len >> 1;
    if ((int)threadIdx.x < half) list[threadIdx.x] += list[threadIdx.x + half];
    __syncthreads();
  }
  return list[0];
}

// output_lv1 + output_lv3 of device_func.cu:49-167 (2D), over caller arrays:
// sigma[i*row_stride + j] in physical azimuth order, rot_j[i] the ring's FARGO
// offset (storage index j_s holds physical (j_s + rot_j) mod jmax).  rot_j
// may be any int: it is reduced into [0, jmax) once per ring, which for the
// offsets output_lv1 wraps (device_func.cu:71-73, -jmax < rot_j < 2 jmax)
// gives the same column.  With imax <= 1024 the ring partials are summed in
// output_lv3's single 1024-wide tree; above that they are summed 1024 at a
// time, an extension with no reference counterpart (output_lv3 holds 1024).
__global__ void __launch_bounds__(1024) k_reduce_noalloc(
    const double *sigma, long long row_stride, const double *xc, const double *xvol, const int *rot_j,
    const double *yc, const double *yvol, int imax, int jmax, pgd::Body pl, double exclude, int mode,
    double p_alpha, double *part, unsigned int *done, double *out) {
  __shared__ double list[1024];
  __shared__ bool is_last;
  const int i = blockIdx.x, tt = threadIdx.x;
  int rot = rot_j[i] % jmax;
  if (rot < 0) rot += jmax;
  const double rad = xc[i], xv = xvol[i];
  const double *row = sigma + (size_t)i * row_stride;
  const int loop = jmax / 1024 + (jmax % 1024 != 0);
  double val = 0.0;
  for (int l = 0; l < loop; l++) {
    int j = tt + 1024 * l;
    double v = 0.0;
    if (j < jmax) {
      int j0 = j + rot;
      if (j0 >= jmax) j0 -= jmax;
      double phi = yc[j0];
      double r = row[j0];
      if (mode == 0) {
        v = r * xv * yvol[j0] * 1.0;
      } else if ((rad - pl.x) * (rad - pl.x) + rad * rad * (phi - pl.y) * (phi - pl.y) > exclude * exclude) {
        if (mode == 8) {
          double t = -pgd::grav_rad_cyl(rad, phi, 0.0, pl, 0.0);
          t *= (r - pow(rad, -p_alpha)) * xv * yvol[j0];
          v = t;
        } else {
          double t = -pgd::grav_azi_cyl(rad, phi, 0.0, pl, 0.0);
          t *= rad * (r - pow(rad, -p_alpha)) * xv * yvol[j0];
          v = t;
        }
      }
    }
    list[tt] = v;
    __syncthreads();
    double s = tree1024(list);
    if (tt == 0) val += s;
    __syncthreads();
  }
  if (tt == 0) {
    part[i] = val;
    __threadfence();
    unsigned int prev = atomicAdd(done, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  const volatile double *pv = part;
  double total = 0.0;
  for (int b = 0; b < imax; b += 1024) {
    int ii = b + tt;
    list[tt] = (ii < imax) ? pv[ii] : 0.0;
    __syncthreads();
    double s = tree1024(list);
    if (tt == 0) total += s;
    __syncthreads();
  }
  if (tt == 0) *out = 0.0 + total;
}

int setup_device(int dev) {
  if (dev < 0 || dev >= 64) return PG_ERR_ARG;
  Scratch &s = g_scratch[dev];
  if (s.ready.load(std::memory_order_acquire)) return PG_OK;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (s.ready.load(std::memory_order_relaxed)) return PG_OK;
  void *a = nullptr, *b = nullptr;
  if (cudaGetSymbolAddress(&a, g_ring_part) != cudaSuccess) return PG_ERR_CUDA;
  if (cudaGetSymbolAddress(&b, g_done) != cudaSuccess) return PG_ERR_CUDA;
  s.part = (double *)a;
  s.done = (unsigned int *)b;
  s.ready.store(true, std::memory_order_release);
  return PG_OK;
}

}  // namespace

extern "C" int pg_reduce_noalloc(const double *sigma, int64_t row_stride, const double *xc,
                                 const double *xvol, const int *rot_j, const double *yc,
                                 const double *yvol, int imax, int jmax, const pg_body *planet,
                                 double exclude, int mode, double p_alpha, double sc_h,
                                 double *out, void *stream) {
  if (!sigma || !xc || !xvol || !rot_j || !yc || !yvol || !planet || !out) return PG_ERR_ARG;
  if (mode != 0 && mode != 8 && mode != 9) return PG_ERR_ARG;
  if (imax < 1 || jmax < 1 || row_stride < jmax) return PG_ERR_ARG;
  if (imax > PG_NOALLOC_MAX_RINGS) {
    std::fprintf(stderr, "pg_reduce_noalloc: imax = %d exceeds the static scratch of %d rings\n", imax,
                 PG_NOALLOC_MAX_RINGS);
    return PG_ERR_PARAMS;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PG_ERR_CUDA;
  int st = setup_device(dev);
  if (st) return st;
  const Scratch &s = g_scratch[dev];
  cudaStream_t cs = (cudaStream_t)stream;
  if (cudaMemsetAsync(s.done, 0, sizeof(unsigned int), cs) != cudaSuccess) return PG_ERR_CUDA;
  pgd::Body b{planet->m, planet->x, planet->y, planet->vx, planet->vy, planet->fx, planet->fy, planet->rs};
  exclude *= sc_h;                          // GPU_output_reduction device_func.cu:171
  k_reduce_noalloc<<<imax, 1024, 0, cs>>>(sigma, (long long)row_stride, xc, xvol, rot_j, yc, yvol, imax, jmax, b,
                                          exclude, mode, p_alpha, s.part, s.done, out);
  return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}
