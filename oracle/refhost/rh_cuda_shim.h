// rh_cuda_shim.h -- force-included (g++ -include) ahead of the reference's
// own .cu translation units when they are compiled for the host (TEST
// INFRASTRUCTURE; see rh_fiber.h).  It supplies what nvcc and the CUDA
// runtime would: the execution-space keywords, the thread indices, the
// block barrier, the vector types and the runtime calls the reference's host
// code makes, acting on host memory.  The reference's arithmetic is compiled
// as written, by the host compiler and against the host libm.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "rh_fiber.h"

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static thread_local
#define __syncthreads() ::rh::syncthreads()

struct uint3 {
  unsigned x, y, z;
};
struct dim3 {
  unsigned x, y, z;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct double2 {
  double x, y;
};

#define threadIdx (::rh::tl_threadIdx)
#define blockIdx (::rh::tl_blockIdx)
#define blockDim (::rh::g_blockDim)
#define gridDim (::rh::g_gridDim)

// CUDA's max/min overloads for the argument types the reference mixes
inline double max(double a, double b) { return std::fmax(a, b); }
inline double min(double a, double b) { return std::fmin(a, b); }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline double max(double a, int b) { return std::fmax(a, (double)b); }
inline double max(int a, double b) { return std::fmax((double)a, b); }
inline double min(double a, int b) { return std::fmin(a, (double)b); }
inline double min(int a, double b) { return std::fmin((double)a, b); }

// ---- runtime API subset used by the reference's host code: host memory,
// synchronous execution (every launch has finished when it returns) ----------
typedef int cudaError;
typedef int cudaError_t;
typedef void *cudaStream_t;
typedef void *cudaEvent_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                      cudaMemcpyDeviceToDevice, cudaMemcpyDefault };
enum cudaFuncCache { cudaFuncCachePreferNone, cudaFuncCachePreferShared, cudaFuncCachePreferL1,
                     cudaFuncCachePreferEqual };

inline const char *cudaGetErrorString(int) { return "no error"; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaDeviceSetCacheConfig(cudaFuncCache) { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaGetDevice(int *d) { *d = 0; return cudaSuccess; }
inline cudaError_t cudaDeviceReset() { return cudaSuccess; }
inline cudaError_t cudaDeviceEnablePeerAccess(int, unsigned) { return cudaSuccess; }
inline cudaError_t cudaDeviceDisablePeerAccess(int) { return cudaSuccess; }
inline cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned) { return cudaSuccess; }
inline cudaError_t cudaStreamCreate(cudaStream_t *s) { *s = nullptr; return cudaSuccess; }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaMalloc(void **p, size_t n) { *p = std::calloc(1, n ? n : 1); return *p ? 0 : 2; }
inline cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
inline cudaError_t cudaFree(void *p) { std::free(p); return cudaSuccess; }
inline cudaError_t cudaFreeHost(void *p) { std::free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) {
  std::memmove(d, s, n);
  return cudaSuccess;
}
inline cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, cudaMemcpyKind k, cudaStream_t = nullptr) {
  return cudaMemcpy(d, s, n, k);
}
// events time on the host clock (rh_fiber.cpp)
cudaError_t cudaEventCreate(cudaEvent_t *e);
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t = nullptr);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b);

// kernel<<<grid, block, shmem, stream>>>(args) is rewritten by the build
// recipe (oracle/refhost/launch_rewrite.py) into
// RH_LAUNCH(grid, block, [&] { kernel(args); })
template <class F>
inline void RH_LAUNCH(dim3 g, dim3 b, F &&f) {
  const std::function<void()> body(f);
  ::rh::launch(g.x, g.y, g.z, b.x, b.y, b.z, body);
}
