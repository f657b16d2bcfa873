// rh_fiber.cpp -- fibers and the per-block barrier scheduler (see rh_fiber.h).
// The context switch is a few lines of x86-64 assembly: it saves the
// callee-saved registers of the SysV ABI on the current stack, swaps stack
// pointers and restores the other context's registers.
#include "rh_fiber.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" void rh_swap(void **save_sp, void *load_sp);
asm(R"(
.text
.globl rh_swap
.type rh_swap, @function
rh_swap:
  pushq %rbp
  pushq %rbx
  pushq %r12
  pushq %r13
  pushq %r14
  pushq %r15
  movq %rsp, (%rdi)
  movq %rsi, %rsp
  popq %r15
  popq %r14
  popq %r13
  popq %r12
  popq %rbx
  popq %rbp
  ret
.size rh_swap, .-rh_swap
.section .note.GNU-stack,"",@progbits
.text
)");

namespace rh {

thread_local dim3_t tl_threadIdx, tl_blockIdx;
dim3_t g_blockDim{1, 1, 1}, g_gridDim{1, 1, 1};

namespace {

// Bytes of stack per CUDA thread.  The stacks sit in one arena at a stride
// that is not a power of two, so the hot tops of 128 or 1024 stacks fall in
// different cache sets (at a 64 KiB stride they all share one).
constexpr size_t kStack = 64 * 1024 + 7 * 64;

struct Fiber {
  void *sp = nullptr;
  char *stack = nullptr;
  bool done = true;
  dim3_t tid{0, 0, 0};
};

// one per OS thread: the block being run
struct Block {
  std::vector<Fiber> f;
  std::vector<char *> arenas;
  void *sched_sp = nullptr;
  int cur = -1;
  int n = 0;
  const std::function<void()> *body = nullptr;
};
thread_local Block *tl_block = nullptr;

// The fiber after t (round robin) that has not returned, or -1.  Fibers run
// in index order, each up to its next barrier, so when the last one of a
// round yields every fiber has arrived and the first one may go on.
int next_live(const Block &b, int t, int n) {
  for (int k = t + 1; k < n; k++)
    if (!b.f[k].done) return k;
  for (int k = 0; k <= t; k++)
    if (!b.f[k].done) return k;
  return -1;
}

[[noreturn]] void fiber_entry() {
  Block *b = tl_block;
  (*b->body)();
  b->f[b->cur].done = true;
  const int nx = next_live(*b, b->cur, b->n);
  void *dummy;
  if (nx < 0) {
    rh_swap(&dummy, b->sched_sp);   // block finished; never resumed
  } else {
    b->cur = nx;
    tl_threadIdx = b->f[nx].tid;
    rh_swap(&dummy, b->f[nx].sp);
  }
  std::abort();
}

void prepare(Fiber &fb) {
  uintptr_t top = (reinterpret_cast<uintptr_t>(fb.stack) + kStack) & ~uintptr_t(15);
  void **s = reinterpret_cast<void **>(top);
  *--s = nullptr;                                   // fake return address of fiber_entry
  *--s = reinterpret_cast<void *>(&fiber_entry);    // rh_swap returns here
  for (int r = 0; r < 6; r++) *--s = nullptr;       // rbp rbx r12-r15
  fb.sp = s;
  fb.done = false;
}

void run_block(Block &b, unsigned nthreads, const std::function<void()> &body) {
  if (b.f.size() < nthreads) {
    const size_t have = b.f.size();
    b.f.resize(nthreads);
    char *arena = static_cast<char *>(std::malloc((nthreads - have) * kStack + 64));
    if (!arena) { std::fprintf(stderr, "rh: out of memory for fiber stacks\n"); std::abort(); }
    b.arenas.push_back(arena);
    for (size_t t = have; t < nthreads; t++) b.f[t].stack = arena + (t - have) * kStack;
  }
  b.body = &body;
  const unsigned bx = g_blockDim.x, by = g_blockDim.y;
  for (unsigned t = 0; t < nthreads; t++) {
    prepare(b.f[t]);
    b.f[t].tid = dim3_t{t % bx, (t / bx) % by, t / (bx * by)};
  }
  // the fibers hand over to each other at barriers (syncthreads) and come
  // back here when the last one returns
  b.n = (int)nthreads;
  b.cur = 0;
  tl_threadIdx = b.f[0].tid;
  rh_swap(&b.sched_sp, b.f[0].sp);
}

}  // namespace

void syncthreads() {
  Block *b = tl_block;
  const int me = b->cur;
  const int nx = next_live(*b, me, b->n);
  if (nx == me) return;   // the only fiber left: the barrier is its own
  b->cur = nx;
  tl_threadIdx = b->f[nx].tid;
  rh_swap(&b->f[me].sp, b->f[nx].sp);
}

void launch(unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by, unsigned bz,
            const std::function<void()> &body) {
  g_gridDim = dim3_t{gx, gy, gz};
  g_blockDim = dim3_t{bx, by, bz};
  const long nblocks = (long)gx * gy * gz;
  const unsigned nthreads = bx * by * bz;
#pragma omp parallel
  {
    if (!tl_block) tl_block = new Block();
    Block &b = *tl_block;
#pragma omp for schedule(dynamic, 1)
    for (long n = 0; n < nblocks; n++) {
      tl_blockIdx = dim3_t{(unsigned)(n % gx), (unsigned)((n / gx) % gy), (unsigned)(n / ((long)gx * gy))};
      run_block(b, nthreads, body);
    }
  }
}

int threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // namespace rh

// ---- host-clock events for the shim's cudaEvent* ---------------------------
#include <chrono>
typedef void *cudaEvent_t;
typedef void *cudaStream_t;
typedef int cudaError_t;

cudaError_t cudaEventCreate(cudaEvent_t *e) {
  *e = new std::chrono::steady_clock::time_point();
  return 0;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
  *static_cast<std::chrono::steady_clock::time_point *>(e) = std::chrono::steady_clock::now();
  return 0;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return 0; }
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b) {
  auto ta = *static_cast<std::chrono::steady_clock::time_point *>(a);
  auto tb = *static_cast<std::chrono::steady_clock::time_point *>(b);
  *ms = std::chrono::duration<float, std::milli>(tb - ta).count();
  return 0;
}
