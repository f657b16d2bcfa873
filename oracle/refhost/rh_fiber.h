// rh_fiber.h -- a CUDA-thread emulator for running the reference's own
// kernels on the host (TEST INFRASTRUCTURE: the timed CPU baseline and a
// host-side pin of the restatement; never part of the product).
//
// Each CUDA thread of a block is a fiber (its own stack, its own locals);
// the fibers of one block run on one OS thread and switch only at
// __syncthreads(), so a barrier is a yield: the block's scheduler resumes the
// next fiber, and a barrier is released once every fiber that has not
// returned has reached one.  __shared__ data become `static thread_local`,
// shared by the fibers of the block running on that OS thread.  Blocks of a
// grid are spread over OS threads with OpenMP; a launch returns when every
// block has finished (the reference synchronises its stream after every
// launch sequence, so stream order is kept).
#pragma once
#include <functional>

namespace rh {

struct dim3_t {
  unsigned x, y, z;
};

// the running fiber's CUDA indices (set by the scheduler before it resumes one)
extern thread_local dim3_t tl_threadIdx, tl_blockIdx;
extern dim3_t g_blockDim, g_gridDim;

void syncthreads();
// Runs body once per CUDA thread of grid x block; body reads the indices above.
void launch(unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by, unsigned bz,
            const std::function<void()> &body);
// OS threads used for blocks (OpenMP)
int threads();

}  // namespace rh
