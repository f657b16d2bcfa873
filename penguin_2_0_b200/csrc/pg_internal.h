// pg_internal.h -- what the batch and serving code (pg_batch.cu, pg_serve.cpp)
// use of a run object.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/penguin_b200.h"
#include "pg_kernels.cuh"

namespace pgi {

struct RunShape {
  int dev, ndim, fp32, loaded, clock_ready, p0_live;
  int moving;              // plnt_flag 2: the planet feels the disk (own step sequence)
  int eos;                 // EOS 1: isentropic sweeps (own step sequence)
  int nr, nphi, nk;
  int tiles_x, tiles_y;    // 2D pencil chunks of the radial and azimuthal sweeps
  int tiles_xs;            // radial last chunks of at most 64 cells, 4 columns per tile
                           // (then not counted in tiles_x)
};
int run_shape(const pg_run *run, RunShape *out);

// Device descriptor of a 2D run whose clock is set (pg_clock_reset).
int run_batch_desc(pg_run *run, pgd::BatchRun *d);
// The batch enqueued steps of this run: the p0 plane is used up, count launches.
void run_batched(pg_run *run, int64_t launches);
// One step of the device-resident loop of this run, enqueued on stream s.
int run_enqueue_on(pg_run *run, cudaStream_t s, int64_t *launches);
// Device clock of the run.
pgd::DevClock *run_clock(pg_run *run);
// which of the two plane copies is current (3D steps flip it)
int run_cur(const pg_run *run);
cudaStream_t run_stream(pg_run *run);

}  // namespace pgi
