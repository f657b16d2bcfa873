// pg_batch.cu -- many disk runs stepped together on one GPU.
//
// The reference runs one disk per process.  Here a batch holds any number of
// runs (each a pg_run with its own planes, tables, clock and dt) and steps
// them together:
//   * 2D members are split by precision into two groups.  For each group a
//     step is one launch per phase: prestep (one CTA per run: dt, Index_Shift,
//     half kick), radial sweep and azimuthal sweep (a tile queue over the
//     pencil chunks of every member; CTA b takes tiles b, b + grid, ...),
//     poststep, mass and torque reductions (one CTA per ring of every member)
//     and the history record.
//   * 3D members, members with a moving planet (plnt_flag 2) and isentropic
//     members (EOS 1) take their own launch sequence (the per-run fused
//     step) in the same stream order; the queue kernels are isothermal 2D.
// The step sequence of `chunk` steps is captured once as a CUDA graph and
// replayed; membership changes rebuild the descriptors and the graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pg_internal.h"
#include "pg_kernels.cuh"

namespace {

// per-member clock snapshot for pg_batch_status and the early exit
__global__ void kb_status(pgd::DevClock *const *clks, int n, pg_batch_member *out, int *halted_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const pgd::DevClock &c = *clks[i];
    out[i].halted = c.halted;
    out[i].status = c.status;
    out[i].ncycle = c.ncycle;
    out[i].simtime = c.simtime;
    if (c.halted) atomicAdd(halted_count, 1);
  }
}

struct Group {
  std::vector<pg_run *> members;
  pgd::BatchRun *d_runs = nullptr;
  int *d_start = nullptr;          // [4][n+1]: radial tiles, azimuthal tiles, rings, short radial tiles
  size_t cap = 0;
  pgd::BatchQueue qx{}, qy{}, qr{}, qxs{};
  pg_batch_shape shape{0, 0, 8, 0};
};

}  // namespace

struct pg_batch {
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<pg_run *> runs;      // in the order added
  Group g[2];                      // 2D members: FP64, FP32
  std::vector<pg_run *> solo;      // members with their own step sequence
  bool dirty = true;
  cudaGraphExec_t gexec = nullptr;
  int gsteps = 0;
  int64_t graph_kernels = 0;
  std::vector<int> solo_cur;       // plane copy of each 3D member at capture
  int64_t launches = 0;
  // status snapshot
  pgd::DevClock **d_clks = nullptr;
  pg_batch_member *d_status = nullptr, *h_status = nullptr;
  int *d_halted = nullptr, *h_halted = nullptr;
  size_t status_cap = 0;
  cudaEvent_t probe[4] = {};
};

#define BK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
      (void)cudaGetLastError(); /* reported: not a later launch's error */    \
      return PG_ERR_CUDA;                                                     \
    }                                                                         \
  } while (0)

static int bfail(pg_batch *b, int code, const std::string &msg) {
  b->err = msg;
  return code;
}

static void drop_graph(pg_batch *b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->gsteps = 0;
}

// descriptors, tile prefix sums and the status arrays for the current members
static int rebuild(pg_batch *b) {
  BK(cudaStreamSynchronize(b->stream));   // in-flight steps read the old descriptors
  drop_graph(b);
  for (auto &g : b->g) g.members.clear();
  b->solo.clear();
  for (pg_run *r : b->runs) {
    pgi::RunShape sh;
    pgi::run_shape(r, &sh);
    if (sh.ndim == 3 || sh.moving || sh.eos) b->solo.push_back(r);
    else b->g[sh.fp32].members.push_back(r);
  }
  for (auto &g : b->g) {
    size_t n = g.members.size();
    if (n > g.cap) {
      cudaFree(g.d_runs);
      cudaFree(g.d_start);
      g.d_runs = nullptr;
      g.d_start = nullptr;
      size_t cap = std::max<size_t>(n, 16);
      BK(cudaMalloc(&g.d_runs, cap * sizeof(pgd::BatchRun)));
      BK(cudaMalloc(&g.d_start, 4 * (cap + 1) * sizeof(int)));
      g.cap = cap;
    }
    std::vector<pgd::BatchRun> h(n);
    std::vector<int> st(4 * (n + 1), 0);
    for (size_t i = 0; i < n; i++) {
      pg_run *r = g.members[i];
      if (int e = pgi::run_batch_desc(r, &h[i])) return bfail(b, e, pg_last_error(r));
      pgi::RunShape sh;
      pgi::run_shape(r, &sh);
      st[i + 1] = st[i] + sh.tiles_x;
      st[(n + 1) + i + 1] = st[(n + 1) + i] + sh.tiles_y;
      st[2 * (n + 1) + i + 1] = st[2 * (n + 1) + i] + sh.nr;
      st[3 * (n + 1) + i + 1] = st[3 * (n + 1) + i] + sh.tiles_xs;
    }
    if (n) {
      BK(cudaMemcpy(g.d_runs, h.data(), n * sizeof(pgd::BatchRun), cudaMemcpyHostToDevice));
      BK(cudaMemcpy(g.d_start, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    int ni = (int)n;
    g.qx = {g.d_runs, g.d_start, ni, st[n]};
    g.qy = {g.d_runs, g.d_start + (n + 1), ni, st[(n + 1) + n]};
    g.qr = {g.d_runs, g.d_start + 2 * (n + 1), ni, st[2 * (n + 1) + n]};
    g.qxs = {g.d_runs, g.d_start + 3 * (n + 1), ni, st[3 * (n + 1) + n]};
  }
  size_t n = b->runs.size();
  if (n > b->status_cap) {
    cudaFree(b->d_clks);
    cudaFree(b->d_status);
    if (b->h_status) cudaFreeHost(b->h_status);
    b->d_clks = nullptr; b->d_status = nullptr; b->h_status = nullptr;
    size_t cap = std::max<size_t>(n, 16);
    BK(cudaMalloc(&b->d_clks, cap * sizeof(pgd::DevClock *)));
    BK(cudaMalloc(&b->d_status, cap * sizeof(pg_batch_member)));
    BK(cudaHostAlloc(&b->h_status, cap * sizeof(pg_batch_member), cudaHostAllocDefault));
    b->status_cap = cap;
  }
  std::vector<pgd::DevClock *> clks(n);
  for (size_t i = 0; i < n; i++) clks[i] = pgi::run_clock(b->runs[i]);
  if (n) BK(cudaMemcpy(b->d_clks, clks.data(), n * sizeof(pgd::DevClock *), cudaMemcpyHostToDevice));
  b->dirty = false;
  return PG_OK;
}

// one step of the members of group gi
static void enqueue_group_step(pg_batch *b, int gi, int64_t *nk) {
  cudaStream_t s = b->stream;
  Group &g = b->g[gi];
  int n = (int)g.members.size();
  if (!n) return;
  pgk::batch_prestep(g.d_runs, n, s);
  if (gi == 1) {
    pgk::batch_sweep_x32(g.qx, g.shape.grid_x, g.shape.minb, s);
    pgk::batch_sweep_x32_short(g.qxs, s);
    pgk::batch_sweep_y32(g.qy, g.shape.grid_y, g.shape.minb, s);
  } else {
    pgk::batch_sweep_x(g.qx, g.shape.grid_x, g.shape.minb, s);
    pgk::batch_sweep_x_short(g.qxs, s);
    pgk::batch_sweep_y(g.qy, g.shape.grid_y, g.shape.minb, s);
  }
  pgk::batch_poststep(g.d_runs, n, s);
  pgk::batch_reduce(g.qr, gi, 0, s);
  pgk::batch_reduce(g.qr, gi, 9, s);
  pgk::batch_record(g.d_runs, n, s);
  *nk += 8 + (g.qxs.total > 0 ? 1 : 0);
}

// one step of every member, on the batch stream
static int enqueue_batch_step(pg_batch *b, int64_t *nk) {
  cudaStream_t s = b->stream;
  for (int gi = 0; gi < 2; gi++) enqueue_group_step(b, gi, nk);
  for (pg_run *r : b->solo)
    if (int e = pgi::run_enqueue_on(r, s, nk)) return bfail(b, e, pg_last_error(r));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(b, PG_ERR_CUDA, cudaGetErrorString(e));
  return PG_OK;
}

// count of halted members, read back through pinned memory
static int snapshot(pg_batch *b) {
  int n = (int)b->runs.size();
  BK(cudaMemsetAsync(b->d_halted, 0, sizeof(int), b->stream));
  if (n) kb_status<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_clks, n, b->d_status, b->d_halted);
  BK(cudaGetLastError());
  if (n) BK(cudaMemcpyAsync(b->h_status, b->d_status, n * sizeof(pg_batch_member), cudaMemcpyDeviceToHost, b->stream));
  BK(cudaMemcpyAsync(b->h_halted, b->d_halted, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  return PG_OK;
}

extern "C" {

int pg_batch_create(int device, pg_batch **out) {
  if (!out) return PG_ERR_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return PG_ERR_CUDA;
  pg_batch *b = new pg_batch();
  b->dev = device;
  b->g[1].shape.minb = 4;   // the FP32 sweeps keep ~80 registers
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->d_halted, sizeof(int)) != cudaSuccess ||
      cudaHostAlloc(&b->h_halted, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
    pg_batch_destroy(b);
    (void)cudaGetLastError();
    return PG_ERR_CUDA;
  }
  for (auto &e : b->probe)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      pg_batch_destroy(b);
      return PG_ERR_CUDA;
    }
  *out = b;
  return PG_OK;
}

int pg_batch_destroy(pg_batch *b) {
  if (!b) return PG_OK;
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (auto &g : b->g) {
    cudaFree(g.d_runs);
    cudaFree(g.d_start);
  }
  cudaFree(b->d_clks);
  cudaFree(b->d_status);
  cudaFree(b->d_halted);
  if (b->h_status) cudaFreeHost(b->h_status);
  if (b->h_halted) cudaFreeHost(b->h_halted);
  for (auto e : b->probe) if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PG_OK;
}

const char *pg_batch_last_error(const pg_batch *b) { return b ? b->err.c_str() : "null batch"; }

int pg_batch_add(pg_batch *b, pg_run *run) {
  if (!b || !run) return PG_ERR_ARG;
  pgi::RunShape sh;
  pgi::run_shape(run, &sh);
  if (sh.dev != b->dev) return bfail(b, PG_ERR_ARG, "run is on another device");
  if (!sh.loaded || !sh.clock_ready) return bfail(b, PG_ERR_STATE, "run needs pg_load_* and pg_clock_reset");
  if (std::find(b->runs.begin(), b->runs.end(), run) != b->runs.end())
    return bfail(b, PG_ERR_ARG, "run is already in the batch");
  BK(cudaSetDevice(b->dev));
  BK(cudaStreamSynchronize(pgi::run_stream(run)));
  b->runs.push_back(run);
  b->dirty = true;
  return PG_OK;
}

int pg_batch_remove(pg_batch *b, pg_run *run) {
  if (!b || !run) return PG_ERR_ARG;
  auto it = std::find(b->runs.begin(), b->runs.end(), run);
  if (it == b->runs.end()) return bfail(b, PG_ERR_ARG, "run is not in the batch");
  BK(cudaSetDevice(b->dev));
  BK(cudaStreamSynchronize(b->stream));
  b->runs.erase(it);
  b->dirty = true;
  return PG_OK;
}

int pg_batch_size(const pg_batch *b) { return b ? (int)b->runs.size() : 0; }

int pg_batch_sync(pg_batch *b) {
  if (!b) return PG_ERR_ARG;
  BK(cudaSetDevice(b->dev));
  BK(cudaStreamSynchronize(b->stream));
  return PG_OK;
}

int pg_batch_advance(pg_batch *b, int nsteps, int chunk) {
  if (!b || nsteps < 0) return PG_ERR_ARG;
  if (chunk < 1) chunk = 1;
  BK(cudaSetDevice(b->dev));
  if (b->runs.empty() || nsteps == 0) return PG_OK;
  if (b->dirty)
    if (int e = rebuild(b)) return e;
  if (!b->solo.empty() && (chunk & 1)) chunk += 1;   // 3D steps alternate the plane copies
  int done = 0;
  // a 3D member with a freshly loaded dump reads its p0 plane in its first
  // step only: take that step outside the graph (2D members select p0 by
  // their step count inside the kernels, so a replay never re-reads it)
  bool p0_solo = false;
  for (pg_run *r : b->solo) {
    pgi::RunShape sh;
    pgi::run_shape(r, &sh);
    if (sh.p0_live) p0_solo = true;
  }
  if (p0_solo) {
    int64_t nk = 0;
    if (int e = enqueue_batch_step(b, &nk)) return e;
    b->launches += nk;
    done = 1;
  }
  // 3D members flip their plane copies once per step: a graph captured with
  // other copies current is stale
  bool stale = false;
  for (size_t i = 0; i < b->solo.size(); i++)
    if (i >= b->solo_cur.size() || pgi::run_cur(b->solo[i]) != b->solo_cur[i]) stale = true;
  if (!b->gexec || b->gsteps != chunk || stale) {
    drop_graph(b);
    b->solo_cur.clear();
    for (pg_run *r : b->solo) b->solo_cur.push_back(pgi::run_cur(r));
    cudaGraph_t gr;
    int64_t nk = 0;
    // an even chunk leaves the 3D members' plane copies where they started
    BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < chunk; i++) {
      if (int e = enqueue_batch_step(b, &nk)) {
        cudaStreamEndCapture(b->stream, &gr);
        return e;
      }
    }
    BK(cudaStreamEndCapture(b->stream, &gr));
    BK(cudaGraphInstantiate(&b->gexec, gr, 0));
    cudaGraphDestroy(gr);
    b->gsteps = chunk;
    b->graph_kernels = nk;
  }
  int64_t unit = 0;
  for (; done + chunk <= nsteps; done += chunk, unit++) {
    // early exit: every 4th replay, read the halted count of 4 replays back
    if (unit >= 4 && (unit & 3) == 0) {
      BK(cudaEventSynchronize(b->probe[(unit / 4 - 1) & 3]));
      if (*b->h_halted == (int)b->runs.size()) break;
    }
    BK(cudaGraphLaunch(b->gexec, b->stream));
    b->launches += b->graph_kernels;
    if ((unit & 3) == 3) {
      if (int e = snapshot(b)) return e;
      BK(cudaEventRecord(b->probe[(unit / 4) & 3], b->stream));
    }
  }
  if (done < nsteps && done + chunk > nsteps) {
    int64_t nk = 0;
    for (; done < nsteps; done++)
      if (int e = enqueue_batch_step(b, &nk)) return e;
    b->launches += nk;
  }
  for (auto &g : b->g)
    for (pg_run *r : g.members) pgi::run_batched(r, 0);
  return PG_OK;
}

int pg_batch_status(pg_batch *b, pg_batch_member *out, int n) {
  if (!b || (!out && n > 0)) return PG_ERR_ARG;
  BK(cudaSetDevice(b->dev));
  if (b->dirty)
    if (int e = rebuild(b)) return e;
  if (int e = snapshot(b)) return e;
  BK(cudaStreamSynchronize(b->stream));
  int m = std::min(n, (int)b->runs.size());
  for (int i = 0; i < m; i++) out[i] = b->h_status[i];
  return PG_OK;
}

int pg_batch_set_shape(pg_batch *b, int group, const pg_batch_shape *shape) {
  if (!b || !shape || group < 0 || group > 1) return PG_ERR_ARG;
  if (shape->grid_x < 0 || shape->grid_y < 0 || (shape->minb != 4 && shape->minb != 8)) return PG_ERR_ARG;
  b->g[group].shape = *shape;
  drop_graph(b);
  return PG_OK;
}

int pg_batch_get_shape(const pg_batch *b, int group, pg_batch_shape *shape) {
  if (!b || !shape || group < 0 || group > 1) return PG_ERR_ARG;
  *shape = b->g[group].shape;
  return PG_OK;
}

int pg_batch_tune(pg_batch *b, int trial_steps) {
  if (!b) return PG_ERR_ARG;
  if (trial_steps < 1) trial_steps = 1;
  BK(cudaSetDevice(b->dev));
  if (b->dirty)
    if (int e = rebuild(b)) return e;
  int sms = 148;
  BK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev));
  cudaEvent_t e0, e1;
  BK(cudaEventCreate(&e0));
  BK(cudaEventCreate(&e1));
  int rc = PG_OK;
  for (int gi = 0; gi < 2 && rc == PG_OK; gi++) {
    Group &g = b->g[gi];
    if (g.members.empty()) continue;
    // candidates: CTAs per SM the sweeps are compiled for, and one CTA per
    // tile or a persistent grid of 1 or 2 waves walking the tile queue
    std::vector<pg_batch_shape> cand;
    for (int minb : {8, 4})
      for (int waves : {0, 1, 2}) {
        int grid = waves ? waves * minb * sms : 0;
        cand.push_back(pg_batch_shape{grid, grid, minb, 0});
      }
    float best = 1e30f;
    pg_batch_shape keep = g.shape;
    for (const pg_batch_shape &c : cand) {
      g.shape = c;
      int64_t nk = 0;
      enqueue_group_step(b, gi, &nk);   // warm-up step
      if (cudaEventRecord(e0, b->stream) != cudaSuccess) { rc = PG_ERR_CUDA; break; }
      for (int i = 0; i < trial_steps; i++) enqueue_group_step(b, gi, &nk);
      if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
        rc = PG_ERR_CUDA;
        break;
      }
      b->launches += nk;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) { best = ms; keep = c; }
    }
    g.shape = keep;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return bfail(b, rc, "tuning launches failed");
  drop_graph(b);
  for (auto &g : b->g)
    for (pg_run *r : g.members) pgi::run_batched(r, 0);
  return PG_OK;
}

int64_t pg_batch_launch_count(const pg_batch *b) { return b ? b->launches : 0; }

void *pg_batch_stream(const pg_batch *b) { return b ? (void *)b->stream : nullptr; }

}  // extern "C"
