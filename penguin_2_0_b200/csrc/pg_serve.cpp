// pg_serve.cpp -- a serving loop for disk runs on one GPU (continuous batching).
//
// Requests (a pg_params each: grid, planet mass, h, alpha, end time) arrive
// over time.  The loop keeps every admitted run's state on the device and
// steps all of them together in one pg_batch; it admits queued requests in
// arrival order whenever a slot and enough of the HBM budget are free (the
// footprint is pg_run_device_bytes), retires runs whose clock halted at their
// end time, and records arrival, admission and completion times.  Host work
// (building a new run's initial state, loading it) overlaps the batch's
// steps: a round enqueues `chunk` steps of the batch, does the admission
// work while they run, then synchronises and retires.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/penguin_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Live {
  int64_t id;
  int req;              // index into the trace
  pg_run *run;
  size_t bytes;
  double admit_s;
};

}  // namespace

struct pg_server {
  int dev = 0;
  size_t budget = 0, used = 0;
  int max_slots = 64;
  int chunk = 32;
  int keep_results = 0;
  pg_batch *batch = nullptr;
  std::string err;
  std::vector<Live> live;
  std::map<int64_t, std::vector<unsigned char>> results;
  int64_t rounds = 0;
};

static int sfail(pg_server *s, int code, const std::string &m) {
  s->err = m;
  return code;
}

extern "C" {

int pg_server_create(int device, size_t hbm_budget, int max_slots, int chunk, int keep_results,
                     pg_server **out) {
  if (!out || hbm_budget == 0 || max_slots < 1 || chunk < 1) return PG_ERR_ARG;
  *out = nullptr;
  pg_server *s = new pg_server();
  s->dev = device;
  s->budget = hbm_budget;
  s->max_slots = max_slots;
  s->chunk = chunk;
  s->keep_results = keep_results;
  int st = pg_batch_create(device, &s->batch);
  if (st) {
    delete s;
    return st;
  }
  *out = s;
  return PG_OK;
}

int pg_server_destroy(pg_server *s) {
  if (!s) return PG_OK;
  for (auto &l : s->live) {
    pg_batch_remove(s->batch, l.run);
    pg_destroy(l.run);
  }
  pg_batch_destroy(s->batch);
  delete s;
  return PG_OK;
}

const char *pg_server_last_error(const pg_server *s) { return s ? s->err.c_str() : "null server"; }

int pg_server_result(pg_server *s, int64_t id, void *rings, size_t bytes) {
  if (!s) return PG_ERR_ARG;
  auto it = s->results.find(id);
  if (it == s->results.end()) return sfail(s, PG_ERR_ARG, "no kept result for this id");
  if (!rings || bytes != it->second.size()) return sfail(s, PG_ERR_ARG, "result buffer size mismatch");
  std::memcpy(rings, it->second.data(), bytes);
  s->results.erase(it);
  return PG_OK;
}

int pg_server_run_trace(pg_server *s, const pg_params *reqs, const double *arrival_s, const int64_t *ids,
                        int n, pg_completion *out) {
  if (!s || (n > 0 && (!reqs || !arrival_s || !ids || !out))) return PG_ERR_ARG;
  for (int i = 1; i < n; i++)
    if (arrival_s[i] < arrival_s[i - 1]) return sfail(s, PG_ERR_ARG, "arrivals must be sorted");
  for (int i = 0; i < n; i++) {
    if (pg_check_params(&reqs[i])) return sfail(s, PG_ERR_PARAMS, "request with invalid parameters");
    // a run retires when its clock halts; a tmovie before the end time would
    // halt it early for a dump
    if (reqs[i].tmovie < reqs[i].endtime) return sfail(s, PG_ERR_PARAMS, "requests need tmovie >= endtime");
    if (pg_run_device_bytes(&reqs[i]) > s->budget) return sfail(s, PG_ERR_NOMEM, "request larger than the budget");
    std::memset(&out[i], 0, sizeof(out[i]));
    out[i].id = ids[i];
    out[i].arrival_s = arrival_s[i];
    out[i].status = -1;
  }
  const auto t0 = Clock::now();
  auto now_s = [&]() { return std::chrono::duration<double>(Clock::now() - t0).count(); };
  std::deque<int> queue;
  int next = 0, done = 0;
  std::vector<pg_batch_member> st;
  std::vector<unsigned char> buf;
  auto admit = [&]() -> int {
    double t = now_s();
    while (next < n && arrival_s[next] <= t) queue.push_back(next++);
    while (!queue.empty() && (int)s->live.size() < s->max_slots) {
      int r = queue.front();
      size_t need = pg_run_device_bytes(&reqs[r]);
      if (s->used + need > s->budget) break;
      pg_run *run = nullptr;
      int e = pg_create(&reqs[r], s->dev, &run);
      if (e) return sfail(s, e, "pg_create failed on admission");
      size_t bytes = pg_ring_bytes(reqs[r].jmax) * (size_t)reqs[r].imax * reqs[r].kmax;
      buf.resize(bytes);
      if ((e = pg_build_ic(&reqs[r], buf.data(), bytes)) || (e = pg_load_rings(run, buf.data(), bytes)) ||
          (e = pg_clock_reset(run, 0)) || (e = pg_batch_add(s->batch, run))) {
        std::string m = pg_last_error(run);
        pg_destroy(run);
        return sfail(s, e, "admission: " + m);
      }
      queue.pop_front();
      s->used += need;
      out[r].admit_s = now_s();
      s->live.push_back(Live{ids[r], r, run, need, out[r].admit_s});
    }
    return PG_OK;
  };
  while (done < n) {
    int e;
    if (s->live.empty()) {
      if ((e = admit())) return e;
      if (s->live.empty()) {
        // idle until the next arrival
        double wait = (next < n) ? arrival_s[next] - now_s() : 0.0;
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
        continue;
      }
    }
    // enqueue `chunk` steps of every live run, admit arrivals while they run
    // (new members join the next round), then synchronise and retire
    if ((e = pg_batch_advance(s->batch, s->chunk, s->chunk)))
      return sfail(s, e, std::string("batch advance: ") + pg_batch_last_error(s->batch));
    s->rounds++;
    size_t stepped = s->live.size();
    if ((e = admit())) return e;
    st.resize(s->live.size());
    if ((e = pg_batch_status(s->batch, st.data(), (int)st.size())))
      return sfail(s, e, std::string("batch status: ") + pg_batch_last_error(s->batch));
    double tf = now_s();
    std::vector<Live> keep, finished;
    for (size_t i = 0; i < s->live.size(); i++) {
      if (i < stepped && st[i].halted) {
        Live &l = s->live[i];
        out[l.req].finish_s = tf;
        out[l.req].steps = st[i].ncycle;
        out[l.req].simtime = st[i].simtime;
        out[l.req].status = st[i].status;
        out[l.req].cells = (int64_t)reqs[l.req].imax * reqs[l.req].jmax * reqs[l.req].kmax;
        finished.push_back(l);
      } else {
        keep.push_back(s->live[i]);
      }
    }
    for (Live &l : finished) {
      if ((e = pg_batch_remove(s->batch, l.run))) return sfail(s, e, "batch remove");
      if (s->keep_results) {
        size_t bytes = pg_ring_bytes(reqs[l.req].jmax) * (size_t)reqs[l.req].imax * reqs[l.req].kmax;
        std::vector<unsigned char> res(bytes);
        if ((e = pg_save_rings(l.run, res.data(), bytes))) return sfail(s, e, "save result");
        s->results[l.id] = std::move(res);
      }
      pg_destroy(l.run);
      s->used -= l.bytes;
      done++;
    }
    s->live.swap(keep);
  }
  return PG_OK;
}

int64_t pg_server_rounds(const pg_server *s) { return s ? s->rounds : 0; }

int pg_server_batch(pg_server *s, pg_batch **out) {
  if (!s || !out) return PG_ERR_ARG;
  *out = s->batch;
  return PG_OK;
}

}  // extern "C"
