// Serving runtime: a worker thread that admits PB solve requests against a
// device-memory budget and keeps many solves in flight at once.
//
// Every admitted request runs in a problem of its own grid and precision
// (pmg_problem: the device hierarchy, a stream, the captured solve graph),
// taken from a pool of idle problems of the same shape when one exists, so a
// steady stream of requests reuses resident hierarchies and captured graphs
// instead of allocating and capturing again. The worker issues a request as
// set_fine -> build_hierarchy -> pmg_solve_start on the problem's stream and
// polls the problem's completion event; solves of different grid sizes
// therefore overlap on the device, each one launch.
//
// Admission is first come, first served: the head request waits while the
// bytes held (busy + idle problems) plus its own would exceed the budget;
// idle problems are evicted (least recently used first) to make room. A
// request that could never fit completes at once with PMG_ERR_BUDGET.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "pmg_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Slot {
  pmg_problem *prob = nullptr;
  int base = 0, nlev = 0, precision = 0;
  double box = 0;
  long long bytes = 0;
  Clock::time_point last_used;
};

struct Flight {
  pmg_request req;
  Slot slot;
  int lane = -1;
  bool copy_queued = false; // the result copy is queued before the event
  double t_submit = 0, t_admit = 0;
};

// A lane: a stream an admitted request runs on, its completion event and a
// pinned staging buffer for the request's atoms. One request per lane at a
// time, so at most `lanes` requests are in flight; with at most as many
// lanes as the device has hardware work queues
// (CUDA_DEVICE_MAX_CONNECTIONS), no request queues behind another's solve.
struct Lane {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  double *pinned = nullptr;
  size_t pinned_doubles = 0;
};

struct Queued {
  pmg_request req;
  double t_submit = 0;
};

} // namespace

struct pmg_server {
  int device = 0;
  long long budget = 0;
  int max_inflight = 1;
  Clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work; // new requests or shutdown
  std::condition_variable cv_done; // new completions
  std::deque<Queued> queue;
  std::vector<pmg_completion> done;
  bool stopping = false;

  // worker-owned (read under mu for stats)
  std::vector<Lane> lanes;
  std::vector<int> free_lanes;
  std::vector<Flight> inflight;
  std::list<Slot> idle; // front = most recently used
  long long held = 0, peak = 0;
  long long completed = 0, created = 0, evicted = 0;
  double issue_s = 0, issue_max_s = 0, retire_s = 0, retire_max_s = 0;

  std::thread worker;

  double now() const {
    return std::chrono::duration<double>(Clock::now() - t0).count();
  }
};

namespace {

void fill_message(pmg_completion &c, int status) {
  if (status == PMG_OK) {
    c.message[0] = '\0';
    return;
  }
  std::snprintf(c.message, sizeof(c.message), "%s", pmg_last_error());
}

pmg_completion make_completion(const pmg_request &r, int status, int cycles,
                               double relres, double t_submit, double t_admit,
                               double t_done) {
  pmg_completion c;
  std::memset(&c, 0, sizeof(c));
  c.tag = r.tag;
  c.status = status;
  c.cycles = cycles;
  c.relres = relres;
  c.t_submit = t_submit;
  c.t_admit = t_admit;
  c.t_done = t_done;
  fill_message(c, status);
  return c;
}

// The request's hierarchy: as given, or the deepest of the same grid.
void resolve_levels(pmg_request &r) {
  if (r.hierarchy != 1)
    return;
  int base = r.base, nlev = r.nlev;
  if (pmg_levels_for(r.base * (1 << r.nlev) + 1, 12, 5, &base, &nlev) ==
      PMG_OK) {
    r.base = base;
    r.nlev = nlev;
  }
}

// True when dst may be written by a copy queued on a stream: device,
// managed or pinned host memory (pageable memory is copied synchronously
// after the solve instead).
bool async_target(const void *dst) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, dst) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged ||
         a.type == cudaMemoryTypeHost;
}

// Issues load -> build -> solve_start (-> result copy) -> lane event for a
// request on its problem, all on the lane's stream; never waits on the GPU.
int issue(const pmg_request &r, pmg_problem *p, Lane &lane, Flight &f) {
  int rc = pmg_problem_set_stream(p, lane.stream);
  if (rc != PMG_OK)
    return rc;
  if (r.atoms) {
    // stage the atoms in pinned memory so their copy is queued, not waited
    // for (the lane's previous request has finished with the buffer)
    const size_t need = 5 * (size_t)(r.natoms > 0 ? r.natoms : 1);
    if (need > lane.pinned_doubles) {
      if (lane.pinned)
        cudaFreeHost(lane.pinned);
      lane.pinned = nullptr;
      lane.pinned_doubles = 0;
      if (cudaMallocHost((void **)&lane.pinned, need * sizeof(double)) !=
          cudaSuccess)
        return PMG_ERR_NOMEM;
      lane.pinned_doubles = need;
    }
    std::memcpy(lane.pinned, r.atoms, sizeof(double) * 5 * r.natoms);
    rc = pmg_problem_set_atoms(p, lane.pinned, r.natoms, &r.physics);
  } else {
    rc = pmg_problem_set_fine(p, r.fine[0], r.fine[1], r.fine[2], r.fine[3],
                              r.fine[4], r.fine[5]);
  }
  if (rc == PMG_OK)
    rc = pmg_build_hierarchy(p, 0);
  if (rc == PMG_OK)
    rc = pmg_solve_start(p, r.tol, r.max_cycles);
  f.copy_queued = false;
  if (rc == PMG_OK && r.potential && async_target(r.potential)) {
    rc = pmg_get_potential_async(p, r.potential);
    f.copy_queued = rc == PMG_OK;
  }
  if (rc == PMG_OK && cudaEventRecord(lane.done, lane.stream) != cudaSuccess)
    rc = PMG_ERR_CUDA;
  return rc;
}

// Takes an idle problem of the request's shape, or makes room and creates
// one. Returns PMG_OK with *slot filled, PMG_ERR_BUDGET when the request
// must wait, or another status on failure. Called by the worker only.
int acquire(pmg_server *s, const pmg_request &r, Slot *slot) {
  for (auto it = s->idle.begin(); it != s->idle.end(); ++it)
    if (it->base == r.base && it->nlev == r.nlev &&
        it->precision == r.precision && it->box == r.box) {
      *slot = *it;
      s->idle.erase(it);
      return PMG_OK;
    }
  const long long need = pmg_problem_bytes(r.base, r.nlev, r.precision);
  if (need < 0)
    return PMG_ERR_ARG;
  while (s->held + need > s->budget && !s->idle.empty()) {
    Slot victim = s->idle.back(); // least recently used
    s->idle.pop_back();
    pmg_problem_destroy(victim.prob);
    s->held -= victim.bytes;
    ++s->evicted;
  }
  if (s->held + need > s->budget)
    return PMG_ERR_BUDGET;
  pmg_problem *p = nullptr;
  int rc = pmg_problem_create(r.base, r.nlev, r.box, r.precision, nullptr, &p);
  if (rc != PMG_OK)
    return rc;
  // many solves share the GPU here: kernels that do not wait for whole SMs
  if ((rc = pmg_problem_set_throughput_mode(p, 1)) != PMG_OK) {
    pmg_problem_destroy(p);
    return rc;
  }
  slot->prob = p;
  slot->base = r.base;
  slot->nlev = r.nlev;
  slot->precision = r.precision;
  slot->box = r.box;
  slot->bytes = need;
  s->held += need;
  s->peak = std::max(s->peak, s->held);
  ++s->created;
  return PMG_OK;
}

void release(pmg_server *s, Slot slot, bool healthy) {
  if (!healthy) { // a failed problem is not reused
    pmg_problem_destroy(slot.prob);
    s->held -= slot.bytes;
    return;
  }
  slot.last_used = Clock::now();
  s->idle.push_front(slot);
}

// One pass of the worker: admit what fits, retire what finished. Returns
// true when anything changed.
bool step(pmg_server *s) {
  bool progress = false;
  // admission (head of line)
  for (;;) {
    Queued q;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->queue.empty() || s->free_lanes.empty())
        break;
      q = s->queue.front();
    }
    const long long need =
        pmg_problem_bytes(q.req.base, q.req.nlev, q.req.precision);
    if (need < 0 || need > s->budget) {
      const int st = need < 0 ? PMG_ERR_ARG : PMG_ERR_BUDGET;
      pmg_completion c = make_completion(q.req, st, 0, 0.0, q.t_submit,
                                         s->now(), s->now());
      std::snprintf(c.message, sizeof(c.message), "%s",
                    need < 0 ? "bad grid shape"
                             : "problem larger than the whole budget");
      std::lock_guard<std::mutex> lk(s->mu);
      s->queue.pop_front();
      s->done.push_back(c);
      ++s->completed;
      s->cv_done.notify_all();
      progress = true;
      continue;
    }
    Slot slot;
    int rc;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      rc = acquire(s, q.req, &slot);
    }
    if (rc == PMG_ERR_BUDGET)
      break; // wait for a completion to free memory
    const double t_admit = s->now();
    Flight f;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      f.lane = s->free_lanes.back();
      s->free_lanes.pop_back();
    }
    if (rc == PMG_OK)
      rc = issue(q.req, slot.prob, s->lanes[f.lane], f);
    const double dt_issue = s->now() - t_admit;
    std::lock_guard<std::mutex> lk(s->mu);
    s->issue_s += dt_issue;
    s->issue_max_s = std::max(s->issue_max_s, dt_issue);
    s->queue.pop_front();
    progress = true;
    if (rc != PMG_OK) {
      if (slot.prob) {
        // let the lane drain what was queued before reusing it
        cudaStreamSynchronize(s->lanes[f.lane].stream);
        release(s, slot, false);
      }
      s->free_lanes.push_back(f.lane);
      s->done.push_back(make_completion(q.req, rc, 0, 0.0, q.t_submit,
                                        t_admit, s->now()));
      ++s->completed;
      s->cv_done.notify_all();
      continue;
    }
    f.req = q.req;
    f.slot = slot;
    f.t_submit = q.t_submit;
    f.t_admit = t_admit;
    s->inflight.push_back(f);
  }
  // retirement
  for (size_t i = 0; i < s->inflight.size();) {
    Flight &f = s->inflight[i];
    const cudaError_t q = cudaEventQuery(s->lanes[f.lane].done);
    if (q == cudaErrorNotReady) {
      ++i;
      continue;
    }
    int rc = q == cudaSuccess ? PMG_OK : PMG_ERR_CUDA;
    if (q != cudaSuccess)
      (void)cudaGetLastError();
    int cycles = 0;
    double relres = 0.0;
    const double t_ret = s->now();
    if (rc == PMG_OK)
      rc = pmg_solve_finish(f.slot.prob, &cycles, &relres, nullptr);
    if ((rc == PMG_OK || rc == PMG_ERR_DIVERGED) && f.req.potential &&
        !f.copy_queued) {
      const int rc2 = pmg_get_potential(f.slot.prob, f.req.potential);
      if (rc == PMG_OK)
        rc = rc2;
    }
    pmg_completion c = make_completion(f.req, rc, cycles, relres, f.t_submit,
                                       f.t_admit, s->now());
    // park the problem on its own stream while the lane is idle, so its next
    // lane does not wait for whatever this lane runs next
    if (pmg_problem_set_stream(f.slot.prob, nullptr) != PMG_OK && rc == PMG_OK)
      rc = PMG_ERR_CUDA;
    const double dt_ret = s->now() - t_ret;
    std::lock_guard<std::mutex> lk(s->mu);
    s->retire_s += dt_ret;
    s->retire_max_s = std::max(s->retire_max_s, dt_ret);
    release(s, f.slot, rc == PMG_OK || rc == PMG_ERR_DIVERGED);
    s->free_lanes.push_back(f.lane);
    s->done.push_back(c);
    ++s->completed;
    s->inflight.erase(s->inflight.begin() + (long)i);
    s->cv_done.notify_all();
    progress = true;
  }
  return progress;
}

void worker_main(pmg_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    const bool progress = step(s);
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stopping && s->queue.empty() && s->inflight.empty())
      break;
    if (progress)
      continue;
    if (s->inflight.empty() && s->queue.empty()) {
      s->cv_work.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
    } else {
      // solves in flight (or a request waiting for memory): poll the GPU
      // again shortly
      s->cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  for (Slot &sl : s->idle) {
    pmg_problem_destroy(sl.prob);
    s->held -= sl.bytes;
  }
  s->idle.clear();
  for (Lane &l : s->lanes) {
    cudaStreamSynchronize(l.stream);
    cudaEventDestroy(l.done);
    cudaStreamDestroy(l.stream);
    if (l.pinned)
      cudaFreeHost(l.pinned);
  }
  s->lanes.clear();
}

} // namespace

extern "C" {

int pmg_levels_for(int n, int max_levels, int min_coarse, int *base,
                   int *nlev) {
  if (!base || !nlev || n < 3)
    return PMG_ERR_ARG;
  for (int L = max_levels < 30 ? max_levels : 30; L >= 2; --L)
    if ((n - 1) % (1 << L) == 0 && ((n - 1) >> L) >= 1) {
      const int b = (n - 1) >> L;
      if (2 * b + 1 >= min_coarse) {
        *base = b;
        *nlev = L;
        return PMG_OK;
      }
    }
  return PMG_ERR_ARG;
}

int pmg_server_create(long long budget_bytes, int max_inflight,
                      pmg_server **out) {
  if (!out || budget_bytes <= 0 || max_inflight < 1 || max_inflight > 256)
    return PMG_ERR_ARG;
  *out = nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return PMG_ERR_CUDA;
  pmg_server *s = new pmg_server();
  s->device = dev;
  s->budget = budget_bytes;
  s->max_inflight = max_inflight;
  s->t0 = Clock::now();
  s->lanes.resize(max_inflight);
  for (int l = 0; l < max_inflight; ++l) {
    Lane &ln = s->lanes[l];
    if (cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking) !=
            cudaSuccess ||
        cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming) !=
            cudaSuccess) {
      for (Lane &x : s->lanes) {
        if (x.done)
          cudaEventDestroy(x.done);
        if (x.stream)
          cudaStreamDestroy(x.stream);
      }
      delete s;
      return PMG_ERR_CUDA;
    }
    s->free_lanes.push_back(max_inflight - 1 - l);
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return PMG_OK;
}

int pmg_server_submit(pmg_server *s, const pmg_request *r) {
  if (!s || !r)
    return PMG_ERR_ARG;
  if (r->max_cycles < 0 || r->max_cycles > 1024 || !(r->tol >= 0.0) ||
      (r->precision != PMG_PREC_FP64 && r->precision != PMG_PREC_MIXED &&
       r->precision != PMG_PREC_FP64_FAST))
    return PMG_ERR_ARG;
  if (r->atoms) {
    if (r->natoms < 0)
      return PMG_ERR_ARG;
  } else {
    for (int q = 0; q < 6; ++q)
      if (!r->fine[q])
        return PMG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping)
    return PMG_ERR_STATE;
  Queued q;
  q.req = *r;
  resolve_levels(q.req);
  q.t_submit = s->now();
  s->queue.push_back(q);
  s->cv_work.notify_one();
  return PMG_OK;
}

int pmg_server_wait(pmg_server *s, pmg_completion *out, int cap, int *n,
                    double timeout_s) {
  if (!s || !n || cap < 0 || (cap > 0 && !out))
    return PMG_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && timeout_s > 0)
    s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                        [&] { return !s->done.empty(); });
  const int k = std::min(cap, (int)s->done.size());
  for (int i = 0; i < k; ++i)
    out[i] = s->done[i];
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return PMG_OK;
}

int pmg_server_get_stats(pmg_server *s, pmg_server_stats *st) {
  if (!s || !st)
    return PMG_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  st->queued = (int)s->queue.size();
  st->inflight = (int)s->inflight.size();
  st->idle_problems = (int)s->idle.size();
  st->held_bytes = s->held;
  st->peak_bytes = s->peak;
  st->budget_bytes = s->budget;
  st->completed = s->completed;
  st->created_problems = s->created;
  st->evicted_problems = s->evicted;
  st->issue_s = s->issue_s;
  st->issue_max_s = s->issue_max_s;
  st->retire_s = s->retire_s;
  st->retire_max_s = s->retire_max_s;
  return PMG_OK;
}

int pmg_server_destroy(pmg_server *s) {
  if (!s)
    return PMG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable())
    s->worker.join();
  delete s;
  return PMG_OK;
}

int pmg_batch_solve(const pmg_request *reqs, int count, long long budget_bytes,
                    int max_inflight, pmg_completion *out) {
  if (count < 0 || (count > 0 && (!reqs || !out)))
    return PMG_ERR_ARG;
  pmg_server *s = nullptr;
  int rc = pmg_server_create(budget_bytes, max_inflight, &s);
  if (rc != PMG_OK)
    return rc;
  // tags are rewritten to indices so completions land in request order
  for (int i = 0; i < count && rc == PMG_OK; ++i) {
    pmg_request r = reqs[i];
    r.tag = i;
    rc = pmg_server_submit(s, &r);
  }
  std::vector<pmg_completion> buf(count > 0 ? count : 1);
  int got = 0;
  while (rc == PMG_OK && got < count) {
    int n = 0;
    pmg_server_wait(s, buf.data(), count, &n, 1.0);
    for (int i = 0; i < n; ++i) {
      const long long idx = buf[i].tag;
      out[idx] = buf[i];
      out[idx].tag = reqs[idx].tag;
    }
    got += n;
  }
  pmg_server_destroy(s);
  return rc;
}

} // extern "C"
