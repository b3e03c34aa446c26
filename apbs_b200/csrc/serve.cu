// Serving loop: many independent PB calculations on one GPU.
//
// The reference runs its ELEC blocks one after another from main()
// (src/main.c:529); this loop is the part that has no counterpart there.
// Requests queue in arrival order.  Each of `max_inflight` worker threads
// owns a CUDA stream; a free worker takes the head of the queue as soon as
// the head's device footprint fits the budget beside the calculations
// already resident (first in, first out: a large head waits rather than
// being overtaken, so no request starves).  Calculations that finish stay
// resident in a pool keyed by grid shape and are reused by later requests of
// the same shape; idle ones are released, least recently used first, when a
// new request needs their memory.  The device work of concurrent requests
// overlaps because every worker drives its own stream.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "apbs_b200.h"
#include "solver_internal.cuh"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  long long id = 0;
  pmgb_params p;
  std::vector<double> xyz, q, r;
  double* u_out = nullptr;
  size_t bytes = 0;
  double t_submit = 0, t_start = 0, t_end = 0;
  long long admit_order = 0;
  int status = 0;  // 0 queued/running, 1 done, -1 failed
  double energy = 0;
  pmgb_stats st;
  std::string err;
};

typedef std::tuple<int, int, int, int> Shape;

struct Pooled {
  void* calc;
  Shape shape;
  size_t bytes;
  double last_used;
};

// ---- device side through the public calculation API ---------------------
size_t cuda_footprint(void*, const pmgb_params* p, int precision, int natoms) {
  return pmgb_footprint(p, precision, natoms);
}
void* cuda_create(void*, const pmgb_params* p, int precision) {
  pmgb_solver* s = nullptr;
  return pmgb_create(p, precision, &s) ? s : nullptr;
}
int cuda_reconfigure(void*, void* calc, const pmgb_params* p) {
  return pmgb_reconfigure((pmgb_solver*)calc, p);
}
void cuda_destroy(void*, void* calc) { pmgb_destroy((pmgb_solver*)calc); }

}  // namespace

struct pmgb_server {
  pmgb_server_config cfg;
  pmgb_server_backend be;
  bool cuda = false;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::map<long long, Request*> reqs;
  std::vector<Pooled> idle;
  std::vector<std::thread> workers;
  size_t in_use = 0, peak = 0, budget = 0;
  bool stop = false;
  long long next_id = 1, submitted = 0, done = 0, failed = 0;
  long long created = 0, reused = 0, evicted = 0, admitted = 0;
  int inflight = 0, inflight_peak = 0;
  std::vector<double> lat, service;
  std::map<Shape, std::vector<std::pair<int, int>>> shape_tune;

  Shape shape_of(const pmgb_params& p) const { return Shape(p.nx, p.ny, p.nz, p.nlev); }

  // idle bytes that could be released to make room (all of them)
  size_t idle_bytes() const {
    size_t b = 0;
    for (const Pooled& q : idle) b += q.bytes;
    return b;
  }
  // the idle calculation admit_at reuses for this shape (most recently
  // used), or -1
  int pick_idle(const Shape& sh) const {
    int pick = -1;
    for (int i = 0; i < (int)idle.size(); i++)
      if (idle[i].shape == sh && (pick < 0 || idle[i].last_used > idle[pick].last_used))
        pick = i;
    return pick;
  }
  // a request can start now.  A pooled calculation is reused when one of
  // the shape is idle; its footprint grows to the request's when the
  // request has more atoms (the fill buffers grow with natoms), and that
  // growth must fit beside everything not evictable.
  bool admissible(const Request* h) const {
    const int pick = pick_idle(shape_of(h->p));
    if (pick >= 0) {
      const size_t b = idle[pick].bytes;
      if (h->bytes <= b) return true;
      return in_use - (idle_bytes() - b) + (h->bytes - b) <= budget;
    }
    return in_use - idle_bytes() + h->bytes <= budget;
  }
  bool head_admissible() const { return !queue.empty() && admissible(queue.front()); }

  struct Slot {
    Request* rq = nullptr;
    void* calc = nullptr;
    size_t held = 0;
  };
  long long batches = 0, batched = 0;
  int batch_peak = 0;

  void worker_main();
  int run_request(Request* rq, void* calc, void* stream);
  Slot admit_at(size_t pos, std::vector<void*>& release);
  bool batchable(const Request* rq) const;
  void* prepare(Slot& sl);
  void* finish(Slot& sl, int status);
};

// Runs one request on its calculation; the status is published by the
// caller under the lock.
int pmgb_server::run_request(Request* rq, void* calc, void* stream) {
  double e = 0.0;
  int ok = 1;
  if (cuda) {
    pmgb_solver* s = (pmgb_solver*)calc;
    ok = pmgb_set_stream(s, stream) &&
         pmgb_fillco(s, (int)rq->q.size(), rq->xyz.data(), rq->q.data(), rq->r.data()) &&
         pmgb_solve(s) && pmgb_energy(s, &e) && pmgb_get_stats(s, &rq->st);
    if (ok && rq->u_out) ok = pmgb_get_potential(s, rq->u_out);
    if (!ok) rq->err = pmgb_last_error();
    // back on its own stream: the worker's stream dies with the worker,
    // while the calculation may outlive it in the pool
    pmgb_set_stream(s, nullptr);
  } else {
    ok = be.run(be.ctx, calc, (int)rq->q.size(), rq->xyz.data(), rq->q.data(), rq->r.data(), &e);
    if (!ok) rq->err = "backend run failed";
  }
  rq->energy = e;
  return ok ? 1 : -1;
}

// Takes request `pos` of the queue (the caller holds the lock and has
// checked it is admissible): a pooled calculation of its shape or reserved
// memory.
pmgb_server::Slot pmgb_server::admit_at(size_t pos, std::vector<void*>& release) {
  Slot sl;
  sl.rq = queue[pos];
  queue.erase(queue.begin() + pos);
  const Shape sh = shape_of(sl.rq->p);
  // a resident calculation of this shape, most recently used first
  const int pick = pick_idle(sh);
  size_t grow = sl.rq->bytes;  // bytes in_use must take on
  if (pick >= 0) {
    sl.calc = idle[pick].calc;
    sl.held = std::max(idle[pick].bytes, sl.rq->bytes);
    grow = sl.held - idle[pick].bytes;
    idle.erase(idle.begin() + pick);
    reused++;
  } else {
    sl.held = sl.rq->bytes;
  }
  // release idle calculations, least recently used first, until it fits
  std::sort(idle.begin(), idle.end(),
            [](const Pooled& a, const Pooled& b) { return a.last_used < b.last_used; });
  while (grow > 0 && in_use + grow > budget && !idle.empty()) {
    in_use -= idle.front().bytes;
    release.push_back(idle.front().calc);
    idle.erase(idle.begin());
    evicted++;
  }
  in_use += grow;
  peak = std::max(peak, in_use);
  inflight++;
  inflight_peak = std::max(inflight_peak, inflight);
  sl.rq->t_start = now_ms();
  sl.rq->admit_order = ++admitted;
  return sl;
}

// Mixed-precision LPBE on a grid whose level 1 fits the one-cluster tail:
// these share one persistent kernel (pmgb_batch_solve).
bool pmgb_server::batchable(const Request* rq) const {
  return cuda && cfg.max_batch > 1 && cfg.precision == PMGB_MIXED && !rq->p.nonlin &&
         rq->p.nx <= 65 && rq->p.ny <= 65 && rq->p.nz <= 65;
}

// A calculation for the slot (pooled one reconfigured, or a new one).
void* pmgb_server::prepare(Slot& sl) {
  void* calc = sl.calc;
  if (!calc) {
    calc = be.create(be.ctx, &sl.rq->p, cfg.precision);
    if (calc) {
      std::vector<std::pair<int, int>> tv;
      {
        std::lock_guard<std::mutex> lk(mu);
        created++;
        auto it = shape_tune.find(shape_of(sl.rq->p));
        if (it != shape_tune.end()) tv = it->second;
      }
      if (cuda)
        for (const auto& kv : tv) pmgb_solver_set_tuning((pmgb_solver*)calc, kv.first, kv.second);
    }
  } else if (!be.reconfigure(be.ctx, calc, &sl.rq->p)) {
    be.destroy(be.ctx, calc);
    calc = be.create(be.ctx, &sl.rq->p, cfg.precision);
  }
  sl.calc = calc;
  if (!calc) sl.rq->err = cuda ? pmgb_last_error() : "backend create failed";
  return calc;
}

// Publishes a finished slot and keeps its calculation resident (or drops it).
void* pmgb_server::finish(Slot& sl, int status) {
  Request* rq = sl.rq;
  void* drop = nullptr;
  rq->status = status;
  rq->t_end = now_ms();
  inflight--;
  if (rq->status == 1) {
    done++;
    lat.push_back(rq->t_end - rq->t_submit);
    service.push_back(rq->t_end - rq->t_start);
  } else {
    failed++;
  }
  // keep the calculation resident unless its shape's pool is full
  const Shape sh = shape_of(rq->p);
  int same = 0;
  for (const Pooled& q : idle) same += (q.shape == sh);
  if (sl.calc && rq->status == 1 && same < cfg.pool_per_shape) {
    idle.push_back(Pooled{sl.calc, sh, sl.held, rq->t_end});
  } else {
    drop = sl.calc;
    in_use -= sl.held;
  }
  return drop;
}

void pmgb_server::worker_main() {
  cudaStream_t stream = nullptr;
  if (cuda) {
    cudaSetDevice(device);
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  }
  for (;;) {
    std::vector<Slot> slots;
    std::vector<void*> release;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return (stop && queue.empty()) || head_admissible(); });
      if (queue.empty()) break;  // stopping
      slots.push_back(admit_at(0, release));
      // continuous batching: small mixed LPBE requests waiting anywhere in
      // the queue join a small head in one persistent kernel (they need
      // little memory; larger requests keep their order among themselves)
      if (batchable(slots[0].rq))
        for (size_t q = 0; q < queue.size() && (int)slots.size() < cfg.max_batch;) {
          if (batchable(queue[q]) && admissible(queue[q]))
            slots.push_back(admit_at(q, release));
          else
            q++;
        }
      batch_peak = std::max(batch_peak, (int)slots.size());
    }
    for (void* c : release) be.destroy(be.ctx, c);
    std::vector<int> status(slots.size(), -1);
    if (slots.size() == 1) {
      if (prepare(slots[0])) status[0] = run_request(slots[0].rq, slots[0].calc, stream);
    } else {
      // fill each on its own stream (the fills overlap on the device), solve
      // all in one launch, then the energies
      std::vector<pmgb_solver*> calcs;
      std::vector<int> member;
      for (size_t b = 0; b < slots.size(); b++) {
        Request* rq = slots[b].rq;
        if (!prepare(slots[b])) continue;
        pmgb_solver* s = (pmgb_solver*)slots[b].calc;
        if (pmgb_set_stream(s, nullptr) &&
            pmgb::fillco_issue(s, (int)rq->q.size(), rq->xyz.data(), rq->q.data(),
                               rq->r.data())) {
          calcs.push_back(s);
          member.push_back((int)b);
        } else {
          rq->err = pmgb_last_error();
        }
      }
      const int ok = calcs.empty() ? 0 : pmgb_batch_solve(calcs.data(), (int)calcs.size(), stream);
      const std::string berr = ok ? "" : pmgb_last_error();
      for (size_t c = 0; c < calcs.size(); c++) {
        Request* rq = slots[member[c]].rq;
        double e = 0.0;
        int good = ok && pmgb_energy(calcs[c], &e) && pmgb_get_stats(calcs[c], &rq->st);
        if (good && rq->u_out) good = pmgb_get_potential(calcs[c], rq->u_out);
        if (!good) rq->err = ok ? pmgb_last_error() : berr;
        rq->energy = e;
        status[member[c]] = good ? 1 : -1;
        pmgb_set_stream(calcs[c], nullptr);
      }
      std::lock_guard<std::mutex> lk(mu);
      batches++;
      batched += (long long)calcs.size();
    }
    std::vector<void*> drops;
    {
      std::lock_guard<std::mutex> lk(mu);
      for (size_t b = 0; b < slots.size(); b++) {
        void* d = finish(slots[b], status[b]);
        if (d) drops.push_back(d);
      }
    }
    for (void* d : drops) be.destroy(be.ctx, d);
    cv_done.notify_all();
    cv_work.notify_all();
  }
  if (stream) cudaStreamDestroy(stream);
}

namespace {

int server_start(pmgb_server* srv, const pmgb_server_config* cfg) {
  srv->cfg = *cfg;
  if (srv->cfg.max_inflight < 1) srv->cfg.max_inflight = 1;
  // by default a shape keeps as many calculations as can run at once, so a
  // burst of one shape never has to release (cudaFree synchronises the device)
  if (cfg->max_batch == 0) srv->cfg.max_batch = 16;
  if (cfg->pool_per_shape == 0)
    srv->cfg.pool_per_shape = std::max(2, srv->cfg.max_inflight) * std::max(1, srv->cfg.max_batch);
  else if (cfg->pool_per_shape < 0) srv->cfg.pool_per_shape = 0;
  srv->budget = cfg->hbm_budget_bytes;
  for (int i = 0; i < srv->cfg.max_inflight; i++)
    srv->workers.emplace_back([srv] { srv->worker_main(); });
  return 1;
}

void fill_result(const Request* rq, pmgb_result* out) {
  memset(out, 0, sizeof(*out));
  out->status = rq->status;
  out->energy_kT = rq->energy;
  if (rq->status != 0) {
    out->latency_ms = rq->t_end - rq->t_submit;
    out->queue_ms = rq->t_start - rq->t_submit;
    out->service_ms = rq->t_end - rq->t_start;
  }
  out->admit_order = rq->admit_order;
  out->stats = rq->st;
  snprintf(out->error, sizeof(out->error), "%s", rq->err.c_str());
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest rank
  size_t k = (size_t)std::ceil(q * (double)v.size());
  if (k < 1) k = 1;
  if (k > v.size()) k = v.size();
  return v[k - 1];
}

}  // namespace

extern "C" int pmgb_server_create(const pmgb_server_config* cfg, pmgb_server** out) {
  if (!cfg || !out) return 0;
  *out = nullptr;
  if (cfg->precision != PMGB_FP64 && cfg->precision != PMGB_MIXED) return 0;
  pmgb_server* srv = new pmgb_server();
  srv->cuda = true;
  if (cudaGetDevice(&srv->device) != cudaSuccess) {
    delete srv;
    return 0;
  }
  srv->be.ctx = nullptr;
  srv->be.footprint = cuda_footprint;
  srv->be.create = cuda_create;
  srv->be.reconfigure = cuda_reconfigure;
  srv->be.run = nullptr;  // the CUDA path runs through run_request
  srv->be.destroy = cuda_destroy;
  pmgb_server_config c = *cfg;
  if (c.hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      delete srv;
      return 0;
    }
    c.hbm_budget_bytes = (size_t)(0.8 * (double)fr);
  }
  server_start(srv, &c);
  *out = srv;
  return 1;
}

extern "C" int pmgb_server_create_ex(const pmgb_server_config* cfg,
                                     const pmgb_server_backend* backend, pmgb_server** out) {
  if (!cfg || !backend || !out || !backend->footprint || !backend->create ||
      !backend->reconfigure || !backend->run || !backend->destroy || cfg->hbm_budget_bytes == 0)
    return 0;
  *out = nullptr;
  pmgb_server* srv = new pmgb_server();
  srv->cuda = false;
  srv->be = *backend;
  server_start(srv, cfg);
  *out = srv;
  return 1;
}

extern "C" long long pmgb_server_submit(pmgb_server* srv, const pmgb_params* params, int natoms,
                                        const double* xyz, const double* charge,
                                        const double* radius, double* u_out) {
  if (!srv || !params || natoms < 0 || (natoms > 0 && (!xyz || !charge || !radius))) return 0;
  Request* rq = new Request();
  rq->p = *params;
  rq->xyz.assign(xyz, xyz + 3 * (size_t)natoms);
  rq->q.assign(charge, charge + natoms);
  rq->r.assign(radius, radius + natoms);
  rq->u_out = u_out;
  memset(&rq->st, 0, sizeof(rq->st));
  rq->bytes = srv->be.footprint(srv->be.ctx, params, srv->cfg.precision, natoms);
  std::lock_guard<std::mutex> lk(srv->mu);
  if (srv->stop || rq->bytes > srv->budget) {
    delete rq;
    return 0;
  }
  rq->id = srv->next_id++;
  rq->t_submit = now_ms();
  srv->reqs[rq->id] = rq;
  srv->queue.push_back(rq);
  srv->submitted++;
  srv->cv_work.notify_one();
  return rq->id;
}

extern "C" int pmgb_server_set_shape_tuning(pmgb_server* srv, const pmgb_params* shape, int key,
                                            int value) {
  if (!srv || !shape || key < 0 || key >= PMGB_TUNE_NKEYS) return 0;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto& v = srv->shape_tune[srv->shape_of(*shape)];
  for (auto& kv : v)
    if (kv.first == key) {
      kv.second = value;
      return 1;
    }
  v.emplace_back(key, value);
  return 1;
}

extern "C" int pmgb_server_poll(pmgb_server* srv, long long id, pmgb_result* result) {
  if (!srv || !result) return -1;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) {
    memset(result, 0, sizeof(*result));
    result->status = -1;
    snprintf(result->error, sizeof(result->error), "unknown request %lld", id);
    return -1;
  }
  fill_result(it->second, result);
  return result->status;
}

extern "C" int pmgb_server_wait(pmgb_server* srv, long long id, pmgb_result* result) {
  if (!srv || !result) return -1;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) {
    memset(result, 0, sizeof(*result));
    result->status = -1;
    snprintf(result->error, sizeof(result->error), "unknown request %lld", id);
    return -1;
  }
  Request* rq = it->second;
  srv->cv_done.wait(lk, [&] { return rq->status != 0; });
  fill_result(rq, result);
  return result->status;
}

extern "C" int pmgb_server_drain(pmgb_server* srv) {
  if (!srv) return 0;
  std::unique_lock<std::mutex> lk(srv->mu);
  srv->cv_done.wait(lk, [&] { return srv->done + srv->failed == srv->submitted; });
  return 1;
}

extern "C" int pmgb_server_get_stats(pmgb_server* srv, pmgb_server_stats* st) {
  if (!srv || !st) return 0;
  std::lock_guard<std::mutex> lk(srv->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = srv->submitted;
  st->done = srv->done;
  st->failed = srv->failed;
  st->p50_ms = percentile(srv->lat, 0.50);
  st->p99_ms = percentile(srv->lat, 0.99);
  double a = 0.0, b = 0.0;
  for (double v : srv->lat) a += v;
  for (double v : srv->service) b += v;
  st->mean_ms = srv->lat.empty() ? 0.0 : a / (double)srv->lat.size();
  st->mean_service_ms = srv->service.empty() ? 0.0 : b / (double)srv->service.size();
  st->bytes_in_use = srv->in_use;
  st->bytes_peak = srv->peak;
  st->budget = srv->budget;
  st->created = srv->created;
  st->reused = srv->reused;
  st->evicted = srv->evicted;
  st->inflight_peak = srv->inflight_peak;
  st->batches = srv->batches;
  st->batched = srv->batched;
  st->batch_peak = srv->batch_peak;
  return 1;
}

extern "C" void pmgb_server_destroy(pmgb_server* srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  for (std::thread& t : srv->workers) t.join();
  for (Pooled& q : srv->idle) srv->be.destroy(srv->be.ctx, q.calc);
  for (auto& kv : srv->reqs) delete kv.second;
  delete srv;
}
