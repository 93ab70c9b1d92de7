// server.cpp -- continuous batching of forward-modelling jobs on one GPU
// (include/salvus_b200.h, "serving").
//
// Threads:
//   scheduler  admits queued jobs while the device-memory budget and the
//              running-job limit allow (any queued job that fits may pass a
//              larger one ahead of it) and keeps every running job two
//              graph-replayed chunks of steps ahead on the job's own stream
//              (so the jobs' kernels overlap on the device and no job waits
//              for another's chunk): each chunk ends with an asynchronous
//              copy of the job's seismogram ring and status word into
//              page-locked host buffers and an event; the scheduler polls
//              the events, streams each finished chunk's samples into the
//              job's result, enqueues the next chunk, and retires finished
//              jobs, freeing their device memory.
//   workers    (up to 8) prepare admitted jobs (mesh flattening on the host,
//              device setup, sources, receivers) while the scheduler keeps
//              running jobs busy.
// Jobs never share device state, so a job's result does not depend on the
// mix it ran in.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace salvus {
const char *last_error();
}

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t id = 0;
  // owned copies of the description
  salvus_mesh_desc mesh{};
  std::vector<double> vertices, params, receivers;
  std::vector<int64_t> cells;
  std::vector<salvus_source> sources;
  int32_t precision = SALVUS_FP32;
  double dt = 0;
  int64_t n_steps = 0;
  int c = 1;
  // lifecycle
  std::atomic<int> state{SALVUS_JOB_QUEUED};
  std::atomic<int64_t> steps_done{0};
  std::atomic<bool> cancel{false};
  int64_t est_bytes = 0, G = 0;
  std::string error;
  std::vector<double> seis;  // [R][c][n_steps]
  Clock::time_point submitted, done;
  salvus_mesh *m = nullptr;
  salvus_problem *p = nullptr;
  // chunks in flight (at most two, in order from `head`): first step, step
  // count, completion event, host copies of the seismogram ring and status
  cudaStream_t stream = nullptr;
  int64_t enq_steps = 0, rows = 0, cap = 0;
  int head = 0, inflight = 0;
  int64_t first[2] = {0, 0}, count[2] = {0, 0};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double *ring[2] = {nullptr, nullptr};
  int *status[2] = {nullptr, nullptr};
};

int64_t estimate_bytes(const salvus_mesh_desc &d, int precision) {
  const int dim = d.shape == SALVUS_QUAD ? 2 : 3;
  const int64_t n = d.order + 1;
  const int64_t P = dim == 2 ? n * n : n * n * n;
  const int64_t c = salvus::physics_components(d.physics);
  const int64_t E = d.n_elements;
  int64_t G = E;
  for (int k = 0; k < dim; ++k) G *= d.order;
  G = G * 5 / 4 + 4 * E;  // interior count plus a generous boundary allowance
  const bool ti = (d.reserved & SALVUS_MESH_ELASTIC_TI) != 0;
  const int64_t rw32 = salvus::record_words(d.shape, d.physics, 0, ti);
  const int64_t rw64 = salvus::record_words(d.shape, d.physics, 1, ti);
  const int64_t rs = precision == SALVUS_FP64 ? 8 : 4;
  int64_t b = 0;
  b += E * P * (4 * rw32 + 4 /*conn*/ + 4 /*incidence*/ + 8 /*setup mass, transient*/);
  if (precision == SALVUS_FP64) b += E * P * 8 * rw64;
  b += G * (4 + 8 + 4 + 8 * c);  // offsets, inverse mass, node coordinates
  b += 4 * G * c * rs;             // u v a a_
  b += E * P * c * rs;             // element-local residual
  b += G * c * 8;                  // host-copy staging
  b += E * 8 * dim * 8 + E * 8 * 6 * 8;  // vertices and vertex material
  return b + (8 << 20);            // per-job slack (graphs, rings)
}

}  // namespace

struct salvus_server {
  int device = 0;
  int64_t budget = 0;
  int max_running = 8;
  int chunk = 32;
  std::mutex mu;
  std::condition_variable cv_sched, cv_work, cv_done;
  std::deque<Job *> queue, to_prepare, ready;
  std::vector<Job *> running;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 1;
  int64_t mem_in_use = 0, peak_mem = 0;
  int n_preparing = 0;
  bool stop = false;
  std::thread sched;
  std::vector<std::thread> workers;  // job preparation pool
  // stats
  std::vector<double> latencies;
  double updates = 0;
  double busy = 0, prep = 0;
  int64_t submitted = 0, completed = 0, failed = 0;
  Clock::time_point busy_since;
  bool busy_now = false;
};

namespace {

void finish_locked(salvus_server *s, Job *j, int state) {
  j->state = state;
  j->done = Clock::now();
  s->mem_in_use -= j->est_bytes;
  if (state == SALVUS_JOB_DONE) {
    s->completed++;
    s->latencies.push_back(std::chrono::duration<double>(j->done - j->submitted).count());
    s->updates += (double)j->G * (double)j->n_steps;
  } else if (state == SALVUS_JOB_FAILED) {
    s->failed++;
  }
  s->cv_done.notify_all();
  s->cv_sched.notify_all();
}

void release_device(Job *j) {
  if (j->stream && j->inflight > 0) cudaStreamSynchronize(j->stream);
  j->inflight = 0;
  for (int k = 0; k < 2; ++k) {
    if (j->ev[k]) cudaEventDestroy(j->ev[k]);
    if (j->ring[k]) cudaFreeHost(j->ring[k]);
    if (j->status[k]) cudaFreeHost(j->status[k]);
    j->ev[k] = nullptr;
    j->ring[k] = nullptr;
    j->status[k] = nullptr;
  }
  if (j->p) salvus_problem_destroy(j->p);
  if (j->m) salvus_mesh_destroy(j->m);
  j->p = nullptr;
  j->m = nullptr;
  j->stream = nullptr;
}

// Host + device preparation of one job (worker thread).
int prepare(salvus_server *s, Job *j) {
  int rc = cudaSetDevice(s->device) == cudaSuccess ? SALVUS_OK : SALVUS_E_CUDA;
  if (rc) return salvus::fail(rc, "cudaSetDevice failed");
  salvus_mesh_desc d = j->mesh;
  d.vertices = j->vertices.data();
  d.cells = j->cells.data();
  d.params = j->params.data();
  if (j->precision == SALVUS_FP32) d.reserved |= SALVUS_MESH_FP32_ONLY;
  if ((rc = salvus_mesh_create(&d, s->device, &j->m))) return rc;
  int32_t c = 1;
  if ((rc = salvus_mesh_info(j->m, &j->G, &c, nullptr))) return rc;
  j->c = c;
  if ((rc = salvus_problem_create(j->m, j->precision, 1, &j->p))) return rc;
  if ((rc = salvus_problem_set_dt(j->p, j->dt))) return rc;
  if ((rc = salvus_problem_set_seismogram_capacity(j->p, 2 * (int64_t)s->chunk + 8))) return rc;
  for (auto &src : j->sources)
    if ((rc = salvus_problem_add_source(j->p, &src))) return rc;
  const int64_t R = (int64_t)j->receivers.size() / 3;
  for (int64_t r = 0; r < R; ++r)
    if ((rc = salvus_problem_add_receiver(j->p, &j->receivers[3 * r]))) return rc;
  j->seis.assign((size_t)(R * j->c * j->n_steps), 0.0);
  // sources and receivers on the device, step form tuned, here rather than
  // in the scheduler's first chunk
  if ((rc = salvus_problem_step_config(j->p, nullptr, nullptr))) return rc;
  void *st = nullptr;
  if ((rc = salvus_problem_stream(j->p, &st))) return rc;
  j->stream = (cudaStream_t)st;
  salvus::seis_ring_shape(j->p, &j->rows, &j->cap);
  for (int k = 0; k < 2; ++k) {
    if (cudaEventCreateWithFlags(&j->ev[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost((void **)&j->status[k], sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void **)&j->ring[k], sizeof(double) * std::max<int64_t>(1, j->rows * j->cap)) !=
            cudaSuccess)
      return salvus::fail(SALVUS_E_CUDA, "job %lld: chunk buffers", (long long)j->id);
  }
  return SALVUS_OK;
}

void worker_loop(salvus_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    Job *j = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->to_prepare.empty(); });
      if (s->stop) return;
      j = s->to_prepare.front();
      s->to_prepare.pop_front();
    }
    const auto t0 = Clock::now();
    int rc = j->cancel ? SALVUS_E_STATE : prepare(s, j);
    std::string err = rc ? salvus::last_error() : "";
    std::lock_guard<std::mutex> lk(s->mu);
    s->prep += std::chrono::duration<double>(Clock::now() - t0).count();
    s->n_preparing--;
    if (rc) {
      release_device(j);
      j->error = j->cancel ? "cancelled" : err;
      finish_locked(s, j, j->cancel ? SALVUS_JOB_CANCELLED : SALVUS_JOB_FAILED);
    } else {
      s->ready.push_back(j);
      s->cv_sched.notify_all();
    }
  }
}

void scheduler_loop(salvus_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Job *> run;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_sched.wait_for(lk, std::chrono::milliseconds(2), [&] {
        return s->stop || !s->ready.empty() || !s->running.empty() || !s->queue.empty();
      });
      if (s->stop) return;
      // admission: any queued job that fits the budget and the slot limit
      for (auto it = s->queue.begin(); it != s->queue.end();) {
        Job *j = *it;
        const int active = (int)s->running.size() + (int)s->ready.size() + s->n_preparing;
        if (active >= s->max_running) break;
        if (j->cancel) {
          j->state = SALVUS_JOB_CANCELLED;
          it = s->queue.erase(it);
          s->cv_done.notify_all();
          continue;
        }
        if (s->mem_in_use + j->est_bytes <= s->budget) {
          s->mem_in_use += j->est_bytes;
          s->peak_mem = std::max(s->peak_mem, s->mem_in_use);
          j->state = SALVUS_JOB_RUNNING;
          s->n_preparing++;
          s->to_prepare.push_back(j);
          s->cv_work.notify_one();
          it = s->queue.erase(it);
        } else {
          ++it;
        }
      }
      while (!s->ready.empty()) {
        s->running.push_back(s->ready.front());
        s->ready.pop_front();
      }
      const bool busy = !s->running.empty() || s->n_preparing > 0;
      if (busy && !s->busy_now) {
        s->busy_now = true;
        s->busy_since = Clock::now();
      } else if (!busy && s->busy_now) {
        s->busy_now = false;
        s->busy += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
      }
      run = s->running;
    }
    if (run.empty()) continue;
    bool progressed = false;
    for (Job *j : run) {
      int rc = SALVUS_OK;
      // collect this job's finished chunks, in order
      while (j->inflight > 0) {
        const int k = j->head;
        const cudaError_t q = cudaEventQuery(j->ev[k]);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) {
          rc = salvus::fail(SALVUS_E_CUDA, "job %lld: %s", (long long)j->id, cudaGetErrorString(q));
          break;
        }
        if ((rc = salvus::status_error(j->p, *j->status[k]))) break;
        const int64_t f = j->first[k], n = j->count[k];
        for (int64_t r = 0; r < j->rows; ++r)
          for (int64_t t = 0; t < n; ++t)
            j->seis[(size_t)(r * j->n_steps + f + t)] = j->ring[k][r * j->cap + (f + t) % j->cap];
        j->steps_done += n;
        j->head ^= 1;
        j->inflight--;
        progressed = true;
      }
      // keep two chunks in flight
      while (rc == SALVUS_OK && !j->cancel && j->inflight < 2 && j->enq_steps < j->n_steps) {
        const int k = (j->head + j->inflight) & 1;
        const int64_t n = std::min<int64_t>(s->chunk, j->n_steps - j->enq_steps);
        if ((rc = salvus_run(j->p, n, SALVUS_RUN_GRAPH))) break;
        if ((rc = salvus::enqueue_seis_copy(j->p, j->ring[k], j->status[k]))) break;
        if (cudaEventRecord(j->ev[k], j->stream) != cudaSuccess) {
          rc = salvus::fail(SALVUS_E_CUDA, "job %lld: event record", (long long)j->id);
          break;
        }
        j->first[k] = j->enq_steps;
        j->count[k] = n;
        j->enq_steps += n;
        j->inflight++;
        progressed = true;
      }
      if (rc != SALVUS_OK) j->error = salvus::last_error();
      const bool cancelled = j->cancel;
      const bool finished = rc != SALVUS_OK || (cancelled && j->inflight == 0) ||
                            j->steps_done >= j->n_steps;
      if (finished) {
        release_device(j);
        std::lock_guard<std::mutex> lk(s->mu);
        s->running.erase(std::find(s->running.begin(), s->running.end(), j));
        finish_locked(s, j, rc != SALVUS_OK ? SALVUS_JOB_FAILED
                               : cancelled  ? SALVUS_JOB_CANCELLED
                                            : SALVUS_JOB_DONE);
      }
    }
    // nothing finished or started: let the device work before polling again
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

Job *find_job(salvus_server *s, int64_t id) {
  auto it = s->jobs.find(id);
  return it == s->jobs.end() ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

int salvus_server_create(int device, int64_t budget, int32_t max_running, int32_t chunk,
                         salvus_server **out) {
  if (!out) return salvus::fail(SALVUS_E_INVALID, "null argument");
  if (budget <= 0 || max_running < 1 || chunk < 1)
    return salvus::fail(SALVUS_E_INVALID, "budget, max_running and chunk must be positive");
  if (cudaSetDevice(device) != cudaSuccess)
    return salvus::fail(SALVUS_E_CUDA, "cannot use device %d", device);
  auto *s = new salvus_server();
  s->device = device;
  s->budget = budget;
  s->max_running = max_running;
  s->chunk = chunk;
  s->sched = std::thread(scheduler_loop, s);
  const unsigned hw = std::thread::hardware_concurrency();
  const int nw = (int)std::max(1u, std::min(8u, hw / 2));
  for (int w = 0; w < nw; ++w) s->workers.emplace_back(worker_loop, s);
  *out = s;
  return SALVUS_OK;
}

int salvus_server_submit(salvus_server *s, const salvus_job_desc *d, int64_t *job_id) {
  if (!s || !d || !job_id) return salvus::fail(SALVUS_E_INVALID, "null argument");
  if (d->n_steps <= 0 || !(d->dt > 0)) return salvus::fail(SALVUS_E_INVALID, "bad dt / n_steps");
  const salvus_mesh_desc &m = d->mesh;
  if (m.n_elements <= 0 || m.n_vertices <= 0 || !m.vertices || !m.cells || !m.params)
    return salvus::fail(SALVUS_E_INVALID, "empty mesh");
  if (m.shape != SALVUS_QUAD && m.shape != SALVUS_HEX)
    return salvus::fail(SALVUS_E_UNSUPPORTED, "shape %d not served", m.shape);
  std::unique_ptr<Job> j(new Job());
  j->mesh = m;
  const int dim = m.shape == SALVUS_QUAD ? 2 : 3, nv = m.shape == SALVUS_QUAD ? 4 : 8;
  const int npar = salvus::physics_params(m.physics, m.reserved);
  j->vertices.assign(m.vertices, m.vertices + m.n_vertices * dim);
  j->cells.assign(m.cells, m.cells + m.n_elements * nv);
  j->params.assign(m.params, m.params + (size_t)npar * m.n_elements * nv);
  if (d->n_sources > 0) j->sources.assign(d->sources, d->sources + d->n_sources);
  if (d->n_receivers > 0) j->receivers.assign(d->receivers, d->receivers + 3 * d->n_receivers);
  j->precision = d->precision;
  j->dt = d->dt;
  j->n_steps = d->n_steps;
  j->est_bytes = estimate_bytes(m, d->precision);
  if (j->est_bytes > s->budget)
    return salvus::fail(SALVUS_E_OOM, "job needs about %lld bytes; the server budget is %lld",
                        (long long)j->est_bytes, (long long)s->budget);
  j->submitted = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  j->id = s->next_id++;
  *job_id = j->id;
  s->queue.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  s->submitted++;
  s->cv_sched.notify_all();
  return SALVUS_OK;
}

int salvus_server_poll(salvus_server *s, int64_t id, int32_t *state, int64_t *steps_done,
                       int64_t *n_nodes) {
  if (!s) return salvus::fail(SALVUS_E_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Job *j = find_job(s, id);
  if (!j) return salvus::fail(SALVUS_E_INVALID, "unknown job %lld", (long long)id);
  if (state) *state = j->state;
  if (steps_done) *steps_done = j->steps_done;
  if (n_nodes) *n_nodes = j->G;
  if (j->state == SALVUS_JOB_FAILED) salvus::set_error("%s", j->error.c_str());
  return SALVUS_OK;
}

int salvus_server_seismograms(salvus_server *s, int64_t id, int64_t first, int64_t count, double *out) {
  if (!s || !out) return salvus::fail(SALVUS_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  Job *j = find_job(s, id);
  if (!j) return salvus::fail(SALVUS_E_INVALID, "unknown job %lld", (long long)id);
  if (first < 0 || count < 0 || first + count > j->steps_done)
    return salvus::fail(SALVUS_E_INVALID, "steps [%lld, %lld) not yet streamed (%lld done)",
                        (long long)first, (long long)(first + count), (long long)j->steps_done.load());
  const int64_t rows = (int64_t)j->receivers.size() / 3 * j->c;
  for (int64_t q = 0; q < rows; ++q)
    std::memcpy(out + q * count, &j->seis[(size_t)(q * j->n_steps + first)], sizeof(double) * count);
  return SALVUS_OK;
}

int salvus_server_wait(salvus_server *s, int64_t id, double timeout_s) {
  if (!s) return salvus::fail(SALVUS_E_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  Job *j = find_job(s, id);
  if (!j) return salvus::fail(SALVUS_E_INVALID, "unknown job %lld", (long long)id);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    const int st = j->state;
    return st == SALVUS_JOB_DONE || st == SALVUS_JOB_FAILED || st == SALVUS_JOB_CANCELLED;
  });
  if (!ok) return salvus::fail(SALVUS_E_TIMEOUT, "job %lld not finished after %.3f s", (long long)id, timeout_s);
  if (j->state == SALVUS_JOB_FAILED) return salvus::fail(SALVUS_E_INVALID, "%s", j->error.c_str());
  return SALVUS_OK;
}

int salvus_server_cancel(salvus_server *s, int64_t id) {
  if (!s) return salvus::fail(SALVUS_E_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Job *j = find_job(s, id);
  if (!j) return salvus::fail(SALVUS_E_INVALID, "unknown job %lld", (long long)id);
  j->cancel = true;
  s->cv_sched.notify_all();
  return SALVUS_OK;
}

int salvus_server_release(salvus_server *s, int64_t id) {
  if (!s) return salvus::fail(SALVUS_E_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Job *j = find_job(s, id);
  if (!j) return salvus::fail(SALVUS_E_INVALID, "unknown job %lld", (long long)id);
  const int st = j->state;
  if (st != SALVUS_JOB_DONE && st != SALVUS_JOB_FAILED && st != SALVUS_JOB_CANCELLED)
    return salvus::fail(SALVUS_E_STATE, "job %lld is still active", (long long)id);
  s->jobs.erase(id);
  return SALVUS_OK;
}

int salvus_server_stats_read(salvus_server *s, salvus_server_stats *o) {
  if (!s || !o) return salvus::fail(SALVUS_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) -> double {
    if (l.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>(l.size() - 1, std::ceil(q * l.size()) - 1);
    return l[k];
  };
  std::memset(o, 0, sizeof(*o));
  o->submitted = s->submitted;
  o->completed = s->completed;
  o->failed = s->failed;
  o->running = (int64_t)s->running.size() + s->n_preparing + (int64_t)s->ready.size();
  o->queued = (int64_t)s->queue.size();
  o->p50_latency_s = pct(0.50);
  o->p99_latency_s = pct(0.99);
  double sum = 0;
  for (double x : l) sum += x;
  o->mean_latency_s = l.empty() ? 0.0 : sum / l.size();
  o->gll_point_updates = s->updates;
  o->busy_seconds = s->busy + (s->busy_now ? std::chrono::duration<double>(Clock::now() - s->busy_since).count() : 0.0);
  o->peak_device_bytes = s->peak_mem;
  o->prep_seconds = s->prep;
  return SALVUS_OK;
}

int salvus_server_destroy(salvus_server *s) {
  if (!s) return SALVUS_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto &kv : s->jobs) kv.second->cancel = true;
  }
  s->cv_sched.notify_all();
  s->cv_work.notify_all();
  if (s->sched.joinable()) s->sched.join();
  for (auto &w : s->workers)
    if (w.joinable()) w.join();
  cudaSetDevice(s->device);
  for (auto &kv : s->jobs) release_device(kv.second.get());
  delete s;
  return SALVUS_OK;
}

}  // extern "C"
