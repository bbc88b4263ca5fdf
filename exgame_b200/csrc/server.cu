// Continuous-batching request loop over a world pool.
//
// The reference funnels every producer into one worker thread that owns all GPU submission
// (crates/newton/src/accelerator/mod.rs:1010-1155) and reports a dead loop as
// EvalError::WorkerGone (crates/newton/src/error.rs:11-28). Here producers submit whole
// simulation requests (a world and a step count) from any thread; one worker thread owns a pool
// (exg_pool_*), admits queued requests in arrival order while the memory budget and the pool's
// ranges allow, gives each admitted world its step budget, and steps the pool in ticks of CUDA
// graph replays. Worlds whose budget is spent hold still on the device until the tick ends, when
// their state is read back and their ranges are released for the next admissions. Every world
// takes exactly its requested steps, with the arithmetic it would have alone.
//
// The loop uses only the public C ABI, so it is also a worked example of serving on top of it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>
#include "../../include/exg.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

struct Request {
  uint64_t id = 0;
  std::vector<exg_body_t> bodies;  // input, then the result
  std::vector<exg_joint_t> joints;
  exg_step_params_t params{};
  int32_t steps = 0;
  int32_t left = 0;  // steps still to take (host mirror of the pool's counter)
  int64_t footprint = 0;
  int32_t slot = -1;
  int status = EXG_PENDING;
  double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct exg_server_s {
  exg_device_t dev = nullptr;
  exg_world_t pool = nullptr;
  exg_server_config_t cfg{};
  Clock::time_point t0 = Clock::now();        // request clocks
  Clock::time_point t_stats = Clock::now();   // start of the statistics window
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;                     // submitted, not yet admitted
  std::unordered_map<uint64_t, std::shared_ptr<Request>> known;  // every request not yet collected
  std::vector<std::shared_ptr<Request>> running;                 // by pool slot (worker only)
  int n_running = 0;
  int64_t resident = 0;
  uint64_t next_id = 1;
  bool stop = false;
  bool worker_gone = false;
  int worker_status = EXG_OK;
  std::thread worker;
  // statistics (under mu)
  int64_t submitted = 0, completed = 0, failed = 0, ticks = 0, steps_launched = 0, body_steps = 0;
  int32_t peak_running = 0;
  int64_t peak_resident = 0;
  double busy_s = 0.0;
  std::vector<double> latencies;
};

namespace {

void finish_locked(exg_server_s* S, const std::shared_ptr<Request>& r, int status) {
  r->status = status;
  r->t_done = seconds_since(S->t0);
  if (status == EXG_OK) {
    ++S->completed;
    S->body_steps += (int64_t)r->bodies.size() * r->steps;
    S->latencies.push_back(r->t_done - r->t_submit);
  } else {
    ++S->failed;
  }
}

// Release a running request's slot and publish its outcome.
void retire(exg_server_s* S, const std::shared_ptr<Request>& r, int status) {
  int st = status;
  if (st == EXG_OK && !r->bodies.empty())
    st = exg_batch_get_world(S->pool, r->slot, r->bodies.data(), (int32_t)r->bodies.size());
  exg_pool_release(S->pool, r->slot);
  std::lock_guard<std::mutex> lk(S->mu);
  S->running[r->slot].reset();
  --S->n_running;
  S->resident -= r->footprint;
  finish_locked(S, r, st);
  S->cv_done.notify_all();
}

// Admit queued requests in arrival order while the budget and the pool allow.
void admit(exg_server_s* S) {
  for (;;) {
    std::shared_ptr<Request> r;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (S->queue.empty()) return;
      r = S->queue.front();
      if (S->n_running > 0 && S->resident + r->footprint > S->cfg.hbm_budget_bytes) return;
      S->queue.pop_front();
    }
    if (r->steps == 0) {  // nothing to step: the result is the input
      std::lock_guard<std::mutex> lk(S->mu);
      r->t_admit = seconds_since(S->t0);
      finish_locked(S, r, EXG_OK);
      S->cv_done.notify_all();
      continue;
    }
    int32_t slot = -1;
    int rc = exg_pool_admit(S->pool, r->bodies.data(), (int32_t)r->bodies.size(), r->joints.data(),
                            (int32_t)r->joints.size(), &r->params, &slot);
    if (rc == EXG_OK) rc = exg_pool_set_steps(S->pool, slot, r->steps);
    std::lock_guard<std::mutex> lk(S->mu);
    if (rc == EXG_ERR_OUT_OF_MEMORY && S->n_running > 0) {  // wait for ranges to free up
      S->queue.push_front(r);
      return;
    }
    if (rc != EXG_OK) {
      if (slot >= 0) exg_pool_release(S->pool, slot);
      finish_locked(S, r, rc);
      S->cv_done.notify_all();
      continue;
    }
    r->slot = slot;
    r->left = r->steps;
    r->t_admit = seconds_since(S->t0);
    S->running[slot] = r;
    ++S->n_running;
    S->resident += r->footprint;
    S->peak_running = std::max<int32_t>(S->peak_running, S->n_running);
    S->peak_resident = std::max(S->peak_resident, S->resident);
  }
}

void run(exg_server_s* S) {
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->stop) break;
      if (S->queue.empty() && S->n_running == 0) {
        S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
    }
    admit(S);
    std::vector<std::shared_ptr<Request>> live;
    for (auto& r : S->running)
      if (r) live.push_back(r);
    if (live.empty()) continue;
    int32_t tick = 0;
    for (auto& r : live) tick = std::max(tick, r->left);
    tick = std::min(tick, S->cfg.steps_per_tick);
    Clock::time_point t_tick = Clock::now();
    int rc = exg_world_step(S->pool, tick);
    for (auto& r : live) r->left = std::max(0, r->left - tick);
    if (rc == EXG_ERR_FATAL) {
      // a guarded site fired in some worlds: those fail, the rest go on
      for (auto& r : live) {
        exg_world_stats_t st;
        if (exg_batch_world_stats(S->pool, r->slot, &st) == EXG_OK && st.fatal) retire(S, r, EXG_ERR_FATAL);
      }
      rc = EXG_OK;
    }
    if (rc != EXG_OK) {  // the device is unusable: fail everything and stop serving
      for (auto& r : live)
        if (S->running[r->slot]) retire(S, r, rc);
      std::lock_guard<std::mutex> lk(S->mu);
      S->worker_gone = true;
      S->worker_status = rc;
      for (auto& q : S->queue) finish_locked(S, q, EXG_ERR_WORKER_GONE);
      S->queue.clear();
      S->cv_done.notify_all();
      return;
    }
    for (auto& r : live)
      if (r->left == 0 && S->running[r->slot]) retire(S, r, EXG_OK);
    std::lock_guard<std::mutex> lk(S->mu);
    ++S->ticks;
    S->steps_launched += tick;
    S->busy_s += seconds_since(t_tick);
  }
}

// Result and info of a finished request; forgets it (under mu).
int collect_locked(exg_server_s* S, uint64_t id, exg_body_t* out, int32_t n, exg_request_info_t* info) {
  auto it = S->known.find(id);
  if (it == S->known.end()) return EXG_ERR_INVALID_ARGUMENT;
  const std::shared_ptr<Request>& r = it->second;
  if (info) {
    info->steps = r->steps;
    info->n_bodies = (int32_t)r->bodies.size();
    info->status = r->status;
    info->queued_s = (r->t_admit > 0 ? r->t_admit : seconds_since(S->t0)) - r->t_submit;
    info->latency_s = (r->status == EXG_PENDING ? seconds_since(S->t0) : r->t_done) - r->t_submit;
  }
  if (r->status == EXG_PENDING) return EXG_PENDING;
  if (out) {
    if (n != (int32_t)r->bodies.size()) return EXG_ERR_INVALID_ARGUMENT;
    std::copy(r->bodies.begin(), r->bodies.end(), out);
  }
  int st = r->status;
  S->known.erase(it);
  return st;
}

}  // namespace

extern "C" {

int exg_server_create(exg_device_t dev, const exg_server_config_t* cfg, exg_server_t* out) {
  if (!dev || !cfg || !out || cfg->hbm_budget_bytes <= 0 || cfg->max_worlds <= 0 || cfg->max_bodies <= 0 ||
      cfg->max_joints < 0 || cfg->steps_per_tick <= 0)
    return EXG_ERR_INVALID_ARGUMENT;
  exg_server_s* S = new (std::nothrow) exg_server_s();
  if (!S) return EXG_ERR_OUT_OF_MEMORY;
  S->dev = dev;
  S->cfg = *cfg;
  exg_pool_config_t pc{};
  pc.max_bodies = cfg->max_bodies;
  pc.max_joints = cfg->max_joints;
  pc.max_worlds = cfg->max_worlds;
  pc.precision = cfg->precision;
  int rc = exg_pool_create(dev, &pc, &S->pool);
  if (rc != EXG_OK) {
    delete S;
    return rc;
  }
  S->running.resize(cfg->max_worlds);
  try {
    S->worker = std::thread(run, S);
  } catch (...) {
    exg_world_destroy(S->pool);
    delete S;
    return EXG_ERR_BACKEND;
  }
  *out = S;
  return EXG_OK;
}

int exg_server_submit(exg_server_t S, const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                      const exg_step_params_t* params, int32_t steps, uint64_t* id) {
  if (!S || !id || !params || n < 0 || nj < 0 || steps < 0 || (n > 0 && !bodies) || (nj > 0 && !joints))
    return EXG_ERR_INVALID_ARGUMENT;
  if (params->precision != S->cfg.precision) return EXG_ERR_INVALID_ARGUMENT;
  if (n > S->cfg.max_bodies || nj > S->cfg.max_joints) return EXG_ERR_OUT_OF_MEMORY;  // can never fit
  int64_t fp = 0;
  int rc = exg_world_footprint(n, nj, params, &fp);
  if (rc != EXG_OK) return rc;
  if (fp > S->cfg.hbm_budget_bytes) return EXG_ERR_OUT_OF_MEMORY;
  auto r = std::make_shared<Request>();
  r->bodies.assign(bodies, bodies + n);
  r->joints.assign(joints, joints + nj);
  r->params = *params;
  r->steps = steps;
  r->footprint = fp;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->worker_gone) return EXG_ERR_WORKER_GONE;
  r->id = S->next_id++;
  r->t_submit = seconds_since(S->t0);
  S->known[r->id] = r;
  S->queue.push_back(r);
  ++S->submitted;
  *id = r->id;
  S->cv_work.notify_one();
  return EXG_OK;
}

int exg_server_poll(exg_server_t S, uint64_t id, exg_body_t* out, int32_t n, exg_request_info_t* info) {
  if (!S) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  return collect_locked(S, id, out, n, info);
}

int exg_server_wait(exg_server_t S, uint64_t id, int32_t timeout_ms, exg_body_t* out, int32_t n,
                    exg_request_info_t* info) {
  if (!S || timeout_ms < 0) return EXG_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->known.find(id);
  if (it == S->known.end()) return EXG_ERR_INVALID_ARGUMENT;
  std::shared_ptr<Request> r = it->second;
  if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->status != EXG_PENDING; }))
    return EXG_ERR_TIMEOUT;
  return collect_locked(S, id, out, n, info);
}

int exg_server_stats(exg_server_t S, exg_server_stats_t* out) {
  if (!S || !out) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = exg_server_stats_t{};
  out->submitted = S->submitted;
  out->completed = S->completed;
  out->failed = S->failed;
  out->ticks = S->ticks;
  out->steps_launched = S->steps_launched;
  out->body_steps = S->body_steps;
  out->queued = (int32_t)S->queue.size();
  out->running = S->n_running;
  out->peak_running = S->peak_running;
  out->resident_bytes = S->resident;
  out->peak_resident_bytes = S->peak_resident;
  out->busy_s = S->busy_s;
  out->elapsed_s = seconds_since(S->t_stats);
  if (!S->latencies.empty()) {
    std::vector<double> v(S->latencies);
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {  // nearest rank
      size_t k = (size_t)std::max<double>(0.0, std::ceil(p * v.size()) - 1.0);
      return v[std::min(k, v.size() - 1)];
    };
    out->p50_latency_s = pct(0.50);
    out->p99_latency_s = pct(0.99);
    double s = 0.0;
    for (double x : v) s += x;
    out->mean_latency_s = s / v.size();
  }
  return S->worker_gone ? S->worker_status : EXG_OK;
}

int exg_server_reset_stats(exg_server_t S) {
  if (!S) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  S->submitted = S->completed = S->failed = S->ticks = S->steps_launched = S->body_steps = 0;
  S->peak_running = S->n_running;
  S->peak_resident = S->resident;
  S->busy_s = 0.0;
  S->latencies.clear();
  S->t_stats = Clock::now();
  return EXG_OK;
}

int exg_server_destroy(exg_server_t S) {
  if (!S) return EXG_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  exg_world_destroy(S->pool);
  delete S;
  return EXG_OK;
}

}  // extern "C"
