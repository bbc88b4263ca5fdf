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
// With cfg.pools = 2 the capacities are split between two pools, each on a CUDA stream of its own
// (EXG_OPT_OWN_STREAM) and stepped by a worker thread of its own; both take requests from the one
// arrival queue under the one memory budget, so one pool's admissions, state uploads and
// read-backs run on the host and its copy engines while the other pool's tick runs on the GPU.
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
  int lane = -1;  // the pool it runs in
  int status = EXG_PENDING;
  double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct ServerLane {  // one pool and the worker thread that steps it
  exg_world_t pool = nullptr;
  std::vector<std::shared_ptr<Request>> running;  // by pool slot (this lane's worker only)
  int n_running = 0;                              // (under the server's mu)
  std::thread worker;
};

struct exg_server_s {
  exg_device_t dev = nullptr;
  std::vector<ServerLane> lanes;
  exg_server_config_t cfg{};
  Clock::time_point t0 = Clock::now();        // request clocks
  Clock::time_point t_stats = Clock::now();   // start of the statistics window
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;                     // submitted, not yet admitted
  std::unordered_map<uint64_t, std::shared_ptr<Request>> known;  // every request not yet collected
  int n_running = 0;                                              // over all lanes
  int n_admitting = 0;  // requests taken off the queue whose pool admission is still under way
  int64_t resident = 0;
  uint64_t next_id = 1;
  bool stop = false;
  bool worker_gone = false;
  int worker_status = EXG_OK;
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
void retire(exg_server_s* S, ServerLane& L, const std::shared_ptr<Request>& r, int status) {
  int st = status;
  if (st == EXG_OK && !r->bodies.empty())
    st = exg_batch_get_world(L.pool, r->slot, r->bodies.data(), (int32_t)r->bodies.size());
  exg_pool_release(L.pool, r->slot);
  std::lock_guard<std::mutex> lk(S->mu);
  L.running[r->slot].reset();
  --L.n_running;
  --S->n_running;
  S->resident -= r->footprint;
  finish_locked(S, r, st);
  S->cv_done.notify_all();
}

// Admit queued requests in arrival order into this lane's pool while the budget and the pool allow.
void admit(exg_server_s* S, ServerLane& L, int lane) {
  for (;;) {
    std::shared_ptr<Request> r;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (S->queue.empty()) return;
      r = S->queue.front();
      const bool others = S->n_running > 0 || S->n_admitting > 0;
      if (others && S->resident + r->footprint > S->cfg.hbm_budget_bytes) return;
      S->queue.pop_front();
      // the budget is taken now, under the lock, so the other lane's admission counts it
      S->resident += r->footprint;
      ++S->n_admitting;
      S->peak_resident = std::max(S->peak_resident, S->resident);
    }
    if (r->steps == 0) {  // nothing to step: the result is the input
      std::lock_guard<std::mutex> lk(S->mu);
      --S->n_admitting;
      S->resident -= r->footprint;
      r->t_admit = seconds_since(S->t0);
      finish_locked(S, r, EXG_OK);
      S->cv_done.notify_all();
      continue;
    }
    int32_t slot = -1;
    int rc = exg_pool_admit(L.pool, r->bodies.data(), (int32_t)r->bodies.size(), r->joints.data(),
                            (int32_t)r->joints.size(), &r->params, &slot);
    if (rc == EXG_OK) rc = exg_pool_set_steps(L.pool, slot, r->steps);
    std::lock_guard<std::mutex> lk(S->mu);
    --S->n_admitting;
    if (rc != EXG_OK) S->resident -= r->footprint;
    if (rc == EXG_ERR_OUT_OF_MEMORY && (L.n_running > 0 || S->n_running > 0 || S->n_admitting > 0)) {
      S->queue.push_front(r);  // wait for ranges to free up
      return;
    }
    if (rc != EXG_OK) {
      if (slot >= 0) exg_pool_release(L.pool, slot);
      finish_locked(S, r, rc);
      S->cv_done.notify_all();
      continue;
    }
    r->slot = slot;
    r->lane = lane;
    r->left = r->steps;
    r->t_admit = seconds_since(S->t0);
    L.running[slot] = r;
    ++L.n_running;
    ++S->n_running;
    S->peak_running = std::max<int32_t>(S->peak_running, S->n_running);
  }
}

void run(exg_server_s* S, int lane) {
  ServerLane& L = S->lanes[lane];
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->stop || S->worker_gone) break;
      if (S->queue.empty() && L.n_running == 0) {
        S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
    }
    admit(S, L, lane);
    std::vector<std::shared_ptr<Request>> live;
    for (auto& r : L.running)
      if (r) live.push_back(r);
    if (live.empty()) {
      std::unique_lock<std::mutex> lk(S->mu);  // the queue head waits for the other lane's memory
      S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
      continue;
    }
    int32_t tick = 0;
    for (auto& r : live) tick = std::max(tick, r->left);
    tick = std::min(tick, S->cfg.steps_per_tick);
    Clock::time_point t_tick = Clock::now();
    int rc = exg_world_step(L.pool, tick);
    for (auto& r : live) r->left = std::max(0, r->left - tick);
    if (rc == EXG_ERR_FATAL) {
      // a guarded site fired in some worlds: those fail, the rest go on
      for (auto& r : live) {
        exg_world_stats_t st;
        if (exg_batch_world_stats(L.pool, r->slot, &st) == EXG_OK && st.fatal) retire(S, L, r, EXG_ERR_FATAL);
      }
      rc = EXG_OK;
    }
    if (rc != EXG_OK) {  // the device is unusable: fail everything and stop serving
      for (auto& r : live)
        if (L.running[r->slot]) retire(S, L, r, rc);
      std::lock_guard<std::mutex> lk(S->mu);
      S->worker_gone = true;
      S->worker_status = rc;
      for (auto& q : S->queue) finish_locked(S, q, EXG_ERR_WORKER_GONE);
      S->queue.clear();
      S->cv_done.notify_all();
      S->cv_work.notify_all();
      return;
    }
    for (auto& r : live)
      if (r->left == 0 && L.running[r->slot]) retire(S, L, r, EXG_OK);
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
  const int pools = cfg->pools == 0 ? 1 : cfg->pools;
  if (pools < 1 || pools > 2 || cfg->max_worlds < pools) return EXG_ERR_INVALID_ARGUMENT;
  exg_server_s* S = new (std::nothrow) exg_server_s();
  if (!S) return EXG_ERR_OUT_OF_MEMORY;
  S->dev = dev;
  S->cfg = *cfg;
  S->cfg.pools = pools;
  S->lanes.resize(pools);
  exg_pool_config_t pc{};
  pc.max_bodies = cfg->max_bodies / pools;
  pc.max_joints = cfg->max_joints / pools;
  pc.max_worlds = cfg->max_worlds / pools;
  pc.precision = cfg->precision;
  int rc = EXG_OK;
  for (int k = 0; k < pools && rc == EXG_OK; ++k) {
    rc = exg_pool_create(dev, &pc, &S->lanes[k].pool);
    if (rc == EXG_OK && pools > 1) rc = exg_world_set_option(S->lanes[k].pool, EXG_OPT_OWN_STREAM, 1);
    S->lanes[k].running.resize(pc.max_worlds);
  }
  auto undo = [&]() {
    for (ServerLane& L : S->lanes)
      if (L.pool) exg_world_destroy(L.pool);
    delete S;
  };
  if (rc != EXG_OK) {
    undo();
    return rc;
  }
  try {
    for (int k = 0; k < pools; ++k) S->lanes[k].worker = std::thread(run, S, k);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stop = true;
    }
    for (ServerLane& L : S->lanes)
      if (L.worker.joinable()) L.worker.join();
    undo();
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
  if (n > S->cfg.max_bodies / S->cfg.pools || nj > S->cfg.max_joints / S->cfg.pools)
    return EXG_ERR_OUT_OF_MEMORY;  // can never fit a pool
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
  S->cv_work.notify_all();
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
  for (ServerLane& L : S->lanes)
    if (L.worker.joinable()) L.worker.join();
  for (ServerLane& L : S->lanes) exg_world_destroy(L.pool);
  delete S;
  return EXG_OK;
}

}  // extern "C"
