// mg_server.cu -- continuous-batching answer loop over the scan workspaces.
//
// The reference serves GPU queries from tokio handlers that each lock the
// matrix and run one scan (crates/morphogen-server/src/network/api/mod.rs:
// 544-838, network/gpu_batch.rs:129-149).  Here a dispatcher thread owns a
// pool of workspaces (one CUDA stream each): whenever a workspace is free it
// folds every request that has arrived since into one pass, so requests that
// arrive while others are on the GPU join the next pass and passes of
// different workspaces overlap on the device.  Work is admitted against free
// device memory (keys, frontier and partial rows of the pass), pausing drains
// the in-flight passes so that an epoch merge can patch the tables, and the
// loop records per-request latency for p50/p95/p99.
//
// Locking: one mutex guards the queues, the request table and the statistics.
// The dispatcher holds it only to decide what to do; key parsing, planning,
// the key upload, the launch and the read-back of a pass run with the mutex
// released, so submit / wait / stats never wait behind a pass being planned.
// A slot whose requests are assigned counts as in flight from the moment it
// is claimed, so a pause waits for it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mg_internal.h"
#include "morphogen_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

// Pass size when the caller sets no key cap: a pass is closed once its
// estimated device time reaches this bound (the p99 target of a lookup), so
// the earliest requests of a backlog are answered after one bounded pass
// instead of after the whole backlog.
constexpr double kPassTargetS = 0.050;

struct Request {
  uint64_t id = 0;
  std::vector<const mg_table*> tables;
  std::vector<std::vector<uint8_t>> keys;
  std::vector<uint8_t> shares;
  size_t share_bytes = 0;
  uint64_t est_bytes = 0;  // device scratch estimate for admission
  double cost = 0;         // tree nodes its keys expand (sum of the tables' rows)
  Clock::time_point t_submit, t_done;
  int status = MG_OK;
  std::string error;
  bool done = false;
};

// Device bytes a key adds to a pass: its device copy (key and warp-kernel
// constants, 1200 B), its frontier (17 B per
// node: at most rows / 2 nodes for tables up to 2^24 rows, rows / 2^8 above,
// where the planner keeps at least 8 depth-first levels) and partial-row
// columns for every persistent warp.
uint64_t key_scratch_bytes(const mg_table* t, int sms) {
  const uint64_t rows = mg_table_rows(t);
  const uint64_t frontier = (rows <= (1ull << 24) ? rows / 2 : rows >> 8) * 17 + 32 * 17;
  const uint64_t partial = (uint64_t)sms * 4 * 8 * (mg_table_row_bytes(t));
  return 1200 + frontier + partial;
}

}  // namespace

struct mg_server {
  mg_context* ctx = nullptr;
  mg_server_config cfg{};
  int sms = 0;
  std::vector<mg_batch*> slots;
  std::vector<std::vector<Request*>> slot_reqs;
  std::vector<Clock::time_point> slot_start;
  std::mutex mu;
  std::condition_variable cv_work;  // dispatcher wake-up
  std::condition_variable cv_done;  // request completion / drain
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  bool paused = false;
  std::thread dispatcher;
  uint32_t waiters = 0;   // threads inside mg_server_wait
  bool closing = false;   // destroy is waiting for the waiters to leave
  // Measured device rate (tree nodes per second) of completed passes, for the
  // latency-aware pass size; 0 until the first pass completes.
  double node_rate = 0;
  std::vector<double> slot_cost;
  // statistics
  std::vector<double> lat_ms;
  uint64_t completed = 0, failed = 0, passes = 0, keys_done = 0;
  Clock::time_point t0;
};

namespace {

uint32_t in_flight(const mg_server* s) {
  uint32_t n = 0;
  for (const auto& r : s->slot_reqs) n += r.empty() ? 0 : 1;
  return n;
}

// Hands a slot's shares (or its error) to its requests; called with the
// mutex held, after the shares were read back with the mutex released.
void finish_slot(mg_server* s, size_t i, int status, const char* err, const std::vector<uint8_t>& all) {
  std::vector<Request*>& rs = s->slot_reqs[i];
  const auto now = Clock::now();
  size_t off = 0;
  for (Request* r : rs) {
    r->status = status;
    if (status == MG_OK) {
      r->shares.assign(all.begin() + off, all.begin() + off + r->share_bytes);
      s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
      ++s->completed;
      s->keys_done += r->keys.size();
    } else {
      r->error = err ? err : "pass failed";
      ++s->failed;
    }
    off += r->share_bytes;
    r->t_done = now;
    r->done = true;
  }
  ++s->passes;
  rs.clear();
}

void run(mg_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    // 1. Completions: the slot stays claimed (in flight) while its shares
    //    are read back with the mutex released.
    for (size_t i = 0; i < s->slots.size(); ++i) {
      if (s->slot_reqs[i].empty()) continue;
      if (!mg::batch_done(s->slots[i])) continue;
      size_t total = 0;
      for (Request* r : s->slot_reqs[i]) total += r->share_bytes;
      std::vector<uint8_t> all(total);
      lk.unlock();
      int status = mg_batch_read(s->slots[i], all.data(), nullptr);
      std::string err = status == MG_OK ? std::string() : std::string(mg_last_error());
      uint64_t ns = 0;
      if (status == MG_OK && mg_batch_last_kernel_ns(s->slots[i], &ns) != MG_OK) ns = 0;
      lk.lock();
      if (status == MG_OK && ns > 0 && s->slot_cost[i] > 0) {
        const double rate = s->slot_cost[i] / ((double)ns * 1e-9);
        s->node_rate = s->node_rate > 0 ? 0.7 * s->node_rate + 0.3 * rate : rate;
      }
      finish_slot(s, i, status, err.c_str(), all);
      s->cv_done.notify_all();
    }
    if (s->stop && in_flight(s) == 0) break;
    // 2. Dispatch: one pass per free workspace from everything pending.
    if (!s->paused && !s->stop) {
      for (size_t i = 0; i < s->slots.size() && !s->pending.empty(); ++i) {
        if (!s->slot_reqs[i].empty()) continue;
        size_t free_b = 0, total_b = 0;
        lk.unlock();  // only this thread claims slots or takes pending requests
        cudaSetDevice(mg::context_device(s->ctx));
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
          cudaGetLastError();
          free_b = 0;
        }
        lk.lock();
        if (s->paused || s->stop) break;
        const uint64_t budget = free_b > s->cfg.memory_reserve ? free_b - s->cfg.memory_reserve : 0;
        // Without an explicit key cap, close the pass at the measured device
        // time bound (always at least one request).
        const double cost_cap = (s->cfg.max_keys_per_pass == 0 && s->node_rate > 0)
                                    ? s->node_rate * kPassTargetS : 0.0;
        std::vector<Request*> take;
        uint64_t need = 0, nk = 0;
        double cost = 0;
        while (!s->pending.empty()) {
          Request* r = s->pending.front();
          const bool first = take.empty();
          if (!first && s->cfg.max_keys_per_pass && nk + r->keys.size() > s->cfg.max_keys_per_pass) break;
          if (!first && cost_cap > 0 && cost + r->cost > cost_cap) break;
          if (!first && need + r->est_bytes > budget) break;
          if (first && r->est_bytes > budget && in_flight(s) > 0) break;  // wait for memory to free up
          take.push_back(r);
          need += r->est_bytes;
          nk += r->keys.size();
          cost += r->cost;
          s->pending.pop_front();
        }
        if (take.empty()) break;
        std::vector<const mg_table*> tabs;
        std::vector<const uint8_t*> kp;
        std::vector<size_t> kl;
        for (Request* r : take)
          for (size_t j = 0; j < r->keys.size(); ++j) {
            tabs.push_back(r->tables[j]);
            kp.push_back(r->keys[j].data());
            kl.push_back(r->keys[j].size());
          }
        // Claim the slot, then plan and launch with the mutex released.  The
        // requests' keys and tables stay valid: a request is released only by
        // its waiter after it is done, and destroy first joins this thread.
        s->slot_reqs[i] = take;
        s->slot_cost[i] = cost;
        lk.unlock();
        int rc = mg_batch_set_keys(s->slots[i], tabs.data(), kp.data(), kl.data(), (uint32_t)kp.size());
        if (rc == MG_OK) rc = mg_batch_launch(s->slots[i], nullptr);
        std::string err = rc == MG_OK ? std::string() : std::string(mg_last_error());
        lk.lock();
        if (rc != MG_OK) {
          if (rc == MG_ENOMEM && in_flight(s) > 1) {
            // Memory is held by other passes: put the requests back in order.
            for (auto it = take.rbegin(); it != take.rend(); ++it) s->pending.push_front(*it);
            s->slot_reqs[i].clear();
            break;
          }
          finish_slot(s, i, rc, err.c_str(), {});
          s->cv_done.notify_all();
          continue;
        }
        s->slot_start[i] = Clock::now();
      }
    }
    // 3. Sleep until new work or (briefly) to poll the GPU.
    if (in_flight(s) > 0)
      s->cv_work.wait_for(lk, std::chrono::microseconds(100));
    else if (!s->stop)
      s->cv_work.wait(lk, [&] { return s->stop || (!s->paused && !s->pending.empty()); });
  }
}

double pct(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q / 100.0 * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" {

int mg_server_create(mg_context* ctx, const mg_server_config* cfg, mg_server** out) {
  if (!ctx || !out) {
    mg::set_last_error("null argument");
    return MG_EINVAL;
  }
  *out = nullptr;
  mg_server* s = new mg_server();
  s->ctx = ctx;
  s->cfg.slots = 2;
  s->cfg.max_keys_per_pass = 0;
  s->cfg.memory_reserve = 1ull << 30;
  if (cfg) {
    s->cfg = *cfg;
    if (s->cfg.slots == 0) s->cfg.slots = 2;
  }
  int sms = 0;
  mg_device_info(ctx, &sms, nullptr, nullptr);
  s->sms = sms;
  for (uint32_t i = 0; i < s->cfg.slots; ++i) {
    mg_batch* b = nullptr;
    if (int rc = mg_batch_create(ctx, &b)) {
      for (mg_batch* x : s->slots) mg_batch_destroy(x);
      delete s;
      return rc;
    }
    s->slots.push_back(b);
  }
  s->slot_reqs.resize(s->slots.size());
  s->slot_start.resize(s->slots.size());
  s->slot_cost.assign(s->slots.size(), 0.0);
  s->t0 = Clock::now();
  s->dispatcher = std::thread(run, s);
  *out = s;
  return MG_OK;
}

int mg_server_destroy(mg_server* s) {
  if (!s) return MG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->paused = false;
  }
  s->cv_work.notify_all();
  // The dispatcher completes the passes already on the GPU (their requests
  // are answered) and exits.
  if (s->dispatcher.joinable()) s->dispatcher.join();
  {
    std::unique_lock<std::mutex> lk(s->mu);
    for (Request* r : s->pending) {
      r->status = MG_EBUSY;
      r->error = "server destroyed before the request was dispatched";
      r->t_done = Clock::now();
      r->done = true;
    }
    s->pending.clear();
    // Threads blocked in mg_server_wait wake up, take their result (MG_EBUSY
    // for undispatched requests), release their request and leave; only
    // then is anything freed.
    s->closing = true;
    s->cv_done.notify_all();
    s->cv_done.wait(lk, [&] { return s->waiters == 0; });
    for (auto& kv : s->reqs) delete kv.second;
    s->reqs.clear();
  }
  for (mg_batch* b : s->slots) mg_batch_destroy(b);
  delete s;
  return MG_OK;
}

int mg_server_submit(mg_server* s, const mg_table* const* tables, const uint8_t* const* keys, const size_t* key_lens,
                     uint32_t nkeys, uint64_t* id) {
  if (!s || !tables || !keys || !key_lens || !id || nkeys == 0) {
    mg::set_last_error("null argument or no keys");
    return MG_EINVAL;
  }
  Request* r = new Request();
  for (uint32_t i = 0; i < nkeys; ++i) {
    uint32_t d = 0;
    if (!tables[i]) {
      delete r;
      mg::set_last_error("null table");
      return MG_EINVAL;
    }
    if (int rc = mg_key_check(keys[i], key_lens[i], &d, nullptr)) {
      delete r;
      return rc;
    }
    if (d < 64 && mg_table_first_row(tables[i]) + mg_table_rows(tables[i]) > (1ull << d)) {
      delete r;
      mg::set_last_error("more rows than domain size");
      return MG_ERANGE;
    }
    r->tables.push_back(tables[i]);
    r->keys.emplace_back(keys[i], keys[i] + key_lens[i]);
    r->share_bytes += mg_table_row_bytes(tables[i]);
    r->est_bytes += key_scratch_bytes(tables[i], s->sms);
    r->cost += (double)mg_table_rows(tables[i]);
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      mg::set_last_error("server is shutting down");
      return MG_EBUSY;
    }
    r->id = s->next_id++;
    s->reqs[r->id] = r;
    s->pending.push_back(r);
    *id = r->id;
  }
  s->cv_work.notify_all();
  return MG_OK;
}

int mg_server_wait(mg_server* s, uint64_t id, uint8_t* out, uint32_t timeout_ms, double* latency_ms) {
  if (!s) {
    mg::set_last_error("null server");
    return MG_EINVAL;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    mg::set_last_error("unknown request id");
    return MG_EINVAL;
  }
  Request* r = it->second;
  ++s->waiters;
  auto leave = [&](int status) {
    --s->waiters;
    if (s->closing) s->cv_done.notify_all();
    return status;
  };
  auto ready = [&] { return r->done; };
  if (timeout_ms == 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    mg::set_last_error("request not answered before the deadline");
    return leave(MG_ETIMEDOUT);
  }
  const int status = r->status;
  if (status == MG_OK) {
    if (out) std::memcpy(out, r->shares.data(), r->shares.size());
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  } else {
    mg::set_last_error(r->error.c_str());
  }
  s->reqs.erase(r->id);
  delete r;
  return leave(status);
}

int mg_server_pause(mg_server* s, uint32_t timeout_ms) {
  if (!s) {
    mg::set_last_error("null server");
    return MG_EINVAL;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  s->paused = true;
  auto drained = [&] { return in_flight(s) == 0; };
  s->cv_work.notify_all();
  if (timeout_ms == 0) {
    s->cv_done.wait(lk, drained);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), drained)) {
    mg::set_last_error("in-flight passes did not drain before the deadline");
    return MG_ETIMEDOUT;
  }
  return MG_OK;
}

int mg_server_resume(mg_server* s) {
  if (!s) {
    mg::set_last_error("null server");
    return MG_EINVAL;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->paused = false;
  }
  s->cv_work.notify_all();
  return MG_OK;
}

int mg_server_get_stats(mg_server* s, mg_server_stats* st) {
  if (!s || !st) {
    mg::set_last_error("null argument");
    return MG_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof *st);
  st->completed = s->completed;
  st->failed = s->failed;
  st->passes = s->passes;
  st->keys_completed = s->keys_done;
  st->pending = (uint32_t)s->pending.size();
  st->in_flight = in_flight(s);
  st->wall_s = std::chrono::duration<double>(Clock::now() - s->t0).count();
  st->p50_ms = pct(s->lat_ms, 50);
  st->p95_ms = pct(s->lat_ms, 95);
  st->p99_ms = pct(s->lat_ms, 99);
  double sum = 0, mx = 0;
  for (double v : s->lat_ms) {
    sum += v;
    mx = std::max(mx, v);
  }
  st->mean_ms = s->lat_ms.empty() ? 0 : sum / (double)s->lat_ms.size();
  st->max_ms = mx;
  return MG_OK;
}

int mg_server_reset_stats(mg_server* s) {
  if (!s) {
    mg::set_last_error("null server");
    return MG_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat_ms.clear();
  s->completed = s->failed = s->passes = s->keys_done = 0;
  s->t0 = Clock::now();
  return MG_OK;
}

}  // extern "C"
