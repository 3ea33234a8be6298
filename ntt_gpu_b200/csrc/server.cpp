// Continuous-batching key-switch server (ntt_b200_server_*, include/ntt_b200.h).
//
// Requests (key switch, relinearization, rotation) arrive from any host thread
// and reference device-resident ciphertexts and keys. One scheduler thread
// forms waves and launches them through ntt_b200_keyswitch_requests:
//  - a wave is the oldest pending request's shape class (context, level) plus
//    every later pending request of that class, up to max_batch;
//  - a wave launches as soon as a lane (a CUDA stream) has fewer than `depth`
//    waves in flight, the waves in flight hold less workspace than
//    max_inflight_bytes (the measure of how much of the GPU they occupy), and
//    its workspace fits the HBM budget next to the waves already in flight, so requests that arrive while others run are admitted
//    as lanes and memory free up, and waves on different lanes overlap on the
//    device (a depth above 1 queues the next wave behind the running one);
//  - each lane owns a workspace arena that its waves reuse in stream order; an
//    arena only grows (stream-ordered free + allocation on its own stream), the
//    sum of all arenas stays within the HBM budget, and idle lanes give their
//    arenas back when a wave needs the room;
//  - an event recorded after each wave marks its completion; the scheduler
//    polls the events of waves in flight (every 20 us while any is in flight),
//    so latency runs from submission to the observed GPU completion, and no
//    host callback ever stalls a lane's stream.
// The reference serves one request per Session transaction (src/resident.cpp,
// include/ntt/openfhe_hybrid_adapter.hpp:163-181) and has no server; the
// admission budget follows its Limits/Reservation model (src/resident.cpp:10-28).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ntt_b200.h"

namespace {

double now_us() {
  using namespace std::chrono;
  return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

// Placeholder key address for the host-side checks (sizes, alignment, overlap)
// of requests that name their key by id: far below any device allocation and
// never dereferenced; the real pointers come from the key cache at launch.
const uint64_t *const kKeyPlaceholder = reinterpret_cast<const uint64_t *>(uintptr_t(256));

struct Ticket {
  ntt_b200_context ctx = nullptr;
  ntt_b200_ks_request req{};
  int status = NTT_B200_NOT_READY;
  std::string error;
  double t_submit = 0, t_launch = 0, t_done = 0;
  uint32_t wave_size = 0;
  int lane = -1;
};

// One launched wave and the event recorded after its work.
struct Wave {
  int lane = -1;
  std::vector<uint64_t> ids;
  size_t bytes = 0;
  cudaEvent_t done = nullptr;
};

struct Lane {
  cudaStream_t stream = nullptr;
  int inflight = 0;  // waves enqueued on this stream and not yet retired
  void *arena = nullptr;
  size_t arena_bytes = 0;
};

}  // namespace

struct ntt_b200_server_s {
  ntt_b200_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, Ticket> tickets;
  std::vector<Lane> lanes;
  std::vector<std::unique_ptr<Wave>> waves_in_flight;
  std::vector<cudaEvent_t> event_pool;
  ntt_b200_keycache keycache = nullptr;  // resolves requests submitted by key id
  int depth = 1;
  uint64_t next_id = 1;
  size_t in_use = 0, peak_in_use = 0;
  size_t work_in_flight = 0;  // workspace bytes of the waves in flight
  bool stopping = false;
  std::string fatal;  // first CUDA failure; the server refuses new work after it
  std::thread sched;
  // statistics since the last reset
  std::vector<double> latencies_us;
  uint64_t waves = 0, wave_requests = 0;
  double first_submit = 0, last_done = 0, queue_us = 0;

  cudaEvent_t take_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
  }

  // Retire waves whose completion event has fired (lock held).
  void retire() {
    for (auto it = waves_in_flight.begin(); it != waves_in_flight.end();) {
      Wave &w = **it;
      const cudaError_t q = cudaEventQuery(w.done);
      if (q == cudaErrorNotReady) {
        ++it;
        continue;
      }
      const double t_done = now_us();
      const bool ok = q == cudaSuccess;
      const std::string why = ok ? "" : std::string("CUDA: wave: ") + cudaGetErrorString(q);
      for (uint64_t id : w.ids) {
        auto t = tickets.find(id);
        if (t == tickets.end()) continue;
        if (!ok) {
          fail_ticket(id, NTT_B200_ERR_CUDA, why);
          continue;
        }
        t->second.status = NTT_B200_OK;
        t->second.t_done = t_done;
        latencies_us.push_back(t_done - t->second.t_submit);
        queue_us += t->second.t_launch - t->second.t_submit;
        last_done = std::max(last_done, t_done);
      }
      if (!ok && fatal.empty()) fatal = why;
      lanes[w.lane].inflight -= 1;
      work_in_flight -= w.bytes;
      event_pool.push_back(w.done);
      it = waves_in_flight.erase(it);
      cv_done.notify_all();
    }
  }

  void fail_ticket(uint64_t id, int status, const std::string &why) {
    auto it = tickets.find(id);
    if (it == tickets.end()) return;
    it->second.status = status;
    it->second.error = why;
    it->second.t_done = now_us();
    cv_done.notify_all();
  }

  void erase_pending(const std::vector<uint64_t> &ids) {
    for (uint64_t id : ids) {
      auto it = std::find(pending.begin(), pending.end(), id);
      if (it != pending.end()) pending.erase(it);
    }
  }

  bool any_busy() const { return !waves_in_flight.empty(); }

  // Form and launch at most one wave. Called with the lock held; the lock is
  // released around the CUDA calls (the completion callback takes it too).
  // Returns true if it made progress.
  bool launch_one(std::unique_lock<std::mutex> &lock) {
    if (pending.empty()) return false;
    if (!fatal.empty()) {
      for (uint64_t id : pending) fail_ticket(id, NTT_B200_ERR_CUDA, fatal);
      pending.clear();
      return false;
    }
    // The lane with the fewest waves in flight, below the depth; among those,
    // the one with the largest arena, so grown arenas are reused rather than
    // new ones grown (an arena's growth can wait on the driver for memory).
    int lane = -1;
    for (size_t i = 0; i < lanes.size(); ++i) {
      if (lanes[i].inflight >= depth) continue;
      if (lane < 0 || lanes[i].inflight < lanes[lane].inflight ||
          (lanes[i].inflight == lanes[lane].inflight && lanes[i].arena_bytes > lanes[lane].arena_bytes))
        lane = (int)i;
    }
    if (lane < 0) return false;
    // Enough work in flight to occupy the GPU: let the pending requests gather
    // into a fuller wave. Nothing in flight means no limit, so this never stalls.
    if (cfg.max_inflight_bytes && work_in_flight >= cfg.max_inflight_bytes) return false;
    const Ticket &head = tickets[pending.front()];
    const ntt_b200_context ctx = head.ctx;
    const uint32_t level = head.req.level;
    std::vector<uint64_t> wave;
    std::vector<ntt_b200_ks_request> reqs;
    for (uint64_t id : pending) {
      if ((int)wave.size() >= cfg.max_batch) break;
      const Ticket &t = tickets[id];
      if (t.ctx != ctx || t.req.level != level) continue;
      wave.push_back(id);
      reqs.push_back(t.req);
    }
    // Shrink the wave until it fits the lane's arena, grown within the budget
    // (idle lanes' arenas are released first when the room is needed).
    size_t need = 0;
    std::vector<int> release;  // idle lanes whose arenas this wave takes over
    while (true) {
      // Requests by key id carry no key pointers yet: size them with the
      // placeholder addresses used at submission.
      std::vector<ntt_b200_ks_request> sized(reqs);
      for (auto &r : sized)
        if (!r.key_b && !r.key_a) r.key_b = r.key_a = kKeyPlaceholder;
      if (ntt_b200_keyswitch_requests_workspace(ctx, sized.data(), sized.size(), &need) != NTT_B200_OK) {
        // Requests are validated at submission; a failure here fails the wave.
        const std::string why = ntt_b200_last_error();
        for (uint64_t id : wave) fail_ticket(id, NTT_B200_ERR_CONTRACT, why);
        erase_pending(wave);
        return true;
      }
      const size_t mine = lanes[lane].arena_bytes;
      if (need <= mine) break;
      size_t others = in_use - mine, idle = 0;
      release.clear();
      for (size_t i = 0; i < lanes.size(); ++i)
        if ((int)i != lane && lanes[i].inflight == 0 && lanes[i].arena_bytes) {
          idle += lanes[i].arena_bytes;
          release.push_back((int)i);
        }
      if (others + need <= cfg.hbm_budget_bytes) {
        release.clear();
        break;
      }
      if (others - idle + need <= cfg.hbm_budget_bytes) break;
      release.clear();
      if (reqs.size() == 1) {
        if (need > cfg.hbm_budget_bytes) {
          fail_ticket(wave[0], NTT_B200_ERR_WORKSPACE, "request workspace exceeds the server's HBM budget");
          erase_pending(wave);
          return true;
        }
        return false;  // wait for in-flight waves to free their lanes
      }
      const size_t keep = reqs.size() / 2;
      reqs.resize(keep);
      wave.resize(keep);
    }
    // Keys by id: acquire them on the lane's stream (uploading what is not
    // resident); they are released in stream order right after the wave.
    // A wave whose keys do not all fit the cache's budget is cut to the
    // requests whose keys were acquired; the rest stay pending.
    std::vector<uint64_t> acquired;
    if (keycache) {
      for (size_t i = 0; i < reqs.size(); ++i) {
        auto &r = reqs[i];
        if (r.key_b || r.key_a) continue;
        const uint64_t *kb = nullptr, *ka = nullptr;
        const int krc = ntt_b200_keycache_acquire(keycache, r.key_id, lanes[lane].stream, &kb, &ka);
        if (krc == NTT_B200_ERR_WORKSPACE && i > 0) {
          reqs.resize(i);
          wave.resize(i);
          break;
        }
        if (krc != NTT_B200_OK) {
          const std::string why = ntt_b200_keycache_last_error();
          for (uint64_t id : acquired) ntt_b200_keycache_release(keycache, id, lanes[lane].stream);
          if (krc == NTT_B200_ERR_WORKSPACE && any_busy()) return false;  // wait for in-flight keys
          fail_ticket(wave[0], krc, why);
          erase_pending({wave[0]});
          return true;
        }
        acquired.push_back(r.key_id);
        r.key_b = kb;
        r.key_a = ka;
      }
    }
    // Reserve the lane and the memory, then launch without the lock.
    erase_pending(wave);
    const double t_launch = now_us();
    for (uint64_t id : wave) {
      Ticket &tk = tickets[id];
      tk.t_launch = t_launch;
      tk.wave_size = (uint32_t)wave.size();
      tk.lane = lane;
    }
    auto owned = std::make_unique<Wave>();
    owned->lane = lane;
    owned->ids = wave;
    owned->bytes = need;  // the lane's arena holds the memory; counted as work in flight
    owned->done = take_event();
    cudaEvent_t done = owned->done;
    lanes[lane].inflight += 1;
    // Arena changes happen under the lock, in stream order on each lane's own
    // stream (frees and allocations are stream-ordered, never synchronous).
    cudaError_t e = done ? cudaSuccess : cudaErrorMemoryAllocation;
    for (int i : release) {
      if (e == cudaSuccess) e = cudaFreeAsync(lanes[i].arena, lanes[i].stream);
      in_use -= lanes[i].arena_bytes;
      lanes[i].arena = nullptr;
      lanes[i].arena_bytes = 0;
    }
    Lane &ln = lanes[lane];
    if (e == cudaSuccess && need > ln.arena_bytes) {
      if (ln.arena) e = cudaFreeAsync(ln.arena, ln.stream);
      in_use -= ln.arena_bytes;
      ln.arena = nullptr;
      ln.arena_bytes = 0;
      if (e == cudaSuccess) e = cudaMallocAsync(&ln.arena, need, ln.stream);
      if (e == cudaSuccess) {
        ln.arena_bytes = need;
        in_use += need;
      }
    }
    peak_in_use = std::max(peak_in_use, in_use);
    const cudaStream_t stream = ln.stream;
    void *ws = ln.arena;
    const size_t ws_bytes = ln.arena_bytes;
    lock.unlock();
    int rc = NTT_B200_OK;
    std::string why;
    if (e != cudaSuccess) {
      rc = NTT_B200_ERR_CUDA;
      why = std::string("CUDA: lane arena: ") + cudaGetErrorString(e);
      for (uint64_t id : acquired) ntt_b200_keycache_release(keycache, id, stream);
    } else {
      rc = ntt_b200_keyswitch_requests(ctx, reqs.data(), reqs.size(), ws, ws_bytes, stream);
      if (rc != NTT_B200_OK) why = ntt_b200_last_error();
      for (uint64_t id : acquired) ntt_b200_keycache_release(keycache, id, stream);
      if (rc == NTT_B200_OK) {
        e = cudaEventRecord(done, stream);
        if (e != cudaSuccess) {
          rc = NTT_B200_ERR_CUDA;
          why = std::string("CUDA: cudaEventRecord: ") + cudaGetErrorString(e);
        }
      }
    }
    lock.lock();
    if (rc != NTT_B200_OK) {
      lanes[lane].inflight -= 1;
      if (done) event_pool.push_back(done);
      for (uint64_t id : wave) fail_ticket(id, rc, why);
      if (rc == NTT_B200_ERR_CUDA && fatal.empty()) fatal = why;
      return true;
    }
    work_in_flight += owned->bytes;
    waves_in_flight.push_back(std::move(owned));
    waves += 1;
    wave_requests += wave.size();
    return true;
  }

  void run() {
    cudaSetDevice(cfg.device);
    std::unique_lock<std::mutex> lock(mu);
    while (true) {
      retire();
      while (launch_one(lock)) retire();
      if (stopping && pending.empty() && !any_busy()) break;
      if (any_busy())
        cv_sched.wait_for(lock, std::chrono::microseconds(20));  // poll the waves in flight
      else
        cv_sched.wait(lock);
    }
  }
};

namespace {
thread_local std::string g_server_error;

template <class F> int server_guard(F f) {
  try {
    return f();
  } catch (const std::exception &e) {
    g_server_error = e.what();
    return NTT_B200_ERR_CUDA;
  }
}

int contract(const char *why) {
  g_server_error = why;
  return NTT_B200_ERR_CONTRACT;
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  const size_t i = (size_t)std::min<double>((double)v.size() - 1, p * (double)(v.size() - 1) + 0.5);
  return v[i];
}
}  // namespace

extern "C" {

const char *ntt_b200_server_last_error(void) { return g_server_error.c_str(); }

int ntt_b200_server_create(ntt_b200_server *out, const ntt_b200_server_config *cfg) {
  return server_guard([&] {
    if (!out || !cfg) return contract("null argument");
    *out = nullptr;
    if (cfg->device < 0 || cfg->lanes < 1 || cfg->lanes > 16 || cfg->max_batch < 1 || cfg->max_batch > 1024 ||
        cfg->hbm_budget_bytes == 0)
      return contract("invalid server configuration (1..16 lanes, 1..1024 batch, nonzero budget)");
    if (cfg->depth < 0 || cfg->depth > 8) return contract("invalid server configuration (depth 0..8)");
    auto *s = new ntt_b200_server_s();
    s->cfg = *cfg;
    s->depth = cfg->depth ? cfg->depth : 1;
    cudaError_t e = cudaSetDevice(cfg->device);
    s->lanes.resize(cfg->lanes);
    for (int i = 0; i < cfg->lanes && e == cudaSuccess; ++i)
      e = cudaStreamCreateWithFlags(&s->lanes[i].stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      cudaMemPool_t pool;
      e = cudaDeviceGetDefaultMemPool(&pool, cfg->device);
      uint64_t keep = UINT64_MAX;  // keep freed workspace cached for the next wave
      if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
      for (Lane &l : s->lanes)
        if (l.stream) cudaStreamDestroy(l.stream);
      delete s;
      g_server_error = std::string("CUDA: server streams: ") + cudaGetErrorString(e);
      return NTT_B200_ERR_CUDA;
    }
    s->sched = std::thread([s] { s->run(); });
    *out = s;
    return NTT_B200_OK;
  });
}

int ntt_b200_server_submit(ntt_b200_server srv, ntt_b200_context ctx, const ntt_b200_ks_request *req,
                           uint64_t *ticket) {
  return server_guard([&] {
    if (!srv || !ctx || !req || !ticket) return contract("null argument");
    // Validate the request alone before it joins a wave: a bad request is
    // refused here and never fails the requests it would have been batched with.
    ntt_b200_ks_request check = *req;
    if (!req->key_b && !req->key_a) {
      ntt_b200_context owner = nullptr;
      ntt_b200_keycache cache = nullptr;
      {
        std::lock_guard<std::mutex> lock(srv->mu);
        cache = srv->keycache;
      }
      if (!cache) return contract("request without key pointers, and no key cache attached");
      if (ntt_b200_keycache_contains(cache, req->key_id, &owner) != NTT_B200_OK || owner != ctx)
        return contract("key id not in the attached key cache for this context");
      check.key_b = check.key_a = kKeyPlaceholder;
    }
    size_t need = 0;
    if (ntt_b200_keyswitch_requests_workspace(ctx, &check, 1, &need) != NTT_B200_OK) {
      g_server_error = ntt_b200_last_error();
      return NTT_B200_ERR_CONTRACT;
    }
    std::lock_guard<std::mutex> lock(srv->mu);
    if (srv->stopping) return contract("server is shutting down");
    if (!srv->fatal.empty()) {
      g_server_error = srv->fatal;
      return NTT_B200_ERR_CUDA;
    }
    if (need > srv->cfg.hbm_budget_bytes) {
      g_server_error = "request workspace exceeds the server's HBM budget";
      return NTT_B200_ERR_WORKSPACE;
    }
    const uint64_t id = srv->next_id++;
    Ticket t;
    t.ctx = ctx;
    t.req = *req;
    t.t_submit = now_us();
    if (srv->first_submit == 0) srv->first_submit = t.t_submit;
    srv->tickets.emplace(id, std::move(t));
    srv->pending.push_back(id);
    *ticket = id;
    srv->cv_sched.notify_all();
    return NTT_B200_OK;
  });
}

int ntt_b200_server_wait(ntt_b200_server srv, uint64_t ticket, uint32_t timeout_ms, ntt_b200_ticket_info *info) {
  return server_guard([&] {
    if (!srv) return contract("null server");
    std::unique_lock<std::mutex> lock(srv->mu);
    auto it = srv->tickets.find(ticket);
    if (it == srv->tickets.end()) return contract("unknown or already collected ticket");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    while (it->second.status == NTT_B200_NOT_READY) {
      const bool timed_out = srv->cv_done.wait_until(lock, deadline) == std::cv_status::timeout;
      it = srv->tickets.find(ticket);
      if (it == srv->tickets.end()) return contract("ticket collected by another waiter");
      if (timed_out && it->second.status == NTT_B200_NOT_READY) {
        g_server_error = "ticket not complete within the timeout";
        return NTT_B200_ERR_TIMEOUT;
      }
    }
    const Ticket &t = it->second;
    if (info) {
      info->status = t.status;
      info->wave_size = t.wave_size;
      info->lane = t.lane;
      info->queue_us = t.t_launch > 0 ? t.t_launch - t.t_submit : 0;
      info->latency_us = t.t_done - t.t_submit;
    }
    const int status = t.status;
    if (status != NTT_B200_OK) g_server_error = t.error;
    srv->tickets.erase(it);
    return status;
  });
}

int ntt_b200_server_drain(ntt_b200_server srv, uint32_t timeout_ms) {
  return server_guard([&] {
    if (!srv) return contract("null server");
    std::unique_lock<std::mutex> lock(srv->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    while (!srv->pending.empty() || srv->any_busy()) {
      if (srv->cv_done.wait_until(lock, deadline) == std::cv_status::timeout &&
          (!srv->pending.empty() || srv->any_busy())) {
        g_server_error = "server did not drain within the timeout";
        return NTT_B200_ERR_TIMEOUT;
      }
    }
    if (!srv->fatal.empty()) {
      g_server_error = srv->fatal;
      return NTT_B200_ERR_CUDA;
    }
    return NTT_B200_OK;
  });
}

int ntt_b200_server_stats(ntt_b200_server srv, ntt_b200_server_report *out, int reset) {
  return server_guard([&] {
    if (!srv || !out) return contract("null argument");
    std::lock_guard<std::mutex> lock(srv->mu);
    std::memset(out, 0, sizeof(*out));
    out->completed = srv->latencies_us.size();
    out->waves = srv->waves;
    out->mean_wave = srv->waves ? (double)srv->wave_requests / (double)srv->waves : 0;
    out->p50_ms = percentile(srv->latencies_us, 0.50) / 1000.0;
    out->p99_ms = percentile(srv->latencies_us, 0.99) / 1000.0;
    out->max_ms = srv->latencies_us.empty()
                      ? 0
                      : *std::max_element(srv->latencies_us.begin(), srv->latencies_us.end()) / 1000.0;
    const double span = srv->last_done - srv->first_submit;
    out->throughput = span > 0 ? (double)out->completed / (span / 1e6) : 0;
    out->mean_queue_ms = out->completed ? srv->queue_us / (double)out->completed / 1000.0 : 0;
    out->peak_bytes = srv->peak_in_use;
    out->in_flight_bytes = srv->in_use;
    if (reset) {
      srv->latencies_us.clear();
      srv->waves = srv->wave_requests = 0;
      srv->first_submit = srv->last_done = srv->queue_us = 0;
      srv->peak_in_use = srv->in_use;
    }
    return NTT_B200_OK;
  });
}

int ntt_b200_server_reserve(ntt_b200_server srv, size_t bytes_per_lane) {
  return server_guard([&] {
    if (!srv) return contract("null server");
    std::lock_guard<std::mutex> lock(srv->mu);
    // Lanes with waves in flight (or a launch being enqueued, which counts as in
    // flight) keep their arenas; the others grow to bytes_per_lane.
    size_t after = srv->in_use;
    for (const Lane &ln : srv->lanes)
      if (ln.inflight == 0 && ln.arena_bytes < bytes_per_lane) after += bytes_per_lane - ln.arena_bytes;
    if (after > srv->cfg.hbm_budget_bytes) return contract("reservation exceeds the server's HBM budget");
    for (Lane &ln : srv->lanes) {
      if (ln.inflight != 0 || ln.arena_bytes >= bytes_per_lane) continue;
      cudaError_t e = ln.arena ? cudaFreeAsync(ln.arena, ln.stream) : cudaSuccess;
      srv->in_use -= ln.arena_bytes;
      ln.arena = nullptr;
      ln.arena_bytes = 0;
      if (e == cudaSuccess) e = cudaMallocAsync(&ln.arena, bytes_per_lane, ln.stream);
      if (e != cudaSuccess) {
        ln.arena = nullptr;
        g_server_error = std::string("CUDA: lane arena: ") + cudaGetErrorString(e);
        return NTT_B200_ERR_CUDA;
      }
      ln.arena_bytes = bytes_per_lane;
      srv->in_use += bytes_per_lane;
    }
    srv->peak_in_use = std::max(srv->peak_in_use, srv->in_use);
    return NTT_B200_OK;
  });
}

int ntt_b200_server_attach_keycache(ntt_b200_server srv, ntt_b200_keycache cache) {
  return server_guard([&] {
    if (!srv) return contract("null server");
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->keycache = cache;
    return NTT_B200_OK;
  });
}

int ntt_b200_server_destroy(ntt_b200_server srv) {
  return server_guard([&] {
    if (!srv) return NTT_B200_OK;
    {
      std::lock_guard<std::mutex> lock(srv->mu);
      srv->stopping = true;
      srv->cv_sched.notify_all();
    }
    srv->sched.join();  // drains pending work first
    for (Lane &l : srv->lanes) {
      if (l.arena) cudaFreeAsync(l.arena, l.stream);
      cudaStreamSynchronize(l.stream);
      cudaStreamDestroy(l.stream);
    }
    for (cudaEvent_t e : srv->event_pool) cudaEventDestroy(e);
    delete srv;
    return NTT_B200_OK;
  });
}

}  // extern "C"
