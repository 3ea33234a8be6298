// Evaluation-key cache (ntt_b200_keycache_*, include/ntt_b200.h).
//
// The reference proposes, but does not implement, an evaluation-key cache with
// a byte budget, pins and eviction of eligible entries
// (include/ntt/backend_api.hpp:51-79, include/ntt/backend_contract.hpp:322-430:
// CacheStats{budget, allocated, pinned}, set_cache_budget evicts eligible
// entries first and rejects a lower budget that pins prevent, trim_cache frees
// every eligible entry). This is that cache for the B200 path:
//  - insert() copies a full-context switching key (digits x (M+K) towers per
//    channel) into pinned host memory owned by the cache;
//  - acquire() makes the key resident in HBM (a stream-ordered allocation and
//    upload on the caller's stream), evicting least-recently-used eligible
//    keys to stay within the budget, pins it and returns its device pointers;
//  - a key acquired on another stream than the one that uploaded it makes that
//    stream wait for the upload (an event recorded after the copy), so no
//    caller reads a key whose upload is still in flight;
//  - release() unpins it in stream order: every release records its own event
//    on the caller's stream, and the key becomes eligible for eviction only
//    once all of them have completed, so work already enqueued on any stream
//    never loses its key;
//  - eviction frees device memory stream-ordered on the cache's own stream,
//    after the host has seen every release event of the key complete (the
//    callers' streams may be gone by then).
// A key is identified by a caller-chosen 64-bit id (the reference's
// EvaluationKeyCacheKey material token plus kind and index).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <list>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ntt_b200.h"

namespace {
thread_local std::string g_cache_error;

int fail(int code, const std::string &why) {
  g_cache_error = why;
  return code;
}
int cuda_fail(cudaError_t e, const char *call) {
  return fail(NTT_B200_ERR_CUDA, std::string("CUDA: ") + call + ": " + cudaGetErrorString(e));
}

struct Entry {
  ntt_b200_context ctx = nullptr;
  size_t words = 0;             // per channel
  uint64_t *host = nullptr;     // pinned: [b | a]
  uint64_t *dev = nullptr;      // resident copy [b | a], or null
  int pins = 0;
  cudaEvent_t uploaded = nullptr;       // recorded after the upload of the resident copy
  cudaStream_t upload_stream = nullptr;  // the stream that upload was enqueued on
  std::vector<cudaEvent_t> releases;     // release points not yet seen complete, one per release
  std::list<uint64_t>::iterator lru;  // position in the resident LRU list
};
}  // namespace

struct ntt_b200_keycache_s {
  int device = 0;
  cudaStream_t free_stream = nullptr;  // stream-ordered frees of evicted keys
  size_t budget = 0, allocated = 0;
  uint64_t hits = 0, misses = 0, evictions = 0;
  std::mutex mu;
  std::unordered_map<uint64_t, Entry> entries;
  std::list<uint64_t> lru;  // resident keys, most recently used at the front

  std::vector<cudaEvent_t> spare;  // completed release events, reused by later releases

  size_t bytes(const Entry &e) const { return 2 * e.words * sizeof(uint64_t); }

  // Drops the release events of `e` that have completed (back to the spare
  // pool); true when none is left pending.
  bool settled(Entry &e) {
    auto pending = e.releases.begin();
    for (cudaEvent_t ev : e.releases) {
      if (cudaEventQuery(ev) == cudaSuccess)
        spare.push_back(ev);
      else
        *pending++ = ev;
    }
    e.releases.erase(pending, e.releases.end());
    return e.releases.empty();
  }

  // Resident, unpinned, and every stream that released it has passed its
  // release point: no enqueued work reads it any more.
  bool eligible(Entry &e) {
    if (!e.dev || e.pins > 0) return false;
    // A release on another stream than the upload's does not order after it.
    if (e.uploaded && cudaEventQuery(e.uploaded) != cudaSuccess) return false;
    return settled(e);
  }

  cudaError_t take_event(cudaEvent_t *ev) {
    if (!spare.empty()) {
      *ev = spare.back();
      spare.pop_back();
      return cudaSuccess;
    }
    return cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  }

  // Evict one entry (lock held; the entry is eligible).
  int evict(uint64_t id, Entry &e) {
    const cudaError_t err = cudaFreeAsync(e.dev, free_stream);
    if (err != cudaSuccess) return cuda_fail(err, "cudaFreeAsync");
    e.dev = nullptr;
    allocated -= bytes(e);
    lru.erase(e.lru);
    evictions += 1;
    (void)id;
    return NTT_B200_OK;
  }

  // Evict least-recently-used eligible entries until `need` more bytes fit
  // under `limit` (lock held).
  int make_room(size_t need, size_t limit) {
    // Snapshot the resident ids, least recently used first: evict() erases list
    // nodes, so the list itself is not walked while evicting.
    const std::vector<uint64_t> order(lru.rbegin(), lru.rend());
    for (uint64_t id : order) {
      if (allocated + need <= limit) break;
      Entry &e = entries.at(id);
      if (!eligible(e)) continue;
      const int rc = evict(id, e);
      if (rc != NTT_B200_OK) return rc;
    }
    return allocated + need <= limit ? NTT_B200_OK
                                     : fail(NTT_B200_ERR_WORKSPACE,
                                            "key cache budget exhausted by pinned or in-use keys");
  }

  size_t pinned_bytes() {
    size_t p = 0;
    for (auto &kv : entries)
      if (kv.second.dev && (kv.second.pins > 0 || !eligible(kv.second))) p += bytes(kv.second);
    return p;
  }
};

extern "C" {

const char *ntt_b200_keycache_last_error(void) { return g_cache_error.c_str(); }

int ntt_b200_keycache_create(ntt_b200_keycache *out, int device, size_t budget_bytes) {
  if (!out || device < 0) return fail(NTT_B200_ERR_CONTRACT, "invalid key cache request");
  int previous = 0;
  cudaGetDevice(&previous);
  cudaError_t err = cudaSetDevice(device);
  cudaStream_t fs = nullptr;
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking);
  cudaSetDevice(previous);
  if (err != cudaSuccess) return cuda_fail(err, "key cache stream");
  auto *c = new ntt_b200_keycache_s();
  c->device = device;
  c->budget = budget_bytes;
  c->free_stream = fs;
  *out = c;
  return NTT_B200_OK;
}

int ntt_b200_keycache_insert(ntt_b200_keycache c, ntt_b200_context ctx, uint64_t key_id, const uint64_t *host_b,
                             const uint64_t *host_a) {
  if (!c || !ctx || !host_b || !host_a) return fail(NTT_B200_ERR_CONTRACT, "null argument");
  size_t words = 0;
  if (ntt_b200_context_key_words(ctx, &words) != NTT_B200_OK) return fail(NTT_B200_ERR_CONTRACT, ntt_b200_last_error());
  std::lock_guard<std::mutex> lock(c->mu);
  if (c->entries.count(key_id)) return fail(NTT_B200_ERR_CONTRACT, "key id already in the cache");
  Entry e;
  e.ctx = ctx;
  e.words = words;
  cudaError_t err = cudaMallocHost(&e.host, 2 * words * sizeof(uint64_t));
  if (err != cudaSuccess) return cuda_fail(err, "cudaMallocHost");
  std::memcpy(e.host, host_b, words * sizeof(uint64_t));
  std::memcpy(e.host + words, host_a, words * sizeof(uint64_t));
  c->entries.emplace(key_id, e);
  return NTT_B200_OK;
}

int ntt_b200_keycache_acquire(ntt_b200_keycache c, uint64_t key_id, void *stream, const uint64_t **key_b,
                              const uint64_t **key_a) {
  if (!c || !key_b || !key_a) return fail(NTT_B200_ERR_CONTRACT, "null argument");
  std::lock_guard<std::mutex> lock(c->mu);
  auto it = c->entries.find(key_id);
  if (it == c->entries.end()) return fail(NTT_B200_ERR_CONTRACT, "unknown key id");
  Entry &e = it->second;
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int previous = 0;
  cudaGetDevice(&previous);
  if (previous != c->device) cudaSetDevice(c->device);
  int rc = NTT_B200_OK;
  if (e.dev) {
    c->hits += 1;
    c->lru.erase(e.lru);
    // The upload may still be in flight on the stream that made the key
    // resident: a caller on another stream waits for it.
    if (e.uploaded && st != e.upload_stream) {
      const cudaError_t err = cudaStreamWaitEvent(st, e.uploaded, 0);
      if (err != cudaSuccess) rc = cuda_fail(err, "cudaStreamWaitEvent");
    }
  } else {
    c->misses += 1;
    const size_t need = c->bytes(e);
    rc = need > c->budget ? fail(NTT_B200_ERR_WORKSPACE, "key larger than the key cache budget")
                          : c->make_room(need, c->budget);
    if (rc == NTT_B200_OK) {
      void *dev = nullptr;
      cudaError_t err = cudaSuccess;
      if (!e.uploaded) err = cudaEventCreateWithFlags(&e.uploaded, cudaEventDisableTiming);
      if (err == cudaSuccess) err = cudaMallocAsync(&dev, need, st);
      if (err == cudaSuccess) err = cudaMemcpyAsync(dev, e.host, need, cudaMemcpyHostToDevice, st);
      if (err == cudaSuccess) err = cudaEventRecord(e.uploaded, st);
      if (err != cudaSuccess) {
        if (dev) cudaFreeAsync(dev, st);
        rc = cuda_fail(err, "key upload");
      } else {
        e.dev = static_cast<uint64_t *>(dev);
        e.upload_stream = st;
        c->allocated += need;
      }
    }
  }
  if (rc == NTT_B200_OK) {
    c->lru.push_front(key_id);
    e.lru = c->lru.begin();
    e.pins += 1;
    *key_b = e.dev;
    *key_a = e.dev + e.words;
  }
  if (previous != c->device) cudaSetDevice(previous);
  return rc;
}

int ntt_b200_keycache_release(ntt_b200_keycache c, uint64_t key_id, void *stream) {
  if (!c) return fail(NTT_B200_ERR_CONTRACT, "null key cache");
  std::lock_guard<std::mutex> lock(c->mu);
  auto it = c->entries.find(key_id);
  if (it == c->entries.end() || it->second.pins <= 0) return fail(NTT_B200_ERR_CONTRACT, "key is not acquired");
  Entry &e = it->second;
  int previous = 0;
  cudaGetDevice(&previous);
  if (previous != c->device) cudaSetDevice(c->device);
  // One event per release: releases on different streams are all waited for
  // before the key can be evicted and its memory freed.
  cudaEvent_t ev = nullptr;
  cudaError_t err = c->take_event(&ev);
  if (err == cudaSuccess) err = cudaEventRecord(ev, reinterpret_cast<cudaStream_t>(stream));
  if (previous != c->device) cudaSetDevice(previous);
  if (err != cudaSuccess) {
    if (ev) c->spare.push_back(ev);
    return cuda_fail(err, "cudaEventRecord");
  }
  e.releases.push_back(ev);
  e.pins -= 1;
  return NTT_B200_OK;
}

int ntt_b200_keycache_contains(ntt_b200_keycache c, uint64_t key_id, ntt_b200_context *ctx) {
  if (!c) return fail(NTT_B200_ERR_CONTRACT, "null key cache");
  std::lock_guard<std::mutex> lock(c->mu);
  auto it = c->entries.find(key_id);
  if (it == c->entries.end()) return fail(NTT_B200_ERR_CONTRACT, "unknown key id");
  if (ctx) *ctx = it->second.ctx;
  return NTT_B200_OK;
}

int ntt_b200_keycache_stats(ntt_b200_keycache c, ntt_b200_keycache_report *out) {
  if (!c || !out) return fail(NTT_B200_ERR_CONTRACT, "null argument");
  std::lock_guard<std::mutex> lock(c->mu);
  std::memset(out, 0, sizeof(*out));
  out->budget_bytes = c->budget;
  out->allocated_bytes = c->allocated;
  out->pinned_bytes = c->pinned_bytes();
  out->keys = c->entries.size();
  out->resident = c->lru.size();
  out->hits = c->hits;
  out->misses = c->misses;
  out->evictions = c->evictions;
  return NTT_B200_OK;
}

int ntt_b200_keycache_set_budget(ntt_b200_keycache c, size_t bytes) {
  if (!c) return fail(NTT_B200_ERR_CONTRACT, "null key cache");
  std::lock_guard<std::mutex> lock(c->mu);
  const int rc = c->make_room(0, bytes);
  if (rc != NTT_B200_OK) return fail(NTT_B200_ERR_CONTRACT, "pinned keys exceed the requested budget");
  c->budget = bytes;
  return NTT_B200_OK;
}

int ntt_b200_keycache_trim(ntt_b200_keycache c, size_t *freed) {
  if (!c) return fail(NTT_B200_ERR_CONTRACT, "null key cache");
  std::lock_guard<std::mutex> lock(c->mu);
  const size_t before = c->allocated;
  const std::vector<uint64_t> order(c->lru.begin(), c->lru.end());
  for (uint64_t id : order) {
    Entry &e = c->entries.at(id);
    if (c->eligible(e)) {
      const int rc = c->evict(id, e);
      if (rc != NTT_B200_OK) return rc;
    }
  }
  if (freed) *freed = before - c->allocated;
  return NTT_B200_OK;
}

int ntt_b200_keycache_destroy(ntt_b200_keycache c) {
  if (!c) return NTT_B200_OK;
  {
    std::lock_guard<std::mutex> lock(c->mu);
    for (auto &kv : c->entries)
      if (kv.second.pins > 0) return fail(NTT_B200_ERR_CONTRACT, "key cache destroyed with acquired keys");
    cudaSetDevice(c->device);
    for (auto &kv : c->entries) {
      Entry &e = kv.second;
      for (cudaEvent_t ev : e.releases) {
        cudaEventSynchronize(ev);
        cudaEventDestroy(ev);
      }
      if (e.uploaded) {
        cudaEventSynchronize(e.uploaded);
        cudaEventDestroy(e.uploaded);
      }
      if (e.dev) cudaFree(e.dev);
      cudaFreeHost(e.host);
    }
    for (cudaEvent_t ev : c->spare) cudaEventDestroy(ev);
    cudaStreamSynchronize(c->free_stream);
    cudaStreamDestroy(c->free_stream);
  }
  delete c;
  return NTT_B200_OK;
}

}  // extern "C"
