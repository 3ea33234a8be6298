/*
 * ntt_b200.h - C ABI of the B200 (sm_100a) CKKS NTT / ModUp / ModDown / Hybrid
 * key-switch path.
 *
 * The reference (minnow54426/ntt-gpu) reaches its CUDA path through the C++
 * transport seam ntt::resident::detail::Driver (include/ntt/resident_driver.hpp:13-57)
 * created by make_cuda_session (include/ntt/resident.hpp:142-143). Each entry
 * point below replaces one Driver primitive or one Session composite; the
 * replaced interface is named in the comment. The C++ Driver in
 * ntt_gpu_b200/host maps these status codes onto the reference's exceptions.
 *
 * Conventions
 *  - Towers are addressed by global id: Q tower i -> i, P tower j -> M + j.
 *  - Polynomials are limb-major u64 arrays: tower t occupies words [t*N, t*N+N).
 *    Coefficient form is natural order; evaluation form is the bit-reversed
 *    order of the reference (evaluation at psi^(2j+1), include/ntt/ntt.hpp:5-35).
 *  - All residues are canonical u64 in [0, q). Inputs must be canonical.
 *  - Pointers named dst/src/... are device pointers on the context's device.
 *    `stream` is a cudaStream_t (NULL = legacy default stream). Work is only
 *    enqueued; callers synchronise on the stream.
 *  - Every call validates its arguments on the host and returns a contract
 *    error BEFORE anything is enqueued (reference: ContractError thrown before
 *    enqueue, include/ntt/backend_contract.hpp:20-26). The host-array
 *    transforms check the arrays' contents while copying them in and compute
 *    nothing before every word has passed (see ntt_b200_host_transform).
 *  - Scratch: composite operations take a caller-provided device workspace whose
 *    size ntt_b200_workspace_bytes reports; they never allocate.
 */
#ifndef NTT_B200_H
#define NTT_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define NTT_B200_OK 0
#define NTT_B200_ERR_CONTRACT 1    /* invalid argument / layout (reference ContractError) */
#define NTT_B200_ERR_CUDA 2        /* CUDA runtime failure ("CUDA: <call>: <msg>") */
#define NTT_B200_ERR_UNSUPPORTED 3 /* valid input outside this build's capability */
#define NTT_B200_ERR_WORKSPACE 4   /* workspace missing or too small */
#define NTT_B200_ERR_TIMEOUT 5     /* a bounded device wait expired */
#define NTT_B200_NOT_READY 6       /* event query: recorded work has not completed yet */

typedef struct ntt_b200_context_s *ntt_b200_context;

/* Message of the last failing call on this host thread. */
const char *ntt_b200_last_error(void);
/* Number of this library's kernels launched by this process so far. */
uint64_t ntt_b200_kernel_launches(void);

/* Build a context: validates parameters as proposal::Parameters::create does
 * (include/ntt/backend_contract.hpp:48-66), builds twiddle, conversion and
 * correction tables and keeps them resident in HBM. Replaces the table setup
 * of the reference's CUDA Context (src/cuda/resident_adapter.inc:60-103) and
 * make_cuda_session (src/cuda/resident_adapter.inc:306-317). k may be 0 for a
 * transform-only context; alpha is the full-context digit width
 * (OpenFHE GetNumPerPartQ). */
int ntt_b200_context_create(ntt_b200_context *out, int device, uint64_t n,
                            const uint64_t *q, const uint64_t *q_psi, size_t m,
                            const uint64_t *p, const uint64_t *p_psi, size_t k,
                            size_t alpha);
int ntt_b200_context_destroy(ntt_b200_context ctx);
/* Bytes of device tables the context holds (Driver::constant_bytes,
 * include/ntt/resident_driver.hpp:28). */
int ntt_b200_context_table_bytes(ntt_b200_context ctx, size_t *out);
/* Build every conversion/correction plan a key switch at `level` needs, so that
 * later calls at that level perform no host work or table upload. */
int ntt_b200_context_prepare(ntt_b200_context ctx, size_t level);
/* Nonzero `count` when a kernel of this context gave up a bounded wait on the
 * GPU (its results are then invalid); a synchronous read, `clear` resets it. */
int ntt_b200_device_errors(ntt_b200_context ctx, int *count, int clear);
/* Words of one channel of a full-context switching key: digits x (M + K) x N
 * (the packing of Session::upload_hybrid_key's source, src/resident.cpp:492-529). */
int ntt_b200_context_key_words(ntt_b200_context ctx, size_t *words);

/* Forward (inverse = 0) or inverse NTT of `polys` polynomials. Slot i of poly p
 * is read at src + p*poly_stride + i*N and written at dst + p*poly_stride + i*N
 * (dst may equal src) with the tables of tower_ids[i]. Replaces
 * Driver::transform (include/ntt/resident_driver.hpp:34; src/cuda/ntt_kernels.cu:286-326). */
int ntt_b200_ntt(ntt_b200_context ctx, uint64_t *dst, const uint64_t *src,
                 const uint32_t *tower_ids, size_t towers, size_t polys,
                 size_t poly_stride, int inverse, void *stream);

/* dst = left * right pointwise (evaluation form). Replaces Driver::pointwise
 * (include/ntt/resident_driver.hpp:35-36). */
int ntt_b200_pointwise(ntt_b200_context ctx, uint64_t *dst, const uint64_t *left,
                       const uint64_t *right, const uint32_t *tower_ids, size_t towers,
                       size_t polys, size_t poly_stride, void *stream);

/* Coefficient-domain approximate CRT switch (unreduced lift) from the source
 * towers (contiguous at src) to the target towers (contiguous at dst).
 * Replaces Driver::switch_basis (include/ntt/resident_driver.hpp:45-47;
 * include/ntt/basis_conversion.hpp:13-30). Sources and targets: 1..40, disjoint. */
int ntt_b200_switch_basis(ntt_b200_context ctx, uint64_t *dst, const uint64_t *src,
                          const uint32_t *source_ids, size_t s, const uint32_t *target_ids,
                          size_t t, void *stream);

/* ModDown tail on the active Q towers: dst = (left - right) * [P^-1]_q.
 * Replaces Driver::correct (include/ntt/resident_driver.hpp:48-50;
 * include/ntt/resident_conversion.hpp:45-49). */
int ntt_b200_correct(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *left,
                     const uint64_t *right, void *stream);

/* Hybrid MAC over all active digits in one pass:
 *   out_b = sum_d digits[d] * key_b[d][row],  out_a likewise,
 * digits: beta x (L+K) towers (evaluation QP); keys: FULL-context digits of
 * (M+K) towers each, rows selected by key_indices (i for Q, M+j for P).
 * Replaces the per-digit Driver::hybrid_mac loop (include/ntt/resident_driver.hpp:37-40;
 * src/resident.cpp:530-570) and Session::upload_hybrid_key's row packing
 * (src/resident.cpp:492-529). */
int ntt_b200_hybrid_mac(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                        const uint64_t *digits, const uint64_t *key_b, const uint64_t *key_a,
                        void *stream);

/* out = automorphism(ext) with P*c0 added on the Q towers of the b channel.
 * automorphism must be odd and < 2N. Replaces Driver::hybrid_rotate
 * (include/ntt/resident_driver.hpp:41-44; src/resident.cpp:571-617). */
int ntt_b200_hybrid_rotate(ntt_b200_context ctx, size_t level, uint64_t *out_b,
                           uint64_t *out_a, const uint64_t *ext_b, const uint64_t *ext_a,
                           const uint64_t *c0, uint32_t automorphism, void *stream);

/* Workspace sizes (bytes) of the composite operations below. */
#define NTT_B200_OP_MOD_UP 1
#define NTT_B200_OP_MOD_DOWN 2
#define NTT_B200_OP_DIGITS 3
#define NTT_B200_OP_KEYSWITCH 4
int ntt_b200_workspace_bytes(ntt_b200_context ctx, int op, size_t level, size_t batch,
                             size_t *out);

/* ModUp: Q_L (coefficient if src_is_eval == 0, else evaluation) -> evaluation
 * QP. Replaces Session::mod_up (src/resident.cpp:431-447). */
int ntt_b200_mod_up(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                    int src_is_eval, void *workspace, size_t workspace_bytes, void *stream);

/* ModDown: evaluation QP -> evaluation Q_L. Replaces Session::mod_down
 * (src/resident.cpp:448-457). */
int ntt_b200_mod_down(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                      void *workspace, size_t workspace_bytes, void *stream);

/* Hybrid digits: evaluation Q_L -> beta evaluation-QP digits (beta x (L+K)
 * towers). Replaces Session::hybrid_digits (src/resident.cpp:458-491). */
int ntt_b200_hybrid_digits(ntt_b200_context ctx, size_t level, uint64_t *digits,
                           const uint64_t *src, void *workspace, size_t workspace_bytes,
                           void *stream);

/* Full Hybrid key switch of one evaluation-Q_L component `src`: digits, MAC
 * with the full-context key, optional rotation (c0 != NULL: P*c0 added and
 * the automorphism applied to the extended QP result), ModDown of both
 * channels. Outputs evaluation Q_L. Replaces run_hybrid_core
 * (include/ntt/openfhe_hybrid_adapter.hpp:163-181). */
int ntt_b200_keyswitch(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                       const uint64_t *src, const uint64_t *key_b, const uint64_t *key_a,
                       const uint64_t *c0, uint32_t automorphism, void *workspace,
                       size_t workspace_bytes, void *stream);

/* Batched key switch: `batch` evaluation-Q_L components src[batch][L][N] at one
 * level with one shared full-context key; outputs out_b/out_a[batch][L][N];
 * c0 (optional) is [batch][L][N] and every request rotates by the same
 * automorphism. Each launch of the pipeline covers the whole batch. The
 * reference has no batch API; per request this equals ntt_b200_keyswitch. */
int ntt_b200_keyswitch_batch(ntt_b200_context ctx, size_t level, size_t batch, uint64_t *out_b,
                             uint64_t *out_a, const uint64_t *src, const uint64_t *key_b,
                             const uint64_t *key_a, const uint64_t *c0, uint32_t automorphism,
                             void *workspace, size_t workspace_bytes, void *stream);

/* One key-switch request of a request list. All pointers are device pointers
 * on the context's device; every polynomial is evaluation form over the
 * request's active Q towers ([level][N]).
 *  - key switch (run_hybrid_core, include/ntt/openfhe_hybrid_adapter.hpp:163-181):
 *      (out_b, out_a) = KeySwitch(src) with the full-context key (key_b, key_a);
 *  - rotation (hybrid_rotate, openfhe_hybrid_adapter.hpp:286-305): c0 set, P*c0
 *      added and the automorphism applied to the extended QP result before ModDown;
 *  - relinearization (hybrid_relinearize_in_place, openfhe_hybrid_adapter.hpp:244-282):
 *      add_b / add_a (c0 / c1 of the ciphertext) are added to the outputs; they may
 *      equal out_b / out_a (in place).
 * Requests that share src at one level share one digit decomposition (the
 * hoisted hybrid_rotate_many, openfhe_hybrid_adapter.hpp:309-361). */
typedef struct ntt_b200_ks_request {
  const uint64_t *src;
  uint64_t *out_b;
  uint64_t *out_a;
  const uint64_t *key_b;
  const uint64_t *key_a;
  const uint64_t *c0;
  const uint64_t *add_b;
  const uint64_t *add_a;
  uint32_t automorphism;
  uint32_t level;
  /* Server only: with key_b == key_a == NULL, the key is taken from the
   * server's key cache under this id (ntt_b200_server_attach_keycache). */
  uint64_t key_id;
} ntt_b200_ks_request;

/* Workspace bytes of ntt_b200_keyswitch_requests for this request list. */
int ntt_b200_keyswitch_requests_workspace(ntt_b200_context ctx, const ntt_b200_ks_request *reqs,
                                          size_t count, size_t *bytes);
/* Key switch a list of requests of mixed levels, keys, rotations and
 * relinearization addends. Requests are grouped by level (shape class) and
 * each group of up to 128 runs as one pass of the fused pipeline; the level
 * groups run concurrently on up to four streams forked from `stream` and
 * joined back into it (each with its own part of the workspace); each result
 * equals the request run alone. Outputs must not overlap any other buffer of
 * the call (except a request's own addend at the same address). The reference
 * has no batch API: per request this equals its Session chain
 * (src/resident.cpp:458-617) and run_hybrid_core. */
int ntt_b200_keyswitch_requests(ntt_b200_context ctx, const ntt_b200_ks_request *reqs, size_t count,
                                void *workspace, size_t workspace_bytes, void *stream);

/* Evaluation-key cache. Keys live in pinned host memory owned by the cache
 * (copied at insert) and are made resident in HBM on demand within a byte
 * budget. acquire() uploads on the caller's stream if needed (stream-ordered),
 * evicting least-recently-used keys that are unpinned and whose last release
 * has completed on the GPU, pins the key and returns its device pointers;
 * release() unpins it in stream order (the key stays in place until the work
 * enqueued before the release has completed). set_budget() evicts eligible keys
 * first and refuses a budget that pinned keys prevent; trim() evicts every
 * eligible key. This is the evaluation-key cache the reference proposes but does
 * not implement (include/ntt/backend_api.hpp:51-79 CacheStats /
 * set_cache_budget / trim_cache; include/ntt/backend_contract.hpp:322-352
 * EvaluationKeyCacheKey, here a caller-chosen 64-bit id). */
typedef struct ntt_b200_keycache_s *ntt_b200_keycache;
typedef struct ntt_b200_keycache_report {
  size_t budget_bytes, allocated_bytes, pinned_bytes;
  uint64_t keys, resident, hits, misses, evictions;
} ntt_b200_keycache_report;
const char *ntt_b200_keycache_last_error(void);
int ntt_b200_keycache_create(ntt_b200_keycache *out, int device, size_t budget_bytes);
int ntt_b200_keycache_destroy(ntt_b200_keycache cache);
/* Host key_b / key_a: full-context digits of ntt_b200_context_key_words each. */
int ntt_b200_keycache_insert(ntt_b200_keycache cache, ntt_b200_context ctx, uint64_t key_id,
                             const uint64_t *host_b, const uint64_t *host_a);
int ntt_b200_keycache_contains(ntt_b200_keycache cache, uint64_t key_id, ntt_b200_context *ctx);
int ntt_b200_keycache_acquire(ntt_b200_keycache cache, uint64_t key_id, void *stream,
                              const uint64_t **key_b, const uint64_t **key_a);
int ntt_b200_keycache_release(ntt_b200_keycache cache, uint64_t key_id, void *stream);
int ntt_b200_keycache_stats(ntt_b200_keycache cache, ntt_b200_keycache_report *out);
int ntt_b200_keycache_set_budget(ntt_b200_keycache cache, size_t bytes);
int ntt_b200_keycache_trim(ntt_b200_keycache cache, size_t *freed);

/* Continuous-batching key-switch server. Requests (ntt_b200_ks_request: key
 * switch, relinearization or rotation) arrive from any host thread and refer to
 * device-resident ciphertexts and keys that the caller keeps alive until the
 * ticket completes. A scheduler thread forms waves of the oldest pending
 * request's (context, level) class, up to max_batch, and launches each on the
 * least-loaded lane (a CUDA stream with fewer than `depth` waves in flight),
 * while the waves in flight hold less than max_inflight_bytes of workspace,
 * once its workspace fits the lane's arena, grown within hbm_budget_bytes
 * (the sum of all lanes' arenas; idle lanes give theirs back when needed): requests arriving while others run join the next
 * wave as lanes and memory free up, and waves on different lanes overlap on
 * the device. Each result equals the request run alone. The reference has no
 * server (one request per Session transaction, src/resident.cpp); admission
 * follows its Limits/Reservation budget model (src/resident.cpp:10-28). */
typedef struct ntt_b200_server_s *ntt_b200_server;
typedef struct ntt_b200_server_config {
  int device;
  int lanes;      /* CUDA streams that run waves concurrently, 1..16 */
  int max_batch;  /* requests per wave, 1..1024 */
  int depth;      /* waves in flight per lane, 1..8 (0 = 1); >1 queues the next wave behind the running one */
  size_t hbm_budget_bytes; /* sum of the lanes' workspace arenas */
  /* 0 = no limit. Otherwise a new wave launches only while the waves in flight
   * hold less than this much workspace: small waves (low levels, small N) then
   * run many at a time, up to lanes x depth, while large ones run a few at a
   * time and the requests behind them gather into fuller waves. */
  size_t max_inflight_bytes;
} ntt_b200_server_config;
typedef struct ntt_b200_ticket_info {
  int status;          /* NTT_B200_OK or the request's error */
  uint32_t wave_size;  /* requests in the wave that carried it */
  int lane;
  int reserved;
  double queue_us;     /* submission -> wave launch */
  double latency_us;   /* submission -> GPU completion of its wave */
} ntt_b200_ticket_info;
typedef struct ntt_b200_server_report {
  uint64_t completed, waves;
  double mean_wave, p50_ms, p99_ms, max_ms;
  double throughput;   /* completed / (last completion - first submission), per second */
  double mean_queue_ms; /* submission -> wave launch, mean */
  size_t peak_bytes, in_flight_bytes; /* workspace arenas held by the lanes: peak and now */
} ntt_b200_server_report;
const char *ntt_b200_server_last_error(void);
int ntt_b200_server_create(ntt_b200_server *out, const ntt_b200_server_config *cfg);
/* Validates the request alone (contract errors return here, before queueing). */
int ntt_b200_server_submit(ntt_b200_server srv, ntt_b200_context ctx, const ntt_b200_ks_request *req,
                           uint64_t *ticket);
/* Waits up to timeout_ms: NTT_B200_OK (ticket released), NTT_B200_ERR_TIMEOUT,
 * or the request's error. */
int ntt_b200_server_wait(ntt_b200_server srv, uint64_t ticket, uint32_t timeout_ms,
                         ntt_b200_ticket_info *info);
/* Waits until nothing is pending or in flight. */
int ntt_b200_server_drain(ntt_b200_server srv, uint32_t timeout_ms);
/* Latency percentiles and throughput of completed requests; reset != 0 clears them. */
int ntt_b200_server_stats(ntt_b200_server srv, ntt_b200_server_report *out, int reset);
/* Finishes pending and in-flight work, then frees the server. */
int ntt_b200_server_destroy(ntt_b200_server srv);
/* Grows every lane's workspace arena that has no wave in flight to at least
 * bytes_per_lane, in stream order on the lane's stream, so that waves up to that
 * size never wait for an arena to grow. A contract error if the arenas would
 * exceed hbm_budget_bytes. (No counterpart in the reference, which has no
 * server; its Limits reserve memory per Session, src/resident.cpp:10-28.) */
int ntt_b200_server_reserve(ntt_b200_server srv, size_t bytes_per_lane);
/* Requests submitted with key_b == key_a == NULL take their key from `cache`
 * by key_id: each wave acquires its keys on its lane's stream at launch and
 * releases them in stream order after it. A wave whose keys do not fit the
 * cache's budget next to the keys of the waves in flight waits for them. The
 * cache must outlive the server. */
int ntt_b200_server_attach_keycache(ntt_b200_server srv, ntt_b200_keycache cache);

/* Host-buffer key switch with overlapped copies. `batch` components at one
 * level from host memory h_src[batch][L][N] into host h_out_b / h_out_a, keys
 * (and the workspace) on the device, optional host h_c0 for rotation. The batch
 * runs in chunks of `chunk` requests through two device staging slots: the copy
 * to the device of one chunk, the key switch of the previous one and the copy
 * back of the one before run concurrently on two internal copy streams and the
 * caller's stream, so the copies in both directions overlap each other and the
 * kernels. The call is stream-ordered: it starts after the work already on
 * `stream`, and work enqueued after it sees every output on the host. Host
 * buffers should be pinned (cudaHostAlloc) for the copies to overlap. Calls on
 * one context serialise their use of its copy streams. This is the
 * host-vector form of the reference's CudaNttTransform / synchronous Session
 * entry points (include/ntt/cuda_ntt.hpp:34-79) for the key switch, which the
 * reference runs as pageable copies around each call. */
int ntt_b200_keyswitch_host_workspace(ntt_b200_context ctx, size_t level, size_t chunk, int rotate,
                                      size_t *bytes);
int ntt_b200_keyswitch_host(ntt_b200_context ctx, size_t level, size_t batch, size_t chunk,
                            const uint64_t *h_src, uint64_t *h_out_b, uint64_t *h_out_a,
                            const uint64_t *key_b, const uint64_t *key_a, const uint64_t *h_c0,
                            uint32_t automorphism, void *workspace, size_t workspace_bytes, void *stream);
/* The same key switch without the final wait: `stream` does not wait for the
 * copies of the outputs to the host, so the next host-buffer call on this
 * context (same workspace) starts copying and switching while this call's last
 * outputs are still leaving, and back-to-back calls keep both copy directions
 * busy. The two staging slots stay ordered across calls. The outputs of every
 * call so far are on the host once ntt_b200_keyswitch_host_wait has made a
 * stream wait for them and that stream has reached that point. */
int ntt_b200_keyswitch_host_async(ntt_b200_context ctx, size_t level, size_t batch, size_t chunk,
                                  const uint64_t *h_src, uint64_t *h_out_b, uint64_t *h_out_a,
                                  const uint64_t *key_b, const uint64_t *key_a, const uint64_t *h_c0,
                                  uint32_t automorphism, void *workspace, size_t workspace_bytes, void *stream);
int ntt_b200_keyswitch_host_wait(ntt_b200_context ctx, void *stream);

/* MAC with per-digit device pointers (count digits of L+K towers each):
 * full_key_rows != 0 -> key pointers are full-context digits (rows chosen by
 * key_indices); 0 -> keys are already packed active QP rows. accumulate != 0
 * adds into out_b/out_a instead of overwriting them. With count = 1 this is
 * the reference's per-digit Driver::hybrid_mac (first_digit = !accumulate;
 * src/cuda/resident_adapter.inc:31-43, 214-231). */
int ntt_b200_hybrid_mac_digits(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                               const uint64_t *const *digits, const uint64_t *const *key_b,
                               const uint64_t *const *key_a, size_t count, int full_key_rows,
                               int accumulate, void *stream);

/* Transport: streams, stream-ordered device memory, copies and events. These
 * replace the reference CUDA Driver's Context stream, Buffer (one cudaMalloc
 * per buffer) and Event plumbing (src/cuda/resident_adapter.inc:60-302).
 * Device memory comes from the device's stream-ordered pool (kept cached).
 * memcpy kind: 1 host->device, 2 device->host, 3 device->device (async). */
int ntt_b200_stream_create(int device, void **stream);
int ntt_b200_stream_destroy(void *stream);
int ntt_b200_stream_synchronize(void *stream);
int ntt_b200_alloc(int device, size_t bytes, void *stream, void **ptr);
int ntt_b200_free(void *ptr, void *stream);
int ntt_b200_memcpy(void *dst, const void *src, size_t bytes, int kind, void *stream);
int ntt_b200_event_create(int device, void **event);
int ntt_b200_event_destroy(void *event);
int ntt_b200_event_record(void *event, void *stream);
/* NTT_B200_OK when the recorded work completed, NTT_B200_NOT_READY otherwise. */
int ntt_b200_event_query(void *event);
int ntt_b200_event_synchronize(void *event);

/* Launch tuning: named choices that never change a result (which NTT pass
 * variant and register budget, which conversion kernel, conversion grid size).
 * ntt_gpu_b200/autotune.py measures them on the device and writes
 * ntt_gpu_b200/tuning.json; the Python loader applies it at load time. Values
 * out of a tunable's range are refused. tuning_name(i) lists the names (NULL
 * past the end). The reference has no tuning interface. */
int ntt_b200_tuning_set(const char *name, int64_t value);
int ntt_b200_tuning_get(const char *name, int64_t *value);
const char *ntt_b200_tuning_name(size_t index);

/* Allocation-free ModDown. For callers that must not allocate device memory:
 * hosts whose HBM is already owned by another caching allocator (a framework
 * process that has reserved the device), latency-critical request threads that
 * cannot afford cudaMalloc's implicit device synchronisation, and FFI hosts
 * that have no way to own or release device buffers across the boundary.
 * Same result as ntt_b200_mod_down, but the scratch is a file-scope device
 * array of ntt_b200_mod_down_static_max_bytes() (8 MiB), which every GPU that
 * loads this library holds until exit; (K + L) * N * 8 bytes must fit in it,
 * larger requests are refused with a contract error. The caller still passes
 * the input and output. The level's tables must exist already
 * (ntt_b200_context_prepare); this call allocates nothing. Its first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and keeps
 * it for the life of the process, so make that first call before any stream
 * capture; the address belongs to the device's primary context, so the entry
 * point must not be used after cudaDeviceReset on that device. All calls share the one array and
 * it keeps the previous call's contents (nothing in it needs to start at zero):
 * calls that overlap on the GPU - on different streams, or on one device from
 * different contexts - race on it. This entry point has no counterpart in the
 * reference. */
size_t ntt_b200_mod_down_static_max_bytes(void);
int ntt_b200_mod_down_static(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                             void *stream);

/* Host-buffer transforms: the reference's CudaNttTransform public calls
 * forward / inverse / pointwise_multiply / multiply (include/ntt/cuda_ntt.hpp:59-66;
 * src/cuda/ntt_kernels.cu:423-488). `values` (and `right`) are limb-major HOST
 * arrays of `towers` towers of N words, tower i using the tables of global tower
 * tower_ids[i]:
 *   FORWARD / INVERSE: values transformed in place (natural coefficients <->
 *     bit-reversed evaluations, as ntt_b200_ntt);
 *   POINTWISE: values *= right (both evaluation form);
 *   MULTIPLY: values = the ring product of values and right mod x^N + 1
 *     (coefficient form in and out).
 * Every residue is checked against its tower's modulus on the host before any
 * result is computed or written (the reference's validate_values; a contract
 * error otherwise): the calling thread checks the towers in chunks and each
 * checked chunk is copied to the device while the next one is checked; the
 * transforms and the copies back to the host run once every residue has
 * passed. On a failed check the call waits for the copies it has started and
 * returns the contract error with `values` unchanged. The call is synchronous,
 * like the reference's: it returns once the results are back in host memory.
 * `workspace` holds every tower of the call, once per operand:
 * ntt_b200_host_transform_workspace reports that size for the context's own
 * towers (a call that repeats tower ids needs more). Host memory should be
 * pinned for the copies to overlap the checks; pageable memory works. */
#define NTT_B200_HOST_FORWARD 0
#define NTT_B200_HOST_INVERSE 1
#define NTT_B200_HOST_POINTWISE 2
#define NTT_B200_HOST_MULTIPLY 3
int ntt_b200_host_transform_workspace(ntt_b200_context ctx, int op, size_t *bytes);
int ntt_b200_host_transform(ntt_b200_context ctx, int op, uint64_t *values, const uint64_t *right,
                            const uint32_t *tower_ids, size_t towers, void *workspace,
                            size_t workspace_bytes, void *stream);

/* Device arithmetic probes: the reference's shoup_kernel / barrett_kernel
 * checks of its device arithmetic against host 128-bit arithmetic
 * (tests/basis_cuda.cu:49-65). `count` queries of 5 words each (device array),
 * one result word each (device array):
 *   op 0: (x, w, floor(w 2^64 / q), q, -)  -> x w mod q, Shoup, canonical
 *         (include/ntt/shoup.hpp:7-27);
 *   op 1: (a, b, q, mu_lo, mu_hi)          -> a b mod q, Barrett with
 *         mu = floor(2^128 / q), canonical (include/ntt/barrett.hpp:10-50);
 *   op 2: (x, w, floor(w 2^64 / q), q, -)  -> the NTT's approximate-quotient
 *         Shoup product, congruent to x w and in [0, 4q) for q < 2^61. */
int ntt_b200_arith_probe(int device, int op, const uint64_t *queries, size_t count, uint64_t *out,
                         void *stream);

/* Test hooks (no counterpart in the reference's public API; its tests reach
 * the same seams through private constructors):
 *  - conv_wait_polls: poll limit of the tensor-core conversion's first bounded
 *    wait (default and maximum 2^20). 0 makes that wait give up at once: the
 *    kernel then waits (bounded, at the full limit) for its own bulk copy,
 *    frees its tensor memory, returns, and reports the timeout through
 *    ntt_b200_device_errors (its outputs are then invalid). Nothing hangs.
 *  - inject_setup_failure: the next ntt_b200_context_create fails with a CUDA
 *    error before its `operation`-th device allocation or upload (1-based; 0
 *    turns it off) and releases everything it had set up, as the reference's
 *    SetupResources unwinds (include/ntt/setup_resources.hpp:19-60);
 *  - setup_operations: the allocations and uploads of the last successful
 *    ntt_b200_context_create. */
int ntt_b200_conv_wait_polls(int polls);
int ntt_b200_inject_setup_failure(size_t operation);
int ntt_b200_setup_operations(size_t *count);

/* Opt-in per-kernel timing: while enabled, every launch of this library is
 * bracketed by CUDA events on its own stream. query() waits for the recorded
 * events and returns the launch count and summed device time of one kernel
 * class ("ntt_fwd_col", "ntt_fwd_row", "ntt_fwd_cluster" (a one-pass forward
 * transform over a thread-block cluster), "ntt_inv_row", "ntt_inv_col",
 * "ntt_small", "conv", "mac", "row_mac" (the digits' forward row pass fused
 * with the key multiplication), "rotate", "correct", "pointwise", "table"). The external
 * clock protocol mirrors the reference's collect_elapsed
 * (include/ntt/measurement.hpp:41-58). */
int ntt_b200_timing_enable(int on);
int ntt_b200_timing_reset(void);
int ntt_b200_timing_query(const char *kernel, uint64_t *launches, double *total_ms);

/* Calibration, with no counterpart in the reference: the running device's
 * rate of the forward NTT's mode-2 butterflies (moduli below 2^61) with every
 * operand in registers and no memory traffic, i.e. the integer-multiply
 * ceiling the NTT passes are measured against. Runs about 10 ms of work on a
 * private stream of `device`, allocates 8 bytes of device memory for the
 * duration, and waits for the result. */
int ntt_b200_butterfly_rate(int device, double *butterflies_per_second);

#ifdef __cplusplus
}
#endif
#endif
