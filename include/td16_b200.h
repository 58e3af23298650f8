/*
 * td16_b200.h -- C ABI of the B200 witness-search engine (libtd16b200.so).
 *
 * Drop-in for the td16 emitter's native boundary.  The reference binds two
 * JNI entry points of class br.unb.cic.tdp.base.GPUSortingSearch
 * (emitter/src/main/java/br/unb/cic/tdp/base/GPUSortingSearch.java:115-117):
 *   initSlots(int totalSlots, int[] devices, long queueBytesBudget)
 *   searchForSortingSeq(byte[] beta, byte[] omega, int initialEvenCycles,
 *                       float minRate, int maxMoves, boolean fullSorting, int slot)
 * td_init_slots and td_search replace them one for one; the batch, serving
 * and codec entry points are additions.  All buffers are plain host or device
 * pointers; no entry point takes or returns a C++ or framework type.
 */
#ifndef TD16_B200_H
#define TD16_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (return values of the entry points) ------------------ */
#define TD_OK 0            /* search ran and found a witness               */
#define TD_NOT_FOUND 1     /* search ran to exhaustion without a witness   */
#define TD_OVERFLOW 2      /* work budget exhausted before a verdict
                              (the reference's "GPU sorting search queue
                              overflow", sorting_search.cu:960-962)         */
#define TD_CUDA_ERROR 3    /* a CUDA call failed; message in err           */
#define TD_INVALID_ARG 4   /* rejected input; message in err               */
#define TD_TIMEOUT 5       /* deadline or abort request reached            */

/* ---- per-instance records ------------------------------------------------ */

/* One search in pinned form (16 bytes).  Build it with td_prepare_pairs or
 * td_prepare_perms; the layout is documented for callers that keep
 * instances resident on the device. */
typedef struct td_instance {
    uint64_t perm;      /* nibble m = L[m] (m < N-1); nibble m >= N-1 holds m */
    float min_rate;     /* minRate (f32), as passed by the reference's callers */
    uint8_t n_symbols;  /* N = length of beta, <= 17 */
    uint8_t offset;     /* pinned position of the caller's beta[0] */
    uint8_t max_moves;  /* 1..9 */
    uint8_t packed;     /* bits 0-4 initialEvenCycles, bit 7 fullSorting */
} td_instance;

/* One result (32 bytes).  moves[] are position triples into the caller's
 * evolving beta array packed as i | j<<5 | k<<10, the reference's PackedMove
 * (core/common.cuh:42-54). */
typedef struct td_result {
    int32_t status;       /* 1 found, 0 not found, <0 error (-2 budget, -4 argument, -5 timeout) */
    int32_t depth;        /* number of moves */
    uint16_t moves[9];
    uint16_t reserved;
    uint32_t expansions;  /* nodes whose children were evaluated */
} td_result;

/* batch flags */
#define TD_FLAG_ORDERED 1u     /* reference single-queue move order: witness
                                  identical to the reference run with one queue */
#define TD_FLAG_PLAIN 2u       /* one launch, one warp per instance, no work
                                  distribution (the baseline form) */
#define TD_FLAG_VERIFY 4u      /* replay every witness on the device after the
                                  search; a witness that fails the replay gets
                                  status -6 */

typedef struct td_batch_stats {
    uint64_t expansions;   /* total nodes expanded */
    uint64_t found;        /* instances with a witness */
    uint64_t not_found;    /* instances exhausted */
    uint64_t errors;       /* instances with status < 0 */
    float kernel_ms;       /* device time of the search launch(es) */
    uint32_t launches;     /* reserved */
    uint64_t donations;    /* free-order engine: donation events */
    uint64_t donated_items;/* free-order engine: subtrees handed between warps */
    uint64_t races;        /* free-order engine: searches raced against their
                              inverse (td_configure_race) */
} td_batch_stats;

/* ---- slots: the reference's JNI boundary --------------------------------- */

/* Replaces Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots
 * (emitter/src/native/jni/jni_sorter.cu:24-47 -> slot_manager.cu:44-128).
 * Slot s runs on devices[s % device_count], each with its own stream,
 * completion event and `queue_bytes_budget` bytes of device scratch.  Fails
 * with TD_INVALID_ARG on an empty, duplicate or out-of-range device list,
 * total_slots <= 0 or a zero budget, and when a device has less free memory
 * than budget x its slots.  Re-initialises: previous slots are destroyed. */
int td_init_slots(int total_slots, const int *devices, int device_count,
                  uint64_t queue_bytes_budget, char *err, size_t errlen);

/* Replaces Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq
 * (jni_sorter.cu:49-117 -> sorting_search.cu:811-972).  beta and omega hold
 * n unsigned bytes each (n <= 17), 1 <= max_moves <= 9.  Blocking; one caller
 * per slot at a time, different slots run concurrently.  On TD_OK writes
 * *out_depth position triples (i,j,k), i<j<k, to out_ijk[3*d..3*d+2]; on
 * TD_NOT_FOUND *out_depth = 0 (also for n < 3). */
int td_search(int slot, const uint8_t *beta, const uint8_t *omega, int n,
              int initial_even_cycles, float min_rate, int max_moves,
              int full_sorting, int16_t *out_ijk, int *out_depth, char *err,
              size_t errlen);

/* Same search with the reference's single-queue move order (its
 * performGpuSortingSearch with maxWarps = 1, sorting_search.cu:842): the
 * witness is the one that order finds first. */
int td_search_ordered(int slot, const uint8_t *beta, const uint8_t *omega, int n,
                      int initial_even_cycles, float min_rate, int max_moves,
                      int full_sorting, int16_t *out_ijk, int *out_depth,
                      char *err, size_t errlen);

/* How td_search and td_search_ordered run (no counterpart in the reference,
 * which launches per call).  mode 1 (default): through one resident serving
 * launch per device; the calling thread writes its request into pinned,
 * device-mapped memory and polls for the result, so a search costs no CUDA
 * API call.  The launch holds half of each SM's block slots while per-call
 * searches run; batch entry points stop it first when none is in flight, and
 * it exits by itself once it has had no request for idle_exit_s and has no
 * work left (default 0.005 s), so a device-wide synchronisation elsewhere
 * (cudaDeviceSynchronize, cudaFree) waits for it at most that long after the
 * last per-call search.  mode 0: one launch per call on the slot's stream.
 * rotate_after_s > 0 sets the age at which a busy server launch is replaced
 * by a fresh one (default 300; every wait of a launch is bounded by its
 * deadline).  A value of 0 keeps that setting. */
int td_configure_percall(int mode, double rotate_after_s, double idle_exit_s);

int td_slot_count(void);
int td_slot_device(int slot);           /* -1 for an invalid slot */
void *td_slot_stream(int slot);         /* cudaStream_t of the slot */
int td_destroy(void);                   /* releases every slot */

/* Launch shape of the engine (the autotuner's knobs): warps per block and
 * instances per ticket of the ordered persistent kernel. */
int td_configure(int warps_per_block, int grain);
/* Deadline of every later launch in seconds (default TD16_TIME_LIMIT_S or
 * 300): searches and device waits that pass it end with a timeout status. */
int td_set_time_limit(double seconds);
/* Work donation of the free-order engine: items per donation, deepest level
 * whose children may be donated, expansions between idle checks (default
 * 4, 2, 64: the best setting for one blocking search per call; the
 * autotuner's tuned.json holds the batch settings). */
int td_configure_steal(int grain, int split_level, int check_every);
/* The same for later serving launches (td_serve_open), kept apart because a
 * serving launch trades throughput for latency (default 1, 2, 32). */
int td_configure_serve(int grain, int split_level, int check_every);
/* Free order only: each warp keeps a table of the states it explored in its
 * current search and skips a child already explored with at least its depth
 * budget.  2^bits entries of 8 bytes per resident warp (6..16; default 12),
 * or 0 for none.  Verdicts do not depend on it. */
int td_configure_table(int bits);
/* Free-order batch searches restart with another child order after
 * base x 1, 1, 2, 1, 1, 2, 4, ... expansions (the Luby sequence; after 32
 * attempts the search runs to the end, in the first attempt's order).
 * base >= 16 (default 16), or 0 for no restarts.  Verdicts do not depend on
 * it. */
int td_configure_restart(int base);
/* Free-order batch searches of full-sorting instances with restarts on and
 * no expansion budget: a search that starts restart attempt `attempt`
 * (1..32, the 32nd being the last, unbounded one) also queues the search of
 * its inverse permutation, which another warp runs alongside; the first
 * witness (turned into the instance's positions) or the first side searched
 * to the end decides.  A permutation and its inverse are equally far from
 * sorted, and a witness found there is kept only if it also keeps the
 * reference's move filter on the instance's side, so verdicts do not depend
 * on it.  Default 8; 0 turns the race off.  The per-call server
 * (td_search), whose warps mostly idle, races from the first restart whenever
 * the race is on.  No counterpart in the reference, whose search runs one
 * order to the end. */
int td_configure_race(int attempt);
/* Reference-order batches (TD_FLAG_ORDERED, no expansion budget) run every
 * walk on one warp for first_pass_expansions (default 64), then split each
 * walk left over into the subtrees of its root's children, searched at once
 * and joined in the walk's order: witness and expansion count are the
 * one-warp walk's.  records (default 2^20, at most 2^24; 34 bytes each per
 * slot) bounds the subtrees of one launch; a root whose children find no
 * room runs whole.  first_pass_expansions = 0: no split. */
int td_configure_split(int first_pass_expansions, int records);

/* ---- instance preparation (host, no GPU needed) -------------------------- */

/* count pairs, beta/omega with a stride of 17 bytes per instance.  Returns
 * TD_OK or TD_INVALID_ARG (index of the first bad instance in *bad). */
int td_prepare_pairs(int count, const uint8_t *beta, const uint8_t *omega,
                     const uint8_t *n, const int32_t *initial_even_cycles,
                     const float *min_rate, const int32_t *max_moves,
                     const uint8_t *full_sorting, td_instance *out, int *bad);

/* count permutations of S_n (int8, stride 16): the reference pair over n+1
 * symbols with beta = (0 1 ... n) and rho = (0, pi0+1, ..., pi_{n-1}+1);
 * initialEvenCycles is computed. */
int td_prepare_perms(int count, const int8_t *perms, const uint8_t *n,
                     const int32_t *max_moves, float min_rate, int full_sorting,
                     td_instance *out, int *bad);

/* Seeded synthetic permutations: instance i uses splitmix64 seeded with
 * seed ^ i; n uniform in [n_min, n_max]; with probability hard_pct/100 the
 * reverse permutation composed with hard_min..hard_max uniform block
 * transpositions, else Fisher-Yates uniform.  perms int8 stride 16. */
int td_synth_perms(uint64_t seed, int count, int n_min, int n_max, int hard_pct,
                   int hard_min, int hard_max, int8_t *perms, uint8_t *n);

/* ---- batch search -------------------------------------------------------- */

/* Host buffers in and out; copies, launches and waits on the slot's stream.
 * max_expansions (all batch forms): 0 = no budget; otherwise a search that
 * expands more nodes without finding a witness ends with status -2 (budget).
 * In the free order the budget bounds each unit of work, i.e. the root search
 * and each subtree donated to another warp.  stats may be NULL; its totals are
 * reduced on the device. */
int td_search_batch(int slot, int count, const td_instance *instances,
                    td_result *results, unsigned flags,
                    uint64_t max_expansions, td_batch_stats *stats, char *err,
                    size_t errlen);

/* Many reference pairs per call: the batch form of td_search, for a case
 * producer that hands pairs over in groups instead of one blocking call per
 * pair (the enumerator's Consumer<CyclicTargetPair>,
 * DirectTwistedBraceletGenerator.java:105-156, calls searchForSortingSeq once
 * per pair through GPUSortingSearch.java:134-162).  Pair i: beta/omega at
 * stride 17 bytes, n[i] <= 17 symbols, init[i], min_rate[i], max_moves[i],
 * full[i].  flags: 0 or TD_FLAG_ORDERED.  Per pair: status[i] is TD_OK
 * (found; depth[i] position triples at out_ijk[27 i + 3 d ..]),
 * TD_NOT_FOUND (also for n < 3), or the per-call error class
 * (TD_INVALID_ARG, TD_OVERFLOW, TD_TIMEOUT).  Returns TD_OK when the batch
 * ran, else the error of the whole call (invalid slot, CUDA error). */
int td_search_pairs(int slot, int count, const uint8_t *beta, const uint8_t *omega,
                    const uint8_t *n, const int32_t *init, const float *min_rate,
                    const int32_t *max_moves, const uint8_t *full, unsigned flags,
                    int32_t *status, int32_t *depth, int16_t *out_ijk, char *err,
                    size_t errlen);

/* ---- pair consumer: the enumerator's Consumer<CyclicTargetPair> --------- */

/* A thread-safe consumer that many producer threads feed one pair at a time
 * (DirectTwistedBraceletGenerator.java:105-156 calls its consumer from every
 * generator thread) and that searches the pairs in batches: one worker thread
 * per slot (slots first_slot .. first_slot + slots - 1) takes a full batch
 * and searches it with one call of `search` (td_search_pairs when NULL; any
 * function of its signature, e.g. a test double).  A batch is handed over when
 * it holds batch_size pairs, when its oldest pair has waited max_delay_s and a
 * worker is idle (while all are busy it keeps filling), at td_batcher_flush,
 * or at close.  td_batcher_accept blocks while max_pending
 * full batches wait for a worker (0 = 2 x slots), as the reference's bounded
 * queue of slots + tdp.gpuQueueCapacity jobs does (GPUSortingSearch.java:46-52).
 * Results: found witnesses go to cert_writer (a td_cert_writer_open handle, or
 * NULL), and done (or NULL) receives every searched batch on a worker thread:
 * the tags given to accept, and per pair the status, depth and position
 * triples td_search_pairs returns.  Batches complete in any order.  Producer
 * threads spread over 16 filling batches with a lock each, so a batch holds
 * pairs of the threads sharing its shard, in their order of arrival. */
typedef void (*td_batcher_done_fn)(void *user, int count, const uint64_t *tags,
                                   const int32_t *status, const int32_t *depth,
                                   const int16_t *out_ijk);

typedef int (*td_batcher_search_fn)(int slot, int count, const uint8_t *beta,
                                    const uint8_t *omega, const uint8_t *n,
                                    const int32_t *init, const float *min_rate,
                                    const int32_t *max_moves, const uint8_t *full,
                                    unsigned flags, int32_t *status, int32_t *depth,
                                    int16_t *out_ijk, char *err, size_t errlen);

typedef struct td_batcher_stats {
    uint64_t pairs, batches, found, not_found, errors, certificates;
    double search_s;  /* summed over workers: time inside td_search_pairs */
} td_batcher_stats;

int td_batcher_open(int first_slot, int slots, int batch_size, double max_delay_s,
                    int max_pending, unsigned flags, td_batcher_search_fn search,
                    void *cert_writer, td_batcher_done_fn done, void *user,
                    void **handle, char *err, size_t errlen);
/* Copies the pair (n <= 17 bytes each of beta and omega); TD_INVALID_ARG for
 * a null handle or pointer or n > 17.  Per-pair errors (bad max_moves, ...)
 * come back as that pair's status. */
int td_batcher_accept(void *handle, uint64_t tag, const uint8_t *beta,
                      const uint8_t *omega, int n, int initial_even_cycles,
                      float min_rate, int max_moves, int full_sorting);
int td_batcher_flush(void *handle);
/* Hands over the filling batches, waits for every batch to be searched and
 * delivered, and frees the consumer.  Call it once every td_batcher_accept
 * has returned (the producers have stopped).  Returns TD_OK, or the first
 * error of a whole batch call (its message in err). */
int td_batcher_close(void *handle, td_batcher_stats *stats, char *err,
                     size_t errlen);

/* Device buffers; enqueues on `stream` (a cudaStream_t, or NULL for the
 * slot's stream) and returns without waiting. */
int td_search_batch_device(int slot, int count, const td_instance *d_instances,
                           td_result *d_results, unsigned flags,
                           uint64_t max_expansions, void *stream, char *err,
                           size_t errlen);

/* Batch search that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc/cudaFree: a slot worker
 * that must not stall on the device-wide synchronisation those calls can
 * imply while other searches run, or a process whose device memory is held by
 * another allocator.  The caller passes device buffers for instances and
 * results; all scratch is a fixed 3.25 MiB static device array per GPU, kept
 * until the process exits.  Runs on the calling thread's current device and
 * enqueues on `stream`.  At most 65536 instances per call (more returns
 * TD_INVALID_ARG).  The first call on a device does a one-time set-up (table
 * uploads and an address query), so make it before any stream capture.  Calls
 * share the scratch: launches that overlap on the GPU race, so serialise them. */
int td_search_batch_noalloc(int count, const td_instance *d_instances,
                            td_result *d_results, unsigned flags,
                            uint64_t max_expansions, void *stream, char *err,
                            size_t errlen);

/* CUDA-graph form of a batch over fixed device buffers: capture once, replay
 * with one graph launch per batch (scratch epochs advance on the device). */
int td_batch_graph_create(int slot, int count, const td_instance *d_instances,
                          td_result *d_results, unsigned flags,
                          uint64_t max_expansions, void **graph, char *err,
                          size_t errlen);
int td_batch_graph_launch(void *graph, void *stream, char *err, size_t errlen);
int td_batch_graph_destroy(void *graph);

/* Replays witnesses on the device with the reference checker's rules
 * (CertificateValidator.java:14-50): d_ok[i] = 1 when results[i] is a found
 * witness that sorts instance i within its max_moves, 0 otherwise. */
int td_validate_batch_device(int count, const td_instance *d_instances,
                             const td_result *d_results, uint8_t *d_ok,
                             void *stream, char *err, size_t errlen);

/* Measures the device's integer issue peaks in warp instructions per second,
 * the denominators of the search kernel's roofline: *issue_per_s with LOP3
 * and IMAD interleaved (ALU and FMA pipes, the full issue rate) and
 * *alu_per_s with LOP3 alone (the ALU pipe), each from independent chains at
 * full occupancy over about target_ms. */
int td_int_issue_peak(int device, float target_ms, double *issue_per_s,
                      double *alu_per_s, char *err, size_t errlen);

/* ---- serving: continuous batching ---------------------------------------- */

/* Starts a resident serving launch on `device`: requests published with
 * td_serve_submit join the running launch as they arrive; each is searched
 * by one warp with its DFS frames resident in shared memory.  The launch
 * ends at td_serve_close (after draining) or after time_limit_s. */
int td_serve_open(int device, unsigned ring_size, unsigned flags,
                  double time_limit_s, void **handle, char *err, size_t errlen);
int td_serve_workers(void *handle);
/* TD_OVERFLOW while ring_size requests are unfinished */
/* Publishes one request; *ticket numbers it.  Returns TD_OVERFLOW while the
 * request's ring slot (ticket mod ring_size) still holds the result of the
 * request ring_size tickets earlier that has not been taken by td_serve_poll. */
int td_serve_submit(void *handle, const td_instance *instance,
                    unsigned long long *ticket);
/* 1 (result copied; the slot may then be reused) when done, else 0 */
int td_serve_poll(void *handle, unsigned long long ticket, td_result *out);
int td_serve_close(void *handle, char *err, size_t errlen);

typedef struct td_serve_stats {
    double p50_ms, p99_ms, p999_ms, mean_ms, max_ms;
    double offered_per_s, served_per_s, wall_s;
    double admission_wait_ms_mean;
    uint64_t served, found;
    int workers, max_inflight;
} td_serve_stats;

/* Open-loop Poisson experiment over `instances` at `rate` requests/s:
 * admission when in-flight frame bytes (max_moves x frame) fit pool_bytes
 * and a worker is free; latency from arrival to result on the host. */
int td_serve_open_loop(int device, const td_instance *instances, int count,
                       double rate, uint64_t seed, uint64_t pool_bytes,
                       unsigned flags, td_result *results, td_serve_stats *stats,
                       char *err, size_t errlen);

/* Open-loop Poisson stream of `count` requests at `rate` per second through
 * the per-call server (no counterpart in the reference): `clients` host
 * threads each wait for their requests' arrival times, submit them as
 * td_search does and poll only their own tickets, so the latency (arrival to
 * result in the client) includes any wait for a free client.  Admission is by
 * client count.  Results land in results[i]. */
int td_percall_open_loop(int device, const td_instance *instances, int count, double rate,
                         uint64_t seed, int clients, td_result *results, td_serve_stats *stats,
                         char *err, size_t errlen);

/* ---- certificates (emitter/src/main/java/br/unb/cic/tdp/base/CertificateCodec.java) */

/* key = omega one-line, 5 bits per symbol, MSB first (CertificateCodec.java:22-36);
 * returns the byte length or -1 */
int td_codec_key(const uint8_t *omega, int n, uint8_t *out, int cap);
/* value = 15-bit (a,b,c) fields (CertificateCodec.java:56-72) */
int td_codec_value(const uint8_t *abc, int count, uint8_t *out, int cap);
/* decoders reject wrong lengths and nonzero padding (CertificateCodec.java:38-50,75-129) */
int td_codec_decode_key(const uint8_t *in, int len, int n, uint8_t *omega);
int td_codec_decode_value(const uint8_t *in, int len, uint8_t *abc, int cap_moves);

/* Replays symbol witnesses on the device with CertificateValidator's rules
 * (CertificateValidator.java:14-50).  Device pointers: beta/omega stride 17,
 * n, max_moves, depth one byte each, abc stride 27. */
int td_replay_symbols_device(int count, const uint8_t *d_beta, const uint8_t *d_omega,
                             const uint8_t *d_n, const uint8_t *d_max_moves,
                             const uint8_t *d_depth, const uint8_t *d_abc,
                             uint8_t *d_ok, void *stream, char *err, size_t errlen);

/* Batched certificate sink with AsyncCertificateWriter's queue-and-flush
 * behaviour (AsyncCertificateWriter.java:50-116), writing flat records
 * [key_len][value_len][key][value] (RocksDB is not linked into this library). */
void *td_cert_writer_open(const char *path, double flush_seconds);
int td_cert_writer_enqueue(void *writer, const uint8_t *omega, int n,
                           const uint8_t *abc, int count);
long long td_cert_writer_close(void *writer);

/* Queues the found witnesses of a batch (caller pairs, stride 17) as
 * certificates; returns the number queued. */
long long td_cert_writer_enqueue_batch(void *writer, int count, const uint8_t *beta,
                                       const uint8_t *omega, const uint8_t *n,
                                       const td_result *results);
/* Reads a certificate file for n-symbol domains: omega (stride 17), symbol
 * triples (stride 27), move counts.  Returns the record count or -1. */
long long td_cert_read_file(const char *path, int n, long long cap, uint8_t *omega,
                            uint8_t *abc, uint8_t *depth);
/* Caller pairs of S_n permutations: beta = (0..n), omega (stride 17). */
void td_pairs_from_perms(int count, const int8_t *perms, const uint8_t *n,
                         uint8_t *beta, uint8_t *omega);

/* Position triples -> symbol triples on a copy of beta
 * (GPUSortingSearch.java:229-238). */
void td_positions_to_symbols(const uint8_t *beta, int n, const int16_t *ijk,
                             int depth, uint8_t *out_abc);

#ifdef __cplusplus
}
#endif
#endif
