// td_slot_threads.cc -- drives a blocking search entry point from native host
// threads, one thread per slot, the way the emitter's Java slot workers call
// searchForSortingSeq (GPUSortingSearch.java:134-147: one worker thread per
// slot, each taking the next queued case and blocking in the native call);
// and feeds a pair consumer from native producer threads, the way the
// enumerator's generator threads call theirs (td_producer_threads_run).
//
// Built as libtd16_slot_threads.so.  It links nothing: the search entry point
// is passed as a function pointer, so the same driver runs this engine's
// td_search / td_search_ordered (include/td16_b200.h) and any other entry of
// the same shape.  Python threads would serialise such calls on the
// interpreter lock; these do not.
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

// td_search's signature
typedef int (*slot_search_fn)(int slot, const uint8_t *beta, const uint8_t *omega, int n, int init, float rate,
                              int maxd, int full, int16_t *out, int *depth, char *err, size_t errlen);
// the reference driver's signature (slot and maxWarps after the search inputs)
typedef int (*ref_search_fn)(const uint8_t *beta, const uint8_t *omega, int n, int init, float rate, int maxd,
                             int full, int slot, int max_warps, int16_t *out, int *depth, char *err, size_t errlen);

}  // namespace

// Runs `count` searches from `threads` threads; thread t uses slot
// first_slot + t and takes the next instance until none is left.  Instance i:
// beta/omega at stride 17 bytes, n[i] symbols, init[i], rate[i], maxd[i],
// full[i].  kind 0: `fn` has td_search's signature (status 0 found, 1 not
// found); kind 1: the reference driver's (status 0 with a depth; no depth is
// not found).  Outputs: status[i] = 1 found, 0 not found, -1 error (the
// engine's return code in code[i] when code is given); depth[i] and
// moves[27 i ..] the witness; latency_s[i] the call's wall time (each may be
// null).  Returns the wall time of the whole run in seconds.
extern "C" __attribute__((visibility("default"))) double td_slot_threads_run(
    int kind, void *fn, int count, const uint8_t *beta, const uint8_t *omega, const int32_t *n,
    const int32_t *init, const float *rate, const int32_t *maxd, const uint8_t *full, int threads, int first_slot,
    int32_t *status, int32_t *code, int32_t *depth, int16_t *moves, double *latency_s) {
    std::atomic<int> next{0};
    auto worker = [&](int slot) {
        int16_t out[27];
        char err[256];
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= count) return;
            int d = 0, rc;
            const auto t0 = std::chrono::steady_clock::now();
            if (kind == 0)
                rc = reinterpret_cast<slot_search_fn>(fn)(slot, beta + 17 * (size_t)i, omega + 17 * (size_t)i, n[i],
                                                          init[i], rate[i], maxd[i], full[i], out, &d, err,
                                                          sizeof err);
            else
                rc = reinterpret_cast<ref_search_fn>(fn)(beta + 17 * (size_t)i, omega + 17 * (size_t)i, n[i],
                                                         init[i], rate[i], maxd[i], full[i], slot, -1, out, &d,
                                                         err, sizeof err);
            const auto t1 = std::chrono::steady_clock::now();
            int st;
            if (kind == 0) st = rc == 0 ? 1 : rc == 1 ? 0 : -1;
            else st = rc == 0 ? (d > 0 ? 1 : 0) : -1;
            if (st != 1) d = 0;
            status[i] = st;
            if (code) code[i] = rc;
            if (depth) depth[i] = d;
            if (moves)
                for (int q = 0; q < 27; ++q) moves[27 * (size_t)i + q] = q < 3 * d ? out[q] : 0;
            if (latency_s) latency_s[i] = std::chrono::duration<double>(t1 - t0).count();
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(worker, first_slot + t);
    for (auto &t : th) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

namespace {

// td_batcher_accept's signature
typedef int (*pair_accept_fn)(void *handle, uint64_t tag, const uint8_t *beta, const uint8_t *omega, int n,
                              int init, float rate, int maxd, int full);

}  // namespace

// Feeds `count` pairs to a pair consumer from `threads` native producer
// threads, the way the enumerator's generator threads call their consumer
// (DirectTwistedBraceletGenerator.java:105-156): thread t hands over pairs t,
// t + threads, ... one call each, with the pair's index as its tag.  `fn` has
// td_batcher_accept's signature.  *first_rc receives the first non-zero
// return code (0 when every call succeeded).  Returns the producers' wall
// time in seconds.
extern "C" __attribute__((visibility("default"))) double td_producer_threads_run(
    void *fn, void *handle, int threads, int count, const uint8_t *beta, const uint8_t *omega, const int32_t *n,
    const int32_t *init, const float *rate, const int32_t *maxd, const uint8_t *full, int32_t *first_rc) {
    std::atomic<int> rc_seen{0};
    auto producer = [&](int t) {
        for (int i = t; i < count; i += threads) {
            const int rc = reinterpret_cast<pair_accept_fn>(fn)(handle, (uint64_t)i, beta + 17 * (size_t)i,
                                                                omega + 17 * (size_t)i, n[i], init[i], rate[i],
                                                                maxd[i], full[i]);
            if (rc != 0) {
                int expect = 0;
                rc_seen.compare_exchange_strong(expect, rc);
                return;
            }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(producer, t);
    for (auto &t : th) t.join();
    if (first_rc) *first_rc = rc_seen.load();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
