// td_batcher.cc -- a native pair consumer: the enumerator's
// Consumer<CyclicTargetPair> in C++, searching pairs in batches.
//
// The reference's case enumerator hands every canonical pair to a thread-safe
// consumer from many generator threads
// (emitter/src/main/java/br/unb/cic/tdp/DirectTwistedBraceletGenerator.java:105-156),
// and that consumer makes one blocking searchForSortingSeq call per pair
// through the slot queue (GPUSortingSearch.java:134-162: `slots` worker
// threads draining a bounded queue of slots + tdp.gpuQueueCapacity jobs).
// This consumer keeps the queue model but moves batches instead of pairs:
//
//   accept      copies the pair into its thread's filling batch (16 of
//               them, each under its own lock, so that many producer threads
//               do not queue on one mutex; no allocation in the common case)
//               and returns; it blocks while
//               max_pending full batches wait for a worker, like the
//               reference's bounded queue;
//   delay       an idle worker takes the filling batch once its oldest pair
//               has waited max_delay_s, so a slow producer still sees results;
//               while every worker is busy the batch keeps filling up to
//               batch_size, since handing it over early would not start it
//               sooner and small batches use the GPU worse;
//   workers     one per slot, each searching a whole batch with one
//               td_search_pairs call (the per-pair statuses of td_search; a
//               caller may pass another function of that signature), then
//               passing the found witnesses to a certificate writer and/or the
//               whole batch to a completion callback.
//
// Only the public C ABI is used; a batch's search runs on its worker's slot.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "td16_b200.h"

#define TD_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int kStride = 17;  // bytes per beta / omega row (the batch forms' stride)

// One batch of pairs, struct of arrays in the layout td_search_pairs takes.
struct PairBatch {
    std::vector<uint64_t> tag;
    std::vector<uint8_t> beta, omega, n, full;
    std::vector<int32_t> init, max_moves;
    std::vector<float> rate;

    void reserve(int cap) {
        tag.reserve(cap);
        beta.reserve((size_t)cap * kStride);
        omega.reserve((size_t)cap * kStride);
        n.reserve(cap);
        full.reserve(cap);
        init.reserve(cap);
        max_moves.reserve(cap);
        rate.reserve(cap);
    }
    int size() const { return (int)tag.size(); }
    void clear() {
        tag.clear();
        beta.clear();
        omega.clear();
        n.clear();
        full.clear();
        init.clear();
        max_moves.clear();
        rate.clear();
    }
};

// Producer threads spread over this many filling batches, each under its own
// lock, so that many producers do not queue on one mutex.
constexpr int kShards = 16;

struct alignas(64) Shard {
    std::mutex mu;
    std::unique_ptr<PairBatch> filling;
    std::chrono::steady_clock::time_point opened_at;
    uint64_t pairs = 0;
};

// a producer thread's shard, assigned round-robin at its first accept
std::atomic<unsigned> g_next_shard{0};
thread_local int tl_shard = -1;

struct Batcher {
    // configuration
    std::vector<int> slots;
    int batch_size = 0;
    std::chrono::nanoseconds max_delay{0};
    size_t max_pending = 0;
    unsigned flags = 0;
    td_batcher_search_fn search = nullptr;
    void *cert_writer = nullptr;
    td_batcher_done_fn done = nullptr;
    void *user = nullptr;

    // Locks: `mu` (the ready queue) may be held while taking a shard's lock,
    // never the other way round; `spare_mu` is taken alone.
    std::mutex mu;
    std::condition_variable cv_ready;  // idle workers: a batch is ready or started filling, or closing
    std::condition_variable cv_space;  // producers: a ready batch was taken
    std::deque<std::unique_ptr<PairBatch>> ready;
    std::atomic<size_t> ready_count{0};  // ready.size(), read without the lock by producers
    bool closed = false;
    std::atomic<bool> closing{false};
    int idle = 0;  // workers waiting for a batch
    Shard shards[kShards];
    std::mutex spare_mu;
    std::vector<std::unique_ptr<PairBatch>> spare;  // recycled buffers

    // statistics
    std::atomic<uint64_t> batches{0}, found{0}, not_found{0}, errors{0}, certificates{0};
    std::atomic<uint64_t> search_ns{0};
    std::atomic<int> first_error{TD_OK};
    char first_message[256] = {0};

    std::vector<std::thread> workers;

    std::unique_ptr<PairBatch> fresh() {
        {
            std::lock_guard<std::mutex> g(spare_mu);
            if (!spare.empty()) {
                auto b = std::move(spare.back());
                spare.pop_back();
                return b;
            }
        }
        auto b = std::make_unique<PairBatch>();
        b->reserve(batch_size);
        return b;
    }

    // queues a batch for the workers (under mu)
    void push_ready(std::unique_ptr<PairBatch> b) {
        ready.push_back(std::move(b));
        ready_count.store(ready.size(), std::memory_order_relaxed);
        cv_ready.notify_one();
    }

    // Moves the shards' filling batches that are due (all non-empty ones when
    // `all`) to the ready queue; returns the earliest due time of those left.
    // Under mu.
    std::chrono::steady_clock::time_point sweep(bool all) {
        const auto now = std::chrono::steady_clock::now();
        auto earliest = std::chrono::steady_clock::time_point::max();
        for (Shard &sh : shards) {
            std::unique_ptr<PairBatch> b;
            {
                std::lock_guard<std::mutex> g(sh.mu);
                if (!sh.filling || sh.filling->size() == 0) continue;
                const auto due = sh.opened_at + max_delay;
                if (all || now >= due) b = std::move(sh.filling);
                else earliest = std::min(earliest, due);
            }
            if (b) push_ready(std::move(b));
        }
        return earliest;
    }

    void record_error(int rc, const char *msg) {
        int expect = TD_OK;
        if (first_error.compare_exchange_strong(expect, rc)) {
            std::lock_guard<std::mutex> g(mu);
            std::snprintf(first_message, sizeof first_message, "%s", msg ? msg : "");
        }
    }

    // Waits (under lk) until a batch is ready for this worker: a full one, a
    // filling one once it is due, or what is left at close.  Returns null
    // when the consumer is closed and drained.
    std::unique_ptr<PairBatch> next_batch(std::unique_lock<std::mutex> &lk) {
        ++idle;
        for (;;) {
            if (ready.empty()) {
                const auto earliest = sweep(closed);
                if (ready.empty()) {
                    if (closed) {
                        --idle;
                        return nullptr;
                    }
                    if (earliest != std::chrono::steady_clock::time_point::max()) cv_ready.wait_until(lk, earliest);
                    else cv_ready.wait(lk);
                    continue;
                }
            }
            break;
        }
        --idle;
        auto b = std::move(ready.front());
        ready.pop_front();
        ready_count.store(ready.size(), std::memory_order_relaxed);
        cv_space.notify_all();
        if (idle > 0) cv_ready.notify_one();  // another idle worker takes over the delays
        return b;
    }

    void run_worker(int slot) {
        std::vector<int32_t> status, depth;
        std::vector<int16_t> ijk;
        std::vector<td_result> records;
        char err[256];
        for (;;) {
            std::unique_ptr<PairBatch> b;
            {
                std::unique_lock<std::mutex> lk(mu);
                b = next_batch(lk);
                if (!b) return;  // closed and drained
            }
            const int c = b->size();
            status.assign(c, TD_OK);
            depth.assign(c, 0);
            ijk.assign((size_t)c * 27, 0);
            err[0] = 0;
            const auto t0 = std::chrono::steady_clock::now();
            const int rc = search(slot, c, b->beta.data(), b->omega.data(), b->n.data(), b->init.data(),
                                  b->rate.data(), b->max_moves.data(), b->full.data(), flags, status.data(),
                                  depth.data(), ijk.data(), err, sizeof err);
            search_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                             std::chrono::steady_clock::now() - t0).count();
            if (rc != TD_OK) {  // the whole call failed: every pair of the batch carries its code
                record_error(rc, err);
                for (int i = 0; i < c; ++i) {
                    status[i] = rc;
                    depth[i] = 0;
                }
            }
            uint64_t f = 0, nf = 0, e = 0;
            for (int i = 0; i < c; ++i) {
                if (status[i] == TD_OK) ++f;
                else if (status[i] == TD_NOT_FOUND) ++nf;
                else ++e;
            }
            found += f;
            not_found += nf;
            errors += e;
            if (cert_writer && f > 0) {
                records.assign(c, td_result{});
                for (int i = 0; i < c; ++i) {
                    td_result &r = records[i];
                    if (status[i] != TD_OK) continue;
                    r.status = 1;
                    r.depth = depth[i];
                    for (int d = 0; d < depth[i]; ++d) {
                        const int16_t *m = &ijk[(size_t)i * 27 + 3 * d];
                        r.moves[d] = (uint16_t)(m[0] | (m[1] << 5) | (m[2] << 10));
                    }
                }
                const long long q = td_cert_writer_enqueue_batch(cert_writer, c, b->beta.data(), b->omega.data(),
                                                                 b->n.data(), records.data());
                if (q < 0) record_error(TD_INVALID_ARG, "certificate writer rejected a batch");
                else certificates += (uint64_t)q;
            }
            if (done) done(user, c, b->tag.data(), status.data(), depth.data(), ijk.data());
            batches += 1;
            b->clear();
            std::lock_guard<std::mutex> g(spare_mu);
            spare.push_back(std::move(b));
        }
    }
};

void set_err(char *err, size_t errlen, const char *msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg);
}

}  // namespace

TD_API int td_batcher_open(int first_slot, int slots, int batch_size, double max_delay_s, int max_pending,
                           unsigned flags, td_batcher_search_fn search, void *cert_writer, td_batcher_done_fn done,
                           void *user, void **handle, char *err, size_t errlen) {
    if (!handle) {
        set_err(err, errlen, "td_batcher_open: handle is null");
        return TD_INVALID_ARG;
    }
    *handle = nullptr;
    if (first_slot < 0 || slots <= 0 || batch_size <= 0 || !(max_delay_s > 0.0) || max_delay_s > 3600.0 ||
        max_pending < 0 || (flags & ~TD_FLAG_ORDERED) != 0) {
        set_err(err, errlen, "td_batcher_open: needs slots, a positive batch size and delay, and flags 0 or ordered");
        return TD_INVALID_ARG;
    }
    auto *b = new Batcher();
    for (int s = 0; s < slots; ++s) b->slots.push_back(first_slot + s);
    b->batch_size = batch_size;
    b->max_delay = std::chrono::nanoseconds((long long)(max_delay_s * 1e9));
    b->max_pending = max_pending > 0 ? (size_t)max_pending : 2 * (size_t)slots;
    b->flags = flags;
    b->search = search ? search : &td_search_pairs;
    b->cert_writer = cert_writer;
    b->done = done;
    b->user = user;
    for (int s : b->slots) b->workers.emplace_back(&Batcher::run_worker, b, s);
    *handle = b;
    return TD_OK;
}

TD_API int td_batcher_accept(void *handle, uint64_t tag, const uint8_t *beta, const uint8_t *omega, int n,
                             int initial_even_cycles, float min_rate, int max_moves, int full_sorting) {
    auto *b = static_cast<Batcher *>(handle);
    if (!b || n < 0 || n > kStride || (n > 0 && (!beta || !omega))) return TD_INVALID_ARG;
    if (b->ready_count.load(std::memory_order_relaxed) >= b->max_pending ||
        b->closing.load(std::memory_order_relaxed)) {
        // the bounded queue: wait for a worker to take a batch
        std::unique_lock<std::mutex> lk(b->mu);
        while (b->ready.size() >= b->max_pending && !b->closed) b->cv_space.wait(lk);
        if (b->closed) return TD_INVALID_ARG;
    }
    if (tl_shard < 0) tl_shard = (int)(g_next_shard.fetch_add(1) % kShards);
    Shard &sh = b->shards[tl_shard];
    std::unique_ptr<PairBatch> full;
    bool started = false;
    {
        std::lock_guard<std::mutex> g(sh.mu);
        if (!sh.filling) {
            sh.filling = b->fresh();
            sh.opened_at = std::chrono::steady_clock::now();
            started = true;
        }
        PairBatch &p = *sh.filling;
        p.tag.push_back(tag);
        const size_t at = p.beta.size();
        p.beta.resize(at + kStride, 0);
        p.omega.resize(at + kStride, 0);
        if (n > 0) {
            std::memcpy(&p.beta[at], beta, (size_t)n);
            std::memcpy(&p.omega[at], omega, (size_t)n);
        }
        p.n.push_back((uint8_t)n);
        p.init.push_back(initial_even_cycles);
        p.rate.push_back(min_rate);
        p.max_moves.push_back(max_moves);
        p.full.push_back(full_sorting ? 1 : 0);
        ++sh.pairs;
        if (p.size() >= b->batch_size) full = std::move(sh.filling);
    }
    if (full) {
        std::lock_guard<std::mutex> g(b->mu);
        b->push_ready(std::move(full));
    } else if (started) {
        // an idle worker starts this batch's delay
        std::lock_guard<std::mutex> g(b->mu);
        if (b->idle > 0) b->cv_ready.notify_one();
    }
    return TD_OK;
}

TD_API int td_batcher_flush(void *handle) {
    auto *b = static_cast<Batcher *>(handle);
    if (!b) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(b->mu);
    b->sweep(true);
    return TD_OK;
}

TD_API int td_batcher_close(void *handle, td_batcher_stats *stats, char *err, size_t errlen) {
    auto *b = static_cast<Batcher *>(handle);
    if (!b) {
        set_err(err, errlen, "td_batcher_close: handle is null");
        return TD_INVALID_ARG;
    }
    b->closing.store(true);
    {
        std::lock_guard<std::mutex> g(b->mu);
        b->sweep(true);
        b->closed = true;
    }
    b->cv_ready.notify_all();
    b->cv_space.notify_all();
    for (auto &t : b->workers) t.join();
    const int rc = b->first_error.load();
    if (stats) {
        stats->pairs = 0;
        for (Shard &sh : b->shards) stats->pairs += sh.pairs;
        stats->batches = b->batches;
        stats->found = b->found;
        stats->not_found = b->not_found;
        stats->errors = b->errors;
        stats->certificates = b->certificates;
        stats->search_s = (double)b->search_ns.load() * 1e-9;
    }
    if (rc != TD_OK) set_err(err, errlen, b->first_message);
    delete b;
    return rc;
}
