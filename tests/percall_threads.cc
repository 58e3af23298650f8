// percall_threads.cc -- native host threads for the per-call speed comparison.
//
// TEST INFRASTRUCTURE ONLY (built and loaded by tests/ref_kernel_speed.py).
// The emitter calls the search from Java threads, one blocking call per slot
// (GPUSortingSearch.java:134-147); Python threads would serialise those calls
// on the interpreter lock.  This runs `nthreads` native threads, thread t on
// slot t, each taking the next instance until all `count` are done, through a
// search function pointer of either form:
//   kind 0: td_search (include/td16_b200.h) of this engine;
//   kind 1: ref_search (oracle/ref_driver.cu) around the reference kernel.
// Returns the wall time in seconds; status[i] = 1 found, 0 not found, -1 error.
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

typedef int (*td_search_fn)(int slot, const uint8_t *beta, const uint8_t *omega, int n, int init, float rate,
                            int maxd, int full, int16_t *out, int *depth, char *err, size_t errlen);
typedef int (*ref_search_fn)(const uint8_t *beta, const uint8_t *omega, int n, int init, float rate, int maxd,
                             int full, int slot, int max_warps, int16_t *out, int *depth, char *err, size_t errlen);

extern "C" double percall_run(int kind, void *fn, int count, const uint8_t *beta, const uint8_t *omega,
                              const int32_t *n, const int32_t *init, int maxd, int nthreads, int32_t *status) {
    std::atomic<int> next{0};
    auto worker = [&](int slot) {
        int16_t out[27];
        char err[256];
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= count) return;
            int depth = 0;
            int rc;
            if (kind == 0)
                rc = reinterpret_cast<td_search_fn>(fn)(slot, beta + 17 * (size_t)i, omega + 17 * (size_t)i, n[i],
                                                        init[i], 0.0f, maxd, 1, out, &depth, err, sizeof err);
            else
                rc = reinterpret_cast<ref_search_fn>(fn)(beta + 17 * (size_t)i, omega + 17 * (size_t)i, n[i],
                                                         init[i], 0.0f, maxd, 1, slot, -1, out, &depth, err,
                                                         sizeof err);
            // this engine: 0 found, 1 not found; reference driver: 0 with a depth
            status[i] = kind == 0 ? (rc == 0 ? 1 : rc == 1 ? 0 : -1) : (rc == 0 ? (depth > 0 ? 1 : 0) : -1);
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) th.emplace_back(worker, t);
    for (auto &t : th) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
