// td_cert.cu -- certificate records: the reference's on-disk byte format, a
// batched file sink, and a device replay of symbol witnesses with the
// checker's rules.
//
// Format (emitter/src/main/java/br/unb/cic/tdp/base/CertificateCodec.java:22-147):
//   key   = omega in one-line notation, 5 bits per symbol, most significant
//           bit first, zero padding to a whole byte
//   value = the witness as consecutive 15-bit fields (a, b, c), same bit order
// Replay (CertificateValidator.java:14-50): 1 <= moves <= maxMoves; each move
// holds three distinct symbols at increasing positions of the current beta
// array; omega <- omega . (a b c)^-1; beta <- block swap; omega . beta stays
// rho; omega ends as the identity.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#define TD_API extern "C" __attribute__((visibility("default")))

#include "td_core.cuh"
#define TD_CERT_MAX_N 17
#define TD_CERT_MAX_MOVES 9

namespace {

inline void put5(uint8_t *buf, int bit, int v) {
    for (int b = 0; b < 5; ++b) {
        const int o = bit + b;
        buf[o >> 3] |= (uint8_t)(((v >> (4 - b)) & 1) << (7 - (o & 7)));
    }
}

inline int get5(const uint8_t *buf, int bit) {
    int v = 0;
    for (int b = 0; b < 5; ++b) {
        const int o = bit + b;
        v = (v << 1) | ((buf[o >> 3] >> (7 - (o & 7))) & 1);
    }
    return v;
}

inline bool padding_zero(const uint8_t *in, int len, int payload_bits) {
    if (len != (payload_bits + 7) / 8) return false;
    const int pad = 8 * len - payload_bits;
    return pad == 0 || (in[len - 1] & ((1 << pad) - 1)) == 0;
}

}  // namespace

// Key bytes for omega over n symbols (1 <= n <= 32, symbols < 32).  Returns
// the length or -1.
TD_API int td_codec_key(const uint8_t *omega, int n, uint8_t *out, int cap) {
    if (n <= 0 || n > 32) return -1;
    const int len = (5 * n + 7) / 8;
    if (cap < len) return -1;
    std::memset(out, 0, (size_t)len);
    for (int x = 0; x < n; ++x) {
        if (omega[x] >= 32) return -1;
        put5(out, 5 * x, omega[x]);
    }
    return len;
}

// Value bytes for `count` symbol triples (abc[3*m..3*m+2]).
TD_API int td_codec_value(const uint8_t *abc, int count, uint8_t *out, int cap) {
    if (count <= 0) return -1;
    const int len = (15 * count + 7) / 8;
    if (cap < len) return -1;
    std::memset(out, 0, (size_t)len);
    for (int m = 0; m < 3 * count; ++m) {
        if (abc[m] >= 32) return -1;
        put5(out, 5 * m, abc[m]);
    }
    return len;
}

TD_API int td_codec_decode_key(const uint8_t *in, int len, int n, uint8_t *omega) {
    if (!in || n <= 0 || n > 32 || !padding_zero(in, len, 5 * n)) return -1;
    for (int x = 0; x < n; ++x) omega[x] = (uint8_t)get5(in, 5 * x);
    return n;
}

// Decodes a value into symbol triples; returns the move count or -1 for a
// truncated value or nonzero padding (CertificateCodec.java:75-97,120-129).
TD_API int td_codec_decode_value(const uint8_t *in, int len, uint8_t *abc, int cap_moves) {
    if (!in || len <= 0) return -1;
    const int count = (8 * len) / 15;
    if (count == 0 || !padding_zero(in, len, 15 * count) || count > cap_moves) return -1;
    for (int m = 0; m < 3 * count; ++m) abc[m] = (uint8_t)get5(in, 5 * m);
    return count;
}

// ---- device replay of symbol witnesses ------------------------------------

__global__ void td_replay_symbols_kernel(const uint8_t *__restrict__ beta, const uint8_t *__restrict__ omega,
                                         const uint8_t *__restrict__ n_arr, const uint8_t *__restrict__ maxm,
                                         const uint8_t *__restrict__ depth, const uint8_t *__restrict__ abc,
                                         uint8_t *__restrict__ ok, int count) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const int n = n_arr[idx], mm = maxm[idx], dep = depth[idx];
    uint8_t b[TD_CERT_MAX_N], o[TD_CERT_MAX_N], rho[TD_CERT_MAX_N], nb[TD_CERT_MAX_N];
    bool good = n >= 3 && n <= TD_CERT_MAX_N && dep >= 1 && dep <= mm && dep <= TD_CERT_MAX_MOVES;
    if (good) {
        for (int x = 0; x < n; ++x) {
            b[x] = beta[idx * TD_CERT_MAX_N + x];
            o[x] = omega[idx * TD_CERT_MAX_N + x];
            if (b[x] >= n || o[x] >= n) good = false;
        }
    }
    if (good) {
        // rho = omega . beta (beta read as the cycle b0 -> b1 -> ...)
        for (int x = 0; x < n; ++x) rho[b[x]] = o[b[(x + 1) % n]];
    }
    for (int m = 0; good && m < dep; ++m) {
        const int a = abc[(size_t)idx * 27 + 3 * m], c2 = abc[(size_t)idx * 27 + 3 * m + 1],
                  c3 = abc[(size_t)idx * 27 + 3 * m + 2];
        if (a == c2 || c2 == c3 || a == c3 || a >= n || c2 >= n || c3 >= n) { good = false; break; }
        int pa = -1, pb = -1, pc = -1;
        for (int x = 0; x < n; ++x) {
            if (b[x] == a) pa = x;
            if (b[x] == c2) pb = x;
            if (b[x] == c3) pc = x;
        }
        if (!(pa >= 0 && pa < pb && pb < pc)) { good = false; break; }
        // omega <- omega . (a b c)^-1
        const uint8_t oa = o[a], ob = o[c2], oc = o[c3];
        o[a] = oc;
        o[c2] = oa;
        o[c3] = ob;
        int w = 0;
        for (int x = 0; x < pa; ++x) nb[w++] = b[x];
        for (int x = pb; x < pc; ++x) nb[w++] = b[x];
        for (int x = pa; x < pb; ++x) nb[w++] = b[x];
        for (int x = pc; x < n; ++x) nb[w++] = b[x];
        for (int x = 0; x < n; ++x) b[x] = nb[x];
        for (int x = 0; x < n && good; ++x)
            if (o[b[(x + 1) % n]] != rho[b[x]]) good = false;  // target preserved
    }
    for (int x = 0; good && x < n; ++x)
        if (o[x] != x) good = false;
    ok[idx] = good ? 1 : 0;
}

// Replays `count` symbol witnesses on the device (all pointers are device
// pointers): beta/omega stride 17, abc stride 27 (9 triples).  ok[i] = 1
// when witness i is accepted.
TD_API int td_replay_symbols_device(int count, const uint8_t *d_beta, const uint8_t *d_omega, const uint8_t *d_n,
                                    const uint8_t *d_max_moves, const uint8_t *d_depth, const uint8_t *d_abc,
                                    uint8_t *d_ok, void *stream, char *err, size_t errlen) {
    if (count <= 0) return 0;
    td_replay_symbols_kernel<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_beta, d_omega, d_n,
                                                                                     d_max_moves, d_depth, d_abc,
                                                                                     d_ok, count);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        if (err && errlen) std::snprintf(err, errlen, "td_replay_symbols_device: %s", cudaGetErrorString(e));
        return 3;
    }
    return 0;
}

// Loads the replay kernel on the current device (called when the engine sets
// a device up, so that its first launch never waits for loading while the
// per-call server's resident launch runs).  Returns a cudaError_t.
int td_cert_preload(void) {
    cudaFuncAttributes a;
    return (int)cudaFuncGetAttributes(&a, td_replay_symbols_kernel);
}

// ---- batched certificate sink ----------------------------------------------
//
// AsyncCertificateWriter semantics (AsyncCertificateWriter.java:50-116): one
// writer thread drains a queue of (key, value) records in batches and flushes
// on a period; the first write failure is kept and reported to every later
// call.  Without RocksDB the store is a flat file of records
// [u8 key_len][u8 value_len][key][value].

namespace {

struct CertWriter {
    FILE *f = nullptr;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::vector<uint8_t>> q;
    std::thread th;
    bool stop = false;
    int failed = 0;
    double flush_s = 5.0;
    uint64_t written = 0;

    void run() {
        auto last = std::chrono::steady_clock::now();
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait_for(lk, std::chrono::milliseconds(50), [&] { return stop || !q.empty(); });
            std::deque<std::vector<uint8_t>> batch;
            batch.swap(q);
            const bool done = stop;
            lk.unlock();
            for (auto &r : batch)
                if (!failed && std::fwrite(r.data(), 1, r.size(), f) != r.size()) failed = 1;
            const auto now = std::chrono::steady_clock::now();
            if (done || std::chrono::duration<double>(now - last).count() >= flush_s) {
                if (std::fflush(f) != 0) failed = 1;
                last = now;
            }
            lk.lock();
            written += batch.size();
            if (done && q.empty()) break;
        }
    }
};

}  // namespace

TD_API void *td_cert_writer_open(const char *path, double flush_seconds) {
    FILE *f = std::fopen(path, "ab");
    if (!f) return nullptr;
    auto *w = new CertWriter();
    w->f = f;
    w->flush_s = flush_seconds > 0 ? flush_seconds : 5.0;
    w->th = std::thread([w] { w->run(); });
    return w;
}

// Queues one certificate: omega one-line over n symbols and `count` symbol
// triples.  Returns 0, -1 for an unencodable record, -2 after a write failure.
TD_API int td_cert_writer_enqueue(void *handle, const uint8_t *omega, int n, const uint8_t *abc, int count) {
    auto *w = static_cast<CertWriter *>(handle);
    if (!w) return -1;
    uint8_t key[32], val[64];
    const int kl = td_codec_key(omega, n, key, sizeof key);
    const int vl = td_codec_value(abc, count, val, sizeof val);
    if (kl < 0 || vl < 0) return -1;
    std::vector<uint8_t> rec(2 + kl + vl);
    rec[0] = (uint8_t)kl;
    rec[1] = (uint8_t)vl;
    std::memcpy(&rec[2], key, kl);
    std::memcpy(&rec[2 + kl], val, vl);
    std::lock_guard<std::mutex> g(w->mu);
    if (w->failed) return -2;
    w->q.push_back(std::move(rec));
    w->cv.notify_one();
    return 0;
}

// Drains, flushes and closes; returns the number of records written or -2.
TD_API long long td_cert_writer_close(void *handle) {
    auto *w = static_cast<CertWriter *>(handle);
    if (!w) return -1;
    {
        std::lock_guard<std::mutex> g(w->mu);
        w->stop = true;
    }
    w->cv.notify_one();
    w->th.join();
    const int failed = w->failed || std::fclose(w->f) != 0;
    const long long n = (long long)w->written;
    delete w;
    return failed ? -2 : n;
}

// Queues the found witnesses of a batch: omega/beta stride 17 (the caller's
// pair), n symbols each, results as td_result records (caller positions).
// Returns the number queued, -1 for an unencodable record, -2 after a write
// failure.
TD_API long long td_cert_writer_enqueue_batch(void *handle, int count, const uint8_t *beta, const uint8_t *omega,
                                              const uint8_t *n, const td_result *results) {
    auto *w = static_cast<CertWriter *>(handle);
    if (!w) return -1;
    std::deque<std::vector<uint8_t>> recs;
    for (int i = 0; i < count; ++i) {
        const td_result &r = results[i];
        if (r.status != TD_FOUND || r.depth <= 0 || r.depth > TD_CERT_MAX_MOVES) continue;
        const int N = n[i];
        if (N < 3 || N > TD_CERT_MAX_N) return -1;
        uint8_t cur[TD_CERT_MAX_N], nxt[TD_CERT_MAX_N], abc[3 * TD_CERT_MAX_MOVES];
        std::memcpy(cur, beta + (size_t)i * TD_CERT_MAX_N, (size_t)N);
        for (int d = 0; d < r.depth; ++d) {  // GPUSortingSearch.java:229-238
            const int a = r.moves[d] & 31, b = (r.moves[d] >> 5) & 31, c = (r.moves[d] >> 10) & 31;
            if (!(a < b && b < c && c < N)) return -1;
            abc[3 * d] = cur[a];
            abc[3 * d + 1] = cur[b];
            abc[3 * d + 2] = cur[c];
            int k = 0;
            for (int x = 0; x < a; ++x) nxt[k++] = cur[x];
            for (int x = b; x < c; ++x) nxt[k++] = cur[x];
            for (int x = a; x < b; ++x) nxt[k++] = cur[x];
            for (int x = c; x < N; ++x) nxt[k++] = cur[x];
            std::memcpy(cur, nxt, (size_t)N);
        }
        uint8_t key[32], val[64];
        const int kl = td_codec_key(omega + (size_t)i * TD_CERT_MAX_N, N, key, sizeof key);
        const int vl = td_codec_value(abc, r.depth, val, sizeof val);
        if (kl < 0 || vl < 0) return -1;
        std::vector<uint8_t> rec(2 + kl + vl);
        rec[0] = (uint8_t)kl;
        rec[1] = (uint8_t)vl;
        std::memcpy(&rec[2], key, kl);
        std::memcpy(&rec[2 + kl], val, vl);
        recs.push_back(std::move(rec));
    }
    std::lock_guard<std::mutex> g(w->mu);
    if (w->failed) return -2;
    const long long q = (long long)recs.size();
    for (auto &r : recs) w->q.push_back(std::move(r));
    w->cv.notify_one();
    return q;
}

// Reads up to `cap` records of a certificate file written for domains of n
// symbols into omega (stride 17), abc (stride 27) and depth.  Returns the
// number read, or -1 for a malformed record.
TD_API long long td_cert_read_file(const char *path, int n, long long cap, uint8_t *omega, uint8_t *abc,
                                   uint8_t *depth) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return -1;
    long long k = 0;
    uint8_t hdr[2], buf[96];
    while (k < cap && std::fread(hdr, 1, 2, f) == 2) {
        const int kl = hdr[0], vl = hdr[1];
        if (kl + vl > (int)sizeof buf || std::fread(buf, 1, (size_t)(kl + vl), f) != (size_t)(kl + vl)) {
            std::fclose(f);
            return -1;
        }
        if (td_codec_decode_key(buf, kl, n, omega + (size_t)k * TD_CERT_MAX_N) < 0) {
            std::fclose(f);
            return -1;
        }
        const int m = td_codec_decode_value(buf + kl, vl, abc + (size_t)k * 27, TD_CERT_MAX_MOVES);
        if (m < 0) {
            std::fclose(f);
            return -1;
        }
        depth[k] = (uint8_t)m;
        ++k;
    }
    std::fclose(f);
    return k;
}

// Caller pairs of S_n permutations (perms int8 stride 16): beta = (0..n),
// omega one-line over n+1 symbols (stride 17).
TD_API void td_pairs_from_perms(int count, const int8_t *perms, const uint8_t *n, uint8_t *beta, uint8_t *omega) {
    for (int i = 0; i < count; ++i) {
        int init;
        if (n[i] > TD_CERT_MAX_N - 1) continue;
        td_perm_to_pair(perms + (size_t)i * 16, n[i], beta + (size_t)i * TD_CERT_MAX_N,
                        omega + (size_t)i * TD_CERT_MAX_N, &init);
    }
}
