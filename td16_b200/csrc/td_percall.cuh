// td_percall.cuh -- the per-call server behind td_search and td_search_ordered
// (included by td_engine.cu after td_serve.cuh).
//
// The reference runs one blocking search per JNI call: four small copies, two
// launches and an event wait per search (sorting_search.cu:811-972), which is
// why its host keeps 7-16 slots in flight.  Here every per-call search goes
// to one resident serving launch per device (td_serve_kernel in per-request
// mode): the calling slot thread writes its request into a pinned,
// device-mapped ring, the launch's dispatcher picks it up, a worker warp
// searches it while idle warps take donated subtrees, and the result lands in
// mapped host memory that the caller polls.  A search costs no CUDA API call
// at all once the launch runs.
//
// Sharing the device.  The launch holds half of each SM's block slots, so a
// batch launch started while per-call searches run still gets SMs and makes
// progress.  A batch entry point first stops the device's server when no
// per-call search is in flight, so a batch alone has the whole GPU; the next
// per-call search starts it again.
//
// Lifetime.  Every wait in the launch is bounded by its deadline, so the
// launch cannot serve forever.  A server that has run for the rotation age
// (td_configure_percall, default 300 s) is replaced: new requests go to a fresh launch on the second server of the
// device, and the old one is stopped when its last request has been read.
// Each request's search is bounded by the engine's time limit
// (td_set_time_limit), and the old launch lives long enough for any request
// it accepted.
#pragma once

namespace {

constexpr unsigned kPercallRing = 1u << 16;   // requests in flight per launch, at most
constexpr int kPercallItems = 1 << 18;        // donated subtrees in flight
constexpr int kPercallDevices = 64;

struct PercallServer {
    bool allocated = false, running = false, retiring = false;
    int device = -1;
    cudaStream_t stream = nullptr;
    td_instance *h_ring = nullptr, *d_ring = nullptr;
    td_result *h_res = nullptr, *d_res = nullptr;
    unsigned long long *h_done = nullptr, *d_done = nullptr;
    td_serve_host_ctl *h_ctl = nullptr, *d_hctl = nullptr;
    td_serve_dev_ctl *d_ctl = nullptr;
    td_instance *d_queue = nullptr;
    td_inst_state *d_state = nullptr;
    td_pool *d_pool = nullptr;
    td_item *d_items = nullptr;
    uint32_t *d_ready = nullptr;
    uint64_t *d_tt = nullptr;
    uint32_t *d_tt_gen = nullptr;
    size_t tt_warps = 0;
    int tt_bits = 0;
    // tickets are numbered across the launches of this server, so a stamp of
    // one launch never matches a request of another
    unsigned long long published = 0;
    unsigned long long *taken = nullptr;  // per ring slot: ticket + 1 of the last result read
    int inflight = 0;
    std::atomic<unsigned> generation{0};  // launches started; a waiting client compares it
    std::chrono::steady_clock::time_point started;
    int grid = 0, warps = 0;
};

struct PercallDevice {
    std::mutex mu;
    PercallServer srv[2];
    int cur = 0;
};

PercallDevice g_percall[kPercallDevices];
std::atomic<int> g_percall_mode{1};  // 1: resident server, 0: one launch per call
std::atomic<long long> g_percall_rotate_ns{300000000000ll};
std::atomic<long long> g_percall_idle_ns{5000000ll};  // a launch idle this long exits by itself

// rotation age of a launch; its deadline leaves every accepted request the
// full search time limit on top
std::chrono::nanoseconds percall_rotate_after() { return std::chrono::nanoseconds(g_percall_rotate_ns.load()); }

void percall_free(PercallServer &ps) {
    if (!ps.allocated) return;
    cudaSetDevice(ps.device);
    if (ps.stream) cudaStreamSynchronize(ps.stream);
    if (ps.h_ring) cudaFreeHost(ps.h_ring);
    if (ps.h_res) cudaFreeHost(ps.h_res);
    if (ps.h_done) cudaFreeHost(ps.h_done);
    if (ps.h_ctl) cudaFreeHost(ps.h_ctl);
    if (ps.d_ctl) cudaFree(ps.d_ctl);
    if (ps.d_queue) cudaFree(ps.d_queue);
    if (ps.d_state) cudaFree(ps.d_state);
    if (ps.d_pool) cudaFree(ps.d_pool);
    if (ps.d_items) cudaFree(ps.d_items);
    if (ps.d_ready) cudaFree(ps.d_ready);
    if (ps.d_tt) cudaFree(ps.d_tt);
    if (ps.d_tt_gen) cudaFree(ps.d_tt_gen);
    if (ps.stream) cudaStreamDestroy(ps.stream);
    delete[] ps.taken;
    ps.allocated = ps.running = ps.retiring = false;
    ps.device = -1;
    ps.stream = nullptr;
    ps.h_ring = ps.d_ring = nullptr;
    ps.h_res = ps.d_res = nullptr;
    ps.h_done = ps.d_done = nullptr;
    ps.h_ctl = ps.d_hctl = nullptr;
    ps.d_ctl = nullptr;
    ps.d_queue = nullptr;
    ps.d_state = nullptr;
    ps.d_pool = nullptr;
    ps.d_items = nullptr;
    ps.d_ready = nullptr;
    ps.d_tt = nullptr;
    ps.d_tt_gen = nullptr;
    ps.tt_warps = 0;
    ps.tt_bits = 0;
    ps.published = 0;
    ps.taken = nullptr;
    ps.inflight = 0;
    ps.generation.fetch_add(1);
}

int percall_alloc(PercallServer &ps, int device, char *err, size_t errlen) {
    if (ps.allocated) return TD_OK;
    ps.device = device;
    ps.allocated = true;  // percall_free releases whatever was obtained
    const unsigned R = kPercallRing;
    const unsigned mapped = cudaHostAllocMapped | cudaHostAllocPortable;
    cudaError_t e = cudaStreamCreateWithFlags(&ps.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc(&ps.h_ring, sizeof(td_instance) * R, mapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&ps.h_res, sizeof(td_result) * R, mapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&ps.h_done, sizeof(unsigned long long) * R, mapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&ps.h_ctl, sizeof(td_serve_host_ctl), mapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&ps.d_ring, ps.h_ring, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&ps.d_res, ps.h_res, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&ps.d_done, ps.h_done, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&ps.d_hctl, ps.h_ctl, 0);
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_ctl, sizeof(td_serve_dev_ctl));
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_queue, sizeof(td_instance) * R);
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_state, sizeof(td_inst_state) * R);
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_pool, sizeof(td_pool));
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_items, sizeof(td_item) * kPercallItems);
    if (e == cudaSuccess) e = cudaMalloc(&ps.d_ready, sizeof(uint32_t) * kPercallItems);
    if (e != cudaSuccess) {
        set_err(err, errlen, cuda_msg(e, __FILE__, __LINE__));
        percall_free(ps);
        return TD_CUDA_ERROR;
    }
    ps.taken = new unsigned long long[R];
    std::memset(ps.taken, 0, sizeof(unsigned long long) * R);
    std::memset((void *)ps.h_done, 0, sizeof(unsigned long long) * R);
    ps.published = 0;
    return TD_OK;
}

// Stops a running launch: it serves what was published, then exits.
void percall_stop(PercallServer &ps) {
    if (!ps.running) return;
    __atomic_store_n(const_cast<int *>(&ps.h_ctl->stop), 1, __ATOMIC_RELEASE);
    cudaSetDevice(ps.device);
    cudaStreamSynchronize(ps.stream);
    ps.running = false;
    ps.retiring = false;
}

// Starts the launch of `ps` on `device` (current).  Called with the device's
// lock held and `ps` stopped.
int percall_start(PercallServer &ps, int device, char *err, size_t errlen) {
    int rc = percall_alloc(ps, device, err, errlen);
    if (rc != TD_OK) return rc;
    LaunchCfg cfg;
    rc = launch_cfg(device, &cfg, err, errlen);
    if (rc != TD_OK) return rc;
    const int warps = cfg.warps;
    const size_t smem = smem_bytes(warps);
    int per_sm = 0;
    TD_CHECK(cudaFuncSetAttribute(td_serve_kernel<TD_SERVE_PER_REQUEST>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TD_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, td_serve_kernel<TD_SERVE_PER_REQUEST>,
                                                           warps * 32, smem));
    // half of each SM's block slots: batch launches keep the other half
    const int grid = cfg.sms * std::max(1, per_sm / 2);
    if (cfg.tt_bits > 0 && ((size_t)grid * warps > ps.tt_warps || cfg.tt_bits != ps.tt_bits)) {
        // in stream order: a cudaFree would wait for the device's other
        // server launch, which may be draining
        if (ps.d_tt) TD_CHECK(cudaFreeAsync(ps.d_tt, ps.stream));
        if (ps.d_tt_gen) TD_CHECK(cudaFreeAsync(ps.d_tt_gen, ps.stream));
        ps.d_tt = nullptr;
        ps.d_tt_gen = nullptr;
        ps.tt_warps = 0;
        const size_t words = (size_t)grid * warps << cfg.tt_bits;
        TD_CHECK(cudaMallocAsync(&ps.d_tt, words * sizeof(uint64_t), ps.stream));
        TD_CHECK(cudaMallocAsync(&ps.d_tt_gen, (size_t)grid * warps * sizeof(uint32_t), ps.stream));
        TD_CHECK(cudaMemsetAsync(ps.d_tt, 0, words * sizeof(uint64_t), ps.stream));
        TD_CHECK(cudaMemsetAsync(ps.d_tt_gen, 0, (size_t)grid * warps * sizeof(uint32_t), ps.stream));
        ps.tt_warps = (size_t)grid * warps;
        ps.tt_bits = cfg.tt_bits;
    }
    // the launch starts at the next ticket: its dispatcher and workers begin
    // there, and the item tags of the previous launch are cleared
    td_serve_dev_ctl ctl;
    std::memset(&ctl, 0, sizeof ctl);
    ctl.available = ctl.claimed = ps.published;
    ps.h_ctl->stop = 0;
    ps.h_ctl->exit_reason = 0;
    __atomic_store_n(const_cast<unsigned long long *>(&ps.h_ctl->published), ps.published, __ATOMIC_RELEASE);
    TD_CHECK(cudaMemcpyAsync(ps.d_ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, ps.stream));
    TD_CHECK(cudaStreamSynchronize(ps.stream));  // `ctl` lives on this stack
    TD_CHECK(cudaMemsetAsync(ps.d_pool, 0, sizeof(td_pool), ps.stream));
    TD_CHECK(cudaMemsetAsync(ps.d_ready, 0, sizeof(uint32_t) * kPercallItems, ps.stream));
    const uint64_t request_ns = time_limit_ns();
    const uint64_t life_ns = (uint64_t)percall_rotate_after().count() + request_ns + 60000000000ull;
    td_serve_kernel<TD_SERVE_PER_REQUEST><<<grid, warps * 32, smem, ps.stream>>>(
        ps.d_ring, ps.d_res, ps.d_done, kPercallRing, ps.d_hctl, ps.d_ctl, ps.d_queue, ps.d_state, ps.d_pool,
        ps.d_items, ps.d_ready, kPercallItems, cfg.serve_grain, cfg.serve_split_level, cfg.serve_check_every, 0,
        life_ns, cfg.tt_bits > 0 ? ps.d_tt : nullptr, ps.d_tt_gen, cfg.tt_bits, cfg.restart_base, request_ns,
        (uint64_t)g_percall_idle_ns.load(), cfg.race ? 1 : 0);  // mostly idle warps: race from the first restart
    TD_CHECK(cudaGetLastError());
    ps.grid = grid;
    ps.warps = warps;
    ps.running = true;
    ps.retiring = false;
    ps.started = std::chrono::steady_clock::now();
    ps.generation.fetch_add(1);
    return TD_OK;
}

// Stops the device's per-call launches that have no request in flight (before
// a batch launch, so that it has the whole GPU).
void percall_park(int device) {
    if (device < 0 || device >= kPercallDevices) return;
    PercallDevice &pd = g_percall[device];
    std::lock_guard<std::mutex> g(pd.mu);
    for (auto &ps : pd.srv)
        if (ps.running && ps.inflight == 0) percall_stop(ps);
}

// Stops and frees every per-call launch (td_destroy, td_init_slots).
void percall_shutdown() {
    // every launch is stopped before anything is freed: a free waits for all
    // work on its device
    for (auto &pd : g_percall) {
        std::lock_guard<std::mutex> g(pd.mu);
        for (auto &ps : pd.srv) percall_stop(ps);
    }
    for (auto &pd : g_percall) {
        std::lock_guard<std::mutex> g(pd.mu);
        for (auto &ps : pd.srv) percall_free(ps);
        pd.cur = 0;
    }
}

// Publishes `x` to the device's current launch (starting or replacing it as
// needed).  Called with the device's lock held.
int percall_submit(PercallDevice &pd, int device, const td_instance &x, PercallServer **out_ps,
                   unsigned long long *out_ticket, unsigned *out_gen, char *err, size_t errlen) {
    TD_CHECK(cudaSetDevice(device));
    PercallServer *ps = &pd.srv[pd.cur];
    // the launch has ended (idle or its deadline; its dispatcher says so in
    // mapped memory, so no CUDA call is needed to see it): start afresh.  A
    // launch that failed is seen by its clients' own checks.
    if (ps->running && __atomic_load_n(&ps->h_ctl->exit_reason, __ATOMIC_ACQUIRE) != 0) {
        cudaStreamSynchronize(ps->stream);
        ps->running = false;
        ps->retiring = false;
    }
    if (ps->running && std::chrono::steady_clock::now() - ps->started > percall_rotate_after()) {
        PercallServer &next = pd.srv[1 - pd.cur];
        if (next.running && __atomic_load_n(&next.h_ctl->exit_reason, __ATOMIC_ACQUIRE) != 0) {
            cudaStreamSynchronize(next.stream);
            next.running = false;
            next.retiring = false;
        }
        if (!next.running) {
            const int rc = percall_start(next, device, err, errlen);
            if (rc != TD_OK) return rc;
            if (ps->inflight == 0) percall_stop(*ps);
            else ps->retiring = true;
            pd.cur = 1 - pd.cur;
            ps = &next;
        }
    }
    if (!ps->running) {
        const int rc = percall_start(*ps, device, err, errlen);
        if (rc != TD_OK) return rc;
    }
    const unsigned long long ticket = ps->published;
    const unsigned slot = (unsigned)(ticket % kPercallRing);
    // the ring slot's previous request must have been read (a ring of 2^16
    // requests makes this wait practically never happen)
    if (ticket >= kPercallRing)
        while (__atomic_load_n(&ps->taken[slot], __ATOMIC_ACQUIRE) != ticket - kPercallRing + 1)
            std::this_thread::yield();
    ps->h_ring[slot] = x;
    __atomic_store_n(&ps->h_done[slot], 0ull, __ATOMIC_RELAXED);
    __atomic_thread_fence(__ATOMIC_SEQ_CST);
    ps->published = ticket + 1;
    __atomic_store_n(const_cast<unsigned long long *>(&ps->h_ctl->published), ticket + 1, __ATOMIC_RELEASE);
    ++ps->inflight;
    *out_ps = ps;
    *out_ticket = ticket;
    *out_gen = ps->generation.load();
    return TD_OK;
}

// One blocking search through the device's per-call server.  `x` is the
// prepared instance (TD_PACKED_ORDERED set for the reference order).
int percall_search(int device, const td_instance &x, td_result *out, char *err, size_t errlen) {
    if (device < 0 || device >= kPercallDevices) {
        set_err(err, errlen, "device ordinal out of range for the per-call server");
        return TD_INVALID_ARG;
    }
    PercallDevice &pd = g_percall[device];
    // a launch that exits for being idle just as a request is published does
    // not serve it; the request then goes to a fresh launch (a few tries)
    for (int attempt = 0;; ++attempt) {
        PercallServer *ps;
        unsigned long long ticket;
        unsigned gen;
        {
            std::lock_guard<std::mutex> g(pd.mu);
            const int rc = percall_submit(pd, device, x, &ps, &ticket, &gen, err, errlen);
            if (rc != TD_OK) return rc;
        }
        const unsigned slot = (unsigned)(ticket % kPercallRing);
        int rc = TD_OK;
        bool again = false;
        for (unsigned spin = 1;; ++spin) {
            if (__atomic_load_n(&ps->h_done[slot], __ATOMIC_ACQUIRE) == ticket + 1) {
                std::memcpy(out, (const void *)&ps->h_res[slot], sizeof(td_result));
                break;
            }
            if ((spin & 1023u) == 0) {
                // the launch this request went to has ended, or been replaced
                // after it ended, without serving it
                const cudaError_t q = ps->generation.load() != gen ? cudaSuccess : cudaStreamQuery(ps->stream);
                if (q != cudaErrorNotReady) {
                    if (__atomic_load_n(&ps->h_done[slot], __ATOMIC_ACQUIRE) == ticket + 1) continue;
                    // a launch that exits for being idle has served everything
                    // it copied, so this request was published after its last
                    // look; after any other end (its deadline) searching again
                    // is harmless, since a search has no side effects
                    if (q == cudaSuccess && attempt < 8) {
                        again = true;
                    } else if (q == cudaSuccess) {
                        set_err(err, errlen, "GPU sorting search deadline reached (the per-call server ended)");
                        rc = TD_TIMEOUT;
                    } else {
                        set_err(err, errlen, cuda_msg(q, __FILE__, __LINE__));
                        rc = TD_CUDA_ERROR;
                    }
                    break;
                }
            }
            // spin briefly (a typical search answers within tens of us), then yield
            if (spin < 4096) __builtin_ia32_pause();
            else std::this_thread::yield();
        }
        __atomic_store_n(&ps->taken[slot], ticket + 1, __ATOMIC_RELEASE);
        {
            std::lock_guard<std::mutex> g(pd.mu);
            --ps->inflight;
            if (ps->retiring && ps->inflight == 0) percall_stop(*ps);
        }
        if (!again) return rc;
    }
}

}  // namespace

// Per-call searches (td_search, td_search_ordered): mode 1 (default) through
// the device's resident server, 0 with one launch per call on the slot's
// stream.  rotate_after_s > 0 sets the age at which a server launch is
// replaced by a fresh one (default 300 s); idle_exit_s > 0 the idle time after
// which a launch with no work left exits by itself (default 0.005 s); 0 keeps
// the current setting.
TD_API int td_configure_percall(int mode, double rotate_after_s, double idle_exit_s) {
    if ((mode != 0 && mode != 1) || rotate_after_s < 0 || idle_exit_s < 0) return TD_INVALID_ARG;
    if (rotate_after_s > 0) g_percall_rotate_ns.store((long long)(rotate_after_s * 1e9));
    if (idle_exit_s > 0) g_percall_idle_ns.store((long long)(idle_exit_s * 1e9));
    g_percall_mode.store(mode);
    if (mode == 0)
        for (int d = 0; d < kPercallDevices; ++d) percall_park(d);
    return TD_OK;
}

// Open-loop Poisson stream through the per-call server, measured from the
// clients' side: `clients` host threads, client c owning requests c,
// c + clients, ...; each waits for its request's arrival time, submits it the
// way td_search does and polls only its own ticket.  Latency runs from the
// arrival to the client holding the result, so it includes the time a request
// waited for its client.  Results land in results[i]; stats as for
// td_serve_open_loop (max_inflight = clients, workers = the server's warps).
TD_API int td_percall_open_loop(int device, const td_instance *instances, int count, double rate, uint64_t seed,
                                int clients, td_result *results, td_serve_stats *stats, char *err, size_t errlen) {
    if (count <= 0 || rate <= 0 || clients <= 0 || !instances || !results || device < 0 ||
        device >= kPercallDevices) {
        set_err(err, errlen, "invalid open-loop arguments");
        return TD_INVALID_ARG;
    }
    {
        std::lock_guard<std::mutex> g(g_mu);
        const int rc = ensure_device(device, err, errlen);
        if (rc != TD_OK) return rc;
    }
    // start the server before the clock runs
    td_result warm;
    td_instance probe = instances[0];
    int rc = percall_search(device, probe, &warm, err, errlen);
    if (rc != TD_OK) return rc;
    std::vector<double> arrive(count), submitted(count), completed(count);
    uint64_t st = seed;
    double t = 0;
    for (int i = 0; i < count; ++i) {
        const double u = ((splitmix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        t += -std::log(u) / rate;
        arrive[i] = t;
    }
    std::atomic<int> failed{0};
    std::string first_err;
    std::mutex err_mu;
    const auto t0 = std::chrono::steady_clock::now();
    auto now_s = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    auto client = [&](int c) {
        char cerr[256];
        for (int i = c; i < count && !failed.load(); i += clients) {
            while (now_s() < arrive[i]) {
            }
            submitted[i] = now_s();
            const int r = percall_search(device, instances[i], &results[i], cerr, sizeof cerr);
            completed[i] = now_s();
            if (r != TD_OK) {
                std::lock_guard<std::mutex> g(err_mu);
                if (!failed.exchange(1)) first_err = cerr;
            }
        }
    };
    std::vector<std::thread> th;
    for (int c = 0; c < clients; ++c) th.emplace_back(client, c);
    for (auto &x : th) x.join();
    const double wall = now_s();
    if (failed.load()) {
        set_err(err, errlen, first_err);
        return TD_TIMEOUT;
    }
    std::vector<double> lat(count);
    double wait = 0, sum = 0;
    uint64_t found = 0;
    for (int i = 0; i < count; ++i) {
        lat[i] = (completed[i] - arrive[i]) * 1e3;
        wait += (submitted[i] - arrive[i]) * 1e3;
        sum += lat[i];
        found += results[i].status == TD_FOUND;
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) { return lat[std::min<size_t>(lat.size() - 1, (size_t)(q * (lat.size() - 1) + 0.5))]; };
    if (stats) {
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        stats->p999_ms = pct(0.999);
        stats->mean_ms = sum / count;
        stats->max_ms = lat.back();
        stats->offered_per_s = count / arrive[count - 1];
        stats->served_per_s = count / wall;
        stats->wall_s = wall;
        stats->admission_wait_ms_mean = wait / count;
        stats->served = (uint64_t)count;
        stats->found = found;
        stats->max_inflight = clients;
        std::lock_guard<std::mutex> g(g_percall[device].mu);
        const PercallServer &ps = g_percall[device].srv[g_percall[device].cur];
        stats->workers = ps.grid * ps.warps - 1;
    }
    return TD_OK;
}
