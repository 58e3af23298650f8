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
    int grid = 0;
};

struct PercallDevice {
    std::mutex mu;
    PercallServer srv[2];
    int cur = 0;
};

PercallDevice g_percall[kPercallDevices];
std::atomic<int> g_percall_mode{1};  // 1: resident server, 0: one launch per call
std::atomic<long long> g_percall_rotate_ns{300000000000ll};

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
        if (ps.d_tt) TD_CHECK(cudaFree(ps.d_tt));
        if (ps.d_tt_gen) TD_CHECK(cudaFree(ps.d_tt_gen));
        ps.d_tt = nullptr;
        ps.d_tt_gen = nullptr;
        ps.tt_warps = 0;
        const size_t words = (size_t)grid * warps << cfg.tt_bits;
        TD_CHECK(cudaMalloc(&ps.d_tt, words * sizeof(uint64_t)));
        TD_CHECK(cudaMalloc(&ps.d_tt_gen, (size_t)grid * warps * sizeof(uint32_t)));
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
        life_ns, cfg.tt_bits > 0 ? ps.d_tt : nullptr, ps.d_tt_gen, cfg.tt_bits, cfg.restart_base, request_ns);
    TD_CHECK(cudaGetLastError());
    ps.grid = grid;
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
    for (auto &pd : g_percall) {
        std::lock_guard<std::mutex> g(pd.mu);
        for (auto &ps : pd.srv) {
            percall_stop(ps);
            percall_free(ps);
        }
        pd.cur = 0;
    }
}

// One blocking search through the device's per-call server.  `x` is the
// prepared instance (TD_PACKED_ORDERED set for the reference order).
int percall_search(int device, const td_instance &x, td_result *out, char *err, size_t errlen) {
    if (device < 0 || device >= kPercallDevices) {
        set_err(err, errlen, "device ordinal out of range for the per-call server");
        return TD_INVALID_ARG;
    }
    PercallDevice &pd = g_percall[device];
    PercallServer *ps;
    unsigned long long ticket;
    unsigned gen;
    {
        std::lock_guard<std::mutex> g(pd.mu);
        TD_CHECK(cudaSetDevice(device));
        ps = &pd.srv[pd.cur];
        if (ps->running && cudaStreamQuery(ps->stream) != cudaErrorNotReady) {
            // the launch has ended (its deadline, or an error): start afresh
            cudaStreamSynchronize(ps->stream);
            ps->running = false;
        }
        if (ps->running && std::chrono::steady_clock::now() - ps->started > percall_rotate_after()) {
            PercallServer &next = pd.srv[1 - pd.cur];
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
        ticket = ps->published;
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
        gen = ps->generation.load();
    }
    const unsigned slot = (unsigned)(ticket % kPercallRing);
    int rc = TD_OK;
    for (unsigned spin = 1;; ++spin) {
        if (__atomic_load_n(&ps->h_done[slot], __ATOMIC_ACQUIRE) == ticket + 1) {
            std::memcpy(out, (const void *)&ps->h_res[slot], sizeof(td_result));
            break;
        }
        if ((spin & 1023u) == 0) {
            // the launch this request went to has ended (its deadline, an
            // error) or been replaced after it ended: the request is lost
            const cudaError_t q = ps->generation.load() != gen ? cudaSuccess : cudaStreamQuery(ps->stream);
            if (q != cudaErrorNotReady) {
                if (__atomic_load_n(&ps->h_done[slot], __ATOMIC_ACQUIRE) == ticket + 1) continue;
                if (q == cudaSuccess) {
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
    return rc;
}

}  // namespace

// Per-call searches (td_search, td_search_ordered): mode 1 (default) through
// the device's resident server, 0 with one launch per call on the slot's
// stream.  rotate_after_s > 0 sets the age at which a server launch is
// replaced by a fresh one (default 300 s); 0 keeps the current setting.
TD_API int td_configure_percall(int mode, double rotate_after_s) {
    if ((mode != 0 && mode != 1) || rotate_after_s < 0) return TD_INVALID_ARG;
    if (rotate_after_s > 0) g_percall_rotate_ns.store((long long)(rotate_after_s * 1e9));
    g_percall_mode.store(mode);
    if (mode == 0)
        for (int d = 0; d < kPercallDevices; ++d) percall_park(d);
    return TD_OK;
}
