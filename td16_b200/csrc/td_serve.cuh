// td_serve.cuh -- continuous-batching serving loop (included by td_engine.cu).
//
// A resident kernel serves search requests as they arrive.  The host publishes
// request r into slot r % R of a pinned, device-mapped ring and advances
// `published`; one dispatcher warp polls that counter (one PCIe read per
// poll), copies new requests into a device queue and raises `available`.
// Worker warps claim requests in arrival order, run the search with their DFS
// frames resident in shared memory, write the result into the mapped result
// ring and stamp done[r % R] = r + 1.  Requests that arrive while others run
// join the same launch: there is no batch boundary.  Every wait is bounded by
// the launch deadline; the launch ends when the host raises `stop` and every
// published request has been served.
#pragma once

struct td_serve_host_ctl {     // pinned, mapped: written by the host
    volatile unsigned long long published;
    volatile int stop;
    volatile int exit_reason;  // written by the dispatcher as it exits (TD_SERVE_EXIT_*)
};

// Why a serving launch's dispatcher stopped.
#define TD_SERVE_EXIT_IDLE 1      // no request for the idle time and no work left
#define TD_SERVE_EXIT_STOP 2      // the host asked
#define TD_SERVE_EXIT_DEADLINE 3  // the launch deadline passed

struct td_serve_dev_ctl {      // device memory: scheduler state of the launch
    unsigned long long available;
    unsigned long long claimed;
    int stop;
    int error;
    unsigned long long served;
    // where the first bounded wait gave up (1 dispatcher at the deadline,
    // 2 a taker waiting for a donated item, 3 a donor waiting for a ring slot),
    // the item index it waited for, and the pool counters at that moment
    int where;
    int snap_produced, snap_consumed, snap_active, snap_idle;
    int pad;
    long long index;
};

// Records the first wait that gave up (see td_serve_dev_ctl).
__device__ __forceinline__ void td_serve_record(td_serve_dev_ctl *dctl, const td_pool *pool, int where,
                                                long long index) {
    if (atomicCAS(&dctl->where, 0, where) == 0) {
        dctl->index = index;
        dctl->snap_produced = *(volatile const int *)&pool->produced;
        dctl->snap_consumed = *(volatile const int *)&pool->consumed;
        dctl->snap_active = *(volatile const int *)&pool->active;
        dctl->snap_idle = *(volatile const int *)&pool->idle;
    }
    atomicCAS(&dctl->error, 0, TD_ERR_TIMEOUT);
}

// Longest sleep of a polling warp between two polls (ns): the dispatcher
// waiting for requests and the workers waiting for work.
#ifndef TD_SERVE_BACKOFF_CAP
#define TD_SERVE_BACKOFF_CAP 2048u
#endif

// Move order of a serving launch: every request in the free order, every
// request in the reference order, or per request (TD_PACKED_ORDERED in the
// request's packed byte; the per-call server of td_search and
// td_search_ordered).
#define TD_SERVE_FREE 0
#define TD_SERVE_ORDERED 1
#define TD_SERVE_PER_REQUEST 2

// Worker warps take fresh requests in arrival order and, in free order, also
// donated subtrees of requests that others are searching (the batch engine's
// donation scheme over a ring of items), so one hard request does not hold a
// single warp for its whole search.  The warp that finishes a request last
// writes its result and stamps done[slot] = request + 1.  A free-order request
// restarts with another child order after restart_base x Luby expansions (0:
// never), as in the batch engine.  Each request's search also ends
// request_limit_ns after it starts (0: only the launch deadline).
template <int MODE>
__global__ void __launch_bounds__(256, 3) td_serve_kernel(const td_instance *ring, td_result *results,
                                                      volatile unsigned long long *done, unsigned ring_size,
                                                      td_serve_host_ctl *hctl, td_serve_dev_ctl *dctl,
                                                      td_instance *queue, td_inst_state *state, td_pool *pool,
                                                      td_item *items, uint32_t *ready, int item_capacity,
                                                      int grain, int max_level, int check_every, uint64_t max_exp,
                                                      uint64_t time_limit_ns, uint64_t *tt, uint32_t *tt_gen,
                                                      int tt_bits, uint32_t restart_base,
                                                      uint64_t request_limit_ns, uint64_t idle_exit_ns, int race) {
    constexpr bool ALL_ORDERED = MODE == TD_SERVE_ORDERED;
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *lut = td_smem;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem + TD_LUT_BYTES);
    td_block_init(lut, ws, warps);
    const uint64_t deadline = td_globaltimer() + time_limit_ns;
    if (blockIdx.x == 0 && warp == 0) {
        // dispatcher: host ring -> device queue, from the launch's first
        // ticket (0, or where the previous launch of a per-call server ended)
        unsigned long long avail = *(volatile unsigned long long *)&dctl->available;
        unsigned backoff = 256;
        uint64_t last_request = td_globaltimer();
        for (;;) {
            const int hstop = hctl->stop;
            const unsigned long long pub = hctl->published;  // read after stop: a stop is never ahead of its requests
            if (pub > avail) {
                for (unsigned long long r = avail + lane; r < pub; r += 32) {
                    const uint4 v = __ldcv(reinterpret_cast<const uint4 *>(&ring[r % ring_size]));
                    *reinterpret_cast<uint4 *>(&queue[r % ring_size]) = v;
                }
                __threadfence();
                __syncwarp();
                if (lane == 0) atomicExch(&dctl->available, pub);
                avail = pub;
                backoff = 256;
                last_request = td_globaltimer();
                continue;
            }
            int reason = 0;
            const uint64_t now = td_globaltimer();
            if (hstop) {
                reason = TD_SERVE_EXIT_STOP;
            } else if (now > deadline) {
                reason = TD_SERVE_EXIT_DEADLINE;
            } else if (idle_exit_ns && now - last_request > idle_exit_ns) {
                // idle: leave once every request copied so far is finished, so
                // that a device-wide synchronisation elsewhere in the process
                // waits for this launch no longer than the idle time.  A
                // request published after the last read above is not served;
                // its client sees the launch end without its result and
                // submits it again to a fresh launch.
                int quiet = 0;
                if (lane == 0)
                    quiet = *(volatile unsigned long long *)&dctl->claimed >= avail &&
                            *(volatile int *)&pool->active == 0 &&
                            *(volatile int *)&pool->consumed >= *(volatile int *)&pool->produced;
                if (__shfl_sync(TD_FULL, quiet, 0)) reason = TD_SERVE_EXIT_IDLE;
            }
            if (reason) {
                if (lane == 0) {
                    if (reason == TD_SERVE_EXIT_DEADLINE) td_serve_record(dctl, pool, 1, -1);
                    hctl->exit_reason = reason;
                    __threadfence_system();
                    atomicExch(&dctl->stop, 1);
                }
                break;
            }
            __nanosleep(backoff);
            backoff = min(backoff * 2u, (unsigned)TD_SERVE_BACKOFF_CAP);
        }
        return;
    }
    td_warp_smem &s = ws[warp];
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    td_search_limits lim;
    lim.max_expansions = max_exp ? max_exp : ~0ull;
    lim.deadline_ns = deadline;
    lim.abort_flag = nullptr;
    lim.tt = (!ALL_ORDERED && tt) ? tt + ((size_t)(blockIdx.x * warps + warp) << tt_bits) : nullptr;
    lim.tt_gen = lim.tt ? tt_gen + blockIdx.x * warps + warp : nullptr;
    lim.tt_bits = tt_bits;
    lim.restart_base = 0;  // serving searches are not restarted
    lim.cutoff = nullptr;
    lim.rank = 0;
    td_donate_ctx dc;
    dc.ring = 1;
    dc.tickets = 0;
    dc.side = 0;
    dc.race = 0;  // set per fresh request (the per-call server's race)
    dc.spawn_base = 0;
    dc.spawn_capacity = 0;
    dc.deadline_ns = deadline;
    dc.pool = pool;
    dc.items = items;
    dc.ready = ready;
    dc.epoch = 0;
    dc.capacity = item_capacity;
    dc.grain = grain;
    dc.max_level = max_level;
    dc.check_every = check_every > 0 ? check_every : 1;
    bool idle = false;
    unsigned backoff = 128;
    for (;;) {
        int kind = 0;
        long long unit = -1;
        if (lane == 0) {
            // donated subtrees of requests in flight come before fresh
            // requests: under load, fresh arrivals would otherwise keep every
            // warp busy while a started request waits for its subtrees
            if (!ALL_ORDERED) {
                const int P = *(volatile int *)&pool->produced;
                int C = *(volatile int *)&pool->consumed;
                while (C < P) {
                    const int prev = atomicCAS(&pool->consumed, C, C + 1);
                    if (prev == C) { kind = 2; unit = C; break; }
                    C = prev;
                }
            }
            if (!kind) {
                const unsigned long long av = *(volatile unsigned long long *)&dctl->available;
                unsigned long long c = *(volatile unsigned long long *)&dctl->claimed;
                while (c < av) {
                    const unsigned long long prev = atomicCAS(&dctl->claimed, c, c + 1);
                    if (prev == c) { kind = 1; unit = (long long)c; break; }
                    c = prev;
                }
            }
            if (kind) atomicAdd(&pool->active, 1);  // counts holders only
        }
        kind = __shfl_sync(TD_FULL, kind, 0);
        unit = __shfl_sync(TD_FULL, unit, 0);
        if (!kind) {
            int stop = 0;
            if (lane == 0) {
                stop = *(volatile int *)&dctl->stop;
                if (stop) {  // drain: every published request claimed and no unit left
                    const unsigned long long av2 = *(volatile unsigned long long *)&dctl->available;
                    const unsigned long long c2 = *(volatile unsigned long long *)&dctl->claimed;
                    stop = c2 >= av2 && *(volatile int *)&pool->active == 0 &&
                           *(volatile int *)&pool->consumed >= *(volatile int *)&pool->produced;
                }
                if (td_globaltimer() > deadline) stop = 1;
                if (!stop && !idle) { atomicAdd(&pool->idle, 1); idle = true; }
            }
            if (__shfl_sync(TD_FULL, stop, 0)) break;
            __nanosleep(backoff);
            backoff = min(backoff * 2u, (unsigned)TD_SERVE_BACKOFF_CAP);
            continue;
        }
        if (lane == 0 && idle) { atomicSub(&pool->idle, 1); idle = false; }
        backoff = 128;
        long long req = unit;
        td_dfs_out r;
        r.status = TD_DFS_ABORTED;
        r.depth = 0;
        r.found_move = 0;
        r.expansions = 0;
        bool run = false;
        bool ord = ALL_ORDERED;  // this unit's move order (donated subtrees: free)
        int d0 = 0;
        int side = 0;  // 1: a unit of the request's inverse (the per-call server's race)
        if (kind == 1) {
            const unsigned slot = (unsigned)(req % ring_size);
            const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(&queue[slot]));
            const td_instance x = *reinterpret_cast<const td_instance *>(&v);
            td_inst_state *st = &state[slot];
            if (lane == 0) {  // the slot's previous request is done: start afresh
                st->found = 0;
                st->expansions = 0;
                st->error = 0;
                st->pending = 1;
                __threadfence();
            }
            __syncwarp();
            if (!td_instance_ok(x) || td_triple_count(x.n_symbols) == 0) {
                td_write_result(&results[slot], td_instance_ok(x) ? TD_NOT_FOUND : TD_ERR_ARG, 0, 0, s.path, 0,
                                0, 8);
                __threadfence_system();
                __syncwarp();
                if (lane == 0) {
                    done[slot] = (unsigned long long)req + 1ull;
                    atomicAdd(&dctl->served, 1ull);
                }
            } else {
                if (MODE == TD_SERVE_PER_REQUEST) ord = (x.packed & TD_PACKED_ORDERED) != 0;
                if (ord) td_setup_root<true>(s, x, code, codeN);
                else td_setup_root<false>(s, x, code, codeN);
                run = true;
            }
        } else {
            // a donated subtree: wait until it is written, copy it, free the slot
            const int phys = (int)(unit % item_capacity);
            const uint32_t tag = td_ring_tag(unit);
            int ok = 0;
            if (lane == 0) {
                for (unsigned spin = 0; spin < (1u << 30); ++spin) {
                    if (*(volatile uint32_t *)&ready[phys] == tag) { ok = 1; break; }
                    if ((spin & 1023u) == 0 && td_globaltimer() > deadline) break;
                    __nanosleep(32);
                }
                if (!ok) td_serve_record(dctl, pool, 2, unit);
                __threadfence();
            }
            ok = __shfl_sync(TD_FULL, ok, 0);
            if (ok) {
                td_item it;
                {
                    const uint4 *src = reinterpret_cast<const uint4 *>(&items[phys]);
                    uint4 *dst = reinterpret_cast<uint4 *>(&it);
                    dst[0] = __ldcg(src);
                    dst[1] = __ldcg(src + 1);
                }
                __syncwarp();
                if (lane == 0) {
                    __threadfence();
                    atomicExch(&ready[phys], tag | 0x80000000u);
                }
                req = it.inst;
                const unsigned slot = (unsigned)(req % ring_size);
                const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(&queue[slot]));
                const td_instance x = *reinterpret_cast<const td_instance *>(&v);
                td_setup_root<false>(s, x, code, codeN);
                d0 = it.depth & 0x7f;
                side = it.depth >> 7;
                if (lane == 0) {
                    s.L[d0] = it.L;
                    s.off[d0] = it.off;
                    for (int d = 0; d < d0; ++d) s.path[d] = it.path[d];
                }
                __syncwarp();
                int stop = 0;
                if (lane == 0) stop = *(volatile int *)&state[slot].found;
                run = !__shfl_sync(TD_FULL, stop, 0);
                if (!run) {  // the request already has its witness
                    if (td_finish_unit<true>(r, &state[slot], &results[slot], s.path, side) && lane == 0) {
                        done[slot] = (unsigned long long)req + 1ull;
                        atomicAdd(&dctl->served, 1ull);
                    }
                }
            }
        }
        if (run) {
            const unsigned slot = (unsigned)(req % ring_size);
            const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(&queue[slot]));
            const td_instance x = *reinterpret_cast<const td_instance *>(&v);
            dc.inst = (uint32_t)req;
            dc.state = &state[slot];
            td_search_limits ulim = lim;
            if (request_limit_ns) ulim.deadline_ns = min(deadline, td_globaltimer() + request_limit_ns);
            // a fresh request may restart, and so may the root of its inverse; a
            // donated subtree is searched once.  A fresh free-order request of
            // the per-call server with full sorting races the search of its
            // inverse from restart attempt `race` (td_steal_kernel's race).
            ulim.restart_base = kind == 1 || d0 == 0 ? restart_base : 0;
            dc.side = side;
            dc.race = MODE == TD_SERVE_PER_REQUEST && kind == 1 && !ord && restart_base && td_inst_full(x) ? race : 0;
            if (ord) r = td_dfs<true>(s, lut, code, x.n_symbols, x.max_moves, d0, ulim, nullptr);
            else r = td_dfs<false>(s, lut, code, x.n_symbols, x.max_moves, d0, ulim, &dc);
            dc.side = 0;
            dc.race = 0;
            // a witness of the inverse becomes one of the request; one that does
            // not convert is reported as a failed replay, and one that leaves the
            // reference's move filter on the request's side is dropped
            if (side && r.status == TD_DFS_FOUND) {
                if (!td_inverse_result(s, x, r)) {
                    r.status = TD_DFS_EXHAUSTED;
                    if (lane == 0) atomicCAS(&state[slot].error, 0, TD_ERR_VERIFY);
                } else if (!td_filtered_witness(s, x, r)) {
                    r.status = TD_DFS_EXHAUSTED;
                }
            }
            if (td_finish_unit<true>(r, &state[slot], &results[slot], s.path, side) && lane == 0) {
                done[slot] = (unsigned long long)req + 1ull;
                atomicAdd(&dctl->served, 1ull);
            }
        }
        if (lane == 0) atomicSub(&pool->active, 1);
    }
    if (lane == 0 && idle) atomicSub(&pool->idle, 1);
}

// ============================================================================
// host side of the serving loop
// ============================================================================

namespace {

struct Server {
    int device = -1;
    unsigned flags = 0;
    cudaStream_t stream = nullptr;
    unsigned R = 0;
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
    int item_capacity = 0;
    uint64_t *d_tt = nullptr;  // tables of explored states, one per worker warp (free order)
    uint32_t *d_tt_gen = nullptr;  // their generation counters
    unsigned long long published = 0;
    int workers = 0;
    // per slot: ticket + 1 of the last request whose result the client took
    // (td_serve_poll); a slot is reused only after that, so a result stamp
    // is never overwritten before the client has read it
    std::vector<unsigned long long> taken;
};

void server_free(Server *sv) {
    if (!sv) return;
    if (sv->device >= 0) cudaSetDevice(sv->device);
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    if (sv->h_ring) cudaFreeHost(sv->h_ring);
    if (sv->h_res) cudaFreeHost(sv->h_res);
    if (sv->h_done) cudaFreeHost(sv->h_done);
    if (sv->h_ctl) cudaFreeHost(sv->h_ctl);
    if (sv->d_ctl) cudaFree(sv->d_ctl);
    if (sv->d_queue) cudaFree(sv->d_queue);
    if (sv->d_state) cudaFree(sv->d_state);
    if (sv->d_pool) cudaFree(sv->d_pool);
    if (sv->d_items) cudaFree(sv->d_items);
    if (sv->d_ready) cudaFree(sv->d_ready);
    if (sv->d_tt) cudaFree(sv->d_tt);
    if (sv->d_tt_gen) cudaFree(sv->d_tt_gen);
    if (sv->stream) cudaStreamDestroy(sv->stream);
    delete sv;
}

}  // namespace

// Starts a resident serving launch on `device` with a ring of `ring_size`
// requests.  flags: TD_FLAG_ORDERED for the reference order.  The launch ends
// after td_serve_close or after time_limit_s.
TD_API int td_serve_open(int device, unsigned ring_size, unsigned flags, double time_limit_s, void **handle,
                         char *err, size_t errlen) {
    if (!handle || ring_size < 2 || ring_size > (1u << 24)) {
        set_err(err, errlen, "invalid serving arguments");
        return TD_INVALID_ARG;
    }
    {
        std::lock_guard<std::mutex> g(g_mu);
        const int rc = ensure_device(device, err, errlen);
        if (rc != TD_OK) return rc;
    }
    percall_park(device);
    auto *sv = new Server();
    sv->device = device;
    sv->flags = flags;
    sv->R = ring_size;
    sv->taken.assign(ring_size, 0ull);
    auto fail = [&](cudaError_t e, int line) {
        set_err(err, errlen, cuda_msg(e, __FILE__, line));
        server_free(sv);
        return TD_CUDA_ERROR;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, __LINE__);
    const unsigned mapped = cudaHostAllocMapped | cudaHostAllocPortable;
    if ((e = cudaHostAlloc(&sv->h_ring, sizeof(td_instance) * ring_size, mapped)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostAlloc(&sv->h_res, sizeof(td_result) * ring_size, mapped)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostAlloc(&sv->h_done, sizeof(unsigned long long) * ring_size, mapped)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostAlloc(&sv->h_ctl, sizeof(td_serve_host_ctl), mapped)) != cudaSuccess) return fail(e, __LINE__);
    std::memset((void *)sv->h_done, 0, sizeof(unsigned long long) * ring_size);
    std::memset((void *)sv->h_ctl, 0, sizeof(td_serve_host_ctl));
    if ((e = cudaHostGetDevicePointer(&sv->d_ring, sv->h_ring, 0)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostGetDevicePointer(&sv->d_res, sv->h_res, 0)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostGetDevicePointer(&sv->d_done, sv->h_done, 0)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaHostGetDevicePointer(&sv->d_hctl, sv->h_ctl, 0)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMalloc(&sv->d_ctl, sizeof(td_serve_dev_ctl))) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMalloc(&sv->d_queue, sizeof(td_instance) * ring_size)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMemsetAsync(sv->d_ctl, 0, sizeof(td_serve_dev_ctl), sv->stream)) != cudaSuccess) return fail(e, __LINE__);
    // donation ring: 64 items per ring slot of requests, at least 2^16
    sv->item_capacity = (int)std::min<size_t>(1u << 24, std::max<size_t>(1u << 16, (size_t)ring_size * 64));
    if ((e = cudaMalloc(&sv->d_state, sizeof(td_inst_state) * ring_size)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMalloc(&sv->d_pool, sizeof(td_pool))) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMalloc(&sv->d_items, sizeof(td_item) * sv->item_capacity)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMalloc(&sv->d_ready, sizeof(uint32_t) * sv->item_capacity)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMemsetAsync(sv->d_pool, 0, sizeof(td_pool), sv->stream)) != cudaSuccess) return fail(e, __LINE__);
    if ((e = cudaMemsetAsync(sv->d_ready, 0, sizeof(uint32_t) * sv->item_capacity, sv->stream)) != cudaSuccess)
        return fail(e, __LINE__);
    LaunchCfg cfg;
    {
        const int rc = launch_cfg(device, &cfg, err, errlen);
        if (rc != TD_OK) {
            server_free(sv);
            return rc;
        }
    }
    const int warps = cfg.warps;
    const size_t smem = smem_bytes(warps);
    int per_sm = 0;
    const bool ordered = flags & TD_FLAG_ORDERED;
    if (ordered) {
        if ((e = cudaFuncSetAttribute(td_serve_kernel<TD_SERVE_ORDERED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return fail(e, __LINE__);
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, td_serve_kernel<TD_SERVE_ORDERED>, warps * 32, smem)) != cudaSuccess) return fail(e, __LINE__);
    } else {
        if ((e = cudaFuncSetAttribute(td_serve_kernel<TD_SERVE_FREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return fail(e, __LINE__);
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, td_serve_kernel<TD_SERVE_FREE>, warps * 32, smem)) != cudaSuccess) return fail(e, __LINE__);
    }
    const int grid = g_dev[device].sms * std::max(1, per_sm);
    sv->workers = grid * warps - 1;
    const int tt_bits = ordered ? 0 : cfg.tt_bits;
    if (tt_bits > 0) {
        const size_t tt_bytes = ((size_t)grid * warps << tt_bits) * sizeof(uint64_t);
        if ((e = cudaMalloc(&sv->d_tt, tt_bytes)) != cudaSuccess) return fail(e, __LINE__);
        if ((e = cudaMalloc(&sv->d_tt_gen, (size_t)grid * warps * sizeof(uint32_t))) != cudaSuccess)
            return fail(e, __LINE__);
        if ((e = cudaMemsetAsync(sv->d_tt, 0, tt_bytes, sv->stream)) != cudaSuccess) return fail(e, __LINE__);
        if ((e = cudaMemsetAsync(sv->d_tt_gen, 0, (size_t)grid * warps * sizeof(uint32_t), sv->stream)) !=
            cudaSuccess)
            return fail(e, __LINE__);
    }
    const uint64_t limit_ns = (uint64_t)((time_limit_s > 0 ? time_limit_s : 60.0) * 1e9);
    if (ordered)
        td_serve_kernel<TD_SERVE_ORDERED><<<grid, warps * 32, smem, sv->stream>>>(
            sv->d_ring, sv->d_res, sv->d_done, ring_size, sv->d_hctl, sv->d_ctl, sv->d_queue, sv->d_state,
            sv->d_pool, sv->d_items, sv->d_ready, sv->item_capacity, cfg.serve_grain, cfg.serve_split_level,
            cfg.serve_check_every, 0, limit_ns, nullptr, nullptr, 0, 0u, 0ull, 0ull, 0);
    else
        td_serve_kernel<TD_SERVE_FREE><<<grid, warps * 32, smem, sv->stream>>>(
            sv->d_ring, sv->d_res, sv->d_done, ring_size, sv->d_hctl, sv->d_ctl, sv->d_queue, sv->d_state,
            sv->d_pool, sv->d_items, sv->d_ready, sv->item_capacity, cfg.serve_grain, cfg.serve_split_level,
            cfg.serve_check_every, 0, limit_ns, sv->d_tt, sv->d_tt_gen, tt_bits, 0u, 0ull, 0ull, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, __LINE__);
    *handle = sv;
    return TD_OK;
}

TD_API int td_serve_workers(void *handle) { return handle ? static_cast<Server *>(handle)->workers : 0; }

// Publishes one request; *ticket receives its sequence number.  Returns
// TD_OVERFLOW when the ring still holds ring_size unfinished requests.
TD_API int td_serve_submit(void *handle, const td_instance *x, unsigned long long *ticket) {
    auto *sv = static_cast<Server *>(handle);
    const unsigned long long r = sv->published;
    const unsigned slot = (unsigned)(r % sv->R);
    if (r >= sv->R && __atomic_load_n(&sv->taken[slot], __ATOMIC_ACQUIRE) != r - sv->R + 1) return TD_OVERFLOW;
    sv->h_ring[slot] = *x;
    __atomic_store_n(&sv->h_done[slot], 0ull, __ATOMIC_RELAXED);
    __atomic_thread_fence(__ATOMIC_SEQ_CST);
    sv->published = r + 1;
    __atomic_store_n(const_cast<unsigned long long *>(&sv->h_ctl->published), r + 1, __ATOMIC_RELEASE);
    if (ticket) *ticket = r;
    return TD_OK;
}

// 1 and the result when request `ticket` is done, 0 while it runs.
TD_API int td_serve_poll(void *handle, unsigned long long ticket, td_result *out) {
    auto *sv = static_cast<Server *>(handle);
    const unsigned slot = (unsigned)(ticket % sv->R);
    if (__atomic_load_n(&sv->h_done[slot], __ATOMIC_ACQUIRE) != ticket + 1) return 0;
    if (out) std::memcpy(out, (const void *)&sv->h_res[slot], sizeof(td_result));
    __atomic_store_n(&sv->taken[slot], ticket + 1, __ATOMIC_RELEASE);
    return 1;
}

// Stops the launch after every published request is served; returns
// TD_TIMEOUT if the launch hit its deadline.
TD_API int td_serve_close(void *handle, char *err, size_t errlen) {
    auto *sv = static_cast<Server *>(handle);
    if (!sv) return TD_INVALID_ARG;
    __atomic_store_n(const_cast<int *>(&sv->h_ctl->stop), 1, __ATOMIC_RELEASE);
    cudaSetDevice(sv->device);
    cudaError_t e = cudaStreamSynchronize(sv->stream);
    td_serve_dev_ctl ctl;
    td_pool pool;
    std::memset(&ctl, 0, sizeof ctl);
    std::memset(&pool, 0, sizeof pool);
    if (e == cudaSuccess) e = cudaMemcpy(&ctl, sv->d_ctl, sizeof ctl, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&pool, sv->d_pool, sizeof pool, cudaMemcpyDeviceToHost);
    server_free(sv);
    if (e != cudaSuccess) {
        set_err(err, errlen, cuda_msg(e, __FILE__, __LINE__));
        return TD_CUDA_ERROR;
    }
    if (ctl.error || pool.error) {
        char msg[320];
        std::snprintf(msg, sizeof msg,
                      "serving launch deadline reached (wait %d, item %lld; produced %d consumed %d active %d "
                      "idle %d; requests available %llu claimed %llu served %llu; donor ring wait %s)",
                      ctl.where, ctl.index, ctl.snap_produced, ctl.snap_consumed, ctl.snap_active, ctl.snap_idle,
                      ctl.available, ctl.claimed, ctl.served, pool.error ? "expired" : "ok");
        set_err(err, errlen, msg);
        return TD_TIMEOUT;
    }
    return TD_OK;
}

struct td_serve_stats {
    double p50_ms, p99_ms, p999_ms, mean_ms, max_ms;
    double offered_per_s, served_per_s, wall_s;
    double admission_wait_ms_mean;
    uint64_t served, found;
    int workers, max_inflight;
};

// Open-loop experiment: `count` requests (instances[]) arrive as a Poisson
// process of `rate` per second (seeded); each is admitted when the in-flight
// frame bytes (max_moves x frame_bytes per request) fit `pool_bytes` and a
// worker slot is free, then served by the resident launch.  Latency runs from
// arrival to the host observing the result.  Results land in results[i].
TD_API int td_serve_open_loop(int device, const td_instance *instances, int count, double rate, uint64_t seed,
                              uint64_t pool_bytes, unsigned flags, td_result *results, td_serve_stats *stats,
                              char *err, size_t errlen) {
    if (count <= 0 || rate <= 0) {
        set_err(err, errlen, "invalid open-loop arguments");
        return TD_INVALID_ARG;
    }
    void *h = nullptr;
    const unsigned R = 1u << 16;
    const double limit_s = std::max(30.0, 4.0 * count / rate + 30.0);
    int rc = td_serve_open(device, R, flags, limit_s, &h, err, errlen);
    if (rc != TD_OK) return rc;
    auto *sv = static_cast<Server *>(h);
    const size_t frame = sizeof(td_warp_smem) / TD_MAX_DEPTH;
    const int max_inflight = std::min<int>(sv->workers, (int)R - 1);
    // Poisson arrivals: exponential gaps from splitmix64 draws
    std::vector<double> arrive(count);
    uint64_t st = seed;
    double t = 0;
    for (int i = 0; i < count; ++i) {
        const double u = ((splitmix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        t += -std::log(u) / rate;
        arrive[i] = t;
    }
    std::vector<double> admitted(count, 0), completed(count, 0);
    std::vector<unsigned long long> ticket(count, 0);
    std::atomic<int> next_done{0};
    std::atomic<long long> inflight_bytes{0};
    std::atomic<int> inflight{0};
    std::atomic<bool> failed{false};
    const auto t0 = std::chrono::steady_clock::now();
    auto now_s = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    std::vector<char> is_done(count, 0);
    std::atomic<int> submitted{0};
    std::thread poller([&] {
        int remaining = count;
        int lo = 0;
        while (remaining > 0 && !failed.load()) {
            const int hi = submitted.load(std::memory_order_acquire);
            bool progress = false;
            for (int i = lo; i < hi; ++i) {
                if (is_done[i]) continue;
                if (td_serve_poll(h, ticket[i], &results[i])) {
                    completed[i] = now_s();
                    is_done[i] = 1;
                    --remaining;
                    inflight_bytes.fetch_sub((long long)(instances[i].max_moves * frame));
                    inflight.fetch_sub(1);
                    progress = true;
                }
            }
            while (lo < hi && is_done[lo]) ++lo;
            if (!progress) std::this_thread::yield();
            if (now_s() > limit_s) failed = true;
        }
        next_done = count - remaining;
    });
    for (int i = 0; i < count && !failed.load(); ++i) {
        while (now_s() < arrive[i]) {
        }
        const long long need = (long long)(instances[i].max_moves * frame);
        // a request larger than the pool still runs once nothing else is in flight
        while (!failed.load() && inflight.load() > 0 &&
               (inflight.load() >= max_inflight || inflight_bytes.load() + need > (long long)pool_bytes)) {
        }
        admitted[i] = now_s();
        inflight.fetch_add(1);
        inflight_bytes.fetch_add(need);
        unsigned long long tk;
        while (td_serve_submit(h, &instances[i], &tk) != TD_OK && !failed.load()) {
        }
        ticket[i] = tk;
        submitted.store(i + 1, std::memory_order_release);
    }
    poller.join();
    const double wall = now_s();
    rc = td_serve_close(h, err, errlen);
    if (failed.load() && rc == TD_OK) {
        set_err(err, errlen, "open-loop run exceeded its time limit");
        rc = TD_TIMEOUT;
    }
    if (rc != TD_OK) return rc;
    std::vector<double> lat(count);
    double wait = 0;
    uint64_t found = 0;
    for (int i = 0; i < count; ++i) {
        lat[i] = (completed[i] - arrive[i]) * 1e3;
        wait += (admitted[i] - arrive[i]) * 1e3;
        found += results[i].status == TD_FOUND;
    }
    std::vector<double> sorted = lat;
    std::sort(sorted.begin(), sorted.end());
    auto pct = [&](double q) { return sorted[std::min<size_t>(sorted.size() - 1, (size_t)(q * (sorted.size() - 1) + 0.5))]; };
    if (stats) {
        double sum = 0;
        for (double v : lat) sum += v;
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        stats->p999_ms = pct(0.999);
        stats->mean_ms = sum / count;
        stats->max_ms = sorted.back();
        stats->offered_per_s = count / arrive[count - 1];
        stats->served_per_s = count / wall;
        stats->wall_s = wall;
        stats->admission_wait_ms_mean = wait / count;
        stats->served = (uint64_t)count;
        stats->found = found;
        stats->workers = sv->workers;
        stats->max_inflight = max_inflight;
    }
    return TD_OK;
}
