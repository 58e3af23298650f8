// td_engine.cu -- kernels and host C ABI of the B200 witness-search engine.
//
// Kernels
//   td_plain_kernel       one warp per instance, one launch per batch
//   td_persistent_kernel  resident grid; warps claim instances with an atomic
//                         ticket (steal granularity = instances per claim)
//   td_validate_kernel    replays witnesses in pinned form
// Host
//   slots (stream + completion event + device scratch per slot) with the
//   reference's initSlots / searchForSortingSeq semantics, batch entry points,
//   instance preparation and the seeded synthetic generator.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "td_kernels.cuh"

#define TD_API extern "C" __attribute__((visibility("default")))

// mirrors include/td16_b200.h
#define TD_OK 0
#define TD_NOT_FOUND_RC 1
#define TD_OVERFLOW 2
#define TD_CUDA_ERROR 3
#define TD_INVALID_ARG 4
#define TD_TIMEOUT 5
#define TD_FLAG_PLAIN 2u
#define TD_FLAG_VERIFY 4u
#define TD_ERR_VERIFY (-6)

struct td_batch_stats {
    uint64_t expansions, found, not_found, errors;
    float kernel_ms;
    uint32_t launches;
    uint64_t donations, donated_items;
    uint64_t races;
};

static_assert(sizeof(td_instance) == 16, "td_instance layout");
static_assert(sizeof(td_result) == 32, "td_result layout");

// ============================================================================
// kernels
// ============================================================================

#define TD_LUT_BYTES 4096
#define TD_TT_BITS 12  // default: 4096 explored-state entries (32 KiB) per warp of a free-order launch
#define TD_RESTART_BASE 16  // default base of the free order's restart budgets (expansions)

// Class table (td_class_of_index for every 12-bit index), filled by the host.
__device__ __align__(16) uint8_t td_lut_global[TD_LUT_BYTES];

// Copies the class table into shared memory (kernels of the reference order;
// `lut` is null in the free-order batch kernel, which does not use it).
__device__ __forceinline__ void td_block_init(uint8_t *lut, td_warp_smem *ws, int warps) {
    if (lut) {
        const uint4 *src = reinterpret_cast<const uint4 *>(td_lut_global);
        uint4 *dst = reinterpret_cast<uint4 *>(lut);
        for (int i = threadIdx.x; i < TD_LUT_BYTES / 16; i += blockDim.x) dst[i] = src[i];
    }
    for (int w = 0; w < warps; ++w)
        for (int b = threadIdx.x; b < TD_PT_STRIDE; b += blockDim.x) ws[w].pt[TD_PT_DUMMY + b] = 0;
    __syncthreads();
}

__device__ __forceinline__ td_search_limits td_make_limits(uint64_t max_exp, uint64_t time_limit_ns,
                                                           const int *abort_flag) {
    td_search_limits lim;
    lim.max_expansions = max_exp ? max_exp : ~0ull;
    lim.deadline_ns = time_limit_ns ? td_globaltimer() + time_limit_ns : 0;
    lim.abort_flag = abort_flag;
    lim.tt = nullptr;
    lim.tt_gen = nullptr;
    lim.tt_bits = 0;
    lim.restart_base = 0;
    lim.cutoff = nullptr;
    lim.rank = 0;
    return lim;
}

template <bool ORDERED>
__global__ void __launch_bounds__(256) td_plain_kernel(const td_instance *__restrict__ in,
                                                      td_result *__restrict__ out, int count,
                                                      uint64_t max_exp, uint64_t time_limit_ns) {
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5;
    uint8_t *lut = td_smem;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem + TD_LUT_BYTES);
    td_block_init(lut, ws, warps);
    const int idx = blockIdx.x * warps + warp;
    if (idx >= count) return;
    const td_search_limits lim = td_make_limits(max_exp, time_limit_ns, nullptr);
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    const td_instance x = in[idx];
    td_warp_search<ORDERED>(x, &out[idx], ws[warp], lut, code, codeN, lim);
}

// hard_count / hard_list (or null): instances that end with TD_ERR_BUDGET are
// listed there, for the split pass of the reference order (td_split_*).
template <bool ORDERED>
__global__ void __launch_bounds__(256) td_persistent_kernel(const td_instance *__restrict__ in,
                                                           td_result *__restrict__ out, int count,
                                                           int *ticket, int grain, uint64_t max_exp,
                                                           uint64_t time_limit_ns, int *hard_count = nullptr,
                                                           int *hard_list = nullptr) {
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *lut = td_smem;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem + TD_LUT_BYTES);
    td_block_init(lut, ws, warps);
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    const td_search_limits lim = td_make_limits(max_exp, time_limit_ns, nullptr);
    for (;;) {
        int first = 0;
        if (lane == 0) first = atomicAdd(ticket, grain);
        first = __shfl_sync(TD_FULL, first, 0);
        if (first >= count) break;
        const int last = min(count, first + grain);
        for (int idx = first; idx < last; ++idx) {
            const td_instance x = in[idx];
            const int st = td_warp_search<ORDERED>(x, &out[idx], ws[warp], lut, code, codeN, lim);
            if (hard_list && st == TD_ERR_BUDGET && lane == 0) hard_list[atomicAdd(hard_count, 1)] = idx;
        }
    }
}

// ---- the reference order, split below the root ------------------------------
//
// The reference's single-queue order is one depth-first walk, so a search
// that runs long is a long serial chain on one warp while the rest of the GPU
// idles: the tail of an ordered batch.  The walk visits the root's children
// c_0, c_1, ... in a fixed order and exhausts each subtree before the next, so
// its witness is the one it meets in the first subtree that holds any, and it
// meets it there exactly as that subtree's own walk does.  The subtrees can
// therefore be searched at once, one warp each, and joined in rank order: the
// witness is the found one of lowest rank r, and the walk's expansion count
// is 1 (the root) plus the expansions of subtrees 0..r, the earlier ones run
// to exhaustion.  Both equal the one-warp walk's, bit for bit.  A subtree
// that ranks after a found one stops early; its result is never read.
//
// Only instances that a first one-warp pass did not finish within
// TD_SPLIT_BUDGET expansions take this path (td_persistent_kernel lists
// them); the rest keep the first pass's results.  Passes: td_split_roots_kernel
// lists each such root's children in visiting order, td_split_kernel searches
// the subtrees rank-major (the first subtree of every instance, then the
// second, ...), td_split_join_kernel writes the joined results.

#define TD_SPLIT_BUDGET 64        // default expansions of the one-warp first pass (td_configure_split)
#define TD_SPLIT_RECORDS (1 << 20)  // default subtree records per launch (32 MiB)
#define TD_SPLIT_SKIPPED 2        // a subtree result that is never read

struct td_split_ctl {
    int hard;                   // instances the first pass did not finish
    int max_rank;               // most children of a split root
    int items_used;             // subtree records reserved
    unsigned long long ticket;  // units of td_split_kernel claimed
};

// Per listed instance h (grid-stride over warps): its root's children in the
// walk's visiting order, as position triples with bit 15 set for a child
// accepted on visit, at kids[base[h] ..], nkids[h] of them; nkids[h] = -1
// when the record space is full (that instance then runs whole).  Also
// clears the instance's cutoff.
__global__ void __launch_bounds__(256) td_split_roots_kernel(const td_instance *__restrict__ in,
                                                            const int *__restrict__ hard_list, td_split_ctl *ctl,
                                                            uint16_t *__restrict__ kids, int *__restrict__ base,
                                                            int *__restrict__ nkids, int *__restrict__ cutoff,
                                                            int records) {
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *lut = td_smem;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem + TD_LUT_BYTES);
    td_block_init(lut, ws, warps);
    td_warp_smem &s = ws[warp];
    const int H = *(volatile int *)&ctl->hard;
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    for (int h = blockIdx.x * warps + warp; h < H; h += gridDim.x * warps) {
        const td_instance x = in[hard_list[h]];
        td_setup_root<true>(s, x, code, codeN);
        const int N = x.n_symbols, T = td_triple_count(N), tb = td_tri_base(N);
        // count the children, reserve their records, then list them (the
        // walk consumes the root's outcome words, so the root is evaluated twice)
        int c = 0, at = -1;
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && at < 0) break;
            const int odd = td_prepare_node(s, s.L[0], s.off[0], N);
            td_evaluate(s, lut, code, (T + 31) >> 5, 0, odd, x.max_moves);
            int k = 0;
            for (;;) {
                int accepted;
                const int u = td_next_child(s, 0, &accepted);
                if (u < 0) break;
                if (pass == 1 && lane == 0)
                    kids[at + k] = (uint16_t)(td_tri_table[tb + T - 1 - u] | (accepted ? 0x8000u : 0u));
                ++k;
            }
            if (pass == 0) {
                c = k;
                if (lane == 0) {
                    at = atomicAdd(&ctl->items_used, c);
                    if (at > records - c) at = -1;
                }
                at = __shfl_sync(TD_FULL, at, 0);
            }
        }
        if (lane == 0) {
            base[h] = at;
            nkids[h] = at < 0 ? -1 : c;
            cutoff[h] = 0x7fffffff;  // no witness yet
            if (at >= 0) atomicMax(&ctl->max_rank, c);
        }
        __syncwarp();
    }
}

// Resident grid over the units of the split, rank-major: unit u is rank
// r = u / H of listed instance h = u % H, i.e. subtree r of its root, or for
// an instance without records (nkids[h] < 0) the whole search at r = 0 (so
// the longest units start first).
__global__ void __launch_bounds__(256) td_split_kernel(const td_instance *__restrict__ in,
                                                      td_result *__restrict__ out, const int *__restrict__ hard_list,
                                                      td_split_ctl *ctl, const uint16_t *__restrict__ kids,
                                                      const int *__restrict__ base, const int *__restrict__ nkids,
                                                      int *cutoff, td_result *__restrict__ items,
                                                      uint64_t time_limit_ns) {
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *lut = td_smem;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem + TD_LUT_BYTES);
    td_block_init(lut, ws, warps);
    td_warp_smem &s = ws[warp];
    const int H = *(volatile int *)&ctl->hard;
    const int R = max(1, *(volatile int *)&ctl->max_rank);
    const unsigned long long units = (unsigned long long)H * (unsigned long long)R;
    td_search_limits lim = td_make_limits(0, time_limit_ns, nullptr);
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    for (;;) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(&ctl->ticket, 1ull);
        u = __shfl_sync(TD_FULL, u, 0);
        if (u >= units) break;
        const int r = (int)(u / (unsigned long long)H), h = (int)(u % (unsigned long long)H);
        const int nk = nkids[h];
        if (nk < 0) {
            if (r == 0) {
                const int idx = hard_list[h];
                lim.cutoff = nullptr;
                td_warp_search<true>(in[idx], &out[idx], s, lut, code, codeN, lim);
            }
            continue;
        }
        if (r >= nk) continue;  // that root has fewer children; the join reads only nkids[h]
        td_result *it = &items[base[h] + r];
        if (*(volatile int *)&cutoff[h] < r) {
            td_write_result(it, TD_SPLIT_SKIPPED, 0, 0, s.path, 0, 0, 8);
            continue;
        }
        const uint32_t kid = kids[base[h] + r];
        const uint32_t t = kid & 0x7fffu;
        const td_instance x = in[hard_list[h]];
        td_setup_root<true>(s, x, code, codeN);
        const int N = x.n_symbols;
        if (lane == 0) s.path[0] = (uint16_t)t;
        __syncwarp();
        if (kid & 0x8000u) {  // accepted on visit: the one-move witness
            td_write_result(it, TD_FOUND, 1, (uint16_t)t, s.path, 0, 0, 8);
            if (lane == 0) atomicMin(&cutoff[h], r);
            continue;
        }
        uint64_t nL;
        int noff;
        td_apply_move(s.L[0], s.off[0], N, t & 31, (t >> 5) & 31, (t >> 10) & 31, &nL, &noff);
        if (lane == 0) {
            s.L[1] = nL;
            s.off[1] = (uint8_t)noff;
        }
        __syncwarp();
        lim.cutoff = &cutoff[h];
        lim.rank = r;
        const td_dfs_out d = td_dfs<true>(s, lut, code, N, x.max_moves, 1, lim, nullptr);
        int status = TD_NOT_FOUND;
        if (d.status == TD_DFS_FOUND) status = TD_FOUND;
        else if (d.status == TD_DFS_ABORTED) status = TD_SPLIT_SKIPPED;
        else if (d.status == TD_DFS_TIMEOUT) status = TD_ERR_TIMEOUT;
        td_write_result(it, status, status == TD_FOUND ? d.depth : 0, d.found_move, s.path, d.expansions, 0, 8);
        if (status == TD_FOUND && lane == 0) atomicMin(&cutoff[h], r);
    }
}

// The joined result of each split instance, as the one-warp walk would give it.
__global__ void td_split_join_kernel(const int *__restrict__ hard_list, const td_split_ctl *ctl,
                                     const int *__restrict__ base, const int *__restrict__ nkids,
                                     const td_result *__restrict__ items, td_result *__restrict__ out) {
    const int H = *(volatile const int *)&ctl->hard;
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < H; h += gridDim.x * blockDim.x) {
        const int nk = nkids[h];
        if (nk < 0) continue;  // searched whole
        td_result res;
        memset(&res, 0, sizeof res);
        res.status = TD_NOT_FOUND;
        uint64_t exp = 1;  // the root
        for (int r = 0; r < nk; ++r) {
            const td_result it = items[base[h] + r];
            if (it.status == TD_FOUND) {
                res = it;
                exp += it.expansions;
                break;
            }
            if (it.status != TD_NOT_FOUND) {  // a subtree before any witness timed out
                res.status = TD_ERR_TIMEOUT;
                break;
            }
            exp += it.expansions;
        }
        res.expansions = exp > 0xffffffffull ? 0xffffffffu : (uint32_t)exp;
        out[hard_list[h]] = res;
    }
}

// Resident grid with work donation (free move order).  Warps take fresh
// instances by ticket; a warp that finds neither tickets nor items counts
// itself idle, and busy warps then hand the remaining children of their
// shallowest DFS level to the item array.  Every wait is bounded by the
// launch deadline; the launch ends when no ticket, item or unit is left.
// Ends one unit of a shared search: records a found witness (first finder
// wins), and the unit that finishes the search last writes the final status
// and the summed expansions.  Returns 1 in the warp that finished last.
// `side` 1 marks a unit of the inverse instance's search (td_steal_kernel's
// race; its witness is already in the instance's positions and keeps the
// reference's move filter there).  When the last unit of the instance's own
// side ends with no witness and no error recorded, its whole filtered tree
// was searched: the instance has no witness within the bound, and found = 2
// stops the inverse's side.  The inverse's side never decides "no witness":
// the filter applies to a different tree there.
// HOST_OUT: `out` is host memory mapped into the device (the serving loop), so
// the fences are system-scope; the batch engine's results are device memory,
// where device-scope fences order the same writes at a fraction of the cost.
template <bool HOST_OUT>
__device__ __forceinline__ void td_unit_fence() {
    if (HOST_OUT) __threadfence_system();
    else __threadfence();
}

template <bool HOST_OUT>
__device__ __forceinline__ int td_finish_unit(const td_dfs_out &r, td_inst_state *st, td_result *out,
                                              const uint16_t *path, int side = 0) {
    const int lane = threadIdx.x & 31;
    int win = 0, last = 0;
    if (lane == 0) {
        atomicAdd(&st->expansions, r.expansions);
        if (r.status == TD_DFS_FOUND) win = atomicCAS(&st->found, 0, 1) == 0;
        if (r.status == TD_DFS_TIMEOUT) atomicCAS(&st->error, 0, TD_ERR_TIMEOUT);
        if (r.status == TD_DFS_BUDGET) atomicCAS(&st->error, 0, TD_ERR_BUDGET);
    }
    win = __shfl_sync(TD_FULL, win, 0);
    if (win) td_write_result(out, TD_FOUND, r.depth, r.found_move, path, 0, 0, 7);
    __syncwarp();
    if (lane == 0) {
        td_unit_fence<HOST_OUT>();
        const int unit = side ? 1 << 16 : 1;
        const int before = atomicSub(&st->pending, unit);
        last = before == unit;
        if (last) td_unit_fence<HOST_OUT>();
        else if (!side && ((before - unit) & 0x0000ffff) == 0 && *(volatile int *)&st->found == 0 &&
                 *(volatile int *)&st->error == 0)
            atomicCAS(&st->found, 0, 2);
    }
    last = __shfl_sync(TD_FULL, last, 0);
    if (last) {
        int found = 0, err = 0;
        unsigned exp = 0;
        if (lane == 0) {
            found = *(volatile int *)&st->found;
            err = *(volatile int *)&st->error;
            exp = *(volatile unsigned *)&st->expansions;
        }
        found = __shfl_sync(TD_FULL, found, 0);
        err = __shfl_sync(TD_FULL, err, 0);
        exp = __shfl_sync(TD_FULL, exp, 0);
        if (found == 1) td_write_result(out, TD_FOUND, 0, 0, path, exp, 7, 8);
        else td_write_result(out, found == 2 || !err ? TD_NOT_FOUND : err, 0, 0, path, exp, 0, 8);
        __syncwarp();
    }
    return last;
}

#ifndef TD_STEAL_MIN_BLOCKS
#define TD_STEAL_MIN_BLOCKS 4  // resident blocks of 8 warps per SM the register budget is sized for
#endif
__global__ void __launch_bounds__(256, TD_STEAL_MIN_BLOCKS) td_steal_kernel(const td_instance *__restrict__ in,
                                                      td_result *__restrict__ out, int count, td_pool *pool,
                                                      td_item *items, uint32_t *ready, const uint32_t *epoch_ptr,
                                                      int capacity, td_inst_state *state, int grain,
                                                      int max_level, int check_every, uint64_t time_limit_ns,
                                                      uint64_t *tt, uint32_t *tt_gen, int tt_bits,
                                                      uint32_t restart_base, uint64_t max_exp,
                                                      unsigned max_backoff_ns, int race, int spawn_base) {
    extern __shared__ __align__(16) uint8_t td_smem[];
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // free order only: no class table, the warp frames start the block's shared memory
    const uint8_t *lut = nullptr;
    td_warp_smem *ws = reinterpret_cast<td_warp_smem *>(td_smem);
    td_block_init(nullptr, ws, warps);
    td_warp_smem &s = ws[warp];
    uint32_t code[TD_MAX_STEPS];
    int codeN = -1;
    // the expansion budget bounds each unit (the root search and each donated
    // subtree); an instance without a witness whose unit ran out reports
    // TD_ERR_BUDGET
    td_search_limits lim = td_make_limits(max_exp, time_limit_ns, nullptr);
    lim.restart_base = restart_base;
    if (tt) {
        lim.tt = tt + ((size_t)(blockIdx.x * warps + warp) << tt_bits);
        lim.tt_gen = tt_gen + blockIdx.x * warps + warp;
        lim.tt_bits = tt_bits;
    }
    td_donate_ctx dc;
    dc.pool = pool;
    dc.items = items;
    dc.ready = ready;
    const uint32_t epoch = *epoch_ptr;  // bumped by td_epoch_kernel before this launch
    dc.epoch = epoch;
    // race: donated items use slots [0, spawn_base), queued inverse roots the rest
    dc.capacity = race ? spawn_base : capacity;
    dc.spawn_base = spawn_base;
    dc.spawn_capacity = race ? capacity - spawn_base : 0;
    dc.side = 0;
    dc.race = 0;
    dc.grain = grain;
    dc.max_level = max_level;
    dc.check_every = check_every > 0 ? check_every : 1;
    dc.ring = 0;
    dc.tickets = 1;
    dc.deadline_ns = lim.deadline_ns;
    unsigned backoff = 64;
    // Claims.  A warp takes fresh instances by ticket while any are left, then
    // one item ticket (fetch-and-add: it never fails) and waits until item
    // `ticket` has been produced; items go to the waiting warps in ticket
    // order.  (One compare-and-swap per claim attempt instead made thousands
    // of idle warps fail on one counter, so the long searches at the end of a
    // launch, split into thousands of items, were served a few hundred
    // thousand items per second.)  `outstanding` counts the root units in
    // progress plus the items not yet finished: it is raised before an
    // instance ticket is taken and by a donor before its items can be
    // claimed, and lowered when a unit ends.  With no instance ticket left
    // and nothing outstanding no unit can start again, so a waiting warp may
    // leave: its ticket is past every item there will be.
    //
    // Race (`race` = a, 0: off): a root search of a full-sorting instance
    // that starts its restart attempt a queues the instance's inverse
    // (td_spawn_inverse).  Queued inverses are claimed once no fresh instance
    // is left, before donated items, by their own tickets (fetch-and-add,
    // taken only while some are queued).  While fresh instances remain every
    // warp is busy, and a second search of an instance would only displace
    // other work; at the end of the launch, where warps idle, it shortens the
    // longest searches.  Most queued inverses belong to instances decided by
    // then and end at once.  A ticket taken past the last inverse queued is
    // kept until one is queued for it.
    int my_ticket = -1;  // lane 0: this warp's item ticket, -1 = none
    int my_spawn = -1;   // lane 0: this warp's ticket of the queue of inverses, -1 = none
    for (;;) {
        int kind = 0, unit = -1;
        if (lane == 0) {
            if (*(volatile int *)&pool->inst_ticket < count) {
                atomicAdd(&pool->outstanding, 1);
                const int t = atomicAdd(&pool->inst_ticket, 1);
                if (t < count) { kind = 1; unit = t; }
                else atomicSub(&pool->outstanding, 1);
            }
            if (!kind && race) {
                // slots past the queue's capacity are never claimed
                const int queued = min(*(volatile int *)&pool->spawn_produced, dc.spawn_capacity);
                if (my_spawn < 0 && *(volatile int *)&pool->spawn_consumed < queued)
                    my_spawn = atomicAdd(&pool->spawn_consumed, 1);
                if (my_spawn >= 0 && my_spawn < min(*(volatile int *)&pool->spawn_produced, dc.spawn_capacity)) {
                    kind = 3;
                    unit = my_spawn;
                    my_spawn = -1;
                }
            }
            if (!kind) {
                if (my_ticket < 0) my_ticket = atomicAdd(&pool->consumed, 1);
                if (my_ticket < *(volatile int *)&pool->produced) {
                    kind = 2;
                    unit = my_ticket;
                    my_ticket = -1;
                }
            }
        }
        kind = __shfl_sync(TD_FULL, kind, 0);
        unit = __shfl_sync(TD_FULL, unit, 0);
        if (!kind) {
            int done = 0;
            unsigned cap = max_backoff_ns;
            if (lane == 0) {
                // the instance tickets first: once they are gone, an
                // outstanding count of zero stays zero
                const int tk = *(volatile int *)&pool->inst_ticket;
                done = tk >= count && *(volatile int *)&pool->outstanding == 0;
                if (!done && lim.deadline_ns && td_globaltimer() > lim.deadline_ns) {
                    atomicCAS(&pool->error, 0, TD_ERR_TIMEOUT);
                    done = 1;
                }
                // the next few tickets in line are served first: they poll often
                if (my_ticket >= 0 && my_ticket - *(volatile int *)&pool->produced < 64) cap = min(cap, 512u);
            }
            if (__shfl_sync(TD_FULL, done, 0)) break;
            // waiting warps back off (to 32 us in a batch) so that their
            // counter reads do not crowd the L2 slices the busy warps'
            // atomics go to; a single search (one per call) caps it lower,
            // since there the launch ends only when every waiting warp has
            // woken up and seen that the work is done
            cap = __shfl_sync(TD_FULL, cap, 0);
            __nanosleep(min(backoff, cap));
            backoff = min(backoff * 2u, cap);
            continue;
        }
        backoff = 64;
        if (kind == 1) {
            const td_instance x = in[unit];
            td_inst_state *st = &state[unit];
            if (!td_instance_ok(x) || td_triple_count(x.n_symbols) == 0) {
                td_write_result(&out[unit], td_instance_ok(x) ? TD_NOT_FOUND : TD_ERR_ARG, 0, 0, s.path, 0, 0, 8);
            } else {
                if (lane == 0) atomicAdd(&st->pending, 1);
                td_setup_root<false>(s, x, code, codeN);
                dc.inst = (uint32_t)unit;
                dc.state = st;
                dc.side = 0;
                dc.race = td_inst_full(x) ? race : 0;
                const td_dfs_out r = td_dfs<false>(s, lut, code, x.n_symbols, x.max_moves, 0, lim, &dc);
                dc.race = 0;
                td_finish_unit<false>(r, st, &out[unit], s.path);
            }
        } else {
            // a donated item (kind 2) or a queued inverse root (kind 3); wait
            // until its producer has written it (bounded)
            const int phys = kind == 3 ? spawn_base + unit : unit;
            int ok = 0;
            if (lane == 0) {
                for (unsigned spin = 0; spin < (1u << 30); ++spin) {
                    if (*(volatile uint32_t *)&ready[phys] == epoch) { ok = 1; break; }
                    if ((spin & 1023u) == 0 && lim.deadline_ns && td_globaltimer() > lim.deadline_ns) break;
                    __nanosleep(32);
                }
                if (!ok) atomicCAS(&pool->error, 0, TD_ERR_TIMEOUT);
                __threadfence();
            }
            ok = __shfl_sync(TD_FULL, ok, 0);
            if (ok) {
                td_item it;  // read through L2: the donor wrote it from another SM
                {
                    const uint4 *src = reinterpret_cast<const uint4 *>(&items[phys]);
                    uint4 *dst = reinterpret_cast<uint4 *>(&it);
                    dst[0] = __ldcg(src);
                    dst[1] = __ldcg(src + 1);
                }
                const uint32_t idx = it.inst;
                const int d0 = it.depth & 0x7f;
                const int side = it.depth >> 7;
                // an item names an instance of this launch and a level of the
                // frame; one that does not is a launch error, never followed
                if (idx >= (uint32_t)count || d0 >= TD_MAX_DEPTH || (kind == 3) != (side && d0 == 0)) {
                    if (lane == 0) {
                        atomicCAS(&pool->error, 0, TD_ERR_VERIFY);
                        atomicSub(&pool->outstanding, 1);
                    }
                    continue;
                }
                const td_instance x = in[idx];
                td_inst_state *st = &state[idx];
                td_setup_root<false>(s, x, code, codeN);
                if (lane == 0) {
                    s.L[d0] = it.L;
                    s.off[d0] = it.off;
                    for (int d = 0; d < d0; ++d) s.path[d] = it.path[d];
                }
                __syncwarp();
                int stop = 0;
                if (lane == 0) stop = *(volatile int *)&st->found;
                stop = __shfl_sync(TD_FULL, stop, 0);
                td_dfs_out r;
                if (stop) {
                    r.status = TD_DFS_ABORTED;
                    r.depth = 0;
                    r.found_move = 0;
                    r.expansions = 0;
                } else {
                    // a donated subtree is searched once, to the end: restarting it
                    // would only repeat work when it holds no witness; the root of
                    // an inverse instance restarts like any root search
                    td_search_limits ilim = lim;
                    if (d0 > 0) ilim.restart_base = 0;
                    dc.inst = idx;
                    dc.state = st;
                    dc.side = side;
                    r = td_dfs<false>(s, lut, code, x.n_symbols, x.max_moves, d0, ilim, &dc);
                    dc.side = 0;
                    // a witness of the inverse becomes one of the instance; one that
                    // does not convert is reported as a failed replay, and one that
                    // leaves the reference's move filter on the instance's side is
                    // dropped (this side then stops; the instance's own search decides)
                    if (side && r.status == TD_DFS_FOUND) {
                        if (!td_inverse_result(s, x, r)) {
                            r.status = TD_DFS_EXHAUSTED;
                            if (lane == 0) atomicCAS(&st->error, 0, TD_ERR_VERIFY);
                        } else if (!td_filtered_witness(s, x, r)) {
                            r.status = TD_DFS_EXHAUSTED;
                        }
                    }
                }
                td_finish_unit<false>(r, st, &out[idx], s.path, side);
            }
        }
        if (lane == 0) atomicSub(&pool->outstanding, 1);
    }
}

// Advances the launch epoch that tags donated items as written; a launch
// replayed from a CUDA graph therefore never mistakes an item of an earlier
// launch for one of its own.
__global__ void td_epoch_kernel(uint32_t *epoch) {
    uint32_t e = *epoch + 1;
    *epoch = e ? e : 1;
}

// Runs after td_steal_kernel on the same stream.  When a bounded wait of the
// launch gave up (pool->error), some instances may have no result record: one
// never claimed, or one whose donated subtree a taker never received (its
// pending count stays above zero, so no unit wrote the final status).  Those
// get a timeout record, so a caller never reads a stale record of an earlier
// launch.  Without an error every thread returns at once.
__global__ void __launch_bounds__(256) td_finalize_kernel(const td_pool *__restrict__ pool,
                                                          const td_inst_state *__restrict__ state,
                                                          td_result *__restrict__ out, int count) {
    if (*(volatile const int *)&pool->error == 0) return;
    const int claimed = min(count, *(volatile const int *)&pool->inst_ticket);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        if (i < claimed && state[i].pending == 0) continue;
        td_result r;
        r.status = TD_ERR_TIMEOUT;
        r.depth = 0;
        for (int m = 0; m < TD_MAX_DEPTH; ++m) r.moves[m] = 0;
        r.reserved = 0;
        r.expansions = i < claimed ? state[i].expansions : 0;
        out[i] = r;
    }
}

// The totals of td_batch_stats, reduced on the device so that the host does
// not walk the result array (2^20 results are 32 MiB of host memory).  Reads
// only the status and expansion words of each record.
struct td_counts {
    unsigned long long expansions, found, not_found, errors;
};

__global__ void __launch_bounds__(256) td_count_kernel(const td_result *__restrict__ res, int count,
                                                       td_counts *__restrict__ c) {
    unsigned long long e = 0;
    uint32_t f = 0, nf = 0, er = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int st = res[i].status;
        e += res[i].expansions;
        f += st == TD_FOUND;
        nf += st == TD_NOT_FOUND;
        er += st != TD_FOUND && st != TD_NOT_FOUND;
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(TD_FULL, e, o);
    f = __reduce_add_sync(TD_FULL, f);
    nf = __reduce_add_sync(TD_FULL, nf);
    er = __reduce_add_sync(TD_FULL, er);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c->expansions, e);
        atomicAdd(&c->found, (unsigned long long)f);
        atomicAdd(&c->not_found, (unsigned long long)nf);
        atomicAdd(&c->errors, (unsigned long long)er);
    }
}

// Witness replay in pinned form with the search's own rules: every move is an
// in-range position triple i<j<k whose symbols omega does not fix and whose
// odd-cycle change is 0 or +2 (sorting_search.cu:375-380,608-610), there are
// at most max_moves of them, and the last node passes the acceptance test of
// the instance (satisfies_rate, sorting_search.cu:336-346: with full sorting,
// omega = id).  With full sorting this is CertificateValidator's replay
// (CertificateValidator.java:14-50) in pinned form.
__global__ void td_validate_kernel(const td_instance *__restrict__ in, td_result *__restrict__ res,
                                   uint8_t *__restrict__ ok, int count, int mark) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const td_instance x = in[idx];
    const td_result r = res[idx];
    const uint8_t good = (uint8_t)td_witness_ok(x, r);
    if (ok) ok[idx] = good;
    if (mark && r.status == TD_FOUND && !good) res[idx].status = TD_ERR_VERIFY;
}

// Integer issue peaks at full occupancy.  Each thread runs `iters` iterations
// of 16 operations over 8 independent chains.  MIX = 0: LOP3 only (ALU pipe
// alone, 16 lanes per SM sub-partition, so at most half a warp instruction per
// clock per sub-partition).  MIX = 1: LOP3 and IMAD alternate (ALU and FMA
// pipes side by side), which can reach one warp instruction per clock per
// sub-partition: the full issue rate.
template <int MIX>
__global__ void __launch_bounds__(256) td_int_peak_kernel(uint32_t *sink, int iters) {
    uint32_t a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = threadIdx.x * 0x9E3779B9u + c * 0x85EBCA6Bu + blockIdx.x;
    const uint32_t m = 0x01000193u | (blockIdx.x << 1);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                if (MIX && (c & 1))
                    asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(m), "r"(a[(c + 3) & 7]));
                else
                    asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[c]) : "r"(a[(c + 1) & 7]), "r"(a[(c + 3) & 7]));
            }
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) x ^= a[c];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}

// ============================================================================
// host side
// ============================================================================

namespace {

struct Slot {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr, t0 = nullptr, t1 = nullptr;
    size_t budget = 0;
    td_instance *d_inst = nullptr;
    td_result *d_res = nullptr;
    td_instance *h_inst = nullptr;
    td_result *h_res = nullptr;
    int *d_ticket = nullptr;
    void *d_batch = nullptr;
    size_t d_batch_bytes = 0;
    // donation scratch: pool counters, item array + ready flags, instance state
    td_pool *d_pool = nullptr;
    td_item *d_items = nullptr;
    uint32_t *d_ready = nullptr;
    int item_capacity = 0;
    uint64_t *d_tt = nullptr;  // tables of explored states, one per resident warp
    uint32_t *d_tt_gen = nullptr;  // their generation counters
    size_t tt_warps = 0;
    int tt_bits = 0;
    td_inst_state *d_state = nullptr;
    size_t state_count = 0;
    uint32_t *d_epoch = nullptr;
    // split pass of the reference order: the listed instances, the pass's
    // counters, each root's children, the subtree results and the cutoffs
    int *d_hard = nullptr;
    size_t hard_cap = 0;
    td_split_ctl *d_split = nullptr;
    uint16_t *d_kids = nullptr;
    int *d_base = nullptr;
    int *d_nkids = nullptr;
    int *d_cutoff = nullptr;
    td_result *d_split_items = nullptr;
    int split_records = 0;
    // td_batch_stats of host-buffer batches: device totals and their pinned copy
    td_counts *d_counts = nullptr;
    struct HostStats {
        td_counts counts;
        td_pool pool;
    } *h_stats = nullptr;
    int slots_on_device = 1;
    std::mutex *mu = nullptr;
};

struct DeviceInfo {
    bool ready = false;
    int sms = 0;
    int blocks_per_sm = 0;
    int steal_blocks_per_sm = 0;
};

std::mutex g_mu;
std::vector<Slot> g_slots;
std::vector<DeviceInfo> g_dev;

int g_warps_per_block = 4;
int g_grain = 1;            // instances per ticket (ordered persistent kernel)
// defaults: the best per-call setting (one blocking search per slot call,
// 16 slots, S_16) measured from native threads; batch callers use tuned ones
int g_steal_grain = 4;      // items per donation
int g_split_level = 2;      // donate children of levels <= this
int g_check_every = 64;     // expansions between idle checks
// the same for serving launches, where latency rather than throughput counts
int g_serve_grain = 1;
int g_serve_split_level = 2;
int g_serve_check_every = 32;
int g_tt_bits = TD_TT_BITS;  // log2 entries of the explored-state tables; 0 = no table
uint32_t g_restart_base = TD_RESTART_BASE;  // free-order restart budget base; 0 = no restarts
int g_split_budget = TD_SPLIT_BUDGET;       // reference order: first-pass expansions before a split; 0 = none
int g_split_records = TD_SPLIT_RECORDS;     // reference order: subtree records per launch
int g_race = 8;  // free-order batches: attempt at which a search starts racing its inverse, 0 = off (td_configure_race)

void set_err(char *err, size_t len, const std::string &msg) {
    if (err && len) {
        std::snprintf(err, len, "%s", msg.c_str());
    }
}

std::string cuda_msg(cudaError_t e, const char *file, int line) {
    return std::string(file) + ":" + std::to_string(line) + ": CUDA error " + cudaGetErrorName(e) + " (" +
           cudaGetErrorString(e) + ")";
}

#define TD_CHECK(call)                                                   \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) {                                         \
            set_err(err, errlen, cuda_msg(e_, __FILE__, __LINE__));      \
            return TD_CUDA_ERROR;                                        \
        }                                                                \
    } while (0)

size_t smem_bytes(int warps) { return TD_LUT_BYTES + (size_t)warps * sizeof(td_warp_smem); }
// td_steal_kernel keeps no class table
size_t steal_smem_bytes(int warps) { return (size_t)warps * sizeof(td_warp_smem); }

std::atomic<uint64_t> g_time_limit_ns{0};

// Launch deadline: td_set_time_limit, else TD16_TIME_LIMIT_S, else 300 s.
uint64_t time_limit_ns() {
    uint64_t v = g_time_limit_ns.load(std::memory_order_relaxed);
    if (v) return v;
    const char *s = std::getenv("TD16_TIME_LIMIT_S");
    double secs = s ? std::atof(s) : 300.0;
    if (!(secs > 0)) secs = 300.0;
    v = (uint64_t)(secs * 1e9);
    g_time_limit_ns.store(v, std::memory_order_relaxed);
    return v;
}

// Loads every kernel of the library on the current device (defined at the
// end of this file).  With lazy module loading a kernel's code would
// otherwise be loaded at its first launch, which may wait for the work
// already on the device, the per-call server's resident launch included.
int preload_kernels(char *err, size_t errlen);

// The launch settings of one launch, read together under g_mu so that a
// concurrent td_configure_* call never hands a launch half of its change.
struct LaunchCfg {
    int warps, grain, steal_grain, split_level, check_every, tt_bits;
    uint32_t restart_base;
    int race;
    int split_budget, split_records;
    int serve_grain, serve_split_level, serve_check_every;
    int sms, steal_blocks_per_sm, blocks_per_sm;  // of the device, for `warps`
};

// Snapshot of the settings and of `device`'s occupancy for them; the device
// must be current and set up (ensure_device).
int launch_cfg(int device, LaunchCfg *c, char *err, size_t errlen) {
    std::lock_guard<std::mutex> g(g_mu);
    c->warps = g_warps_per_block;
    c->grain = g_grain;
    c->steal_grain = g_steal_grain;
    c->split_level = g_split_level;
    c->check_every = g_check_every;
    c->tt_bits = g_tt_bits;
    c->restart_base = g_restart_base;
    c->race = g_race;
    c->split_budget = g_split_budget;
    c->split_records = g_split_records;
    c->serve_grain = g_serve_grain;
    c->serve_split_level = g_serve_split_level;
    c->serve_check_every = g_serve_check_every;
    DeviceInfo &d = g_dev[device];
    const int threads = c->warps * 32;
    if (d.steal_blocks_per_sm == 0) {
        int b = 0;
        TD_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, td_steal_kernel, threads,
                                                               steal_smem_bytes(c->warps)));
        d.steal_blocks_per_sm = std::max(1, b);
    }
    if (d.blocks_per_sm == 0) {
        int b = 0;
        TD_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, td_persistent_kernel<false>, threads,
                                                               smem_bytes(c->warps)));
        d.blocks_per_sm = std::max(1, b);
    }
    c->sms = d.sms;
    c->steal_blocks_per_sm = d.steal_blocks_per_sm;
    c->blocks_per_sm = d.blocks_per_sm;
    return TD_OK;
}

int ensure_device(int device, char *err, size_t errlen) {
    if ((int)g_dev.size() <= device) g_dev.resize(device + 1);
    DeviceInfo &d = g_dev[device];
    if (d.ready) return TD_OK;
    TD_CHECK(cudaSetDevice(device));
    std::vector<uint16_t> tri(TD_TRI_TABLE, 0);
    for (int N = 3; N <= TD_MAX_N; ++N) {
        int base = N < 4 ? 0 : N * (N - 1) * (N - 2) * (N - 3) / 24, t = 0;
        for (int i = 0; i < N - 2; ++i)
            for (int j = i + 1; j < N - 1; ++j)
                for (int k = j + 1; k < N; ++k) tri[base + t++] = td_pack_move(i, j, k);
    }
    TD_CHECK(cudaMemcpyToSymbol(td_tri_table, tri.data(), tri.size() * sizeof(uint16_t)));
    std::vector<uint8_t> lut(TD_LUT_BYTES);
    for (int i = 0; i < TD_LUT_BYTES; ++i) lut[i] = (uint8_t)td_class_of_index(i);
    TD_CHECK(cudaMemcpyToSymbol(td_lut_global, lut.data(), lut.size()));
    TD_CHECK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device));
    const int max_warps = 8;
    const size_t max_smem = smem_bytes(max_warps);
    TD_CHECK(cudaFuncSetAttribute(td_plain_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_plain_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_persistent_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_steal_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_split_roots_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    TD_CHECK(cudaFuncSetAttribute(td_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    const int rc = preload_kernels(err, errlen);
    if (rc != TD_OK) return rc;
    d.ready = true;
    return TD_OK;
}

void release_slot(Slot &s) {
    if (s.device >= 0) cudaSetDevice(s.device);
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.d_inst) cudaFree(s.d_inst);
    if (s.d_res) cudaFree(s.d_res);
    if (s.d_ticket) cudaFree(s.d_ticket);
    if (s.d_batch) cudaFree(s.d_batch);
    if (s.d_pool) cudaFree(s.d_pool);
    if (s.d_items) cudaFree(s.d_items);
    if (s.d_ready) cudaFree(s.d_ready);
    if (s.d_tt) cudaFree(s.d_tt);
    if (s.d_tt_gen) cudaFree(s.d_tt_gen);
    if (s.d_epoch) cudaFree(s.d_epoch);
    if (s.d_state) cudaFree(s.d_state);
    if (s.d_hard) cudaFree(s.d_hard);
    if (s.d_split) cudaFree(s.d_split);
    if (s.d_kids) cudaFree(s.d_kids);
    if (s.d_base) cudaFree(s.d_base);
    if (s.d_nkids) cudaFree(s.d_nkids);
    if (s.d_cutoff) cudaFree(s.d_cutoff);
    if (s.d_split_items) cudaFree(s.d_split_items);
    if (s.d_counts) cudaFree(s.d_counts);
    if (s.h_stats) cudaFreeHost(s.h_stats);
    if (s.h_inst) cudaFreeHost(s.h_inst);
    if (s.h_res) cudaFreeHost(s.h_res);
    if (s.done) cudaEventDestroy(s.done);
    if (s.t0) cudaEventDestroy(s.t0);
    if (s.t1) cudaEventDestroy(s.t1);
    if (s.stream) cudaStreamDestroy(s.stream);
    delete s.mu;
    s = Slot{};
}

// the per-call server (td_percall.cuh)
void percall_shutdown();
void percall_park(int device);
int percall_search(int device, const td_instance &x, td_result *out, char *err, size_t errlen);
extern std::atomic<int> g_percall_mode;

void destroy_all() {
    percall_shutdown();
    for (auto &s : g_slots) release_slot(s);
    g_slots.clear();
}

// Launch one batch on `stream`.  Instances and results are device pointers.
int launch_batch(Slot &s, int count, const td_instance *d_in, td_result *d_out, unsigned flags,
                 uint64_t max_exp, cudaStream_t stream, char *err, size_t errlen) {
    if (count <= 0) return TD_OK;
    const bool ordered = flags & TD_FLAG_ORDERED;
    LaunchCfg cfg;
    const int rc = launch_cfg(s.device, &cfg, err, errlen);
    if (rc != TD_OK) return rc;
    const int warps = cfg.warps;
    const size_t smem = smem_bytes(warps);
    const int threads = warps * 32;
    if (flags & TD_FLAG_PLAIN) {
        const int blocks = (count + warps - 1) / warps;
        if (ordered) td_plain_kernel<true><<<blocks, threads, smem, stream>>>(d_in, d_out, count, max_exp, time_limit_ns());
        else td_plain_kernel<false><<<blocks, threads, smem, stream>>>(d_in, d_out, count, max_exp, time_limit_ns());
    } else if (!ordered) {
        // item space: the slot budget (the reference's queue budget) less the
        // per-instance state, at 36 bytes per item (record + ready flag)
        if (s.d_pool == nullptr) {
            TD_CHECK(cudaMalloc(&s.d_pool, sizeof(td_pool)));
            const size_t cap = std::max<size_t>(1024, std::min<size_t>(s.budget / 36, 1u << 26));
            TD_CHECK(cudaMalloc(&s.d_items, cap * sizeof(td_item)));
            TD_CHECK(cudaMalloc(&s.d_ready, cap * sizeof(uint32_t)));
            TD_CHECK(cudaMemsetAsync(s.d_ready, 0, cap * sizeof(uint32_t), stream));
            TD_CHECK(cudaMalloc(&s.d_epoch, sizeof(uint32_t)));
            TD_CHECK(cudaMemsetAsync(s.d_epoch, 0, sizeof(uint32_t), stream));
            s.item_capacity = (int)cap;
        }
        // buffers grow in stream order: a cudaFree would wait for all work on
        // the device, the per-call server's resident launch included
        if ((size_t)count > s.state_count) {
            if (s.d_state) TD_CHECK(cudaFreeAsync(s.d_state, stream));
            s.d_state = nullptr;
            s.state_count = 0;
            TD_CHECK(cudaMallocAsync(&s.d_state, (size_t)count * sizeof(td_inst_state), stream));
            s.state_count = (size_t)count;
        }
        // at least the slot's share of the resident grid, so that a small batch
        // (one search from td_search) is spread over that many warps by donation
        const int resident = cfg.sms * cfg.steal_blocks_per_sm;
        const int share = std::max(1, resident / std::max(1, s.slots_on_device));
        const int grid = std::max(1, std::min(resident, std::max(share, (count + warps - 1) / warps)));
        if (cfg.tt_bits > 0 && ((size_t)resident * warps > s.tt_warps || cfg.tt_bits != s.tt_bits)) {
            // one table (8 bytes x 2^tt_bits) per resident warp, sized for
            // the whole resident grid so that it never moves under a captured
            // graph; replaced in stream order after the previous launch
            if (s.d_tt) TD_CHECK(cudaFreeAsync(s.d_tt, stream));
            if (s.d_tt_gen) TD_CHECK(cudaFreeAsync(s.d_tt_gen, stream));
            s.d_tt = nullptr;
            s.d_tt_gen = nullptr;
            s.tt_warps = 0;
            const size_t tt_words = (size_t)resident * warps << cfg.tt_bits;
            TD_CHECK(cudaMallocAsync(&s.d_tt, tt_words * sizeof(uint64_t), stream));
            TD_CHECK(cudaMallocAsync(&s.d_tt_gen, (size_t)resident * warps * sizeof(uint32_t), stream));
            // zero words are empty, and generations start at 1
            TD_CHECK(cudaMemsetAsync(s.d_tt, 0, tt_words * sizeof(uint64_t), stream));
            TD_CHECK(cudaMemsetAsync(s.d_tt_gen, 0, (size_t)resident * warps * sizeof(uint32_t), stream));
            s.tt_warps = (size_t)resident * warps;
            s.tt_bits = cfg.tt_bits;
        }
        TD_CHECK(cudaMemsetAsync(s.d_pool, 0, sizeof(td_pool), stream));
        TD_CHECK(cudaMemsetAsync(s.d_state, 0, (size_t)count * sizeof(td_inst_state), stream));
        td_epoch_kernel<<<1, 1, 0, stream>>>(s.d_epoch);
        // the race needs restarts, and an expansion budget per unit would make
        // one side's budget decide the other's; its queue of inverse roots
        // holds one slot per instance (each queues its inverse at most once),
        // at the top of the item space, which keeps at least half for donation
        const int race = cfg.restart_base > 0 && max_exp == 0 && count <= s.item_capacity / 2 ? cfg.race : 0;
        const int spawn_base = race ? s.item_capacity - count : s.item_capacity;
        td_steal_kernel<<<grid, threads, steal_smem_bytes(warps), stream>>>(
            d_in, d_out, count, s.d_pool, s.d_items, s.d_ready, s.d_epoch, s.item_capacity, s.d_state,
            cfg.steal_grain, cfg.split_level, cfg.check_every, time_limit_ns(), cfg.tt_bits > 0 ? s.d_tt : nullptr,
            s.d_tt_gen, cfg.tt_bits, cfg.restart_base, max_exp, count == 1 ? 4096u : 32768u, race, spawn_base);
        TD_CHECK(cudaGetLastError());
        td_finalize_kernel<<<std::max(1, std::min((count + 255) / 256, 2 * cfg.sms)), 256, 0, stream>>>(
            s.d_pool, s.d_state, d_out, count);
    } else {
        const int grid_max = cfg.sms * cfg.blocks_per_sm;
        const int grid = std::max(1, std::min(grid_max, (count + warps - 1) / warps));
        TD_CHECK(cudaMemsetAsync(s.d_ticket, 0, sizeof(int), stream));
        if (ordered && max_exp == 0 && cfg.split_budget > 0) {
            // one warp per instance within split_budget expansions, then the
            // split pass for the instances left (stream-ordered buffers)
            if (s.d_split == nullptr) TD_CHECK(cudaMallocAsync(&s.d_split, sizeof(td_split_ctl), stream));
            if (cfg.split_records > s.split_records) {
                if (s.d_kids) TD_CHECK(cudaFreeAsync(s.d_kids, stream));
                if (s.d_split_items) TD_CHECK(cudaFreeAsync(s.d_split_items, stream));
                s.d_kids = nullptr;
                s.d_split_items = nullptr;
                s.split_records = 0;
                TD_CHECK(cudaMallocAsync(&s.d_kids, sizeof(uint16_t) * (size_t)cfg.split_records, stream));
                TD_CHECK(cudaMallocAsync(&s.d_split_items, sizeof(td_result) * (size_t)cfg.split_records, stream));
                s.split_records = cfg.split_records;
            }
            if ((size_t)count > s.hard_cap) {
                for (int *p : {s.d_hard, s.d_base, s.d_nkids, s.d_cutoff})
                    if (p) TD_CHECK(cudaFreeAsync(p, stream));
                s.d_hard = s.d_base = s.d_nkids = s.d_cutoff = nullptr;
                s.hard_cap = 0;
                TD_CHECK(cudaMallocAsync(&s.d_hard, sizeof(int) * (size_t)count, stream));
                TD_CHECK(cudaMallocAsync(&s.d_base, sizeof(int) * (size_t)count, stream));
                TD_CHECK(cudaMallocAsync(&s.d_nkids, sizeof(int) * (size_t)count, stream));
                TD_CHECK(cudaMallocAsync(&s.d_cutoff, sizeof(int) * (size_t)count, stream));
                s.hard_cap = (size_t)count;
            }
            TD_CHECK(cudaMemsetAsync(s.d_split, 0, sizeof(td_split_ctl), stream));
            td_persistent_kernel<true><<<grid, threads, smem, stream>>>(d_in, d_out, count, s.d_ticket, cfg.grain,
                                                                        (uint64_t)cfg.split_budget, time_limit_ns(),
                                                                        &s.d_split->hard, s.d_hard);
            td_split_roots_kernel<<<grid_max, threads, smem, stream>>>(d_in, s.d_hard, s.d_split, s.d_kids, s.d_base,
                                                                       s.d_nkids, s.d_cutoff, cfg.split_records);
            td_split_kernel<<<grid_max, threads, smem, stream>>>(d_in, d_out, s.d_hard, s.d_split, s.d_kids, s.d_base,
                                                                 s.d_nkids, s.d_cutoff, s.d_split_items,
                                                                 time_limit_ns());
            td_split_join_kernel<<<std::max(1, std::min((count + 255) / 256, 2 * cfg.sms)), 256, 0, stream>>>(
                s.d_hard, s.d_split, s.d_base, s.d_nkids, s.d_split_items, d_out);
        } else if (ordered)
            td_persistent_kernel<true><<<grid, threads, smem, stream>>>(d_in, d_out, count, s.d_ticket, cfg.grain,
                                                                        max_exp, time_limit_ns());
        else
            td_persistent_kernel<false><<<grid, threads, smem, stream>>>(d_in, d_out, count, s.d_ticket, cfg.grain,
                                                                         max_exp, time_limit_ns());
    }
    TD_CHECK(cudaGetLastError());
    if (flags & TD_FLAG_VERIFY) {
        td_validate_kernel<<<(count + 255) / 256, 256, 0, stream>>>(d_in, d_out, nullptr, count, 1);
        TD_CHECK(cudaGetLastError());
    }
    return TD_OK;
}

Slot *get_slot(int slot, char *err, size_t errlen) {
    if (slot < 0 || slot >= (int)g_slots.size() || g_slots[slot].device < 0) {
        set_err(err, errlen, "invalid GPU sorting slot");
        return nullptr;
    }
    return &g_slots[slot];
}

int search_one(int slot, const uint8_t *beta, const uint8_t *omega, int n, int init, float min_rate,
               int max_moves, int full, int16_t *out_ijk, int *out_depth, unsigned flags, char *err,
               size_t errlen) {
    if (out_depth) *out_depth = 0;
    // the reference's order of checks: null arrays, the slot
    // (jni_sorter.cu:59-92), then n, the depth and n < 3
    // (sorting_search.cu:821-827)
    if (!beta || !omega) {
        set_err(err, errlen, "beta and omega must not be null");
        return TD_INVALID_ARG;
    }
    Slot *s;
    {
        std::lock_guard<std::mutex> g(g_mu);
        s = get_slot(slot, err, errlen);
        if (!s) return TD_INVALID_ARG;
    }
    if (n > TD_MAX_N) {
        set_err(err, errlen, "performGpuSortingSearch: n exceeds MAX_N");
        return TD_INVALID_ARG;
    }
    if (max_moves <= 0 || max_moves > TD_MAX_DEPTH) {
        set_err(err, errlen, "performGpuSortingSearch: invalid maximumDepth");
        return TD_INVALID_ARG;
    }
    if (td_triple_count(n) == 0) return TD_NOT_FOUND_RC;
    td_instance x;
    if (td_prepare_pair(beta, omega, n, init, min_rate, max_moves, full, &x) != 0) {
        set_err(err, errlen, "beta/omega are not permutations whose product omega.beta is an n-cycle");
        return TD_INVALID_ARG;
    }
    td_result r;
    if (g_percall_mode.load(std::memory_order_relaxed) == 1) {
        // the device's resident per-call server: no CUDA call per search
        if (flags & TD_FLAG_ORDERED) x.packed |= TD_PACKED_ORDERED;
        const int rc = percall_search(s->device, x, &r, err, errlen);
        if (rc != TD_OK) return rc;
    } else {
        std::lock_guard<std::mutex> g(*s->mu);
        TD_CHECK(cudaSetDevice(s->device));
        *s->h_inst = x;
        TD_CHECK(cudaMemcpyAsync(s->d_inst, s->h_inst, sizeof(td_instance), cudaMemcpyHostToDevice, s->stream));
        // free order: the donation engine over the slot's share of the GPU (as
        // the reference gives each slot SMs x resident blocks / slots queues,
        // sorting_search.cu:740-752); the reference order keeps one warp
        const unsigned how = (flags & TD_FLAG_ORDERED) ? (flags | TD_FLAG_PLAIN) : flags;
        percall_park(s->device);
        int rc = launch_batch(*s, 1, s->d_inst, s->d_res, how, 0, s->stream, err, errlen);
        if (rc != TD_OK) return rc;
        TD_CHECK(cudaMemcpyAsync(s->h_res, s->d_res, sizeof(td_result), cudaMemcpyDeviceToHost, s->stream));
        TD_CHECK(cudaEventRecord(s->done, s->stream));
        TD_CHECK(cudaEventSynchronize(s->done));
        r = *s->h_res;
    }
    if (r.status == TD_FOUND) {
        for (int d = 0; d < r.depth; ++d) {
            out_ijk[3 * d + 0] = (int16_t)(r.moves[d] & 31);
            out_ijk[3 * d + 1] = (int16_t)((r.moves[d] >> 5) & 31);
            out_ijk[3 * d + 2] = (int16_t)((r.moves[d] >> 10) & 31);
        }
        if (out_depth) *out_depth = r.depth;
        return TD_OK;
    }
    if (r.status == TD_NOT_FOUND) return TD_NOT_FOUND_RC;
    if (r.status == TD_ERR_BUDGET) {
        set_err(err, errlen, "GPU sorting search queue overflow");
        return TD_OVERFLOW;
    }
    if (r.status == TD_ERR_TIMEOUT) {
        set_err(err, errlen, "GPU sorting search deadline reached");
        return TD_TIMEOUT;
    }
    set_err(err, errlen, "GPU sorting search rejected its input");
    return TD_INVALID_ARG;
}

// ---- seeded synthetic instances ----------------------------------------------

inline uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Lemire's multiply-shift bounded draw on the upper 32 bits, with rejection.
inline uint32_t bounded(uint64_t &s, uint32_t range) {
    uint32_t x = (uint32_t)(splitmix64(s) >> 32);
    uint64_t m = (uint64_t)x * range;
    uint32_t l = (uint32_t)m;
    if (l < range) {
        const uint32_t t = (0u - range) % range;
        while (l < t) {
            x = (uint32_t)(splitmix64(s) >> 32);
            m = (uint64_t)x * range;
            l = (uint32_t)m;
        }
    }
    return (uint32_t)(m >> 32);
}

// lexicographic unranking of r over triples x<y<z of {0..n}
void unrank_triple(int n, uint32_t r, int *x, int *y, int *z) {
    const int M = n + 1;
    for (int a = 0; a < M - 2; ++a) {
        const uint32_t c = (uint32_t)((M - a - 1) * (M - a - 2) / 2);
        if (r < c) {
            for (int b = a + 1; b < M - 1; ++b) {
                const uint32_t cb = (uint32_t)(M - b - 1);
                if (r < cb) {
                    *x = a;
                    *y = b;
                    *z = b + 1 + (int)r;
                    return;
                }
                r -= cb;
            }
        }
        r -= c;
    }
    *x = 0;
    *y = 1;
    *z = 2;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================

TD_API int td_init_slots(int total_slots, const int *devices, int device_count, uint64_t budget, char *err,
                         size_t errlen) {
    if (!devices || device_count <= 0) {
        set_err(err, errlen, "devices must contain at least one CUDA device ordinal");
        return TD_INVALID_ARG;
    }
    if (total_slots <= 0) {
        set_err(err, errlen, "totalSlots must be positive");
        return TD_INVALID_ARG;
    }
    if (budget == 0) {
        set_err(err, errlen, "queueBytesBudget must be positive");
        return TD_INVALID_ARG;
    }
    int ndev = 0;
    TD_CHECK(cudaGetDeviceCount(&ndev));
    std::vector<int> per(ndev > 0 ? ndev : 1, 0);
    for (int i = 0; i < device_count; ++i) {
        if (devices[i] < 0 || devices[i] >= ndev) {
            set_err(err, errlen, "devices contains a CUDA device ordinal outside the available range");
            return TD_INVALID_ARG;
        }
        for (int j = 0; j < i; ++j)
            if (devices[j] == devices[i]) {
                set_err(err, errlen, "devices must contain distinct CUDA device ordinals");
                return TD_INVALID_ARG;
            }
    }
    for (int i = 0; i < total_slots; ++i) per[devices[i % device_count]]++;
    std::lock_guard<std::mutex> g(g_mu);
    destroy_all();
    for (int i = 0; i < device_count; ++i) {
        const int dev = devices[i];
        TD_CHECK(cudaSetDevice(dev));
        size_t free_b = 0, total_b = 0;
        TD_CHECK(cudaMemGetInfo(&free_b, &total_b));
        const uint64_t need = budget * (uint64_t)per[dev];
        if (per[dev] > 0 && (budget > UINT64_MAX / (uint64_t)per[dev] || need > free_b)) {
            set_err(err, errlen, "CUDA device " + std::to_string(dev) + " has " + std::to_string(free_b) +
                                     " free bytes, but its search queues require at least " +
                                     std::to_string(need) + " bytes");
            return TD_INVALID_ARG;
        }
        int rc = ensure_device(dev, err, errlen);
        if (rc != TD_OK) return rc;
    }
    g_slots.resize(total_slots);
    for (int i = 0; i < total_slots; ++i) {
        Slot &s = g_slots[i];
        s.device = devices[i % device_count];
        s.budget = budget;
        s.slots_on_device = per[s.device];
        s.mu = new std::mutex();
        cudaError_t e = cudaSetDevice(s.device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreate(&s.t0);
        if (e == cudaSuccess) e = cudaEventCreate(&s.t1);
        if (e == cudaSuccess) e = cudaMalloc(&s.d_inst, sizeof(td_instance));
        if (e == cudaSuccess) e = cudaMalloc(&s.d_res, sizeof(td_result));
        if (e == cudaSuccess) e = cudaMalloc(&s.d_ticket, sizeof(int));
        if (e == cudaSuccess) e = cudaMallocHost(&s.h_inst, sizeof(td_instance));
        if (e == cudaSuccess) e = cudaMallocHost(&s.h_res, sizeof(td_result));
        if (e != cudaSuccess) {
            set_err(err, errlen, cuda_msg(e, __FILE__, __LINE__));
            destroy_all();
            return TD_CUDA_ERROR;
        }
    }
    return TD_OK;
}

TD_API int td_search(int slot, const uint8_t *beta, const uint8_t *omega, int n, int init, float min_rate,
                     int max_moves, int full, int16_t *out_ijk, int *out_depth, char *err, size_t errlen) {
    return search_one(slot, beta, omega, n, init, min_rate, max_moves, full, out_ijk, out_depth, 0u, err, errlen);
}

TD_API int td_search_ordered(int slot, const uint8_t *beta, const uint8_t *omega, int n, int init,
                             float min_rate, int max_moves, int full, int16_t *out_ijk, int *out_depth,
                             char *err, size_t errlen) {
    return search_one(slot, beta, omega, n, init, min_rate, max_moves, full, out_ijk, out_depth,
                      TD_FLAG_ORDERED, err, errlen);
}

TD_API int td_slot_count(void) {
    std::lock_guard<std::mutex> g(g_mu);
    return (int)g_slots.size();
}

TD_API int td_slot_device(int slot) {
    std::lock_guard<std::mutex> g(g_mu);
    if (slot < 0 || slot >= (int)g_slots.size()) return -1;
    return g_slots[slot].device;
}

TD_API void *td_slot_stream(int slot) {
    std::lock_guard<std::mutex> g(g_mu);
    if (slot < 0 || slot >= (int)g_slots.size()) return nullptr;
    return (void *)g_slots[slot].stream;
}

TD_API int td_destroy(void) {
    std::lock_guard<std::mutex> g(g_mu);
    destroy_all();
    return TD_OK;
}

TD_API int td_configure(int warps_per_block, int grain) {
    if (warps_per_block < 1 || warps_per_block > 8 || grain < 1) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_warps_per_block = warps_per_block;
    g_grain = grain;
    for (auto &d : g_dev) d.blocks_per_sm = d.steal_blocks_per_sm = 0;
    return TD_OK;
}

// Sets the deadline of every later launch (seconds > 0); every device wait
// and search ends with a timeout status once it passes.
TD_API int td_set_time_limit(double seconds) {
    if (!(seconds > 0)) return TD_INVALID_ARG;
    g_time_limit_ns.store((uint64_t)(seconds * 1e9), std::memory_order_relaxed);
    return TD_OK;
}

// Work-donation parameters of the free-order engine: items per donation,
// deepest level whose children may be donated, expansions between checks.
TD_API int td_configure_steal(int grain, int split_level, int check_every) {
    if (grain < 1 || split_level < 0 || split_level >= TD_MAX_DEPTH || check_every < 1) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_steal_grain = grain;
    g_split_level = split_level;
    g_check_every = check_every;
    return TD_OK;
}

// Size of the per-warp tables of explored states of later free-order launches:
// 2^bits entries of 8 bytes per resident warp (6 <= bits <= 16), or 0 to
// search without them.
TD_API int td_configure_table(int bits) {
    if (bits != 0 && (bits < 6 || bits > 16)) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_tt_bits = bits;
    return TD_OK;
}

// Restarts of later free-order batch searches: a search that has spent
// base x luby(a) expansions in attempt a starts again with another child order
// (td_attempt_budget, td_order_variant); 0 turns restarts off.  Verdicts do
// not depend on it.
// The split pass of reference-order batches: expansions of the one-warp first
// pass (0: no split, every walk on one warp) and subtree records per launch
// (a root whose children find no room runs whole).  Results do not depend on
// either.
TD_API int td_configure_split(int first_pass_expansions, int records) {
    if (first_pass_expansions < 0 || records < 1 || records > (1 << 24)) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_split_budget = first_pass_expansions;
    g_split_records = records;
    return TD_OK;
}

TD_API int td_configure_restart(int base) {
    if (base < 0 || (base > 0 && base < 16)) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_restart_base = (uint32_t)base;
    return TD_OK;
}

// Later free-order batches (full sorting) race a search that starts its
// restart attempt `attempt` (1..32; the 32nd is the last, unbounded one)
// against a search of its inverse instance; 0 turns the race off.
TD_API int td_configure_race(int attempt) {
    if (attempt < 0 || attempt > TD_RESTARTS) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_race = attempt;
    return TD_OK;
}

// Work distribution of later serving launches (td_serve_open): items per
// donation, deepest level whose children are donated, expansions between
// idle checks.
TD_API int td_configure_serve(int grain, int split_level, int check_every) {
    if (grain < 1 || split_level < 0 || split_level >= TD_MAX_DEPTH || check_every < 1) return TD_INVALID_ARG;
    std::lock_guard<std::mutex> g(g_mu);
    g_serve_grain = grain;
    g_serve_split_level = split_level;
    g_serve_check_every = check_every;
    return TD_OK;
}

TD_API int td_prepare_pairs(int count, const uint8_t *beta, const uint8_t *omega, const uint8_t *n,
                            const int32_t *init, const float *min_rate, const int32_t *max_moves,
                            const uint8_t *full, td_instance *out, int *bad) {
    for (int i = 0; i < count; ++i) {
        if (td_prepare_pair(beta + (size_t)i * TD_MAX_N, omega + (size_t)i * TD_MAX_N, n[i], init[i], min_rate[i],
                            max_moves[i], full[i], &out[i]) != 0) {
            if (bad) *bad = i;
            return TD_INVALID_ARG;
        }
    }
    return TD_OK;
}

TD_API int td_prepare_perms(int count, const int8_t *perms, const uint8_t *n, const int32_t *max_moves,
                            float min_rate, int full, td_instance *out, int *bad) {
    for (int i = 0; i < count; ++i) {
        const int ni = n[i];
        uint8_t beta[TD_MAX_N], omega[TD_MAX_N];
        int init = 0;
        bool okp = ni >= 0 && ni < TD_MAX_N;
        if (okp) {
            uint32_t seen = 0;
            for (int m = 0; m < ni; ++m) {
                const int v = perms[(size_t)i * 16 + m];
                if (v < 0 || v >= ni || (seen >> v) & 1u) okp = false;
                else seen |= 1u << v;
            }
        }
        if (okp) {
            td_perm_to_pair(perms + (size_t)i * 16, ni, beta, omega, &init);
            okp = td_prepare_pair(beta, omega, ni + 1, init, min_rate, max_moves[i], full, &out[i]) == 0;
        }
        if (!okp) {
            if (bad) *bad = i;
            return TD_INVALID_ARG;
        }
    }
    return TD_OK;
}

TD_API int td_synth_perms(uint64_t seed, int count, int n_min, int n_max, int hard_pct, int hard_min, int hard_max,
                          int8_t *perms, uint8_t *n_out) {
    if (n_min < 1 || n_max > 16 || n_min > n_max || hard_min < 0 || hard_max < hard_min) return TD_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        uint64_t st = seed ^ (uint64_t)i;
        const int n = n_min + (int)bounded(st, (uint32_t)(n_max - n_min + 1));
        int8_t *p = perms + (size_t)i * 16;
        const bool hard = (int)bounded(st, 100) < hard_pct;
        if (hard) {
            for (int m = 0; m < n; ++m) p[m] = (int8_t)(n - 1 - m);
            const int moves = hard_min + (int)bounded(st, (uint32_t)(hard_max - hard_min + 1));
            const uint32_t triples = (uint32_t)((n + 1) * n * (n - 1) / 6);
            for (int mv = 0; mv < moves && triples > 0; ++mv) {
                int x, y, z;
                unrank_triple(n, bounded(st, triples), &x, &y, &z);
                int8_t tmp[16];
                int w = 0;
                for (int q = 0; q < x; ++q) tmp[w++] = p[q];
                for (int q = y; q < z; ++q) tmp[w++] = p[q];
                for (int q = x; q < y; ++q) tmp[w++] = p[q];
                for (int q = z; q < n; ++q) tmp[w++] = p[q];
                std::memcpy(p, tmp, (size_t)n);
            }
        } else {
            for (int m = 0; m < n; ++m) p[m] = (int8_t)m;
            for (int m = n - 1; m > 0; --m) {
                const int j = (int)bounded(st, (uint32_t)(m + 1));
                const int8_t t = p[m];
                p[m] = p[j];
                p[j] = t;
            }
        }
        for (int m = n; m < 16; ++m) p[m] = 0;
        n_out[i] = (uint8_t)n;
    }
    return TD_OK;
}

TD_API int td_search_batch_device(int slot, int count, const td_instance *d_in, td_result *d_out, unsigned flags,
                                  uint64_t max_exp, void *stream, char *err, size_t errlen) {
    Slot *s;
    {
        std::lock_guard<std::mutex> g(g_mu);
        s = get_slot(slot, err, errlen);
        if (!s) return TD_INVALID_ARG;
    }
    if (count < 0 || (count > 0 && (!d_in || !d_out))) {
        set_err(err, errlen, "invalid batch arguments");
        return TD_INVALID_ARG;
    }
    percall_park(s->device);
    std::lock_guard<std::mutex> g(*s->mu);
    TD_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    return launch_batch(*s, count, d_in, d_out, flags, max_exp, st, err, errlen);
}

TD_API int td_search_batch(int slot, int count, const td_instance *in, td_result *out, unsigned flags,
                           uint64_t max_exp, td_batch_stats *stats, char *err, size_t errlen) {
    Slot *s;
    {
        std::lock_guard<std::mutex> g(g_mu);
        s = get_slot(slot, err, errlen);
        if (!s) return TD_INVALID_ARG;
    }
    if (count < 0 || (count > 0 && (!in || !out))) {
        set_err(err, errlen, "invalid batch arguments");
        return TD_INVALID_ARG;
    }
    if (count == 0) {
        if (stats) std::memset(stats, 0, sizeof *stats);
        return TD_OK;
    }
    percall_park(s->device);
    std::lock_guard<std::mutex> g(*s->mu);
    TD_CHECK(cudaSetDevice(s->device));
    const size_t need = (size_t)count * (sizeof(td_instance) + sizeof(td_result));
    if (need > s->d_batch_bytes) {  // grows in stream order (no device-wide wait)
        if (s->d_batch) TD_CHECK(cudaFreeAsync(s->d_batch, s->stream));
        s->d_batch = nullptr;
        s->d_batch_bytes = 0;
        TD_CHECK(cudaMallocAsync(&s->d_batch, need, s->stream));
        s->d_batch_bytes = need;
    }
    if (stats && !s->d_counts) TD_CHECK(cudaMalloc(&s->d_counts, sizeof(td_counts)));
    if (stats && !s->h_stats) TD_CHECK(cudaMallocHost(&s->h_stats, sizeof(Slot::HostStats)));
    td_instance *d_in = (td_instance *)s->d_batch;
    td_result *d_out = (td_result *)((char *)s->d_batch + (size_t)count * sizeof(td_instance));
    TD_CHECK(cudaMemcpyAsync(d_in, in, (size_t)count * sizeof(td_instance), cudaMemcpyHostToDevice, s->stream));
    TD_CHECK(cudaEventRecord(s->t0, s->stream));
    int rc = launch_batch(*s, count, d_in, d_out, flags, max_exp, s->stream, err, errlen);
    if (rc != TD_OK) return rc;
    TD_CHECK(cudaEventRecord(s->t1, s->stream));
    const bool pooled = !(flags & (TD_FLAG_ORDERED | TD_FLAG_PLAIN)) && s->d_pool;
    if (stats) {
        TD_CHECK(cudaMemsetAsync(s->d_counts, 0, sizeof(td_counts), s->stream));
        const int blocks = std::max(1, std::min((count + 255) / 256, g_dev[s->device].sms * 8));
        td_count_kernel<<<blocks, 256, 0, s->stream>>>(d_out, count, s->d_counts);
        TD_CHECK(cudaGetLastError());
        TD_CHECK(cudaMemcpyAsync(&s->h_stats->counts, s->d_counts, sizeof(td_counts), cudaMemcpyDeviceToHost,
                                 s->stream));
        if (pooled)
            TD_CHECK(cudaMemcpyAsync(&s->h_stats->pool, s->d_pool, sizeof(td_pool), cudaMemcpyDeviceToHost,
                                     s->stream));
    }
    TD_CHECK(cudaMemcpyAsync(out, d_out, (size_t)count * sizeof(td_result), cudaMemcpyDeviceToHost, s->stream));
    TD_CHECK(cudaEventRecord(s->done, s->stream));
    TD_CHECK(cudaEventSynchronize(s->done));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        TD_CHECK(cudaEventElapsedTime(&stats->kernel_ms, s->t0, s->t1));
        if (pooled) {
            const td_pool &pool = s->h_stats->pool;
            stats->donations = pool.donations;
            stats->donated_items = pool.donated_items;
            stats->races = (uint64_t)pool.spawn_produced;
            if (pool.error) {
                set_err(err, errlen, "engine launch deadline reached");
                return TD_TIMEOUT;
            }
        }
        const td_counts &c = s->h_stats->counts;
        stats->expansions = c.expansions;
        stats->found = c.found;
        stats->not_found = c.not_found;
        stats->errors = c.errors;
    }
    return TD_OK;
}

// Many reference pairs in one call: the batch form of td_search for a case
// producer that hands over pairs in groups (the enumerator's
// Consumer<CyclicTargetPair>, DirectTwistedBraceletGenerator.java:105-156,
// feeds one pair per call today).  Pair i: beta/omega at stride 17, n[i]
// symbols, init[i], min_rate[i], max_moves[i], full[i].  Outputs per pair:
// status[i] (TD_OK found, TD_NOT_FOUND, or the per-call error class:
// TD_INVALID_ARG, TD_OVERFLOW, TD_TIMEOUT), depth[i] and the position
// triples at out_ijk[27 i ..].  Returns TD_OK when the batch ran (the pair
// statuses say the rest), else the error of the whole call.
TD_API int td_search_pairs(int slot, int count, const uint8_t *beta, const uint8_t *omega, const uint8_t *n,
                           const int32_t *init, const float *min_rate, const int32_t *max_moves,
                           const uint8_t *full, unsigned flags, int32_t *status, int32_t *depth, int16_t *out_ijk,
                           char *err, size_t errlen) {
    if (count < 0 || (count > 0 && (!beta || !omega || !n || !init || !min_rate || !max_moves || !full ||
                                    !status || !depth || !out_ijk))) {
        set_err(err, errlen, "invalid batch arguments");
        return TD_INVALID_ARG;
    }
    std::vector<td_instance> inst;
    std::vector<int> index;  // batch position -> pair
    inst.reserve(count);
    index.reserve(count);
    for (int i = 0; i < count; ++i) {
        depth[i] = 0;
        for (int q = 0; q < 27; ++q) out_ijk[27 * (size_t)i + q] = 0;
        if (n[i] > TD_MAX_N || max_moves[i] <= 0 || max_moves[i] > TD_MAX_DEPTH) {
            status[i] = TD_INVALID_ARG;
            continue;
        }
        if (td_triple_count(n[i]) == 0) {
            status[i] = TD_NOT_FOUND_RC;
            continue;
        }
        td_instance x;
        if (td_prepare_pair(beta + 17 * (size_t)i, omega + 17 * (size_t)i, n[i], init[i], min_rate[i],
                            max_moves[i], full[i], &x) != 0) {
            status[i] = TD_INVALID_ARG;
            continue;
        }
        inst.push_back(x);
        index.push_back(i);
    }
    if (inst.empty()) {
        Slot *s;
        std::lock_guard<std::mutex> g(g_mu);
        s = get_slot(slot, err, errlen);
        return s ? TD_OK : TD_INVALID_ARG;
    }
    std::vector<td_result> res(inst.size());
    const int rc = td_search_batch(slot, (int)inst.size(), inst.data(), res.data(), flags & TD_FLAG_ORDERED, 0,
                                   nullptr, err, errlen);
    if (rc != TD_OK) return rc;
    for (size_t b = 0; b < res.size(); ++b) {
        const int i = index[b];
        const td_result &r = res[b];
        if (r.status == TD_FOUND) {
            status[i] = TD_OK;
            depth[i] = r.depth;
            for (int d = 0; d < r.depth; ++d) {
                out_ijk[27 * (size_t)i + 3 * d + 0] = (int16_t)(r.moves[d] & 31);
                out_ijk[27 * (size_t)i + 3 * d + 1] = (int16_t)((r.moves[d] >> 5) & 31);
                out_ijk[27 * (size_t)i + 3 * d + 2] = (int16_t)((r.moves[d] >> 10) & 31);
            }
        } else if (r.status == TD_NOT_FOUND) {
            status[i] = TD_NOT_FOUND_RC;
        } else if (r.status == TD_ERR_BUDGET) {
            status[i] = TD_OVERFLOW;
        } else if (r.status == TD_ERR_TIMEOUT) {
            status[i] = TD_TIMEOUT;
        } else {
            status[i] = TD_INVALID_ARG;
        }
    }
    return TD_OK;
}

TD_API int td_validate_batch_device(int count, const td_instance *d_in, const td_result *d_res, uint8_t *d_ok,
                                    void *stream, char *err, size_t errlen) {
    if (count <= 0) return TD_OK;
    const int threads = 256;
    td_validate_kernel<<<(count + threads - 1) / threads, threads, 0, (cudaStream_t)stream>>>(
        d_in, const_cast<td_result *>(d_res), d_ok, count, 0);
    TD_CHECK(cudaGetLastError());
    return TD_OK;
}

TD_API void td_positions_to_symbols(const uint8_t *beta, int n, const int16_t *ijk, int depth, uint8_t *out_abc) {
    uint8_t cur[TD_MAX_N], nxt[TD_MAX_N];
    std::memcpy(cur, beta, (size_t)n);
    for (int d = 0; d < depth; ++d) {
        const int i = ijk[3 * d], j = ijk[3 * d + 1], k = ijk[3 * d + 2];
        out_abc[3 * d] = cur[i];
        out_abc[3 * d + 1] = cur[j];
        out_abc[3 * d + 2] = cur[k];
        int w = 0;
        for (int q = 0; q < i; ++q) nxt[w++] = cur[q];
        for (int q = j; q < k; ++q) nxt[w++] = cur[q];
        for (int q = i; q < j; ++q) nxt[w++] = cur[q];
        for (int q = k; q < n; ++q) nxt[w++] = cur[q];
        std::memcpy(cur, nxt, (size_t)n);
    }
}

namespace {

// Times one form of td_int_peak_kernel on the current device, doubling the
// iteration count until a launch lasts `target_ms`; returns warp instructions
// per second.
template <int MIX>
int time_int_peak(int sms, float target_ms, uint32_t *sink, cudaEvent_t a, cudaEvent_t b, double *rate) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, td_int_peak_kernel<MIX>, 256, 0) != cudaSuccess)
        return -1;
    const int blocks = sms * std::max(1, per_sm);
    int iters = 1024;
    float ms = 0;
    for (int attempt = 0; attempt < 12; ++attempt) {
        td_int_peak_kernel<MIX><<<blocks, 256>>>(sink, iters);  // warm-up at this size
        cudaEventRecord(a);
        td_int_peak_kernel<MIX><<<blocks, 256>>>(sink, iters);
        cudaEventRecord(b);
        if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return -1;
        if (ms >= target_ms) break;
        iters *= 2;
    }
    *rate = (double)blocks * (256 / 32) * (double)iters * 16.0 / (ms * 1e-3);
    return 0;
}

}  // namespace

// Measures the integer issue peaks of `device` in warp instructions per
// second: the full issue rate (LOP3 and IMAD interleaved) and the ALU-pipe
// rate (LOP3 only), each over about `target_ms`.
TD_API int td_int_issue_peak(int device, float target_ms, double *issue_per_s, double *alu_per_s, char *err,
                             size_t errlen) {
    TD_CHECK(cudaSetDevice(device));
    int sms = 0;
    TD_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    uint32_t *sink = nullptr;
    TD_CHECK(cudaMalloc(&sink, sizeof(uint32_t) * sms * 32));
    cudaEvent_t a, b;
    TD_CHECK(cudaEventCreate(&a));
    TD_CHECK(cudaEventCreate(&b));
    double issue = 0, alu = 0;
    const int rc = (time_int_peak<1>(sms, target_ms, sink, a, b, &issue) == 0 &&
                    time_int_peak<0>(sms, target_ms, sink, a, b, &alu) == 0) ? 0 : -1;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    TD_CHECK(cudaGetLastError());
    if (rc != 0) {
        set_err(err, errlen, "td_int_issue_peak: a probe launch failed");
        return TD_CUDA_ERROR;
    }
    if (issue_per_s) *issue_per_s = issue;
    if (alu_per_s) *alu_per_s = alu;
    return TD_OK;
}

// ---- batch search without device allocation ----------------------------------
//
// td_search_batch_noalloc is for callers that cannot call cudaMalloc or
// cudaFree: a slot worker that must not stall on the device-wide
// synchronisation those calls can imply while other slots' searches run on
// their own streams, or a host process whose device memory is already held by
// another allocator, so that a new allocation would fail although the caller's
// buffers exist.  The caller passes device buffers for instances and results;
// every other byte the search needs lives in td_noalloc_scratch below, a
// fixed array that each GPU loading this library holds until the process
// exits.  Limits: TD_NOALLOC_MAX_INSTANCES instances per call and
// TD_NOALLOC_ITEMS donated subtrees in flight (when the item space is full the
// donor keeps the work, so a full item space only costs balance, not results).
// All calls share this one array and it keeps the last call's contents, so
// calls whose launches overlap on the GPU race with each other: serialise
// them (e.g. issue them on one stream).

#define TD_NOALLOC_MAX_INSTANCES 65536
#define TD_NOALLOC_ITEMS 65536
#define TD_NOALLOC_HEAD 256                                             // pool, epoch, ticket
#define TD_NOALLOC_STATE_OFF TD_NOALLOC_HEAD
#define TD_NOALLOC_ITEMS_OFF (TD_NOALLOC_STATE_OFF + TD_NOALLOC_MAX_INSTANCES * 16)
#define TD_NOALLOC_READY_OFF (TD_NOALLOC_ITEMS_OFF + TD_NOALLOC_ITEMS * 32)
#define TD_NOALLOC_BYTES (TD_NOALLOC_READY_OFF + TD_NOALLOC_ITEMS * 4)   // 3.25 MiB + 256 B

static_assert(sizeof(td_pool) + 2 * sizeof(uint32_t) <= TD_NOALLOC_HEAD, "scratch head");
static_assert(sizeof(td_inst_state) == 16 && sizeof(td_item) == 32, "scratch records");

static __device__ __align__(256) uint8_t td_noalloc_scratch[TD_NOALLOC_BYTES];

namespace {

constexpr int kNoAllocDevices = 64;

// error reporting without heap use
#define TD_CHECK_NA(call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            if (err && errlen)                                                                     \
                std::snprintf(err, errlen, "%s:%d: CUDA error %s (%s)", __FILE__, __LINE__,         \
                              cudaGetErrorName(e_), cudaGetErrorString(e_));                       \
            return TD_CUDA_ERROR;                                                                  \
        }                                                                                          \
    } while (0)
#define TD_FAIL_NA(...)                                            \
    do {                                                           \
        if (err && errlen) std::snprintf(err, errlen, __VA_ARGS__); \
        return TD_INVALID_ARG;                                     \
    } while (0)

struct NoAllocDevice {
    bool ready;
    uint8_t *scratch;  // device address of td_noalloc_scratch on this device
    int sms;
    int steal_blocks;
    int persistent_blocks;
};

std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[kNoAllocDevices];
uint16_t g_noalloc_tri[TD_TRI_TABLE];  // host copies of the device tables, no heap
uint8_t g_noalloc_lut[TD_LUT_BYTES];

// Once per device, with that device current: uploads the triple and class
// tables and takes the scratch array's device address.  In host code the
// name td_noalloc_scratch is only a host-side stand-in, never a device address.
int noalloc_setup(int device, char *err, size_t errlen) {
    NoAllocDevice &d = g_noalloc[device];
    if (d.ready) return TD_OK;
    for (int N = 3; N <= TD_MAX_N; ++N) {
        int t = 0;
        const int base = td_tri_base(N);
        for (int i = 0; i < N - 2; ++i)
            for (int j = i + 1; j < N - 1; ++j)
                for (int k = j + 1; k < N; ++k) g_noalloc_tri[base + t++] = td_pack_move(i, j, k);
    }
    for (int i = 0; i < TD_LUT_BYTES; ++i) g_noalloc_lut[i] = (uint8_t)td_class_of_index(i);
    TD_CHECK_NA(cudaMemcpyToSymbol(td_tri_table, g_noalloc_tri, sizeof g_noalloc_tri));
    TD_CHECK_NA(cudaMemcpyToSymbol(td_lut_global, g_noalloc_lut, sizeof g_noalloc_lut));
    void *ptr = nullptr;
    TD_CHECK_NA(cudaGetSymbolAddress(&ptr, td_noalloc_scratch));
    TD_CHECK_NA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device));
    const size_t smem = smem_bytes(4);
    TD_CHECK_NA(cudaFuncSetAttribute(td_plain_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TD_CHECK_NA(cudaFuncSetAttribute(td_plain_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TD_CHECK_NA(cudaFuncSetAttribute(td_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    TD_CHECK_NA(cudaFuncSetAttribute(td_steal_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)steal_smem_bytes(4)));
    TD_CHECK_NA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.steal_blocks, td_steal_kernel, 128,
                                                              steal_smem_bytes(4)));
    TD_CHECK_NA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.persistent_blocks, td_persistent_kernel<true>,
                                                              128, smem));
    d.scratch = static_cast<uint8_t *>(ptr);
    d.ready = true;
    return TD_OK;
}

}  // namespace

// Batch search on the calling thread's current device that allocates no
// device memory.  d_instances / d_results: caller-owned device buffers of
// `count` records; flags as for td_search_batch_device (TD_FLAG_ORDERED,
// TD_FLAG_PLAIN, TD_FLAG_VERIFY).  Enqueues on `stream` and returns.  The
// first call on a device performs the one-time set-up above (table uploads
// and a symbol-address query, both synchronous), so make that first call
// before any stream capture.  count > 65536 is rejected.
TD_API int td_search_batch_noalloc(int count, const td_instance *d_instances, td_result *d_results, unsigned flags,
                                   uint64_t max_exp, void *stream, char *err, size_t errlen) {
    if (count < 0 || count > TD_NOALLOC_MAX_INSTANCES)
        TD_FAIL_NA("td_search_batch_noalloc: count %d outside 0..%d (the fixed scratch holds at most %d instances)",
                   count, TD_NOALLOC_MAX_INSTANCES, TD_NOALLOC_MAX_INSTANCES);
    if (count == 0) return TD_OK;
    if (!d_instances || !d_results) TD_FAIL_NA("td_search_batch_noalloc: null instance or result buffer");
    int device = 0;
    TD_CHECK_NA(cudaGetDevice(&device));
    if (device < 0 || device >= kNoAllocDevices)
        TD_FAIL_NA("td_search_batch_noalloc: device ordinal %d out of range", device);
    NoAllocDevice d;
    {
        std::lock_guard<std::mutex> g(g_noalloc_mu);
        const int rc = noalloc_setup(device, err, errlen);
        if (rc != TD_OK) return rc;
        d = g_noalloc[device];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int warps = 4, threads = 128;
    const size_t smem = smem_bytes(warps);
    const bool ordered = flags & TD_FLAG_ORDERED;
    const uint64_t limit = time_limit_ns();
    td_pool *pool = reinterpret_cast<td_pool *>(d.scratch);
    uint32_t *epoch = reinterpret_cast<uint32_t *>(d.scratch + sizeof(td_pool));
    int *ticket = reinterpret_cast<int *>(d.scratch + sizeof(td_pool) + sizeof(uint32_t));
    td_inst_state *state = reinterpret_cast<td_inst_state *>(d.scratch + TD_NOALLOC_STATE_OFF);
    td_item *items = reinterpret_cast<td_item *>(d.scratch + TD_NOALLOC_ITEMS_OFF);
    uint32_t *ready = reinterpret_cast<uint32_t *>(d.scratch + TD_NOALLOC_READY_OFF);
    const int blocks_needed = (count + warps - 1) / warps;
    if (flags & TD_FLAG_PLAIN) {
        if (ordered)
            td_plain_kernel<true><<<blocks_needed, threads, smem, st>>>(d_instances, d_results, count, max_exp, limit);
        else
            td_plain_kernel<false><<<blocks_needed, threads, smem, st>>>(d_instances, d_results, count, max_exp, limit);
    } else if (ordered) {
        TD_CHECK_NA(cudaMemsetAsync(ticket, 0, sizeof(int), st));
        const int grid = std::max(1, std::min(d.sms * std::max(1, d.persistent_blocks), blocks_needed));
        td_persistent_kernel<true><<<grid, threads, smem, st>>>(d_instances, d_results, count, ticket, 1, max_exp,
                                                                limit);
    } else {
        // the donation settings, read together (a concurrent td_configure_steal
        // or td_configure_restart writes them under the same lock)
        int grain, split_level, check_every;
        uint32_t restart_base;
        {
            std::lock_guard<std::mutex> g(g_mu);
            grain = g_steal_grain;
            split_level = g_split_level;
            check_every = g_check_every;
            restart_base = g_restart_base;
        }
        // counters and per-instance state start at zero on every call; items
        // are tagged with a fresh epoch so an earlier call's items never count
        TD_CHECK_NA(cudaMemsetAsync(pool, 0, sizeof(td_pool), st));
        TD_CHECK_NA(cudaMemsetAsync(state, 0, (size_t)count * sizeof(td_inst_state), st));
        td_epoch_kernel<<<1, 1, 0, st>>>(epoch);
        // the whole resident grid (the scratch does not depend on its size):
        // warps without an instance of their own take donated subtrees, so a
        // small batch is spread over the GPU; a single search wakes its
        // waiting warps sooner (backoff cap 4 us instead of 32 us)
        const int grid = d.sms * std::max(1, d.steal_blocks);
        td_steal_kernel<<<grid, threads, steal_smem_bytes(warps), st>>>(
            d_instances, d_results, count, pool, items, ready, epoch, TD_NOALLOC_ITEMS, state, grain, split_level,
            check_every, limit, nullptr, nullptr, 0, restart_base, max_exp, count == 1 ? 4096u : 32768u,
            /*race=*/0, /*spawn_base=*/TD_NOALLOC_ITEMS);
        TD_CHECK_NA(cudaGetLastError());
        td_finalize_kernel<<<std::max(1, std::min((count + 255) / 256, 2 * d.sms)), 256, 0, st>>>(pool, state,
                                                                                                d_results, count);
    }
    TD_CHECK_NA(cudaGetLastError());
    if (flags & TD_FLAG_VERIFY) {
        td_validate_kernel<<<(count + 255) / 256, 256, 0, st>>>(d_instances, d_results, nullptr, count, 1);
        TD_CHECK_NA(cudaGetLastError());
    }
    return TD_OK;
}

// ---- CUDA graphs -------------------------------------------------------------

namespace {
struct BatchGraph {
    int device;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};
}  // namespace

// Captures one batch launch (search, and the device replay when flags has
// TD_FLAG_VERIFY) over fixed device buffers into a CUDA graph.  Replaying it
// with td_batch_graph_launch costs one graph launch per batch.
TD_API int td_batch_graph_create(int slot, int count, const td_instance *d_in, td_result *d_out, unsigned flags,
                                 uint64_t max_exp, void **out_graph, char *err, size_t errlen) {
    Slot *s;
    {
        std::lock_guard<std::mutex> g(g_mu);
        s = get_slot(slot, err, errlen);
        if (!s) return TD_INVALID_ARG;
    }
    if (!out_graph || count <= 0) {
        set_err(err, errlen, "invalid graph arguments");
        return TD_INVALID_ARG;
    }
    percall_park(s->device);
    std::lock_guard<std::mutex> g(*s->mu);
    TD_CHECK(cudaSetDevice(s->device));
    // one eager launch sizes the slot's scratch outside the capture
    int rc = launch_batch(*s, count, d_in, d_out, flags, max_exp, s->stream, err, errlen);
    if (rc != TD_OK) return rc;
    TD_CHECK(cudaStreamSynchronize(s->stream));
    auto *bg = new BatchGraph();
    bg->device = s->device;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = launch_batch(*s, count, d_in, d_out, flags, max_exp, s->stream, err, errlen);
        e = cudaStreamEndCapture(s->stream, &bg->graph);
        if (rc != TD_OK) {
            if (bg->graph) cudaGraphDestroy(bg->graph);
            delete bg;
            return rc;
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&bg->exec, bg->graph, 0);
    if (e != cudaSuccess) {
        if (bg->graph) cudaGraphDestroy(bg->graph);
        delete bg;
        set_err(err, errlen, cuda_msg(e, __FILE__, __LINE__));
        return TD_CUDA_ERROR;
    }
    *out_graph = bg;
    return TD_OK;
}

TD_API int td_batch_graph_launch(void *graph, void *stream, char *err, size_t errlen) {
    auto *bg = static_cast<BatchGraph *>(graph);
    if (!bg) return TD_INVALID_ARG;
    percall_park(bg->device);
    TD_CHECK(cudaSetDevice(bg->device));
    TD_CHECK(cudaGraphLaunch(bg->exec, (cudaStream_t)stream));
    return TD_OK;
}

TD_API int td_batch_graph_destroy(void *graph) {
    auto *bg = static_cast<BatchGraph *>(graph);
    if (!bg) return TD_INVALID_ARG;
    cudaSetDevice(bg->device);
    if (bg->exec) cudaGraphExecDestroy(bg->exec);
    if (bg->graph) cudaGraphDestroy(bg->graph);
    delete bg;
    return TD_OK;
}

#include "td_serve.cuh"
#include "td_percall.cuh"

// defined in td_cert.cu
int td_cert_preload(void);

namespace {

int preload_kernels(char *err, size_t errlen) {
    cudaFuncAttributes a;
    TD_CHECK(cudaFuncGetAttributes(&a, td_plain_kernel<true>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_plain_kernel<false>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_persistent_kernel<true>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_persistent_kernel<false>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_steal_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_split_roots_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_split_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_split_join_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_epoch_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_finalize_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_count_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_validate_kernel));
    TD_CHECK(cudaFuncGetAttributes(&a, td_int_peak_kernel<0>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_int_peak_kernel<1>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_serve_kernel<TD_SERVE_FREE>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_serve_kernel<TD_SERVE_ORDERED>));
    TD_CHECK(cudaFuncGetAttributes(&a, td_serve_kernel<TD_SERVE_PER_REQUEST>));
    TD_CHECK((cudaError_t)td_cert_preload());
    return TD_OK;
}

}  // namespace
