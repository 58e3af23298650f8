// td_kernels.cuh -- the sm_100a witness-search warp engine.
//
// One warp owns one search (a DFS over move sequences).  Per node it
//   1. labels the omega cycles of the pinned state with warp pointer jumping
//      (lane p = pinned position p; leader = smallest position, dist = steps
//      to the leader, len = cycle length; 5 rounds cover cycles up to 32),
//   2. writes the pair table (4 bits per ordered pair of caller positions),
//   3. evaluates every triple: lane l takes u = 32*s + l in step s, reads three
//      pair entries and one class-table byte (no pointer chasing), and keeps
//      one bit per step in per-lane masks (found / first-choice / second-choice),
//   4. picks the next child with a warp max-reduction over the masks in the
//      reference's single-queue order (ordered mode) or +2 moves first.
// Reference: emitter/src/native/backtracking/sorting_search.cu:478-712.
#pragma once

#include "td_core.cuh"

#define TD_FULL 0xffffffffu
#define TD_PT_ROWS 18          // 17 position rows + one zero row for idle lanes
#define TD_PT_DUMMY (17 * TD_PT_STRIDE)
#define TD_TRI_TABLE 3060      // sum over N <= 17 of C(N,3) = C(18,4)
#define TD_G0 0x09249249u      // bit 0 of each 3-bit group
#define TD_G1 0x12492492u      // bit 1 of each group
#define TD_G2 0x24924924u      // bit 2 of each group

// floor(b / 3) for 0 <= b <= 29: the step of a bit inside a packed word
__device__ __forceinline__ int td_group_of(int b) { return (b * 11) >> 5; }

// Per-warp shared state.
struct td_warp_smem {
    uint8_t pt[TD_PT_ROWS * TD_PT_STRIDE];     // pair table of the current node
    // per level, per lane: the outcome of every step in 3-bit groups, ten
    // steps per word (step st in word st/10 at bit 3*(st%10)): bit 0 found
    // (accepted root in ordered mode), bit 1 first-choice child, bit 2
    // second-choice child
    uint32_t pm[TD_MAX_DEPTH][3][32];
    uint64_t L[TD_MAX_DEPTH + 1];              // pinned state per level
    uint32_t acc[TD_MAX_DEPTH + 2];            // accept mask over odd counts, per depth
    uint32_t reach[TD_MAX_DEPTH + 2];          // prune mask over odd counts, per depth
    uint16_t path[TD_MAX_DEPTH];               // caller-position move per level
    uint8_t off[TD_MAX_DEPTH + 1];
    alignas(16) uint8_t lead[32];              // cycle leader by caller position
    alignas(16) uint8_t dist[32];              // omega steps to the leader
};

// Lexicographic position triples i|j<<5|k<<10 for every N, at offset C(N,4).
__device__ uint16_t td_tri_table[TD_TRI_TABLE];

TD_HD int td_tri_base(int N) {
    return N < 4 ? 0 : N * (N - 1) * (N - 2) * (N - 3) / 24;
}

// Load this lane's per-step pair-table offsets for triples of size N.
__device__ __forceinline__ void td_load_codes(int N, uint32_t (&code)[TD_MAX_STEPS]) {
    const int lane = threadIdx.x & 31;
    const int T = td_triple_count(N);
    const int base = td_tri_base(N);
#pragma unroll
    for (int s = 0; s < TD_MAX_STEPS; ++s) {
        const int u = 32 * s + lane;
        uint32_t c = TD_PT_DUMMY | (TD_PT_DUMMY << 10) | (TD_PT_DUMMY << 20);
        if (u < T) {
            const uint32_t t = td_tri_table[base + T - 1 - u];
            const uint32_t i = t & 31, j = (t >> 5) & 31, k = (t >> 10) & 31;
            c = (i * TD_PT_STRIDE + j) | ((j * TD_PT_STRIDE + k) << 10) | ((k * TD_PT_STRIDE + i) << 20);
        }
        code[s] = c;
    }
}

// Cycle labels and pair table for the state (L, off); returns the number of
// odd-length omega cycles.
__device__ __forceinline__ int td_prepare_node(td_warp_smem &s, uint64_t L, int off, int N) {
    const int p = threadIdx.x & 31;
    const bool act = p < N;
    const uint32_t Bp = (p == 0 || !act) ? 0u : td_nib(L, p - 1) + 1u;
    // inverse of L by a warp OR of one nibble per lane
    uint32_t lo = 0, hi = 0;
    if (p < N - 1) {
        const uint64_t c = (uint64_t)p << (4 * td_nib(L, p));
        lo = (uint32_t)c;
        hi = (uint32_t)(c >> 32);
    }
    lo = __reduce_or_sync(TD_FULL, lo);
    hi = __reduce_or_sync(TD_FULL, hi);
    const uint64_t inv = ((uint64_t)hi << 32) | lo;
    // omega(B[p]) = B[p-1] + 1 (mod N): next position along omega
    const uint32_t Bq = __shfl_sync(TD_FULL, Bp, p == 0 ? N - 1 : p - 1);
    uint32_t y = Bq + 1;
    if (y == (uint32_t)N) y = 0;
    const int nx = act ? (y ? (int)td_nib(inv, (int)y - 1) + 1 : 0) : p;
    // leader = smallest position on the cycle and dist = omega steps to it,
    // in one pointer-jumping pass: each lane keeps the minimum of the window
    // p, next(p), ..., next^(w-1)(p) and its distance; windows double per round
    // and 32 >= any cycle length, so the first occurrence of the minimum wins.
    int m = p, d = 0, j = nx;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int mB = __shfl_sync(TD_FULL, m, j);
        const int dB = __shfl_sync(TD_FULL, d, j);
        const int jB = __shfl_sync(TD_FULL, j, j);
        if (mB < m) {
            m = mB;
            d = (1 << r) + dB;
        }
        j = jB;
    }
    const bool leader = m == p;
    const int after_leader = __shfl_sync(TD_FULL, nx, m);
    const int len = __shfl_sync(TD_FULL, d, after_leader) + 1;
    const int odd = __popc(__ballot_sync(TD_FULL, act && leader && (len & 1)));
    // descriptors by caller position, one byte each
    int rp = p - off;
    rp += rp < 0 ? N : 0;
    if (act) {
        s.lead[rp] = (uint8_t)m;
        s.dist[rp] = (uint8_t)d;
    }
    __syncwarp();
    // pair table row of this lane's caller position, four entries per word
    // (byte-SIMD: every byte stays below 0x80, so no borrow crosses a byte)
    const uint32_t H = 0x80808080u, ONE = 0x01010101u;
    const uint32_t Mp = (uint32_t)m * ONE, Dp = (uint32_t)d * ONE;
    const uint32_t O8 = (len & 1) ? 0x08080808u : 0u;
    const uint32_t F4 = len == 1 ? 0x04040404u : 0u;
    const uint32_t Lodd = (len & 1) ? ONE : 0u;
    const uint4 ml = *reinterpret_cast<const uint4 *>(s.lead);
    const uint4 dl = *reinterpret_cast<const uint4 *>(s.dist);
    const uint32_t m4 = *reinterpret_cast<const uint32_t *>(s.lead + 16);
    const uint32_t d4 = *reinterpret_cast<const uint32_t *>(s.dist + 16);
    const uint32_t Mw[5] = {ml.x, ml.y, ml.z, ml.w, m4};
    const uint32_t Dw[5] = {dl.x, dl.y, dl.z, dl.w, d4};
    uint32_t row[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const uint32_t xm = (Mw[k] ^ Mp) | H;
        const uint32_t same = ~(xm - ONE) & H;                          // 0x80 where leaders match
        const uint32_t gt = ((Dp | H) - Dw[k] - ONE) & H;               // 0x80 where dist_p > dist_q
        const uint32_t G = gt >> 7;
        uint32_t P = (Dp ^ Dw[k]) & ONE;                                // parity of the dist difference
        P ^= (G ^ ONE) & Lodd;                                          // wrap of an odd cycle flips it
        const uint32_t sel = (same << 1) - (same >> 7);                 // 0xff in bytes with the same leader
        const uint32_t in_cycle = ONE | (P << 1) | (G << 2) | O8;
        const uint32_t apart = F4 | O8;
        row[k] = (in_cycle & sel) | (apart & ~sel);
    }
    if (act) {
        uint32_t *dst = reinterpret_cast<uint32_t *>(&s.pt[rp * TD_PT_STRIDE]);
        *reinterpret_cast<uint4 *>(dst) = make_uint4(row[0], row[1], row[2], row[3]);
        dst[4] = row[4];
    }
    return odd;
}

// Accept / prune masks of one instance: lane D computes the masks of depth D
// over all odd counts.  With full sorting the accept test only passes at
// odd == N and its f32 rate part depends on D alone, and the prune bound
// D + ceil((N - odd)/2) <= maxDepth is a threshold on odd, so both masks take
// one f32 division per lane.  Partial sorting evaluates every odd count.
__device__ __forceinline__ void td_rate_masks(td_warp_smem &s, const td_instance &x) {
    const int D = threadIdx.x & 31;
    const int N = x.n_symbols, init = td_inst_init(x), full = td_inst_full(x);
    const int maxd = x.max_moves;
    uint32_t a = 0, r = 0;
    if (D <= TD_MAX_DEPTH + 1) {
        if (full) {
            if (td_accepts(N, init, x.min_rate, 1, N, D)) a = 1u << N;
            if (D < maxd) {
                // D + (N - odd + 1) / 2 <= maxd  <=>  odd >= N - 2 * (maxd - D)
                const int lo = N - 2 * (maxd - D);
                r = lo <= 0 ? 0xffffffffu : (0xffffffffu << lo);
            }
        } else {
            for (int o = 0; o < 32; ++o) {
                if (td_accepts(N, init, x.min_rate, 0, o, D)) a |= 1u << o;
                if (D < maxd && td_can_reach(N, init, x.min_rate, maxd, 0, o, D)) r |= 1u << o;
            }
        }
        s.acc[D] = a;
        s.reach[D] = r;
    }
    __syncwarp();
}

struct td_search_limits {
    uint64_t max_expansions;   // per search; TD_ERR_BUDGET when exceeded
    uint64_t deadline_ns;      // %globaltimer value; 0 = none
    const int *abort_flag;     // optional host/device abort request
};

__device__ __forceinline__ uint64_t td_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Evaluate all children of the node at `level`.  Fills the level's packed
// outcome words and returns the found child's u, or -1.
template <bool ORDERED>
__device__ __forceinline__ int td_evaluate(td_warp_smem &s, const uint8_t *lut,
                                           const uint32_t (&code)[TD_MAX_STEPS], int steps,
                                           int level, int odd, int maxd) {
    const int lane = threadIdx.x & 31;
    const int D = level + 1;
    const uint32_t accD = s.acc[D], reachD = s.reach[D];
    const uint32_t f0 = (accD >> odd) & 1u, f2 = (accD >> (odd + 2)) & 1u;
    const uint32_t x0 = ((reachD >> odd) & 1u) & (f0 ^ 1u);
    const uint32_t x2 = ((reachD >> (odd + 2)) & 1u) & (f2 ^ 1u);
    // byte c of nt holds the flags of class c; byte 0 (filtered out) is zero
    const uint32_t flags0 = ORDERED ? (f0 | (x0 << 1)) : (f0 | (x0 << 2));
    const uint32_t flags2 = f2 | (x2 << 1);
    const uint32_t nt = (flags0 << (8 * TD_CLASS_ZERO)) | (flags2 << (8 * TD_CLASS_PLUS2));
    (void)maxd;
    __syncwarp();
    uint32_t P0 = 0, P1 = 0, P2 = 0;
#pragma unroll
    for (int st = 0; st < TD_MAX_STEPS; ++st) {
        if (st < steps) {
            const uint32_t c = code[st];
            const uint32_t A = s.pt[c & 1023u];
            const uint32_t B = s.pt[(c >> 10) & 1023u];
            const uint32_t C = s.pt[c >> 20];
            const uint32_t cls = lut[A | (B << 4) | (C << 8)];
            const uint32_t tb = __byte_perm(nt, 0, cls);  // flags of this child's class
            const uint32_t mul = 1u << (3 * (st % 10));
            if (st < 10) P0 += tb * mul;
            else if (st < 20) P1 += tb * mul;
            else P2 += tb * mul;
        }
    }
    s.pm[level][0][lane] = P0;
    s.pm[level][1][lane] = P1;
    s.pm[level][2][lane] = P2;
    if (ORDERED && level == 0) return -1;  // roots are accepted on visit, not on seeding
    const uint32_t q0 = P0 & TD_G0, q1 = P1 & TD_G0, q2 = P2 & TD_G0;
    if (__any_sync(TD_FULL, (q0 | q1 | q2) != 0)) {
        int st = -1;
        if (q0) st = td_group_of(__ffs(q0) - 1);
        else if (q1) st = 10 + td_group_of(__ffs(q1) - 1);
        else if (q2) st = 20 + td_group_of(__ffs(q2) - 1);
        const uint32_t key = st >= 0 ? ((uint32_t)st << 5) | (uint32_t)lane : 0xffffffffu;
        return (int)__reduce_min_sync(TD_FULL, key);
    }
    return -1;
}

// Next child of `level`; returns u or -1.  *accepted is set for a root that
// is accepted when visited (ordered mode).
template <bool ORDERED>
__device__ __forceinline__ int td_next_child(td_warp_smem &s, int level, int *accepted) {
    const int lane = threadIdx.x & 31;
    const uint32_t P0 = s.pm[level][0][lane], P1 = s.pm[level][1][lane], P2 = s.pm[level][2][lane];
    const bool desc_lanes = ORDERED && level > 0;
    uint32_t cm;
    if (ORDERED) {
        cm = level == 0 ? (TD_G0 | TD_G1) : TD_G1;
    } else {
        const bool any1 = __any_sync(TD_FULL, ((P0 | P1 | P2) & TD_G1) != 0);
        cm = any1 ? TD_G1 : TD_G2;  // +2 children first
    }
    const uint32_t w0 = P0 & cm, w1 = P1 & cm, w2 = P2 & cm;
    int st = -1;
    if (w2) st = 20 + td_group_of(31 - __clz(w2));
    else if (w1) st = 10 + td_group_of(31 - __clz(w1));
    else if (w0) st = td_group_of(31 - __clz(w0));
    uint32_t key = 0;
    if (st >= 0) key = ((uint32_t)st << 5) + (uint32_t)(desc_lanes ? 31 - lane : lane) + 1u;
    key = __reduce_max_sync(TD_FULL, key);
    *accepted = 0;
    if (key == 0) return -1;
    key -= 1;
    st = (int)(key >> 5);
    const int win = desc_lanes ? 31 - (int)(key & 31) : (int)(key & 31);
    const int k = st < 10 ? 0 : (st < 20 ? 1 : 2);
    const int j = st - 10 * k;
    const uint32_t Pk = k == 0 ? P0 : (k == 1 ? P1 : P2);
    if (ORDERED && level == 0) *accepted = __shfl_sync(TD_FULL, (int)((Pk >> (3 * j)) & 1u), win);
    if (lane == win) s.pm[level][k][lane] = Pk & ~(7u << (3 * j));
    __syncwarp();
    return st * 32 + win;
}

// ---- work items (subtree roots handed between warps) ----------------------

// A node that is known to be expandable, with the moves that lead to it.
struct __align__(16) td_item {  // 32 bytes
    uint64_t L;
    uint32_t inst;          // instance index
    uint8_t depth;          // >= 1
    uint8_t off;
    uint16_t path[TD_MAX_DEPTH];
};

// Per-instance bookkeeping when several warps share one search.
struct td_inst_state {
    int found;              // set once by the warp that records the witness
    int pending;            // units (the root search + items) not yet finished
    unsigned expansions;    // summed over units
    int error;              // first error status seen (timeout)
};

// Scheduler counters of one launch.
struct td_pool {
    int inst_ticket;        // next fresh instance
    int produced;           // items reserved by donors
    int consumed;           // items claimed by takers
    int active;             // warps inside a unit or claiming one
    int idle;               // warps waiting for donated work
    int error;              // launch-level error (bounded wait expired)
    unsigned long long donations;
    unsigned long long donated_items;
};

// Donated items live either in a per-launch array (batch launches: index i
// at slot i, ready[i] == epoch once written) or in a ring (the serving launch:
// index i at slot i % capacity, ready == td_ring_tag(i) once written and
// td_ring_tag(i) | 0x80000000 once its taker has read it, which frees the slot).
__device__ __forceinline__ uint32_t td_ring_tag(long long i) { return (uint32_t)((i + 1) & 0x7fffffff); }

struct td_donate_ctx {
    int ring;
    uint64_t deadline_ns;   // bounds the wait for a ring slot to be freed
    td_pool *pool;
    td_item *items;
    uint32_t *ready;
    uint32_t epoch;
    int capacity;
    int grain;              // at most this many items per donation
    int max_level;          // donate only children of levels <= max_level
    int check_every;        // expansions between idle checks
    uint32_t inst;
    td_inst_state *state;
};

#define TD_DFS_FOUND 1
#define TD_DFS_EXHAUSTED 0
#define TD_DFS_BUDGET (-2)
#define TD_DFS_TIMEOUT (-5)
#define TD_DFS_ABORTED (-7)

struct td_dfs_out {
    int status;
    int depth;
    uint16_t found_move;
    uint32_t expansions;
};

// Hands some remaining children of the shallowest level in [d0, level] to the
// pool as items.  Returns the number donated (uniform across the warp).
__device__ __forceinline__ int td_donate(td_warp_smem &s, const td_donate_ctx &dc, int d0, int level, int N,
                                         int T, int tri_base, int want) {
    const int lane = threadIdx.x & 31;
    const uint32_t CAND = TD_G1 | TD_G2;
    int lv = -1;
    for (int l = d0; l <= level && l <= dc.max_level; ++l) {
        const uint32_t w = (s.pm[l][0][lane] | s.pm[l][1][lane] | s.pm[l][2][lane]) & CAND;
        if (__any_sync(TD_FULL, w != 0)) { lv = l; break; }
    }
    if (lv < 0) return 0;
    uint32_t P0 = s.pm[lv][0][lane], P1 = s.pm[lv][1][lane], P2 = s.pm[lv][2][lane];
    uint32_t Q0 = P0 & CAND, Q1 = P1 & CAND, Q2 = P2 & CAND;
    const int cnt = __popc(Q0) + __popc(Q1) + __popc(Q2);
    const int have = __reduce_add_sync(TD_FULL, (unsigned)cnt);
    // leave at least one child to this warp when the level is the current one
    const int give = min(want, have - (lv == level ? 1 : 0));
    if (give <= 0) return 0;
    int before = cnt;  // lanes give in lane order
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(TD_FULL, before, o);
        if (lane >= o) before += v;
    }
    before -= cnt;
    const int mine = max(0, min(cnt, give - before));
    // reserve `give` item slots; the count never passes the capacity and never
    // goes back, so a taker only ever claims slots that a donor will write
    int base = -1;
    if (lane == 0) {
        int cur = *(volatile int *)&dc.pool->produced;
        for (;;) {
            // a ring holds at most `capacity` items that are not yet claimed
            const int used = dc.ring ? cur - *(volatile int *)&dc.pool->consumed : cur;
            if (used + give > dc.capacity) break;
            const int prev = atomicCAS(&dc.pool->produced, cur, cur + give);
            if (prev == cur) { base = cur; break; }
            cur = prev;
        }
        // the pending count must cover the items before any taker can finish one
        if (base >= 0) atomicAdd(&dc.state->pending, give);
        __threadfence();
    }
    base = __shfl_sync(TD_FULL, base, 0);
    if (base < 0) return 0;  // out of item space: keep the work
    if (lane == 0) {
        atomicAdd(&dc.pool->donations, 1ull);
        atomicAdd(&dc.pool->donated_items, (unsigned long long)give);
    }
    int slot = base + before;
    for (int taken = 0; taken < mine; ++taken) {
        int k, b;
        if (Q0) { k = 0; b = __ffs(Q0) - 1; Q0 &= Q0 - 1; }
        else if (Q1) { k = 1; b = __ffs(Q1) - 1; Q1 &= Q1 - 1; }
        else { k = 2; b = __ffs(Q2) - 1; Q2 &= Q2 - 1; }
        const int j = td_group_of(b);
        const uint32_t clear = ~(7u << (3 * j));
        if (k == 0) P0 &= clear;
        else if (k == 1) P1 &= clear;
        else P2 &= clear;
        const int u = 32 * (10 * k + j) + lane;
        const uint32_t t = td_tri_table[tri_base + T - 1 - u];
        uint64_t nL;
        int noff;
        td_apply_move(s.L[lv], s.off[lv], N, t & 31, (t >> 5) & 31, (t >> 10) & 31, &nL, &noff);
        td_item it;
        it.L = nL;
        it.inst = dc.inst;
        it.depth = (uint8_t)(lv + 1);
        it.off = (uint8_t)noff;
#pragma unroll
        for (int d = 0; d < TD_MAX_DEPTH; ++d) it.path[d] = d < lv ? s.path[d] : (d == lv ? (uint16_t)t : 0);
        int phys = slot;
        uint32_t tag = dc.epoch;
        if (dc.ring) {
            phys = slot % dc.capacity;
            tag = td_ring_tag(slot);
            if (slot >= dc.capacity) {
                // the slot's previous item (index slot - capacity) is claimed;
                // wait until its taker has read it (bounded)
                const uint32_t freed = td_ring_tag(slot - dc.capacity) | 0x80000000u;
                for (unsigned spin = 0; *(volatile uint32_t *)&dc.ready[phys] != freed; ++spin) {
                    if ((spin & 255u) == 0 && dc.deadline_ns && td_globaltimer() > dc.deadline_ns) break;
                    __nanosleep(64);
                }
            }
        }
        dc.items[phys] = it;
        __threadfence();
        atomicExch(&dc.ready[phys], tag);
        ++slot;
    }
    s.pm[lv][0][lane] = P0;
    s.pm[lv][1][lane] = P1;
    s.pm[lv][2][lane] = P2;
    __syncwarp();
    return give;
}

// Depth-first search from the node held at level d0 of `s` (state, path and
// rate masks already set).  Leaves the frames intact on TD_DFS_BUDGET.
template <bool ORDERED>
__device__ td_dfs_out td_dfs(td_warp_smem &s, const uint8_t *lut, const uint32_t (&code)[TD_MAX_STEPS],
                             int N, int maxd, int d0, const td_search_limits &lim, const td_donate_ctx *dc) {
    const int lane = threadIdx.x & 31;
    const int T = td_triple_count(N);
    const int steps = (T + 31) >> 5;
    const int tri_base = td_tri_base(N);
    td_dfs_out r;
    r.status = TD_DFS_EXHAUSTED;
    r.depth = 0;
    r.found_move = 0;
    r.expansions = 0;
    int level = d0;
    int odd = td_prepare_node(s, s.L[d0], s.off[d0], N);
    int found = td_evaluate<ORDERED>(s, lut, code, steps, d0, odd, maxd);
    r.expansions = 1;
    for (;;) {
        if (found >= 0) {
            r.found_move = (uint16_t)td_tri_table[tri_base + T - 1 - found];
            r.depth = level + 1;
            r.status = TD_DFS_FOUND;
            break;
        }
        if (r.expansions >= lim.max_expansions) {
            r.status = TD_DFS_BUDGET;
            break;
        }
        if (dc && (r.expansions % (uint32_t)dc->check_every) == 0) {
            int hungry = 0, stop = 0;
            if (lane == 0) {
                hungry = *(volatile int *)&dc->pool->idle;
                stop = *(volatile int *)&dc->state->found;
            }
            stop = __shfl_sync(TD_FULL, stop, 0);
            if (stop) {
                r.status = TD_DFS_ABORTED;
                break;
            }
            hungry = __shfl_sync(TD_FULL, hungry, 0);
            if (hungry > 0) td_donate(s, *dc, d0, level, N, T, tri_base, min(hungry, dc->grain));
        }
        if ((r.expansions & 255u) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (lim.deadline_ns && td_globaltimer() > lim.deadline_ns) stop = 1;
                if (lim.abort_flag && *(volatile const int *)lim.abort_flag) stop = 1;
            }
            if (__shfl_sync(TD_FULL, stop, 0)) {
                r.status = TD_DFS_TIMEOUT;
                break;
            }
        }
        int accepted;
        const int u = td_next_child<ORDERED>(s, level, &accepted);
        if (u < 0) {
            if (level == d0) break;  // this subtree is exhausted
            --level;
            continue;
        }
        const uint32_t t = td_tri_table[tri_base + T - 1 - u];
        if (accepted) {
            r.found_move = (uint16_t)t;
            r.depth = level + 1;
            r.status = TD_DFS_FOUND;
            break;
        }
        uint64_t nL;
        int noff;
        td_apply_move(s.L[level], s.off[level], N, t & 31, (t >> 5) & 31, (t >> 10) & 31, &nL, &noff);
        __syncwarp();
        if (lane == 0) {
            s.path[level] = (uint16_t)t;
            s.L[level + 1] = nL;
            s.off[level + 1] = (uint8_t)noff;
        }
        ++level;
        odd = td_prepare_node(s, nL, noff, N);
        found = td_evaluate<ORDERED>(s, lut, code, steps, level, odd, maxd);
        ++r.expansions;
    }
    __syncwarp();
    return r;
}

__device__ __forceinline__ bool td_instance_ok(const td_instance &x) {
    return x.n_symbols <= TD_MAX_N && x.max_moves >= 1 && x.max_moves <= TD_MAX_DEPTH &&
           td_inst_init(x) <= TD_MAX_N;
}

// Loads codes for N and the instance's rate masks; places its root at level 0.
__device__ __forceinline__ void td_setup_root(td_warp_smem &s, const td_instance &x, uint32_t (&code)[TD_MAX_STEPS],
                                              int &codeN) {
    const int lane = threadIdx.x & 31;
    if (codeN != x.n_symbols) {
        td_load_codes(x.n_symbols, code);
        codeN = x.n_symbols;
    }
    td_rate_masks(s, x);
    if (lane == 0) {
        s.L[0] = x.perm;
        s.off[0] = x.offset;
    }
    __syncwarp();
}

// Writes words [w0, w1) of a 32-byte result from lanes 0..7.
__device__ __forceinline__ void td_write_result(td_result *out, int status, int depth, uint16_t found_move,
                                                const uint16_t *path, uint32_t expansions, int w0, int w1) {
    const int lane = threadIdx.x & 31;
    uint32_t word = 0;
    if (lane == 0) word = (uint32_t)status;
    else if (lane == 1) word = (uint32_t)depth;
    else if (lane >= 2 && lane < 7) {
        const int m0 = 2 * (lane - 2), m1 = m0 + 1;
        uint32_t lo = 0, hi = 0;
        if (status == TD_FOUND) {
            if (m0 < depth) lo = (m0 == depth - 1) ? found_move : path[m0];
            if (m1 < depth && m1 < TD_MAX_DEPTH) hi = (m1 == depth - 1) ? found_move : path[m1];
        }
        word = lo | (hi << 16);
    } else if (lane == 7) {
        word = expansions;
    }
    if (lane >= w0 && lane < w1) reinterpret_cast<volatile uint32_t *>(out)[lane] = word;
}

// One complete search of instance x by the calling warp (no sharing).
template <bool ORDERED>
__device__ void td_warp_search(const td_instance &x, td_result *out, td_warp_smem &s,
                               const uint8_t *lut, uint32_t (&code)[TD_MAX_STEPS], int &codeN,
                               const td_search_limits &lim) {
    int status = TD_NOT_FOUND, depth = 0;
    uint32_t expansions = 0;
    uint16_t found_move = 0;
    if (!td_instance_ok(x)) {
        status = TD_ERR_ARG;
    } else if (td_triple_count(x.n_symbols) > 0) {
        td_setup_root(s, x, code, codeN);
        const td_dfs_out r = td_dfs<ORDERED>(s, lut, code, x.n_symbols, x.max_moves, 0, lim, nullptr);
        expansions = r.expansions;
        if (r.status == TD_DFS_FOUND) {
            status = TD_FOUND;
            depth = r.depth;
            found_move = r.found_move;
        } else if (r.status == TD_DFS_BUDGET) {
            status = TD_ERR_BUDGET;
        } else if (r.status == TD_DFS_TIMEOUT) {
            status = TD_ERR_TIMEOUT;
        }
    }
    __syncwarp();
    td_write_result(out, status, depth, found_move, s.path, expansions, 0, 8);
}
