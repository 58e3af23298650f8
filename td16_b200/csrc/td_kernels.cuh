// td_kernels.cuh -- the sm_100a witness-search warp engine.
//
// One warp owns one search (a DFS over move sequences), or one donated
// subtree of it.  Two node evaluations share the DFS:
//
// Reference order (td_prepare_node, td_evaluate, td_next_child): per node the
// warp labels the omega cycles of the pinned state by pointer jumping (lane p
// = pinned position p), writes the pair table (4 bits per ordered pair of
// caller positions), and evaluates every triple: lane l takes u = 32*s + l in
// step s, reads three pair entries and one class-table byte, and keeps one bit
// per step in per-lane masks.  The next child comes from a warp max-reduction
// in the reference's single-queue order.
//
// Free order (td_prepare_rows, td_evaluate_rows, td_next_child_rows): the
// state is the caller's array, one byte per position; per node the warp builds
// cycle row masks (one per caller position), and each lane classifies all the
// children (i, j, k) of its pair slots at once with LOP3 logic
// (td_row_classes).  The next child, +2 moves first, comes from per-level lane
// summaries.  A table of explored states skips children reached before by
// another move order, and busy warps donate subtrees to idle ones.
//
// Reference: emitter/src/native/backtracking/sorting_search.cu:478-712.
#pragma once

#include "td_core.cuh"

#define TD_FULL 0xffffffffu
#define TD_PT_ROWS 18          // 17 position rows + one zero row for idle lanes
#define TD_PT_DUMMY (17 * TD_PT_STRIDE)
#define TD_TRI_TABLE 3060      // sum over N <= 17 of C(N,3) = C(18,4)
#define TD_G0 0x09249249u      // bit 0 of each 3-bit group
#define TD_G1 0x12492492u      // bit 1 of each group

// floor(b / 3) for 0 <= b <= 29: the step of a bit inside a packed word
__device__ __forceinline__ int td_group_of(int b) { return (b * 11) >> 5; }

// Per-warp shared state.
struct td_warp_smem {
    union {
        struct {  // reference move order (one triple per lane and step)
            uint8_t pt[TD_PT_ROWS * TD_PT_STRIDE];     // pair table of the current node
            // per level, per lane: the outcome of every step in 3-bit groups, ten
            // steps per word (step st in word st/10 at bit 3*(st%10)): bit 0 found
            // (or, at the root level, accepted when visited), bit 1 a child to visit
            uint32_t pm[TD_MAX_DEPTH][3][32];
        };
        struct {  // free move order (bit-sliced: one pair and all its k per lane and round)
            // per caller position c: the row masks S, G, P and H (positions
            // after c), and the odd-cycle / fixed-point flags as full masks
            uint4 rows[TD_MAX_N];
            uint2 flg[TD_MAX_N];
            // per level and lane: the expandable children of the lane's four
            // pair slots (word r = slot R*lane + r), +2 class at bits k-1
            // (1..15), 0 class at bits k+15 (17..31)
            uint4 pw[TD_MAX_DEPTH][32];
            uint32_t m2[TD_MAX_DEPTH];                 // per level: lanes that hold +2 children
            uint32_t m0[TD_MAX_DEPTH];                 // per level: lanes that hold 0 children
            // per level: the caller's array, one pinned label per caller position
            uint8_t A[TD_MAX_DEPTH + 1][32];
            uint8_t inv[32];                           // caller position of each label
        };
    };
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
    uint64_t *tt;              // this warp's table of explored states (free order); null = none
    uint32_t *tt_gen;          // this warp's generation counter of that table (kept across launches)
    int tt_bits;               // log2 of its entries
    uint32_t restart_base;     // free order: base of the restart budgets (td_attempt_budget); 0 = none
    const int *cutoff;         // a split ordered search: lowest rank with a witness so far; null = none
    int rank;                  // that search's own rank (it stops once *cutoff < rank)
};

__device__ __forceinline__ uint64_t td_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Reference order: evaluate all children of the node at `level`.  Fills the
// level's packed outcome words and returns the found child's u, or -1.
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
    const uint32_t flags0 = f0 | (x0 << 1);
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
    if (level == 0) return -1;  // roots are accepted on visit, not on seeding
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

// Reference order: next child of `level`; returns u or -1.  *accepted is set
// for a root that is accepted when visited.
__device__ __forceinline__ int td_next_child(td_warp_smem &s, int level, int *accepted) {
    const int lane = threadIdx.x & 31;
    const uint32_t P0 = s.pm[level][0][lane], P1 = s.pm[level][1][lane], P2 = s.pm[level][2][lane];
    const bool desc_lanes = level > 0;
    const uint32_t cm = level == 0 ? (TD_G0 | TD_G1) : TD_G1;
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
    if (level == 0) *accepted = __shfl_sync(TD_FULL, (int)((Pk >> (3 * j)) & 1u), win);
    if (lane == win) s.pm[level][k][lane] = Pk & ~(7u << (3 * j));
    __syncwarp();
    return st * 32 + win;
}

// ---- free move order: bit-sliced evaluation ---------------------------------
//
// The state of a level is the caller's array, one byte per caller position
// holding the pinned label (A[c] = B[(c + off) mod N]).  In these terms omega
// maps A[c] to A[c-1] + 1 (mod N), and a move (i, j, k) is the plain block swap
// A[:i] + A[j:k] + A[i:j] + A[k:] (the pinned form's start-of-array rule is the
// rotation that keeps label 0 first).  Lane l owns pair slots 4 l + r
// (td_pair_code) and classifies the children (i, j, k) of every k at once
// from the node's row masks (td_row_classes).

// Rounds of the bit-sliced evaluation for N: ceil(C(N-1,2) / 32).
__device__ __forceinline__ int td_pair_rounds(int N) {
    const int NP = N < 3 ? 0 : (N - 1) * (N - 2) / 2;
    return (NP + 31) >> 5;
}

// Lane l owns slots R l + r, r < R = td_pair_rounds(N); code[r] for r >= R
// (and code[TD_MAX_ROUNDS]) holds R.
__device__ __forceinline__ void td_load_pairs(int N, uint32_t (&code)[TD_MAX_STEPS]) {
    const int lane = threadIdx.x & 31;
    const int R = td_pair_rounds(N);
#pragma unroll
    for (int r = 0; r < TD_MAX_ROUNDS; ++r) code[r] = td_pair_code(N, r < R ? R * lane + r : -1);
    code[TD_MAX_ROUNDS] = (uint32_t)R;
}

// Pinned state (L, off) -> the caller's array of `level`.
__device__ __forceinline__ void td_unpack_state(td_warp_smem &s, int level, uint64_t L, int off, int N) {
    const int c = threadIdx.x & 31;
    if (c < N) {
        int p = c + off;
        p -= p >= N ? N : 0;
        s.A[level][c] = (uint8_t)(p ? td_nib(L, p - 1) + 1u : 0u);
    }
    __syncwarp();
}

// The caller's array of `level` -> pinned state (L, off): label 0 sits at
// caller position c0, so off = -c0 mod N and L[m] = A[(m + 1 + c0) mod N] - 1.
__device__ __forceinline__ void td_pack_state(const td_warp_smem &s, int level, int N, uint64_t *L, int *off) {
    const int m = threadIdx.x & 31;
    const uint32_t z = __ballot_sync(TD_FULL, m < N && s.A[level][m] == 0);
    const int c0 = __ffs(z) - 1;
    uint32_t lo = 0, hi = 0;
    if (m < 16) {
        uint32_t v = (uint32_t)m;
        if (m < N - 1) {
            int q = m + 1 + c0;
            q -= q >= N ? N : 0;
            v = s.A[level][q] - 1u;
        }
        const uint64_t w = (uint64_t)v << (4 * m);
        lo = (uint32_t)w;
        hi = (uint32_t)(w >> 32);
    }
    lo = __reduce_or_sync(TD_FULL, lo);
    hi = __reduce_or_sync(TD_FULL, hi);
    *L = ((uint64_t)hi << 32) | lo;
    *off = c0 == 0 ? 0 : N - c0;
}

// The caller's array of level+1 = that of `level` after the move t.
__device__ __forceinline__ void td_apply_bytes(td_warp_smem &s, int level, uint32_t t, int N) {
    const int m = threadIdx.x & 31;
    const int i = t & 31, j = (t >> 5) & 31, k = (t >> 10) & 31;
    if (m < N) {
        int src = m;
        if (m >= i && m < k) src = m < i + (k - j) ? m + (j - i) : m - (k - j);
        s.A[level + 1][m] = s.A[level][src];
    }
    __syncwarp();
}

// Row masks of the node at `level` (lane c = caller position c); returns the
// number of odd-length omega cycles and the odd-cycle and fixed-point masks.
__device__ __forceinline__ int td_prepare_rows(td_warp_smem &s, int level, int N, uint32_t &O, uint32_t &F) {
    const int c = threadIdx.x & 31;
    const bool act = c < N;
    const int a = act ? s.A[level][c] : 0;
    const int am1 = __shfl_sync(TD_FULL, a, c == 0 ? N - 1 : c - 1);
    if (act) s.inv[a] = (uint8_t)c;
    __syncwarp();
    // next caller position along omega: the one holding A[c-1] + 1 (mod N)
    const int y = am1 + 1 == N ? 0 : am1 + 1;
    const int nx = act ? (int)s.inv[y] : c;
    // leader (smallest caller position on the cycle) and dist (omega steps to
    // it) in one pointer-jumping pass: each lane keeps the minimum of the
    // window c, next(c), ..., next^(w-1)(c) and its distance; windows double
    // per round and 32 >= any cycle length, so the first occurrence wins.
    int m = c, d = 0, j = nx;
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
    const int after_leader = __shfl_sync(TD_FULL, nx, m);
    const int len = __shfl_sync(TD_FULL, d, after_leader) + 1;
    const uint32_t ACT = (1u << N) - 1u;
    const uint32_t S = __match_any_sync(TD_FULL, m) & ACT;  // inactive lanes are their own leaders
    // lt bit q: dist(q) < dist(c), by comparing the five bit planes of dist
    uint32_t lt = 0, eq = TD_FULL, D0 = 0;
#pragma unroll
    for (int b = 4; b >= 0; --b) {
        const uint32_t Bb = __ballot_sync(TD_FULL, (d >> b) & 1);
        const uint32_t mb = 0u - (uint32_t)((d >> b) & 1);
        lt |= eq & ~Bb & mb;
        eq &= ~(Bb ^ mb);
        if (b == 0) D0 = Bb;
    }
    const uint32_t lodd = 0u - (uint32_t)(len & 1);
    const uint32_t G = S & lt;
    // walk c -> q: dist(c) - dist(q), plus the cycle length when q is further
    const uint32_t P = S & ((D0 ^ (0u - (uint32_t)(d & 1))) ^ (lodd & ~lt));
    O = __ballot_sync(TD_FULL, act && (len & 1));
    F = __ballot_sync(TD_FULL, act && len == 1);
    const int odd = __popc(__ballot_sync(TD_FULL, act && m == c && (len & 1)));
    if (act) {
        s.rows[c] = make_uint4(S, G, P, ACT & (0xfffffffeu << c));
        s.flg[c] = make_uint2(lodd, len == 1 ? 0xffffffffu : 0u);
    }
    __syncwarp();
    return odd;
}

// Classifies every child of the node at `level`; fills the level's outcome
// words and lane summaries and returns a found move (i | j<<5 | k<<10) or -1.
__device__ __forceinline__ int td_evaluate_rows(td_warp_smem &s, const uint32_t (&code)[TD_MAX_STEPS], int N,
                                                int level, int odd, uint32_t O, uint32_t F) {
    const int lane = threadIdx.x & 31;
    const int D = level + 1;
    const uint32_t accD = s.acc[D], reachD = s.reach[D];
    const uint32_t f0 = 0u - ((accD >> odd) & 1u), f2 = 0u - ((accD >> (odd + 2)) & 1u);
    const uint32_t x0 = (0u - ((reachD >> odd) & 1u)) & ~f0;
    const uint32_t x2 = (0u - ((reachD >> (odd + 2)) & 1u)) & ~f2;
    const bool accepting = (f0 | f2) != 0;  // warp-uniform
    const int R = (int)code[TD_MAX_ROUNDS];  // warp-uniform
    uint32_t key = 0xffffffffu;
    uint32_t W[TD_MAX_ROUNDS] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int r = 0; r < TD_MAX_ROUNDS; ++r) {
        if (r >= R) break;
        const uint32_t pc = code[r];
        const int i = pc & 31, j = (pc >> 5) & 31;
        const uint4 ri = s.rows[i], rj = s.rows[j];
        const uint2 fi = s.flg[i], fj = s.flg[j];
        uint32_t plus, zero;
        td_row_classes_x(ri.x, ri.y, ri.z, rj.x, rj.y, rj.z, O, F, fi.x, fj.x, fi.y, fj.y, (int)(pc >> 15), &plus,
                         &zero);
        const uint32_t km = rj.w;  // k > j (empty slots: j's row with an empty mask is never read)
        // +2 children at bits k-1, 0 children at bits k+15; the fields do not
        // overlap, so the high-half multiply and the add keep this off the ALU pipe
        W[r] = __umulhi(km & x2 & plus, 0x80000000u) + (km & x0 & zero) * 32768u;
        if (accepting) {
            const uint32_t fnd = km & ((f0 & zero) | (f2 & plus));
            if (fnd && key == 0xffffffffu)
                key = ((uint32_t)lane << 17) | ((uint32_t)r << 15) | (pc & 1023u) |
                      ((uint32_t)(31 - __clz(fnd)) << 10);
        }
    }
    s.pw[level][lane] = make_uint4(W[0], W[1], W[2], W[3]);
    const uint32_t any = W[0] | W[1] | W[2] | W[3];
    const uint32_t m2 = __ballot_sync(TD_FULL, (any & 0x0000ffffu) != 0);
    const uint32_t m0 = __ballot_sync(TD_FULL, (any & 0xffff0000u) != 0);
    if (lane == 0) {
        s.m2[level] = m2;
        s.m0[level] = m0;
    }
    if (accepting) {
        key = __reduce_min_sync(TD_FULL, key);
        if (key != 0xffffffffu) {
            __syncwarp();
            return (int)(key & 0x7fffu);
        }
    }
    __syncwarp();
    return -1;
}

// Next child of `level` in the free order: +2 children first; among them, in
// the plain order (ord = 0), the highest pair slot (the lexicographically
// smallest pair) and its smallest k.  `ord` (td_order_variant) rotates the
// lane priority, reverses the round order and takes the largest k first.
// Returns the move or -1.
__device__ __forceinline__ int td_next_child_rows(td_warp_smem &s, const uint32_t (&code)[TD_MAX_STEPS],
                                                  int level, uint32_t ord) {
    const int lane = threadIdx.x & 31;
    const uint32_t m2 = s.m2[level], m0 = s.m0[level];
    if ((m2 | m0) == 0) return -1;
    const bool c2 = m2 != 0;
    const uint32_t lanes = c2 ? m2 : m0;
    const uint32_t rot = ord & 31u;
    // the lane with the largest (lane - rot) mod 32
    const int win = (int)(((31u - (uint32_t)__clz(__funnelshift_r(lanes, lanes, rot))) + rot) & 31u);
    const uint4 Wv = s.pw[level][win];
    const uint32_t cm = c2 ? 0x0000ffffu : 0xffff0000u;
    int r;
    uint32_t w;
    if (ord & 32u) {
        if (Wv.x & cm) { r = 0; w = Wv.x; }
        else if (Wv.y & cm) { r = 1; w = Wv.y; }
        else if (Wv.z & cm) { r = 2; w = Wv.z; }
        else { r = 3; w = Wv.w; }
    } else {
        if (Wv.w & cm) { r = 3; w = Wv.w; }
        else if (Wv.z & cm) { r = 2; w = Wv.z; }
        else if (Wv.y & cm) { r = 1; w = Wv.y; }
        else { r = 0; w = Wv.x; }
    }
    const int b = (ord & 64u) ? 31 - __clz(w & cm) : __ffs(w & cm) - 1;
    const uint32_t nw = w & ~(1u << b);
    const uint32_t mine = r == 3 ? code[3] : (r == 2 ? code[2] : (r == 1 ? code[1] : code[0]));
    const uint32_t pc = __shfl_sync(TD_FULL, mine, win);
    // does the winning lane keep children of this class?
    const uint32_t rest = (r == 0 ? nw : Wv.x) | (r == 1 ? nw : Wv.y) | (r == 2 ? nw : Wv.z) | (r == 3 ? nw : Wv.w);
    if (lane == 0) {
        reinterpret_cast<uint32_t *>(&s.pw[level][win])[r] = nw;
        if (!(rest & cm)) {
            if (c2) s.m2[level] = m2 & ~(1u << win);
            else s.m0[level] = m0 & ~(1u << win);
        }
    }
    __syncwarp();
    const int k = c2 ? b + 1 : b - 15;
    return (int)((pc & 1023u) | ((uint32_t)k << 10));
}

// ---- work items (subtree roots handed between warps) ----------------------

// A node that is known to be expandable, with the moves that lead to it.
struct __align__(16) td_item {  // 32 bytes
    uint64_t L;
    uint32_t inst;          // instance index
    uint8_t depth;          // bits 0-6: DFS depth of the node (0 only for the root of an inverse
                            // instance); bit 7: the node belongs to the inverse instance's search
    uint8_t off;
    uint16_t path[TD_MAX_DEPTH];
};

// Per-instance bookkeeping when several warps share one search.
struct td_inst_state {
    int found;              // 1: a warp recorded the witness; 2: one side of a race was searched
                            // to the end without one (the verdict is known, the other side stops)
    int pending;            // units (the root search + items) not yet finished: the low 16 bits
                            // count the search of the instance, the high 16 bits that of its
                            // inverse (td_steal_kernel's race; elsewhere only the low half is used)
    unsigned expansions;    // summed over units
    int error;              // first error status seen (timeout)
};

// Scheduler counters of one launch.
struct td_pool {
    int inst_ticket;        // next fresh instance
    int produced;           // items reserved by donors
    int consumed;           // items claimed by takers (the batch engine: item tickets taken)
    int active;             // warps inside a unit or claiming one (the serving loop)
    int idle;               // warps waiting for donated work (the serving loop)
    int error;              // launch-level error (bounded wait expired)
    int outstanding;        // the batch engine: units in progress plus items not yet finished
    int spawn_produced;     // the batch engine's race: inverse roots queued
    int spawn_consumed;     // and claimed
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
    int tickets;            // takers hold item tickets (the batch engine), see td_steal_kernel
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
    int side;               // 1: the unit searches the instance's inverse (items carry it on)
    int race;               // > 0: the unit queues its inverse when it starts restart attempt
                            // `race` (root units of full-sorting instances in td_steal_kernel)
    int spawn_base;         // the race's queue: item slots [spawn_base, spawn_base + spawn_capacity)
    int spawn_capacity;
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
// pool as items (free move order).  Returns the number donated (uniform
// across the warp).
__device__ __forceinline__ int td_donate(td_warp_smem &s, const td_donate_ctx &dc,
                                         const uint32_t (&code)[TD_MAX_STEPS], int d0, int level, int N,
                                         int want) {
    const int lane = threadIdx.x & 31;
    int lv = -1;
    for (int l = d0; l <= level && l <= dc.max_level; ++l) {
        if (s.m2[l] | s.m0[l]) { lv = l; break; }
    }
    if (lv < 0) return 0;
    const uint4 Wv = s.pw[lv][lane];
    uint32_t W0 = Wv.x, W1 = Wv.y, W2 = Wv.z, W3 = Wv.w;
    const int cnt = __popc(W0) + __popc(W1) + __popc(W2) + __popc(W3);
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
        // the pending count must cover the items before any taker can finish
        // one (takers wait for the ready flag, written below); with item
        // tickets, so must the launch's outstanding count
        if (base >= 0) {
            atomicAdd(&dc.state->pending, dc.side ? give << 16 : give);
            if (dc.tickets) atomicAdd(&dc.pool->outstanding, give);
        }
        __threadfence();
    }
    base = __shfl_sync(TD_FULL, base, 0);
    if (base < 0) return 0;  // out of item space: keep the work
    if (lane == 0) {
        atomicAdd(&dc.pool->donations, 1ull);
        atomicAdd(&dc.pool->donated_items, (unsigned long long)give);
    }
    uint64_t Lp;
    int offp;
    td_pack_state(s, lv, N, &Lp, &offp);  // the parent in pinned form
    int slot = base + before;
    // a lane gives its lowest slots first (the ones this warp visits last),
    // and 0-class children (high bits) before +2 children
    for (int taken = 0; taken < mine; ++taken) {
        uint32_t pc, b;
        if (W0) { pc = code[0]; b = 31 - __clz(W0); W0 &= ~(1u << b); }
        else if (W1) { pc = code[1]; b = 31 - __clz(W1); W1 &= ~(1u << b); }
        else if (W2) { pc = code[2]; b = 31 - __clz(W2); W2 &= ~(1u << b); }
        else { pc = code[3]; b = 31 - __clz(W3); W3 &= ~(1u << b); }
        const uint32_t k = b < 16 ? b + 1 : b - 15;
        const uint32_t t = (pc & 1023u) | (k << 10);
        uint64_t nL;
        int noff;
        td_apply_move(Lp, offp, N, t & 31, (t >> 5) & 31, (t >> 10) & 31, &nL, &noff);
        td_item it;
        it.L = nL;
        it.inst = dc.inst;
        it.depth = (uint8_t)((lv + 1) | (dc.side << 7));
        it.off = (uint8_t)noff;
#pragma unroll
        for (int d = 0; d < TD_MAX_DEPTH; ++d) it.path[d] = d < lv ? s.path[d] : (d == lv ? (uint16_t)t : 0);
        int phys = slot;
        uint32_t tag = dc.epoch;
        bool freed_ok = true;
        if (dc.ring) {
            phys = slot % dc.capacity;
            tag = td_ring_tag(slot);
            if (slot >= dc.capacity) {
                // the slot's previous item (index slot - capacity) is claimed;
                // wait until its taker has read it (bounded)
                const uint32_t freed = td_ring_tag(slot - dc.capacity) | 0x80000000u;
                for (unsigned spin = 0; *(volatile uint32_t *)&dc.ready[phys] != freed; ++spin) {
                    if ((spin & 255u) == 0 && dc.deadline_ns && td_globaltimer() > dc.deadline_ns) {
                        atomicCAS(&dc.pool->error, 0, TD_ERR_TIMEOUT);
                        freed_ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        // after an expired wait the slot still belongs to an unread item: it
        // is left alone, and this item's taker gives up at the deadline
        if (freed_ok) {
            dc.items[phys] = it;
            __threadfence();
            atomicExch(&dc.ready[phys], tag);
        }
        ++slot;
    }
    s.pw[lv][lane] = make_uint4(W0, W1, W2, W3);
    const uint32_t any = W0 | W1 | W2 | W3;
    const uint32_t m2 = __ballot_sync(TD_FULL, (any & 0x0000ffffu) != 0);
    const uint32_t m0 = __ballot_sync(TD_FULL, (any & 0xffff0000u) != 0);
    if (lane == 0) {
        s.m2[lv] = m2;
        s.m0[lv] = m0;
    }
    __syncwarp();
    return give;
}

// Queues the inverse of the unit's instance (td_inverse_pinned) as a root item
// of the race's queue, so that another warp searches it while this one goes
// on; the first witness on either side ends both, and so does either side
// searched to the end without one (found = 2).  The pending and outstanding
// counts cover the item before it can be claimed.  In the batch engine only an
// instance's root search queues its inverse, once, and the queue holds a slot
// per instance of the launch, so one fetch-and-add reserves a slot: busy
// searches queue their inverses at up to several per microsecond, and a
// compare-and-swap loop on the counter kept them waiting.  In the serving
// loop (dc.ring) the inverse is one more item of its ring.  Returns whether it
// was queued (uniform across the warp).
__device__ __forceinline__ int td_spawn_inverse(const td_warp_smem &s, const td_donate_ctx &dc, int N) {
    int ok = 0;
    if ((threadIdx.x & 31) == 0) {
        int slot = -1, phys = -1;
        uint32_t tag = dc.epoch;
        if (dc.ring) {
            // the serving loop's ring of items: reserved like a donation (one
            // item), and a reused slot is written once its last item was read
            int cur = *(volatile int *)&dc.pool->produced;
            for (;;) {
                if (cur - *(volatile int *)&dc.pool->consumed + 1 > dc.capacity) break;
                const int prev = atomicCAS(&dc.pool->produced, cur, cur + 1);
                if (prev == cur) { slot = cur; break; }
                cur = prev;
            }
            if (slot >= 0) {
                phys = slot % dc.capacity;
                tag = td_ring_tag(slot);
                atomicAdd(&dc.state->pending, 1 << 16);
                if (slot >= dc.capacity) {
                    const uint32_t freed = td_ring_tag(slot - dc.capacity) | 0x80000000u;
                    for (unsigned spin = 0; *(volatile uint32_t *)&dc.ready[phys] != freed; ++spin) {
                        if ((spin & 255u) == 0 && dc.deadline_ns && td_globaltimer() > dc.deadline_ns) {
                            // the slot still holds an unread item: left alone, and
                            // this item's taker gives up at the deadline
                            atomicCAS(&dc.pool->error, 0, TD_ERR_TIMEOUT);
                            phys = -1;
                            break;
                        }
                        __nanosleep(64);
                    }
                }
            }
        } else {
            slot = atomicAdd(&dc.pool->spawn_produced, 1);
            if (slot < dc.spawn_capacity) {
                phys = dc.spawn_base + slot;
                atomicAdd(&dc.state->pending, 1 << 16);
                atomicAdd(&dc.pool->outstanding, 1);
            } else {
                slot = -1;
            }
        }
        if (phys >= 0) {
            td_item it;
            it.L = td_inverse_pinned(s.L[0], N);
            it.inst = dc.inst;
            it.depth = 0x80;
            it.off = 0;
#pragma unroll
            for (int d = 0; d < TD_MAX_DEPTH; ++d) it.path[d] = 0;
            dc.items[phys] = it;
            __threadfence();
            atomicExch(&dc.ready[phys], tag);
        }
        ok = slot >= 0;
    }
    return __shfl_sync(TD_FULL, ok, 0);
}

// After a unit of the inverse's search found a witness (depth moves: path[0 ..
// depth-2] and found_move), rewrites it as the witness of the instance x in
// the caller's positions: td_witness_from_inverse's steps, one lane per
// position (arrays in registers, block swaps by shuffle, cut points by
// ballot).  Returns 0 if it does not convert (then no witness may be
// recorded).  Uniform across the warp.
__device__ __forceinline__ int td_inverse_result(td_warp_smem &s, const td_instance &x, td_dfs_out &r) {
    const int c = threadIdx.x & 31;
    const int N = x.n_symbols, k = r.depth;
    if (k < 1 || k > TD_MAX_DEPTH) return 0;
    // the swap of blocks [i, j) and [j, kk) moves the value at src(c) to c
    auto swap = [&](uint32_t v, uint32_t mv) {
        const int i = mv & 31, j = (mv >> 5) & 31, kk = (mv >> 10) & 31;
        int src = c;
        if (c >= i && c < kk) src = c < i + (kk - j) ? c + (j - i) : c - (kk - j);
        return __shfl_sync(TD_FULL, v, src);
    };
    // lane q holds the inverse's move q, and then the converted move q
    const uint32_t inv = c < k - 1 ? (uint32_t)s.path[c] : (c == k - 1 ? (uint32_t)r.found_move : 0u);
    __syncwarp();
    // X: the caller's array; S: the identity array after all the inverse's moves
    int p = c + x.offset;
    p -= p >= N ? N : 0;
    uint32_t X = c < N ? (p ? td_nib(x.perm, p - 1) + 1u : 0u) : 0xffu;
    uint32_t S = (uint32_t)c;
    for (int q = 0; q < k; ++q) S = swap(S, __shfl_sync(TD_FULL, inv, q));
    const int prev = c == 0 ? N - 1 : c - 1;
    uint32_t mine = 0;  // lane q: move q of the converted witness
    for (int m = k; m >= 1; --m) {
        const uint32_t mv = __shfl_sync(TD_FULL, inv, m - 1);
        const int i = mv & 31, j = (mv >> 5) & 31, kk = (mv >> 10) & 31;
        if (!(i < j && j < kk && kk < N)) return 0;
        const uint32_t Xp = __shfl_sync(TD_FULL, X, prev);
        // the three cut points of s_m^-1 = (i, i + kk - j, kk) in S, found in X
        // (every lane takes part in every shuffle: they are computed before
        // the comparisons, never inside a short-circuited condition)
        const int g0 = i, g1 = i + kk - j, g2 = kk;
        const uint32_t u0 = __shfl_sync(TD_FULL, S, g0 == 0 ? N - 1 : g0 - 1), v0 = __shfl_sync(TD_FULL, S, g0);
        const uint32_t u1 = __shfl_sync(TD_FULL, S, g1 - 1), v1 = __shfl_sync(TD_FULL, S, g1);
        const uint32_t u2 = __shfl_sync(TD_FULL, S, g2 - 1), v2 = __shfl_sync(TD_FULL, S, g2);
        const bool act = c < N;
        const uint32_t h0 = __ballot_sync(TD_FULL, act & (Xp == u0) & (X == v0));
        const uint32_t h1 = __ballot_sync(TD_FULL, act & (Xp == u1) & (X == v1));
        const uint32_t h2 = __ballot_sync(TD_FULL, act & (Xp == u2) & (X == v2));
        // each cut is one neighbouring pair, so each mask has one bit; their
        // union, taken in ascending order, is the move in the caller's array
        const uint32_t cuts = h0 | h1 | h2;
        if (__popc(h0) != 1 || __popc(h1) != 1 || __popc(h2) != 1 || __popc(cuts) != 3) return 0;
        const int a = __ffs(cuts) - 1;
        const uint32_t rest = cuts & (cuts - 1);
        const int b = __ffs(rest) - 1;
        const int e = 31 - __clz(cuts);
        const uint32_t t = td_pack_move(a, b, e);
        if (c == k - m) mine = t;
        X = swap(X, t);
        S = swap(S, (uint32_t)i | ((uint32_t)(i + kk - j) << 5) | ((uint32_t)kk << 10));  // S_{m-1} = S_m . s_m^-1
    }
    // each lane stores its own move into the path, which it alone read above;
    // the record's writers read it after the barrier
    if (c < k - 1) s.path[c] = (uint16_t)mine;
    r.found_move = (uint16_t)__shfl_sync(TD_FULL, mine, k - 1);
    __syncwarp();
    return 1;
}

// Whether a witness of instance x (its caller positions: path[0 .. depth-2],
// found_move) is one the instance's own search could return: every move keeps
// the reference's move filter (it touches no symbol that omega fixes, and it
// changes the odd-cycle count by 0 or +2, sorting_search.cu:375-380,
// 240-332), no node before the last passes the acceptance test, and the last
// does.  A witness of the inverse, turned into the instance's positions, keeps
// the filter on the inverse's side but need not on this one: its path passes
// through other states.  Recording only witnesses that pass keeps the verdict
// that of the instance's own filtered search.  Uses the warp's frame (levels
// 0..depth) as scratch; uniform across the warp.
__device__ __forceinline__ bool td_filtered_witness(td_warp_smem &s, const td_instance &x, const td_dfs_out &r) {
    const int N = x.n_symbols, k = r.depth;
    if (k < 1 || k > TD_MAX_DEPTH) return false;
    td_unpack_state(s, 0, x.perm, x.offset, N);
    uint32_t O, F;
    int odd = td_prepare_rows(s, 0, N, O, F);
    for (int d = 0; d < k; ++d) {
        const uint32_t t = d == k - 1 ? (uint32_t)r.found_move : (uint32_t)s.path[d];
        const int i = t & 31, j = (t >> 5) & 31, kk = (t >> 10) & 31;
        if (!(i < j && j < kk && kk < N)) return false;
        if (((F >> i) | (F >> j) | (F >> kk)) & 1u) return false;
        td_apply_bytes(s, d, t, N);
        const int next = td_prepare_rows(s, d + 1, N, O, F);
        if (next != odd && next != odd + 2) return false;
        odd = next;
        const bool accepted = (s.acc[d + 1] >> odd) & 1u;
        if (accepted != (d == k - 1)) return false;
    }
    return true;
}

// ---- table of explored states (free order) --------------------------------
//
// Different move orders reach the same state: on near-reverse S_16 about 80%
// of the free-order expansions re-expand a state already expanded at the same
// or a smaller depth.  Whether a node's subtree holds a witness depends only
// on its pinned state L (not on where the caller's array starts: a move is the
// same cycle rotation from any start, so the reachable states do not depend
// on it) and on its depth.  Each warp keeps a direct-mapped table of
// (L, depth) for the states it expanded in its current unit, and skips a
// child whose state is in the table at a depth <= the child's.  This is sound:
// the earlier node was explored with at least as much budget, unless it is an
// ancestor still being explored (which has more budget) or its children were
// donated (then their takers explore them).  The search stops at the first
// witness, so every completed entry is a state without one.
//
// An entry is one word.  The state's 57-bit key (td_tt_key) is multiplied by
// an odd constant modulo 2^57, a bijection; the top tt_bits bits of the
// product pick the slot and the other 57 - tt_bits bits are stored as the
// tag, so (slot, tag) still identifies the state.  That leaves tt_bits + 3
// bits for a generation (15 at the default 4096 entries) under the depth in
// the top nibble.  Entries of other generations never match.  Each unit that
// uses the table, and each restart (which abandons the entries of the
// attempt: their subtrees were not all searched), takes the warp's next
// generation from a counter kept in global memory across units and launches,
// so the table is cleared only when that counter wraps (every 32767 units at
// 4096 entries) instead of once per unit.  Zero words are empty (generation 0
// is never used).

// A unit starts using its table after this many expansions: most searches of
// uniform permutations end sooner, and they then never touch the table.
// States expanded before are simply not recorded.
#define TD_TT_AFTER 32
#define TD_TT_KEY 0x01ffffffffffffffull  // the 57 bits of a state key
#define TD_TT_MULT 0x9E3779B97F4A7C15ull  // odd: multiplying by it permutes keys modulo 2^57

__device__ __forceinline__ void td_tt_clear(const td_search_limits &lim) {
    const int lane = threadIdx.x & 31;
    uint4 *t = reinterpret_cast<uint4 *>(lim.tt);
    const int n4 = 1 << (lim.tt_bits - 1);
    for (int q = lane; q < n4; q += 32) t[q] = make_uint4(0u, 0u, 0u, 0u);
    __syncwarp();
}

// The warp's next table generation (uniform across the warp); clears the
// table when the counter wraps.
__device__ __forceinline__ uint32_t td_tt_next_gen(const td_search_limits &lim) {
    const uint32_t gmax = (1u << (lim.tt_bits + 3)) - 1u;
    uint32_t g = *(volatile uint32_t *)lim.tt_gen + 1u;
    __syncwarp();
    if (g > gmax) {
        td_tt_clear(lim);
        g = 1u;
    }
    if ((threadIdx.x & 31) == 0) *lim.tt_gen = g;
    __syncwarp();
    return g;
}

// Looks up the state of level `lv` (depth lv) in generation `gen` of the table
// and records it there; returns whether it was already explored in this
// generation at a depth <= lv (uniform across the warp).
__device__ __forceinline__ bool td_tt_visit(const td_warp_smem &s, const td_search_limits &lim, int lv, int N,
                                            uint32_t gen) {
    const int m = threadIdx.x & 31;
    const int a = m < N ? s.A[lv][m] : 0xff;
    const int c0 = __ffs(__ballot_sync(TD_FULL, a == 0)) - 1;  // caller position of label 0
    // L[m] = A[(m + 1 + c0) mod N] - 1 for m < N - 1
    int src = m + 1 + c0;
    src -= src >= N ? N : 0;
    const int v = __shfl_sync(TD_FULL, a, m < N - 1 ? src : m) - 1;
    uint32_t lo = 0, hi = 0;
    if (m < N - 1) {
        if (m < 8) lo = (uint32_t)v << (4 * m);
        else hi = (uint32_t)v << (4 * (m - 8));
    }
    lo = __reduce_or_sync(TD_FULL, lo);
    hi = __reduce_or_sync(TD_FULL, hi);
    int hit = 0;
    if (m == 0) {
        const uint64_t h = (td_tt_key((((uint64_t)hi) << 32) | lo) * TD_TT_MULT) & TD_TT_KEY;
        const int tag_bits = 57 - lim.tt_bits;
        const uint32_t slot = (uint32_t)(h >> tag_bits);
        const uint64_t want = (h & ((1ull << tag_bits) - 1ull)) | ((uint64_t)gen << tag_bits);
        const uint64_t old = lim.tt[slot];
        hit = (old & ((1ull << 60) - 1ull)) == want && (int)(old >> 60) <= lv;
        if (!hit) lim.tt[slot] = want | ((uint64_t)lv << 60);
    }
    return __shfl_sync(TD_FULL, hit, 0) != 0;
}

// Depth-first search from the node held at level d0 of `s` (state, path and
// rate masks already set).  Leaves the frames intact on TD_DFS_BUDGET.  The
// reference order evaluates one triple per lane and step (`code` holds the
// lane's triple codes); the free order is bit-sliced (`code` holds the lane's
// pair slots) and may donate subtrees through `dc`.
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
    uint32_t O = 0, F = 0;
    int found;
    if constexpr (ORDERED) {
        const int odd = td_prepare_node(s, s.L[d0], s.off[d0], N);
        found = td_evaluate(s, lut, code, steps, d0, odd, maxd);
        if (found >= 0) found = td_tri_table[tri_base + T - 1 - found];
    } else {
        td_unpack_state(s, d0, s.L[d0], s.off[d0], N);
        const int odd = td_prepare_rows(s, d0, N, O, F);
        found = td_evaluate_rows(s, code, N, d0, odd, O, F);
    }
    r.expansions = 1;
    int since_check = 0;
    bool tt_on = false;  // the table is in use (free order, after TD_TT_AFTER expansions)
    uint32_t tt_gen = 0;  // its current generation
    int attempt = 0;     // free order: restarts with another child order (td_attempt_budget)
    uint32_t ord = 0, attempt_exp = 1;
    uint32_t attempt_budget = ORDERED ? ~0u : td_attempt_budget(lim.restart_base, 0);
    // a unit of a raced instance (the inverse's side, or the instance's side
    // once it queued the inverse) looks for the other side's verdict every 16
    // expansions, so that the loser stops soon after the winner
    bool raced = !ORDERED && dc && dc->side;
    for (;;) {
        if (found >= 0) {
            r.found_move = (uint16_t)found;
            r.depth = level + 1;
            r.status = TD_DFS_FOUND;
            break;
        }
        if (r.expansions >= lim.max_expansions) {
            r.status = TD_DFS_BUDGET;
            break;
        }
        if constexpr (!ORDERED) {
            if (attempt_exp >= attempt_budget) {
                // restart the subtree at d0 with the next child order; the table
                // held nodes of the abandoned attempt that were not explored to
                // the end, so it is cleared before its next use
                ++attempt;
                // a root search that may race queues its inverse when it starts
                // attempt dc->race; another warp then searches it alongside
                if (dc && attempt == dc->race && !dc->side && d0 == 0 && td_spawn_inverse(s, *dc, N))
                    raced = true;
                ord = td_order_variant(attempt);
                attempt_budget = td_attempt_budget(lim.restart_base, attempt);
                attempt_exp = 1;
                if (tt_on) tt_gen = td_tt_next_gen(lim);  // the abandoned attempt's entries no longer match
                level = d0;
                const int odd = td_prepare_rows(s, d0, N, O, F);
                found = td_evaluate_rows(s, code, N, d0, odd, O, F);
                ++r.expansions;
                continue;
            }
        }
        if constexpr (!ORDERED) {
            if (dc && ++since_check >= dc->check_every) {
                since_check = 0;
                int hungry = 0, stop = 0;
                if (lane == 0) {
                    // idle warps not yet served by an unclaimed item: without
                    // this, every busy warp would donate to the same few idle ones
                    if (dc->tickets) {
                        // takers holding a ticket past the last item produced
                        hungry = *(volatile int *)&dc->pool->consumed - *(volatile int *)&dc->pool->produced;
                    } else {
                        const int idle = *(volatile int *)&dc->pool->idle;
                        const int unclaimed =
                            *(volatile int *)&dc->pool->produced - *(volatile int *)&dc->pool->consumed;
                        hungry = idle - unclaimed;
                    }
                    stop = *(volatile int *)&dc->state->found;
                }
                stop = __shfl_sync(TD_FULL, stop, 0);
                if (stop) {
                    r.status = TD_DFS_ABORTED;
                    break;
                }
                hungry = __shfl_sync(TD_FULL, hungry, 0);
                // a search that has handed out subtrees no longer restarts: the
                // subtrees of an abandoned attempt would go on being searched,
                // and searching in parallel already varies the order
                if (hungry > 0 && td_donate(s, *dc, code, d0, level, N, min(hungry, dc->grain)) > 0)
                    attempt_budget = ~0u;
            }
        }
        if constexpr (!ORDERED) {
            if (raced && (r.expansions & 15u) == 0) {
                int stop = 0;
                if (lane == 0) stop = *(volatile int *)&dc->state->found;
                if (__shfl_sync(TD_FULL, stop, 0)) {
                    r.status = TD_DFS_ABORTED;
                    break;
                }
            }
        }
        if ((r.expansions & 255u) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (lim.deadline_ns && td_globaltimer() > lim.deadline_ns) stop = 1;
                if (lim.abort_flag && *(volatile const int *)lim.abort_flag) stop = 1;
                // a subtree of a split ordered search: one of lower rank has a witness
                if (lim.cutoff && *(volatile const int *)lim.cutoff < lim.rank) stop = 2;
            }
            stop = __shfl_sync(TD_FULL, stop, 0);
            if (stop) {
                r.status = stop == 2 ? TD_DFS_ABORTED : TD_DFS_TIMEOUT;
                break;
            }
        }
        // walk to the next node to expand: backtracks, and in free order the
        // children skipped through the table, change no expansion count, so
        // the checks above run once per expansion
        uint32_t t = 0;
        int walk = 0;  // 1: the subtree is exhausted, 2: a root accepted on visit (ordered)
        for (;;) {
            if constexpr (ORDERED) {
                int accepted;
                const int u = td_next_child(s, level, &accepted);
                if (u < 0) {
                    if (level == d0) { walk = 1; break; }
                    --level;
                    continue;
                }
                t = td_tri_table[tri_base + T - 1 - u];
                if (accepted) walk = 2;
                break;
            } else {
                const int m = td_next_child_rows(s, code, level, td_level_order(ord, attempt, level));
                if (m < 0) {
                    if (level == d0) { walk = 1; break; }
                    --level;
                    continue;
                }
                t = (uint32_t)m;
                if (lane == 0) s.path[level] = (uint16_t)t;
                td_apply_bytes(s, level, t, N);
                if (lim.tt) {
                    if (!tt_on && r.expansions >= TD_TT_AFTER) {
                        tt_gen = td_tt_next_gen(lim);
                        tt_on = true;
                    }
                    if (tt_on && td_tt_visit(s, lim, level + 1, N, tt_gen)) continue;  // explored with at least this budget
                }
                break;
            }
        }
        if (walk == 1) break;
        if (walk == 2) {
            r.found_move = (uint16_t)t;
            r.depth = level + 1;
            r.status = TD_DFS_FOUND;
            break;
        }
        if constexpr (ORDERED) {
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
            const int odd = td_prepare_node(s, nL, noff, N);
            found = td_evaluate(s, lut, code, steps, level, odd, maxd);
            if (found >= 0) found = td_tri_table[tri_base + T - 1 - found];
        } else {
            ++level;
            const int odd = td_prepare_rows(s, level, N, O, F);
            found = td_evaluate_rows(s, code, N, level, odd, O, F);
            ++attempt_exp;
        }
        ++r.expansions;
    }
    __syncwarp();
    return r;
}

__device__ __forceinline__ bool td_instance_ok(const td_instance &x) {
    return x.n_symbols <= TD_MAX_N && x.max_moves >= 1 && x.max_moves <= TD_MAX_DEPTH &&
           td_inst_init(x) <= TD_MAX_N;
}

// Loads the lane's codes for N (triple codes in the reference order, pair
// slots in the free order) and the instance's rate masks; places its root at
// level 0.  `codeN` caches the N the codes were loaded for (negative for the
// other order's codes).
template <bool ORDERED>
__device__ __forceinline__ void td_setup_root(td_warp_smem &s, const td_instance &x, uint32_t (&code)[TD_MAX_STEPS],
                                              int &codeN) {
    const int lane = threadIdx.x & 31;
    const int want = ORDERED ? x.n_symbols : -1 - x.n_symbols;
    if (codeN != want) {
        if constexpr (ORDERED) td_load_codes(x.n_symbols, code);
        else td_load_pairs(x.n_symbols, code);
        codeN = want;
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

// One complete search of instance x by the calling warp (no sharing); returns
// the status it wrote (uniform across the warp).
template <bool ORDERED>
__device__ int td_warp_search(const td_instance &x, td_result *out, td_warp_smem &s,
                               const uint8_t *lut, uint32_t (&code)[TD_MAX_STEPS], int &codeN,
                               const td_search_limits &lim) {
    int status = TD_NOT_FOUND, depth = 0;
    uint32_t expansions = 0;
    uint16_t found_move = 0;
    if (!td_instance_ok(x)) {
        status = TD_ERR_ARG;
    } else if (td_triple_count(x.n_symbols) > 0) {
        td_setup_root<ORDERED>(s, x, code, codeN);
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
    return status;
}
