// td_emu.cc -- serial host emulation of the engine's warp algorithm.
//
// TEST INFRASTRUCTURE ONLY, and not a parity oracle: it restates the engine's
// own algorithm, not the reference's.  It runs the kernel's per-node steps one
// lane at a time, so that the CPU test suite can check the engine's logic
// against the oracle (td_oracle.c) without a GPU, and so that the benchmark's
// CPU baseline can time the free-order algorithm on host cores
// (td_emu_search_batch):
//   reference order: pinned state, pair table, 12-bit class table, per-lane
//     step bitmasks and the single-queue child order;
//   free order: row masks and bit-sliced classes (td_row_classes), pair slots,
//     the +2-first child order, the table of explored states and the restarts
//     with their child orders (td_attempt_budget, td_level_order).
// It shares the kernel's helpers in td_core.cuh.  The product library does not
// contain or call it.
#include "../td16_b200/csrc/td_core.cuh"

#include <string.h>

#include <atomic>
#include <thread>
#include <vector>

namespace {

struct Emu {
    int N, T, steps, maxd, ordered;
    uint8_t tri_i[TD_MAX_TRIPLES], tri_j[TD_MAX_TRIPLES], tri_k[TD_MAX_TRIPLES];
    uint32_t acc[TD_MAX_DEPTH + 2], reach[TD_MAX_DEPTH + 2];
    uint8_t lut[4096];
    uint8_t pt[TD_MAX_N * TD_PT_STRIDE];
    uint32_t m1[TD_MAX_DEPTH + 1][32], m2[TD_MAX_DEPTH + 1][32];
    // free order (bit-sliced): rows by caller position, masks, pair slots, outcome words
    uint32_t S[32], G[32], P[32], O, F;
    uint32_t pc[TD_MAX_ROUNDS][32];
    uint32_t pw[TD_MAX_DEPTH + 1][TD_MAX_ROUNDS][32];
    int rounds;
    uint64_t L[TD_MAX_DEPTH + 1];
    int off[TD_MAX_DEPTH + 1];
    uint16_t path[TD_MAX_DEPTH];
    uint32_t expansions;
};

int prepare(Emu &e, uint64_t L, int off) {
    const int N = e.N;
    int B[TD_MAX_N], pos[TD_MAX_N], nxt[TD_MAX_N], lead[TD_MAX_N], dist[TD_MAX_N], len[TD_MAX_N];
    for (int p = 0; p < N; ++p) {
        B[p] = p ? (int)td_nib(L, p - 1) + 1 : 0;
        pos[B[p]] = p;
    }
    for (int p = 0; p < N; ++p) {
        const int q = p ? p - 1 : N - 1;
        int y = B[q] + 1;
        if (y == N) y = 0;
        nxt[p] = pos[y];
    }
    for (int p = 0; p < N; ++p) {
        int m = p, x = nxt[p], l = 1;
        while (x != p) { if (x < m) m = x; x = nxt[x]; ++l; }
        lead[p] = m;
        len[p] = l;
        int d = 0;
        x = p;
        while (x != m) { x = nxt[x]; ++d; }
        dist[p] = d;
    }
    int odd = 0;
    for (int p = 0; p < N; ++p) odd += (lead[p] == p) && (len[p] & 1);
    for (int p = 0; p < N; ++p) {
        const int rp = (p - off + N) % N;
        for (int q = 0; q < N; ++q) {
            const int rq = (q - off + N) % N;
            e.pt[rp * TD_PT_STRIDE + rq] =
                (uint8_t)td_pair_entry(lead[p], dist[p], len[p], lead[q], dist[q]);
        }
    }
    return odd;
}

// Rows of the bit-sliced evaluation, computed the way the kernel does: lane c
// is caller position c, its cycle leader the smallest caller position on the
// cycle, dist the omega steps to it.  Returns the number of odd cycles.
int prepare_rows(Emu &e, uint64_t L, int off) {
    const int N = e.N;
    int B[TD_MAX_N], pos[TD_MAX_N], nxt[32], lead[32], dist[32], len[32];
    for (int p = 0; p < N; ++p) {
        B[p] = p ? (int)td_nib(L, p - 1) + 1 : 0;
        pos[B[p]] = p;
    }
    for (int c = 0; c < 32; ++c) nxt[c] = c;
    for (int c = 0; c < N; ++c) {
        const int p = (c + off) % N;
        const int q = p ? p - 1 : N - 1;
        const int y = (B[q] + 1) % N;
        nxt[c] = (pos[y] - off + N) % N;
    }
    for (int c = 0; c < 32; ++c) {
        int m = c, x = nxt[c], l = 1;
        while (x != c) { if (x < m) m = x; x = nxt[x]; ++l; }
        lead[c] = m;
        len[c] = l;
        int d = 0;
        x = c;
        while (x != m) { x = nxt[x]; ++d; }
        dist[c] = d;
    }
    const uint32_t ACT = (1u << N) - 1u;
    e.O = e.F = 0;
    int odd = 0;
    for (int c = 0; c < N; ++c) {
        if (len[c] & 1) e.O |= 1u << c;
        if (len[c] == 1) e.F |= 1u << c;
        odd += lead[c] == c && (len[c] & 1);
    }
    for (int c = 0; c < N; ++c) {
        uint32_t S = 0, lt = 0, D0 = 0;
        for (int q = 0; q < 32; ++q) {
            if (lead[q] == lead[c]) S |= 1u << q;
            if (dist[q] < dist[c]) lt |= 1u << q;
            if (dist[q] & 1) D0 |= 1u << q;
        }
        S &= ACT;
        const uint32_t lodd = 0u - (uint32_t)(len[c] & 1);
        e.S[c] = S;
        e.G[c] = S & lt;
        e.P[c] = S & ((D0 ^ (0u - (uint32_t)(dist[c] & 1))) ^ (lodd & ~lt));
    }
    return odd;
}

// Bit-sliced evaluation of the node at `level`: fills the outcome words and
// returns the found move (i | j<<5 | k<<10) or -1.
int evaluate_rows(Emu &e, int level, int odd) {
    const int D = level + 1;
    const uint32_t f0 = 0u - ((e.acc[D] >> odd) & 1u), f2 = 0u - ((e.acc[D] >> (odd + 2)) & 1u);
    const uint32_t x0 = (D < e.maxd ? 0u - ((e.reach[D] >> odd) & 1u) : 0u) & ~f0;
    const uint32_t x2 = (D < e.maxd ? 0u - ((e.reach[D] >> (odd + 2)) & 1u) : 0u) & ~f2;
    const uint32_t ACT = (1u << e.N) - 1u;
    uint32_t best = 0xffffffffu;
    for (int lane = 0; lane < 32; ++lane) {
        uint32_t key = 0xffffffffu;
        for (int r = 0; r < e.rounds; ++r) {
            const uint32_t code = e.pc[r][lane];
            const int i = code & 31, j = (code >> 5) & 31, ks = (code >> 10) & 31;
            uint32_t plus, zero;
            td_row_classes_x(e.S[i], e.G[i], e.P[i], e.S[j], e.G[j], e.P[j], e.O, e.F, 0u - ((e.O >> i) & 1u),
                             0u - ((e.O >> j) & 1u), 0u - ((e.F >> i) & 1u), 0u - ((e.F >> j) & 1u), (int)(code >> 15),
                             &plus, &zero);
            const uint32_t km = ACT & (0xfffffffeu << ks);
            const uint32_t fnd = km & ((f0 & zero) | (f2 & plus));
            const uint32_t e2 = km & x2 & plus, e0 = km & x0 & zero;
            e.pw[level][r][lane] = (e2 >> 1) | (e0 << 15);
            if (fnd && key == 0xffffffffu)
                key = ((uint32_t)lane << 17) | ((uint32_t)r << 15) | (code & 1023u) | ((uint32_t)(31 - __builtin_clz(fnd)) << 10);
        }
        if (key < best) best = key;
    }
    e.expansions++;
    return best == 0xffffffffu ? -1 : (int)(best & 0x7fffu);
}

// Next child of `level` in the free order: +2 children first; in the plain
// order (ord = 0) the highest pair slot R*lane + r (lexicographically smallest
// pair) and the smallest k.  `ord` (td_order_variant) rotates the lane
// priority, reverses the round order and takes the largest k first, as the
// kernel does.  Returns the move or -1.
int next_child_rows(Emu &e, int level, uint32_t ord) {
    bool any2 = false;
    for (int lane = 0; lane < 32; ++lane)
        for (int r = 0; r < e.rounds; ++r) any2 |= (e.pw[level][r][lane] & 0xffffu) != 0;
    const uint32_t cm = any2 ? 0x0000ffffu : 0xffff0000u;
    const int rot = (int)(ord & 31u);
    int bl = -1, br = -1;
    unsigned bkey = 0;
    for (int lane = 0; lane < 32; ++lane)
        for (int r = 0; r < e.rounds; ++r)
            if (e.pw[level][r][lane] & cm) {
                const unsigned key = ((((unsigned)(lane - rot) & 31u) << 2) | (unsigned)((ord & 32u) ? 3 - r : r)) + 1u;
                if (key > bkey) { bkey = key; bl = lane; br = r; }
            }
    if (bl < 0) return -1;
    const int lane = bl, r = br;
    const uint32_t w = e.pw[level][r][lane] & cm;
    const int b = (ord & 64u) ? 31 - __builtin_clz(w) : __builtin_ctz(w);
    e.pw[level][r][lane] &= ~(1u << b);
    const int k = any2 ? b + 1 : b - 15;
    return (int)((e.pc[r][lane] & 1023u) | ((uint32_t)k << 10));
}

// Evaluate the children of the node at `level` (parent odd count `odd`).
// Returns the found u (>= 0) or -1.
int evaluate(Emu &e, int level, int odd) {
    const int D = level + 1;
    const int f0 = (e.acc[D] >> odd) & 1, f2 = (e.acc[D] >> (odd + 2)) & 1;
    const int x0 = (D < e.maxd) && ((e.reach[D] >> odd) & 1) && !f0;
    const int x2 = (D < e.maxd) && ((e.reach[D] >> (odd + 2)) & 1) && !f2;
    uint32_t nt;  // byte c holds the flags of class c; byte 0 (filtered out) is zero
    if (e.ordered) nt = ((uint32_t)(f0 | (x0 << 1)) << (8 * TD_CLASS_ZERO)) | ((uint32_t)(f2 | (x2 << 1)) << (8 * TD_CLASS_PLUS2));
    else nt = ((uint32_t)(f0 | (x0 << 2)) << (8 * TD_CLASS_ZERO)) | ((uint32_t)(f2 | (x2 << 1)) << (8 * TD_CLASS_PLUS2));
    uint32_t fb[32];
    for (int lane = 0; lane < 32; ++lane) {
        fb[lane] = 0;
        e.m1[level][lane] = 0;
        e.m2[level][lane] = 0;
        for (int s = 0; s < e.steps; ++s) {
            const int u = 32 * s + lane;
            if (u >= e.T) continue;
            const int t = e.T - 1 - u;
            const int i = e.tri_i[t], j = e.tri_j[t], k = e.tri_k[t];
            const int idx = e.pt[i * TD_PT_STRIDE + j] | (e.pt[j * TD_PT_STRIDE + k] << 4) |
                            (e.pt[k * TD_PT_STRIDE + i] << 8);
            const uint32_t tb = (nt >> (8 * e.lut[idx])) & 7u;
            fb[lane] |= (tb & 1u) << s;
            e.m1[level][lane] |= ((tb >> 1) & 1u) << s;
            e.m2[level][lane] |= ((tb >> 2) & 1u) << s;
        }
    }
    e.expansions++;
    if (e.ordered && level == 0) {  // roots are accepted when visited, not when seeded
        for (int lane = 0; lane < 32; ++lane) e.m2[0][lane] = fb[lane];
        return -1;
    }
    int best = -1;
    for (int lane = 0; lane < 32; ++lane) {
        if (!fb[lane]) continue;
        const int u = 32 * __builtin_ctz(fb[lane]) + lane;
        if (best < 0 || u < best) best = u;
    }
    return best;
}

// Next child of `level` in visit order; returns u or -1; *accepted for roots
// that are accepted on visit (ordered mode).
int next_child(Emu &e, int level, int *accepted) {
    *accepted = 0;
    const bool desc_lanes = e.ordered && level > 0;
    int any1 = 0;
    for (int lane = 0; lane < 32; ++lane) any1 |= e.m1[level][lane] != 0;
    uint32_t best = 0;
    for (int lane = 0; lane < 32; ++lane) {
        uint32_t w;
        if (e.ordered) w = level == 0 ? (e.m1[level][lane] | e.m2[level][lane]) : e.m1[level][lane];
        else w = any1 ? e.m1[level][lane] : e.m2[level][lane];
        if (!w) continue;
        const uint32_t s = 31 - __builtin_clz(w);
        const uint32_t key = s * 32 + (desc_lanes ? 31 - lane : lane) + 1;
        if (key > best) best = key;
    }
    if (!best) return -1;
    best -= 1;
    const int s = (int)(best >> 5);
    const int lane = desc_lanes ? 31 - (int)(best & 31) : (int)(best & 31);
    const uint32_t bit = 1u << s;
    if (e.ordered) {
        if (level == 0 && (e.m2[0][lane] & bit)) *accepted = 1;
        e.m1[level][lane] &= ~bit;
        e.m2[level][lane] &= ~bit;
    } else if (any1) {
        e.m1[level][lane] &= ~bit;
    } else {
        e.m2[level][lane] &= ~bit;
    }
    return 32 * s + lane;
}

// The kernel's table of explored states (free order): 2^12 entries, key =
// td_tt_key of the pinned state (nibbles from N-1 on cleared) times an odd
// constant modulo 2^57, the top 12 bits the slot and the rest the tag, a
// 15-bit generation, the depth in the top nibble.  The generation counter
// persists across searches on a thread, as the kernel's does across units.
#define EMU_TT_BITS 12
// restart budget base of the free order (the kernel's default); 0 = none
static uint32_t g_restart_base = 16;
extern "C" void td_emu_set_restart(uint32_t base) { g_restart_base = base; }
// The child order at DFS level `level` of attempt a, its budget for a base,
// and the number of budgeted attempts (td_core.cuh), for the CPU tests.
extern "C" uint32_t td_emu_order(int a, int level) { return td_level_order(td_order_variant(a), a, level); }
extern "C" uint32_t td_emu_budget(uint32_t base, int a) { return td_attempt_budget(base, a); }
extern "C" int td_emu_restarts(void) { return TD_RESTARTS; }
bool tt_visit(uint64_t *tt, uint64_t L, int N, int lv, uint32_t gen) {
    const uint64_t data = N - 1 >= 16 ? ~0ull : ((1ull << (4 * (N - 1))) - 1ull);
    const uint64_t h = (td_tt_key(L & data) * 0x9E3779B97F4A7C15ull) & 0x01ffffffffffffffull;
    const int tag_bits = 57 - EMU_TT_BITS;
    const unsigned slot = (unsigned)(h >> tag_bits);
    const uint64_t want = (h & ((1ull << tag_bits) - 1ull)) | ((uint64_t)gen << tag_bits);
    const uint64_t old = tt[slot];
    if ((old & ((1ull << 60) - 1ull)) == want && (int)(old >> 60) <= lv) return true;
    tt[slot] = want | ((uint64_t)lv << 60);
    return false;
}

// the next generation of the thread's table; clears it when the counter wraps
uint32_t tt_next_gen(uint64_t *tt, uint32_t &counter) {
    if (++counter >= (1u << (EMU_TT_BITS + 3))) {
        for (int q = 0; q < (1 << EMU_TT_BITS); ++q) tt[q] = 0;
        counter = 1;
    }
    return counter;
}

int search_rows(Emu &e, td_result *res) {
    static thread_local uint64_t tt[1 << EMU_TT_BITS];  // zero-initialised: every word empty
    static thread_local uint32_t tt_counter = 0;
    bool tt_on = false;  // in use after 32 expansions, as in the kernel
    uint32_t tt_gen = 0;
    int attempt = 0;     // restarts, as in the kernel
    uint32_t ord = 0, attempt_exp = 1, attempt_budget = td_attempt_budget(g_restart_base, 0);
    const int NP = (e.N - 1) * (e.N - 2) / 2;
    e.rounds = (NP + 31) / 32;
    for (int r = 0; r < TD_MAX_ROUNDS; ++r)
        for (int lane = 0; lane < 32; ++lane) e.pc[r][lane] = td_pair_code(e.N, r < e.rounds ? e.rounds * lane + r : -1);
    int level = 0;
    int odd = prepare_rows(e, e.L[0], e.off[0]);
    int found = evaluate_rows(e, 0, odd);
    for (;;) {
        if (found >= 0) {
            for (int d = 0; d < level; ++d) res->moves[d] = e.path[d];
            res->moves[level] = (uint16_t)found;
            res->depth = level + 1;
            res->status = TD_FOUND;
            break;
        }
        if (attempt_exp >= attempt_budget) {
            ++attempt;
            ord = td_order_variant(attempt);
            attempt_budget = td_attempt_budget(g_restart_base, attempt);
            attempt_exp = 1;
            if (tt_on) tt_gen = tt_next_gen(tt, tt_counter);  // the abandoned attempt's entries no longer match
            level = 0;
            odd = prepare_rows(e, e.L[0], e.off[0]);
            found = evaluate_rows(e, 0, odd);
            continue;
        }
        const int t = next_child_rows(e, level, td_level_order(ord, attempt, level));
        if (t < 0) {
            if (level == 0) { res->status = TD_NOT_FOUND; break; }
            --level;
            continue;
        }
        e.path[level] = (uint16_t)t;
        int noff;
        td_apply_move(e.L[level], e.off[level], e.N, t & 31, (t >> 5) & 31, (t >> 10) & 31, &e.L[level + 1], &noff);
        e.off[level + 1] = noff;
        if (!tt_on && e.expansions >= 32) {
            tt_gen = tt_next_gen(tt, tt_counter);
            tt_on = true;
        }
        if (tt_on && tt_visit(tt, e.L[level + 1], e.N, level + 1, tt_gen)) continue;  // explored with at least this budget
        ++level;
        odd = prepare_rows(e, e.L[level], e.off[level]);
        found = evaluate_rows(e, level, odd);
        ++attempt_exp;
    }
    res->expansions = e.expansions;
    return res->status;
}

}  // namespace

// Compares the bit-sliced classes of every triple of the state (L, off) with
// the 12-bit class table; returns the number of triples that differ.
extern "C" int td_emu_row_check(uint64_t L, int off, int N) {
    static thread_local Emu e;
    e.N = N;
    prepare(e, L, off);
    prepare_rows(e, L, off);
    const uint32_t ACT = (1u << N) - 1u;
    int bad = 0;
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
            uint32_t plus, zero;
            td_row_classes(e.S[i], e.G[i], e.P[i], e.S[j], e.G[j], e.P[j], e.O, e.F, i, j, &plus, &zero);
            plus &= ACT;
            zero &= ACT;
            for (int k = j + 1; k < N; ++k) {
                const int idx = e.pt[i * TD_PT_STRIDE + j] | (e.pt[j * TD_PT_STRIDE + k] << 4) |
                                (e.pt[k * TD_PT_STRIDE + i] << 8);
                const int cls = td_class_of_index(idx);
                const int got = ((plus >> k) & 1) ? TD_CLASS_PLUS2 : (((zero >> k) & 1) ? TD_CLASS_ZERO : TD_CLASS_SKIP);
                if (((plus >> k) & 1) && ((zero >> k) & 1)) ++bad;
                else if (got != cls) ++bad;
            }
        }
    return bad;
}

extern "C" int td_emu_search(const td_instance *x, unsigned flags, td_result *res) {
    static thread_local Emu e;
    memset(res, 0, sizeof *res);
    e.N = x->n_symbols;
    e.maxd = x->max_moves;
    e.ordered = (flags & TD_FLAG_ORDERED) != 0;
    if (e.N > TD_MAX_N || e.maxd < 1 || e.maxd > TD_MAX_DEPTH) { res->status = TD_ERR_ARG; return res->status; }
    e.T = td_triple_count(e.N);
    if (e.T == 0) { res->status = TD_NOT_FOUND; return 0; }
    e.steps = (e.T + 31) / 32;
    int t = 0;
    for (int i = 0; i < e.N - 2; ++i)
        for (int j = i + 1; j < e.N - 1; ++j)
            for (int k = j + 1; k < e.N; ++k) { e.tri_i[t] = i; e.tri_j[t] = j; e.tri_k[t] = k; ++t; }
    for (int idx = 0; idx < 4096; ++idx) e.lut[idx] = (uint8_t)td_class_of_index(idx);
    const int init = td_inst_init(*x), full = td_inst_full(*x);
    for (int D = 0; D <= TD_MAX_DEPTH + 1; ++D) {
        e.acc[D] = e.reach[D] = 0;
        for (int o = 0; o < 32; ++o) {
            if (td_accepts(e.N, init, x->min_rate, full, o, D)) e.acc[D] |= 1u << o;
            if (td_can_reach(e.N, init, x->min_rate, e.maxd, full, o, D)) e.reach[D] |= 1u << o;
        }
    }
    e.expansions = 0;
    e.L[0] = x->perm;
    e.off[0] = x->offset;
    if (!e.ordered) return search_rows(e, res);
    int level = 0;
    int odd = prepare(e, e.L[0], e.off[0]);
    int found = evaluate(e, 0, odd);
    for (;;) {
        if (found >= 0) {
            const int tt = e.T - 1 - found;
            for (int d = 0; d < level; ++d) res->moves[d] = e.path[d];
            res->moves[level] = td_pack_move(e.tri_i[tt], e.tri_j[tt], e.tri_k[tt]);
            res->depth = level + 1;
            res->status = TD_FOUND;
            break;
        }
        int accepted;
        const int u = next_child(e, level, &accepted);
        if (u < 0) {
            if (level == 0) { res->status = TD_NOT_FOUND; break; }
            --level;
            continue;
        }
        const int tt = e.T - 1 - u;
        const int i = e.tri_i[tt], j = e.tri_j[tt], k = e.tri_k[tt];
        e.path[level] = td_pack_move(i, j, k);
        if (accepted) {
            for (int d = 0; d <= level; ++d) res->moves[d] = e.path[d];
            res->depth = level + 1;
            res->status = TD_FOUND;
            break;
        }
        int noff;
        td_apply_move(e.L[level], e.off[level], e.N, i, j, k, &e.L[level + 1], &noff);
        e.off[level + 1] = noff;
        ++level;
        odd = prepare(e, e.L[level], e.off[level]);
        found = evaluate(e, level, odd);
    }
    res->expansions = e.expansions;
    return res->status;
}

extern "C" int td_emu_prepare_pair(const uint8_t *beta, const uint8_t *omega, int N, int init,
                                   float min_rate, int max_moves, int full, td_instance *out) {
    return td_prepare_pair(beta, omega, N, init, min_rate, max_moves, full, out);
}

extern "C" void td_emu_apply_move(uint64_t L, int off, int N, int i, int j, int k, uint64_t *outL, int *outOff) {
    td_apply_move(L, off, N, i, j, k, outL, outOff);
}

// `count` independent searches on `threads` host threads, one instance per
// thread at a time (the CPU baseline of the free order).  flags as for
// td_emu_search.  Returns 0.
extern "C" int td_emu_search_batch(int count, const td_instance *x, unsigned flags, td_result *res, int threads) {
    std::atomic<int> next{0};
    auto work = [&] {
        for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1)) td_emu_search(&x[i], flags, &res[i]);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}

// The engine's device replay of a witness (td_witness_ok, the rule of
// TD_FLAG_VERIFY), for the CPU tests.
extern "C" int td_emu_witness_ok(const td_instance *x, const td_result *r) { return td_witness_ok(*x, *r); }

// The inverse instance and the conversion of its witnesses (td_core.cuh:
// td_inverse_pinned, td_witness_from_inverse), which the batch engine's race
// of a search against the search of its inverse uses; for the CPU tests.
extern "C" void td_emu_inverse_instance(const td_instance *x, td_instance *out) {
    *out = *x;
    out->perm = td_inverse_pinned(x->perm, x->n_symbols);
    out->offset = 0;
}

extern "C" int td_emu_witness_from_inverse(const td_instance *x, const td_result *inv, td_result *out) {
    *out = *inv;
    return td_witness_from_inverse(x->perm, x->offset, x->n_symbols, inv->moves, inv->depth, out->moves);
}

extern "C" int td_emu_pinned_cycles(uint64_t L, int off, int N) {
    uint32_t fixed;
    return td_pinned_cycles(L, off, N, &fixed);
}
