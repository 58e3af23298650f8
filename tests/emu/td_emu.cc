// td_emu.cc -- serial host emulation of the engine's warp algorithm.
//
// TEST INFRASTRUCTURE ONLY.  It runs the kernel's exact per-node steps
// (pinned state, pair table, 12-bit class table, per-lane step bitmasks,
// child selection order) one lane at a time, so the CPU test suite can check
// the engine's logic against the oracle without a GPU.  The product library
// does not contain or call it.
#include "../../td16_b200/csrc/td_core.cuh"

#include <string.h>

namespace {

struct Emu {
    int N, T, steps, maxd, ordered;
    uint8_t tri_i[TD_MAX_TRIPLES], tri_j[TD_MAX_TRIPLES], tri_k[TD_MAX_TRIPLES];
    uint32_t acc[TD_MAX_DEPTH + 2], reach[TD_MAX_DEPTH + 2];
    uint8_t lut[4096];
    uint8_t pt[TD_MAX_N * TD_PT_STRIDE];
    uint32_t m1[TD_MAX_DEPTH + 1][32], m2[TD_MAX_DEPTH + 1][32];
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

}  // namespace

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
