/*
 * td_oracle.c -- CPU oracle for the td16 witness search.
 *
 * TEST INFRASTRUCTURE ONLY (see td_oracle.h).  Everything here is scalar C
 * written for readability; the f32 rate test is compiled without fast-math so
 * that it rounds exactly like the reference's IEEE single-precision division.
 */
#include "td_oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int tdo_triple_count(int n) { return n < 3 ? 0 : n * (n - 1) * (n - 2) / 6; }

/* PackedMove: three 5-bit position fields (core/common.cuh:18-54, MAX_N=17) */
uint16_t tdo_pack_move(int i, int j, int k) {
    return (uint16_t)((i & 31) | ((j & 31) << 5) | ((k & 31) << 10));
}

void tdo_unpack_move(uint16_t m, int *i, int *j, int *k) {
    *i = m & 31;
    *j = (m >> 5) & 31;
    *k = (m >> 10) & 31;
}

/* Odd-length cycles of omega, fixed points included
 * (sorting_search.cu:211-226; Cycle.isEven is "odd size", Cycle.java:149-151). */
int tdo_count_odd_cycles(const uint8_t *omega, int n) {
    uint32_t seen = 0;
    int odd = 0;
    for (int s = 0; s < n; ++s) {
        if (seen & (1u << s)) continue;
        int len = 0;
        int x = s;
        do {
            seen |= 1u << x;
            ++len;
            x = omega[x];
        } while (x != s);
        odd += len & 1;
    }
    return odd;
}

/* Steps from `from` along omega until the first of {a, b, c} is met. */
static int walk_to_marked(const uint8_t *omega, int from, int a, int b, int c,
                          int *met) {
    int steps = 1;
    int x = omega[from];
    while (x != a && x != b && x != c) {
        x = omega[x];
        ++steps;
    }
    *met = x;
    return steps;
}

/* Odd-cycle change when omega becomes omega . (a b c)^-1
 * (sorting_search.cu:240-332).  The three marked symbols cut their cycles into
 * arcs; the new cycle lengths are sums of arcs. */
int tdo_delta_odd_cycles(const uint8_t *omega, int a, int b, int c) {
    int ma, mb, mc;
    const int da = walk_to_marked(omega, a, a, b, c, &ma);
    const int db = walk_to_marked(omega, b, a, b, c, &mb);
    const int dc = walk_to_marked(omega, c, a, b, c, &mc);

    if (ma == a && mb == b && mc == c) return TDO_DELTA_SKIP; /* three cycles */
    if (ma == b && mb == c && mc == a) {                     /* one cycle, split in three */
        const int len = da + db + dc;
        return (da & 1) + (db & 1) + (dc & 1) - (len & 1);
    }
    if (ma == c && mb == a && mc == b) return 0; /* one cycle, stays one */
    if (ma == b && mb == a) {                    /* {a,b} together, c apart */
        const int l1 = da + db, l2 = dc;
        return (da & 1) + ((db + dc) & 1) - (l1 & 1) - (l2 & 1);
    }
    if (mb == c && mc == b) { /* {b,c} together, a apart */
        const int l1 = db + dc, l2 = da;
        return (db & 1) + ((dc + da) & 1) - (l1 & 1) - (l2 & 1);
    }
    if (ma == c && mc == a) { /* {a,c} together, b apart */
        const int l1 = da + dc, l2 = db;
        return (dc & 1) + ((da + db) & 1) - (l1 & 1) - (l2 & 1);
    }
    return TDO_DELTA_SKIP;
}

/* satisfies_rate (sorting_search.cu:336-346) */
int tdo_accepts(int n, int init_odd, float min_rate, int full, int odd, int depth) {
    if (depth <= 0) return 0;
    if (full && odd != n) return 0;
    const int gained = odd - init_odd;
    const float ratio = (float)gained / (float)depth;
    return gained > 0 && ratio >= min_rate;
}

/* can_still_reach (sorting_search.cu:348-373) */
int tdo_can_reach(int n, int init_odd, float min_rate, int max_depth, int full,
                  int odd, int depth) {
    const int missing = n - odd;
    if (full) return depth + (missing + 1) / 2 <= max_depth;
    const int gained = odd - init_odd;
    const int left = max_depth - depth;
    const int required = (int)floorf(min_rate * (float)max_depth);
    if (gained + 2 * left < required) return 0;
    const int best_depth = depth + (missing + 1) / 2;
    if (best_depth > 0) {
        const float best = (float)(gained + missing) / (float)best_depth;
        if (best < min_rate) return 0;
    }
    return 1;
}

/* ---- search ---------------------------------------------------------- */

typedef struct {
    uint8_t depth;
    uint8_t odd;
    uint16_t moves[TDO_MAX_DEPTH];
    uint8_t omega[TDO_MAX_N];
    uint8_t beta[TDO_MAX_N]; /* current beta array, first element = betaStart */
} tdo_node;

typedef struct {
    tdo_node *items;
    size_t size, cap;
} tdo_stack;

static int stack_push(tdo_stack *s, const tdo_node *node) {
    if (s->size == s->cap) {
        size_t cap = s->cap ? 2 * s->cap : 4096;
        tdo_node *grown = (tdo_node *)realloc(s->items, cap * sizeof(tdo_node));
        if (!grown) return -1;
        s->items = grown;
        s->cap = cap;
    }
    s->items[s->size++] = *node;
    return 0;
}

/* block swap of [i,j) and [j,k) in a linear array of n symbols */
static void swap_blocks(const uint8_t *src, int n, int i, int j, int k, uint8_t *dst) {
    int w = 0;
    for (int p = 0; p < i; ++p) dst[w++] = src[p];
    for (int p = j; p < k; ++p) dst[w++] = src[p];
    for (int p = i; p < j; ++p) dst[w++] = src[p];
    for (int p = k; p < n; ++p) dst[w++] = src[p];
}

/* Child of `parent` under the position triple (i,j,k); returns 0 when the move
 * is filtered out (a fixed symbol, or an odd-cycle change outside {0,+2}),
 * else 1 with *delta set.  sorting_search.cu:436-445, 603-611. */
static int make_child(const tdo_node *parent, int n, int i, int j, int k,
                      tdo_node *child, int *delta) {
    const int a = parent->beta[i], b = parent->beta[j], c = parent->beta[k];
    const uint8_t *om = parent->omega;
    if (om[a] == a || om[b] == b || om[c] == c) return 0;
    const int d = tdo_delta_odd_cycles(om, a, b, c);
    if (d != 0 && d != 2) return 0;
    *delta = d;
    memcpy(child->omega, om, (size_t)n);
    child->omega[a] = om[c];
    child->omega[b] = om[a];
    child->omega[c] = om[b];
    swap_blocks(parent->beta, n, i, j, k, child->beta);
    return 1;
}

/* Expansion budget of later searches (0 = none): lets fixture generators
 * drop candidate cases whose trees are too large to search in a test. */
static _Atomic uint64_t g_budget = 0;
void tdo_set_expansion_budget(uint64_t max_expansions) { atomic_store(&g_budget, max_expansions); }

int tdo_search(const uint8_t *beta, const uint8_t *omega, int n, int init_odd,
               float min_rate, int max_depth, int full, uint16_t *out_moves,
               int *out_depth, tdo_stats *stats) {
    const uint64_t budget = atomic_load(&g_budget);
    if (out_depth) *out_depth = 0;
    if (n < 0 || n > TDO_MAX_N) return TDO_EINVAL;
    if (max_depth <= 0 || max_depth > TDO_MAX_DEPTH) return TDO_EINVAL;
    const int T = tdo_triple_count(n);
    if (T == 0) return TDO_NOT_FOUND;

    /* lexicographic position triples (sorting_search.cu:852-860) */
    static __thread uint8_t ti[816], tj[816], tk[816]; /* C(17,3) = 680 */
    {
        int t = 0;
        for (int i = 0; i < n - 2; ++i)
            for (int j = i + 1; j < n - 1; ++j)
                for (int k = j + 1; k < n; ++k) {
                    ti[t] = (uint8_t)i;
                    tj[t] = (uint8_t)j;
                    tk[t] = (uint8_t)k;
                    ++t;
                }
    }

    tdo_stats local = {0, 0, 0};
    tdo_stack st = {NULL, 0, 0};
    int status = TDO_NOT_FOUND;

    tdo_node root;
    memset(&root, 0, sizeof root);
    memcpy(root.beta, beta, (size_t)n);
    memcpy(root.omega, omega, (size_t)n);

    /* Seeding with one queue: roots in reverse triple order, so the owner's
     * LIFO pop visits them in ascending triple order (sorting_search.cu:411-454). */
    for (int fwd = 0; fwd < T; ++fwd) {
        const int t = T - 1 - fwd;
        tdo_node child;
        int delta;
        if (!make_child(&root, n, ti[t], tj[t], tk[t], &child, &delta)) continue;
        child.depth = 1;
        child.odd = (uint8_t)tdo_count_odd_cycles(child.omega, n);
        memset(child.moves, 0, sizeof child.moves);
        child.moves[0] = tdo_pack_move(ti[t], tj[t], tk[t]);
        if (stack_push(&st, &child)) { status = TDO_EINVAL; goto done; }
    }

    while (st.size > 0) {
        const tdo_node node = st.items[--st.size];
        local.pops++;
        if (tdo_accepts(n, init_odd, min_rate, full, node.odd, node.depth)) {
            for (int d = 0; d < node.depth; ++d) out_moves[d] = node.moves[d];
            if (out_depth) *out_depth = node.depth;
            status = TDO_FOUND;
            goto done;
        }
        if (node.depth >= max_depth ||
            !tdo_can_reach(n, init_odd, min_rate, max_depth, full, node.odd, node.depth))
            continue;
        if (budget && local.expansions >= budget) {
            status = TDO_BUDGET;
            goto done;
        }
        local.expansions++;
        const int child_depth = node.depth + 1;

        /* Children in chunks of 32 "lanes", triple index descending
         * (sorting_search.cu:585-590).  Within a chunk the lowest accepting
         * lane wins (:632-641); survivors are pushed highest lane first
         * (:648-686). */
        for (int base = 0; base < T; base += 32) {
            tdo_node chunk[32];
            int keep[32];
            int found_lane = -1;
            for (int lane = 0; lane < 32; ++lane) {
                keep[lane] = 0;
                const int t = T - 1 - base - lane;
                if (t < 0) continue;
                local.triples++;
                int delta;
                if (!make_child(&node, n, ti[t], tj[t], tk[t], &chunk[lane], &delta)) continue;
                const int odd = node.odd + delta;
                if (tdo_accepts(n, init_odd, min_rate, full, odd, child_depth)) {
                    if (found_lane < 0) found_lane = lane;
                    continue;
                }
                if (child_depth < max_depth &&
                    tdo_can_reach(n, init_odd, min_rate, max_depth, full, odd, child_depth)) {
                    chunk[lane].depth = (uint8_t)child_depth;
                    chunk[lane].odd = (uint8_t)odd;
                    memcpy(chunk[lane].moves, node.moves, sizeof node.moves);
                    chunk[lane].moves[node.depth] = tdo_pack_move(ti[t], tj[t], tk[t]);
                    keep[lane] = 1;
                }
            }
            if (found_lane >= 0) {
                const int t = T - 1 - base - found_lane;
                for (int d = 0; d < node.depth; ++d) out_moves[d] = node.moves[d];
                out_moves[node.depth] = tdo_pack_move(ti[t], tj[t], tk[t]);
                if (out_depth) *out_depth = child_depth;
                status = TDO_FOUND;
                goto done;
            }
            for (int lane = 31; lane >= 0; --lane) {
                if (!keep[lane]) continue;
                if (stack_push(&st, &chunk[lane])) { status = TDO_EINVAL; goto done; }
            }
        }
    }

done:
    free(st.items);
    if (stats) {
        stats->expansions += local.expansions;
        stats->pops += local.pops;
        stats->triples += local.triples;
    }
    return status;
}

/* ---- batch on host threads ------------------------------------------- */

typedef struct {
    int count;
    const uint8_t *beta, *omega, *n, *full;
    const int32_t *init_odd, *max_depth;
    const float *min_rate;
    int32_t *out_status, *out_depth;
    uint16_t *out_moves;
    uint64_t *out_expansions;
    atomic_int next;
} batch_job;

static void *batch_worker(void *arg) {
    batch_job *job = (batch_job *)arg;
    for (;;) {
        const int idx = atomic_fetch_add(&job->next, 1);
        if (idx >= job->count) break;
        tdo_stats st = {0, 0, 0};
        int depth = 0;
        const int rc = tdo_search(job->beta + (size_t)idx * TDO_MAX_N,
                                  job->omega + (size_t)idx * TDO_MAX_N, job->n[idx],
                                  job->init_odd[idx], job->min_rate[idx],
                                  job->max_depth[idx], job->full[idx],
                                  job->out_moves + (size_t)idx * TDO_MAX_DEPTH, &depth, &st);
        job->out_status[idx] = rc;
        job->out_depth[idx] = depth;
        if (job->out_expansions) job->out_expansions[idx] = st.expansions;
    }
    return NULL;
}

int tdo_search_batch(int count, const uint8_t *beta, const uint8_t *omega,
                     const uint8_t *n, const int32_t *init_odd,
                     const float *min_rate, const int32_t *max_depth,
                     const uint8_t *full, int32_t *out_status,
                     int32_t *out_depth, uint16_t *out_moves,
                     uint64_t *out_expansions, int threads) {
    if (count < 0 || threads <= 0) return TDO_EINVAL;
    batch_job job = {count, beta, omega, n, full, init_odd, max_depth, min_rate,
                     out_status, out_depth, out_moves, out_expansions, 0};
    atomic_init(&job.next, 0);
    if (threads == 1) {
        batch_worker(&job);
        return 0;
    }
    pthread_t *tids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!tids) return TDO_EINVAL;
    int started = 0;
    for (; started < threads; ++started)
        if (pthread_create(&tids[started], NULL, batch_worker, &job)) break;
    if (started == 0) batch_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tids[t], NULL);
    free(tids);
    return 0;
}

/* ---- instance conversion ---------------------------------------------- */

/* beta = (0 1 ... n), rho = (0, pi0+1, ..., pi_{n-1}+1), omega = rho . beta^-1,
 * i.e. omega(x) = rho((x-1) mod N). */
void tdo_perm_to_pair(const int8_t *pi, int n, uint8_t *beta, uint8_t *omega,
                      int *init_odd) {
    const int N = n + 1;
    uint8_t rho_seq[TDO_MAX_N], rho[TDO_MAX_N];
    rho_seq[0] = 0;
    for (int m = 0; m < n; ++m) rho_seq[m + 1] = (uint8_t)(pi[m] + 1);
    for (int m = 0; m < N; ++m) rho[rho_seq[m]] = rho_seq[(m + 1) % N];
    for (int x = 0; x < N; ++x) {
        beta[x] = (uint8_t)x;
        omega[x] = rho[(x + N - 1) % N];
    }
    if (init_odd) *init_odd = tdo_count_odd_cycles(omega, N);
}

void tdo_positions_to_symbols(const uint8_t *beta, int n, const uint16_t *moves,
                              int count, uint8_t *out_abc) {
    uint8_t cur[TDO_MAX_N], nxt[TDO_MAX_N];
    memcpy(cur, beta, (size_t)n);
    for (int m = 0; m < count; ++m) {
        int i, j, k;
        tdo_unpack_move(moves[m], &i, &j, &k);
        out_abc[3 * m + 0] = cur[i];
        out_abc[3 * m + 1] = cur[j];
        out_abc[3 * m + 2] = cur[k];
        swap_blocks(cur, n, i, j, k, nxt);
        memcpy(cur, nxt, (size_t)n);
    }
}

/* ---- permutation algebra -------------------------------------------- */

void tdo_apply_transposition(const uint8_t *cycle, int n, int a, int b, int c,
                             uint8_t *out) {
    int idx[3] = {0, 0, 0};
    for (int p = 0; p < n; ++p) {
        if (cycle[p] == a) idx[0] = p;
        if (cycle[p] == b) idx[1] = p;
        if (cycle[p] == c) idx[2] = p;
    }
    for (int x = 0; x < 2; ++x) /* sort three */
        for (int y = 0; y < 2 - x; ++y)
            if (idx[y] > idx[y + 1]) {
                int t = idx[y];
                idx[y] = idx[y + 1];
                idx[y + 1] = t;
            }
    swap_blocks(cycle, n, idx[0], idx[1], idx[2], out);
}

void tdo_compose(const uint8_t *p, const uint8_t *q, int n, uint8_t *out) {
    for (int x = 0; x < n; ++x) out[x] = p[q[x]];
}

void tdo_cycle_oneline(const uint8_t *cyc, int len, int n, uint8_t *out) {
    for (int x = 0; x < n; ++x) out[x] = (uint8_t)x;
    for (int m = 0; m < len; ++m) out[cyc[m]] = cyc[(m + 1) % len];
}

/* ---- witness replay (CertificateValidator.validate) ------------------ */

static void set_err(char *err, size_t len, const char *msg) {
    if (err && len) snprintf(err, len, "%s", msg);
}

int tdo_validate(const uint8_t *beta, const uint8_t *omega, int n,
                 const uint8_t *abc, int count, int max_moves, char *err,
                 size_t errlen) {
    if (n <= 0 || n > TDO_MAX_N) {
        set_err(err, errlen, "invalid domain size");
        return -1;
    }
    if (count < 1 || count > max_moves) {
        set_err(err, errlen, "certificate length outside 1..maxMoves");
        return -2;
    }
    uint8_t cur_beta[TDO_MAX_N], cur_omega[TDO_MAX_N], rho[TDO_MAX_N];
    uint8_t beta_fn[TDO_MAX_N], tmp[TDO_MAX_N];
    memcpy(cur_beta, beta, (size_t)n);
    memcpy(cur_omega, omega, (size_t)n);
    tdo_cycle_oneline(beta, n, n, beta_fn);
    tdo_compose(omega, beta_fn, n, rho); /* rho = omega . beta */
    for (int m = 0; m < count; ++m) {
        const int a = abc[3 * m], b = abc[3 * m + 1], c = abc[3 * m + 2];
        if (a == b || b == c || a == c) {
            set_err(err, errlen, "a move must contain three distinct symbols");
            return -3;
        }
        int pa = -1, pb = -1, pc = -1;
        for (int p = 0; p < n; ++p) {
            if (cur_beta[p] == a) pa = p;
            if (cur_beta[p] == b) pb = p;
            if (cur_beta[p] == c) pc = p;
        }
        if (pa < 0 || pb < 0 || pc < 0 || !(pa < pb && pb < pc)) {
            set_err(err, errlen, "move is not an ordered triple in the current cyclic order");
            return -4;
        }
        /* omega <- omega . (a b c)^-1 */
        uint8_t inv[TDO_MAX_N];
        for (int x = 0; x < n; ++x) inv[x] = (uint8_t)x;
        inv[b] = (uint8_t)a;
        inv[c] = (uint8_t)b;
        inv[a] = (uint8_t)c;
        tdo_compose(cur_omega, inv, n, tmp);
        memcpy(cur_omega, tmp, (size_t)n);
        tdo_apply_transposition(cur_beta, n, a, b, c, tmp);
        memcpy(cur_beta, tmp, (size_t)n);
        tdo_cycle_oneline(cur_beta, n, n, beta_fn);
        tdo_compose(cur_omega, beta_fn, n, tmp);
        if (memcmp(tmp, rho, (size_t)n) != 0) {
            set_err(err, errlen, "certificate move does not preserve the cyclic target");
            return -5;
        }
    }
    for (int x = 0; x < n; ++x)
        if (cur_omega[x] != x) {
            set_err(err, errlen, "certificate does not sort the algebraic permutation");
            return -6;
        }
    return 0;
}

/* ---- certificate codec (CertificateCodec.java:22-147) ---------------- */

static int put_symbol(uint8_t *buf, int bit, int symbol) {
    for (int b = 0; b < 5; ++b) {
        const int v = (symbol >> (4 - b)) & 1;
        const int o = bit + b;
        buf[o >> 3] |= (uint8_t)(v << (7 - (o & 7)));
    }
    return bit + 5;
}

static int get_symbol(const uint8_t *buf, int bit) {
    int s = 0;
    for (int b = 0; b < 5; ++b) {
        const int o = bit + b;
        s = (s << 1) | ((buf[o >> 3] >> (7 - (o & 7))) & 1);
    }
    return s;
}

static int padding_ok(const uint8_t *in, int len, int payload_bits) {
    if (len != (payload_bits + 7) / 8) return 0;
    const int pad = 8 * len - payload_bits;
    return pad == 0 || (in[len - 1] & ((1 << pad) - 1)) == 0;
}

int tdo_codec_key(const uint8_t *omega, int n, uint8_t *out, int cap) {
    if (n <= 0 || n > 32) return -1;
    const int len = (5 * n + 7) / 8;
    if (cap < len) return -1;
    memset(out, 0, (size_t)len);
    int bit = 0;
    for (int x = 0; x < n; ++x) {
        if (omega[x] >= 32) return -1;
        bit = put_symbol(out, bit, omega[x]);
    }
    return len;
}

int tdo_codec_value(const uint8_t *abc, int count, uint8_t *out, int cap) {
    if (count <= 0) return -1;
    const int len = (15 * count + 7) / 8;
    if (cap < len) return -1;
    memset(out, 0, (size_t)len);
    int bit = 0;
    for (int m = 0; m < 3 * count; ++m) {
        if (abc[m] >= 32) return -1;
        bit = put_symbol(out, bit, abc[m]);
    }
    return len;
}

int tdo_codec_decode_key(const uint8_t *in, int len, int n, uint8_t *omega) {
    if (n <= 0 || n > 32) return -1;
    if (!in || !padding_ok(in, len, 5 * n)) return -1;
    for (int x = 0; x < n; ++x) omega[x] = (uint8_t)get_symbol(in, 5 * x);
    return n;
}

int tdo_codec_decode_value(const uint8_t *in, int len, uint8_t *abc, int cap) {
    if (!in || len <= 0) return -1;
    const int count = (8 * len) / 15;
    if (count == 0) return -1;
    if (!padding_ok(in, len, 15 * count)) return -1;
    if (cap < count) return -1;
    for (int m = 0; m < 3 * count; ++m) abc[m] = (uint8_t)get_symbol(in, 5 * m);
    return count;
}

/* ---- seeded synthetic instances ------------------------------------------
 *
 * The benchmark's instance generator, restated here so that the CPU baseline
 * and the reference arm of bench.py build their inputs without loading the
 * engine library.  A CPU test checks it bit for bit against the engine's
 * td_synth_perms.  Published methods only:
 *   - splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
 *     generators", OOPSLA 2014), one stream per instance seeded seed ^ index;
 *   - Lemire's multiply-shift bounded integer with rejection ("Fast random
 *     integer generation in an interval", TOMACS 2019) on the top 32 bits of
 *     each draw;
 *   - Fisher-Yates from the last position down for the uniform permutations;
 *   - for the hard ones, the reverse permutation composed with a uniform
 *     number of block transpositions, each a uniform lexicographic rank over
 *     the triples x < y < z of {0..n} (blocks [x,y) and [y,z) swapped). */

static uint64_t synth_next(uint64_t *state) {
    *state += 0x9E3779B97F4A7C15ull;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint32_t synth_below(uint64_t *state, uint32_t bound) {
    uint64_t product = (uint64_t)(uint32_t)(synth_next(state) >> 32) * bound;
    if ((uint32_t)product < bound) {
        const uint32_t floor_rem = (uint32_t)(-bound) % bound;
        while ((uint32_t)product < floor_rem)
            product = (uint64_t)(uint32_t)(synth_next(state) >> 32) * bound;
    }
    return (uint32_t)(product >> 32);
}

/* rank -> (x, y, z), lexicographic over x < y < z <= n */
static void synth_triple(int n, uint32_t rank, int *x, int *y, int *z) {
    for (int a = 0; a <= n - 2; ++a) {
        const int rest = n - a;  /* symbols after a */
        const uint32_t with_a = (uint32_t)(rest * (rest - 1) / 2);
        if (rank >= with_a) {
            rank -= with_a;
            continue;
        }
        for (int b = a + 1; b <= n - 1; ++b) {
            const uint32_t with_b = (uint32_t)(n - b);
            if (rank < with_b) {
                *x = a;
                *y = b;
                *z = b + 1 + (int)rank;
                return;
            }
            rank -= with_b;
        }
    }
    *x = 0;
    *y = 1;
    *z = 2;
}

int tdo_synth_perms(uint64_t seed, int count, int n_min, int n_max, int hard_pct,
                    int hard_min, int hard_max, int8_t *perms, uint8_t *n_out) {
    if (count < 0 || n_min < 1 || n_max > 16 || n_min > n_max || hard_min < 0 ||
        hard_max < hard_min)
        return TDO_EINVAL;
    for (int idx = 0; idx < count; ++idx) {
        uint64_t state = seed ^ (uint64_t)idx;
        const int n = n_min + (int)synth_below(&state, (uint32_t)(n_max - n_min + 1));
        int8_t *p = perms + (size_t)idx * 16;
        const int hard = (int)synth_below(&state, 100) < hard_pct;
        if (hard) {
            for (int m = 0; m < n; ++m) p[m] = (int8_t)(n - 1 - m);
            const int moves = hard_min + (int)synth_below(&state, (uint32_t)(hard_max - hard_min + 1));
            const uint32_t ranks = (uint32_t)((n + 1) * n * (n - 1) / 6);
            for (int mv = 0; mv < moves && ranks > 0; ++mv) {
                int x, y, z;
                synth_triple(n, synth_below(&state, ranks), &x, &y, &z);
                int8_t swapped[16];
                int w = 0;
                for (int q = 0; q < x; ++q) swapped[w++] = p[q];
                for (int q = y; q < z; ++q) swapped[w++] = p[q];
                for (int q = x; q < y; ++q) swapped[w++] = p[q];
                for (int q = z; q < n; ++q) swapped[w++] = p[q];
                memcpy(p, swapped, (size_t)n);
            }
        } else {
            for (int m = 0; m < n; ++m) p[m] = (int8_t)m;
            for (int m = n - 1; m > 0; --m) {
                const int j = (int)synth_below(&state, (uint32_t)(m + 1));
                const int8_t t = p[m];
                p[m] = p[j];
                p[j] = t;
            }
        }
        for (int m = n; m < 16; ++m) p[m] = 0;
        n_out[idx] = (uint8_t)n;
    }
    return 0;
}
