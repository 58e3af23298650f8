// td_core.cuh -- definitions shared by the sm_100a kernels and the host side of
// the witness-search engine.  Everything here is plain integer arithmetic that
// compiles for both host and device (__host__ __device__), so the host can
// prepare instances and tests can exercise the same logic without a GPU.
//
// Vocabulary (reference: emitter/src/native/backtracking/sorting_search.cu):
//   N      number of symbols (n + 1 for a permutation of S_n), N <= 17
//   beta   the current N-cycle, written as an array that starts at betaStart
//   omega  the algebraic permutation; rho = omega . beta stays fixed
//   move   a position triple i < j < k into the beta array; it swaps the blocks
//          [i,j) and [j,k) and sets omega <- omega . (a b c)^-1 with
//          (a,b,c) = (beta[i], beta[j], beta[k])
//
// Engine state ("pinned" form).  Relabel the symbols so that rho becomes
// x -> x+1 (mod N) and write beta as the cyclic sequence B that starts at
// symbol 0.  The remaining n = N-1 entries L[m] = B[m+1]-1 form a linear
// permutation of 0..n-1 that fits 4-bit nibbles of one uint64.  The caller's
// array start (betaStart) is tracked as `off`, the position in B of the
// caller's beta[0]; caller position p is pinned position (p + off) mod N.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define TD_HD __host__ __device__ __forceinline__
#else
#define TD_HD inline
#endif

#define TD_MAX_N 17      // symbols (core/common.cuh:14-16)
#define TD_MAX_DEPTH 9   // moves (core/common.cuh:10-12)
#define TD_MAX_TRIPLES 680
#define TD_MAX_STEPS 22  // ceil(680 / 32)
#define TD_MAX_ROUNDS 4  // ceil(C(16,2) / 32): pair slots of the bit-sliced evaluation
#define TD_PT_STRIDE 32  // pair table row stride (bytes)

// ---- C-ABI records (mirrored in include/td16_b200.h) ----------------------

// One search request in pinned form: 16 bytes.
struct td_instance {
    uint64_t perm;      // nibble m = L[m] for m < N-1; nibbles m >= N-1 hold m
    float min_rate;     // the reference's minRate (f32)
    uint8_t n_symbols;  // N
    uint8_t offset;     // pinned position of the caller's beta[0]
    uint8_t max_moves;  // 1..9
    uint8_t packed;     // bits 0-4: initialEvenCycles, bit 7: fullSorting,
                        // bit 6: reference order (set by the engine on requests
                        // to its per-call server only)
};

// One search result: 32 bytes.
struct td_result {
    int32_t status;      // TD_FOUND / TD_NOT_FOUND / error code (<0)
    int32_t depth;       // witness length
    uint16_t moves[TD_MAX_DEPTH];  // caller positions, i | j<<5 | k<<10
    uint16_t reserved;
    uint32_t expansions; // nodes whose children were evaluated (saturating)
};

#define TD_FOUND 1
#define TD_NOT_FOUND 0
#define TD_ERR_ARG (-4)
#define TD_ERR_BUDGET (-2)
#define TD_ERR_TIMEOUT (-5)

#define TD_FLAG_ORDERED 1u  // reproduce the reference's single-queue move order

// ---- small helpers ---------------------------------------------------------

TD_HD int td_triple_count(int n) { return n < 3 ? 0 : n * (n - 1) * (n - 2) / 6; }

TD_HD uint16_t td_pack_move(int i, int j, int k) {
    return (uint16_t)((i & 31) | ((j & 31) << 5) | ((k & 31) << 10));
}

TD_HD uint32_t td_nib(uint64_t L, int m) { return (uint32_t)(L >> (4 * m)) & 15u; }

TD_HD uint64_t td_low_nibbles(int count) {  // mask of the lowest `count` nibbles
    return count >= 16 ? ~0ull : ((1ull << (4 * count)) - 1ull);
}

TD_HD int td_inst_init(const td_instance &x) { return x.packed & 31; }
TD_HD int td_inst_full(const td_instance &x) { return (x.packed >> 7) & 1; }
#define TD_PACKED_ORDERED 0x40

// Apply the caller-position move (i,j,k) to the pinned state (L, off).
// The three cut points are pinned positions P,Q,R in cyclic order; rotated so
// that the smallest comes first they give (p1,p2,p3).  A block swap of the
// cyclic sequence is the same cycle whichever arc the array starts in, so in
// pinned form it is the linear transposition (x,y,z) = (p1-1,p2-1,p3-1), or
// (p2-1,p3-1,n) when p1 == 0.  The caller's array start moves to beta[j] when
// i == 0 (sorting_search.cu:450-452, 623-625).
TD_HD void td_apply_move(uint64_t L, int off, int N, int i, int j, int k,
                         uint64_t *outL, int *outOff) {
    const int n = N - 1;
    int P = i + off, Q = j + off, R = k + off;
    P -= (P >= N) ? N : 0;
    Q -= (Q >= N) ? N : 0;
    R -= (R >= N) ? N : 0;
    int p1, p2, p3;
    if (P < Q && Q < R) { p1 = P; p2 = Q; p3 = R; }
    else if (Q < R && R < P) { p1 = Q; p2 = R; p3 = P; }
    else { p1 = R; p2 = P; p3 = Q; }
    int x, y, z;
    if (p1 == 0) { x = p2 - 1; y = p3 - 1; z = n; }
    else { x = p1 - 1; y = p2 - 1; z = p3 - 1; }
    const int a = y - x, b = z - y;  // lengths of the swapped blocks
    const uint64_t keep = (L & td_low_nibbles(x)) | (L & ~td_low_nibbles(z));
    const uint64_t blockA = (L >> (4 * x)) & td_low_nibbles(a);
    const uint64_t blockB = (L >> (4 * y)) & td_low_nibbles(b);
    *outL = keep | (blockB << (4 * x)) | (blockA << (4 * (x + b)));
    // new start of the caller's array, followed through the swap
    int S = (i == 0) ? Q : off;
    if (S != 0) {
        int e = S - 1;
        if (e >= x && e < y) e += b;
        else if (e >= y && e < z) e -= a;
        S = e + 1;
    }
    *outOff = S;
}

// ---- triple classification -------------------------------------------------
//
// For a node, every ordered pair (p,q) of caller positions gets a 4-bit entry
//   bit0 S: the symbols at p and q lie in the same omega cycle
//   bit1 P: parity of the walk p -> q along omega (only when S)
//   bit2 G: dist(p) > dist(q) when S, where dist is the number of omega steps
//           to the cycle's smallest position; when !S: p's cycle is a fixed point
//   bit3 O: p's cycle has odd length
// A triple (i,j,k) reads entries (i,j), (j,k), (k,i) and forms a 12-bit index
// into a table that restates delta_even_cycles (sorting_search.cu:240-332) and
// the move filter (:375-380, :607-610).  Table values: 0 = filtered out,
// 1 = odd-cycle change 0, 2 = change +2.  The value is the byte of the
// per-node outcome word that holds that class's flags (byte 0 is zero).

#define TD_CLASS_SKIP 0
#define TD_CLASS_ZERO 1
#define TD_CLASS_PLUS2 2

TD_HD int td_class_of_index(int idx) {
    const int S1 = idx & 1, P1 = (idx >> 1) & 1, G1 = (idx >> 2) & 1, O1 = (idx >> 3) & 1;  // (a,b)
    const int S2 = (idx >> 4) & 1, P2 = (idx >> 5) & 1, G2 = (idx >> 6) & 1, O2 = (idx >> 7) & 1;  // (b,c)
    const int S3 = (idx >> 8) & 1, P3 = (idx >> 9) & 1, G3 = (idx >> 10) & 1, O3 = (idx >> 11) & 1;  // (c,a)
    int delta;
    if (S1 && S2 && S3) {
        // one cycle: split in three when the omega order is a -> b -> c
        if (O1 != O2 || O2 != O3) return TD_CLASS_SKIP;  // inconsistent
        if (G1 + G2 + G3 != 2) return TD_CLASS_ZERO;
        delta = P1 + P2 + P3 - O1;
    } else if (S1 + S2 + S3 == 1) {
        int o1, o2, s, lone_fixed;
        if (S1) { o1 = O1; o2 = O3; s = P1; lone_fixed = G3; }       // {a,b}, c apart
        else if (S2) { o1 = O2; o2 = O1; s = P2; lone_fixed = G1; }  // {b,c}, a apart
        else { o1 = O3; o2 = O2; s = P3; lone_fixed = G2; }          // {c,a}, b apart
        if (lone_fixed) return TD_CLASS_SKIP;
        delta = s + (o1 ^ s ^ o2) - o1 - o2;
    } else {
        return TD_CLASS_SKIP;  // three cycles (or a fixed point alone)
    }
    if (delta == 2) return TD_CLASS_PLUS2;
    if (delta == 0) return TD_CLASS_ZERO;
    return TD_CLASS_SKIP;
}

// ---- bit-sliced classification (free move order) ---------------------------
//
// The same classes for every third position k of a pair (i, j) at once, one
// bit per k, from row masks of the node indexed by caller position:
//   S[p] bit q: p and q lie on one omega cycle
//   G[p] bit q: on one cycle and dist(p) > dist(q)
//   P[p] bit q: on one cycle and the walk p -> q along omega has odd length
//   O bit q:    q's cycle has odd length
//   F bit q:    q is a fixed point
// The entries of the pair table above follow from these: (i,j) = bits j of
// rows i; (j,k) = rows j; and for (k,i), where the rows of i are read at k,
// the walk k -> i is the rest of the cycle after the walk i -> k (its parity
// is P[i] bit k xor O bit i) and dist(k) > dist(i) is the complement of G[i]
// bit k.  With these entries the cases of td_class_of_index become:
//   all three on one cycle: +2 when exactly two of dist(i)>dist(j),
//     dist(j)>dist(k), dist(k)>dist(i) hold and at least two of the three walk
//     parities are odd (their sum has the cycle's parity, so the change
//     P1+P2+P3-O is then 2, else 0); otherwise 0;
//   one pair on a cycle, the third symbol apart (walk parity s, cycle
//     parities o1 of the pair and o2 of the lone symbol): filtered when the
//     lone symbol is a fixed point; +2 when s & !o1 & !o2; filtered when
//     !s & o1 & o2; 0 otherwise;
//   three cycles: filtered.
// Bits of k outside (j, N) are meaningless; the caller masks them.
// The same with the per-lane flags already spread to full masks: oi/oj/fi/fj
// are all-ones when i's/j's cycle is odd / i/j is fixed, and sh = 31 - j.
TD_HD void td_row_classes_x(uint32_t Si, uint32_t Gi, uint32_t Pi, uint32_t Sj, uint32_t Gj, uint32_t Pj,
                            uint32_t O, uint32_t F, uint32_t oi, uint32_t oj, uint32_t fi, uint32_t fj, int sh,
                            uint32_t *plus2, uint32_t *zero) {
    const uint32_t s1 = Si == Sj ? 0xffffffffu : 0u;             // i and j on one cycle (equal rows)
    const uint32_t p1 = (uint32_t)((int32_t)(Pi << sh) >> 31);   // walk i -> j odd
    const uint32_t g1 = (uint32_t)((int32_t)(Gi << sh) >> 31);   // dist(i) > dist(j)
    const uint32_t P3 = Pi ^ oi;                 // walk k -> i odd (k on i's cycle)
    // all three on one cycle (k on the common cycle of i and j)
    const uint32_t G3 = ~Gi;                     // dist(k) > dist(i)
    const uint32_t two = (g1 & Gj & ~G3) | (g1 & ~Gj & G3) | (~g1 & Gj & G3);
    const uint32_t maj = (p1 & Pj) | (p1 & P3) | (Pj & P3);
    const uint32_t all = s1 & Si;
    const uint32_t split = two & maj;
    // exactly one pair on a cycle: with s1 the pair is (i,j) and k lies apart;
    // otherwise the pair is (j,k) where k is on j's cycle, (k,i) where on i's
    const uint32_t sp = (s1 & p1) | (~s1 & ((Sj & Pj) | (~Sj & P3)));
    const uint32_t o1 = (s1 & oi) | (~s1 & ((Sj & oj) | (~Sj & oi)));
    const uint32_t o2 = (s1 & O) | (~s1 & ((Sj & oi) | (~Sj & oj)));
    const uint32_t lf = (s1 & F) | (~s1 & ((Sj & fi) | (~Sj & fj)));
    const uint32_t dom = (s1 & ~Si) | (~s1 & (Si | Sj));
    const uint32_t p_one = dom & sp & ~o1 & ~o2 & ~lf;
    const uint32_t z_one = dom & ~p_one & ~(lf | (~sp & o1 & o2));
    *plus2 = (all & split) | p_one;
    *zero = (all & ~split) | z_one;
}

TD_HD void td_row_classes(uint32_t Si, uint32_t Gi, uint32_t Pi, uint32_t Sj, uint32_t Gj, uint32_t Pj,
                          uint32_t O, uint32_t F, int i, int j, uint32_t *plus2, uint32_t *zero) {
    td_row_classes_x(Si, Gi, Pi, Sj, Gj, Pj, O, F, 0u - ((O >> i) & 1u), 0u - ((O >> j) & 1u),
                     0u - ((F >> i) & 1u), 0u - ((F >> j) & 1u), 31 - j, plus2, zero);
}

// Pair slot q of a node with N positions: the pairs (i, j), i < j <= N-2 (the
// first two positions of a triple), numbered so that higher slots hold
// lexicographically smaller pairs.  Returns i | j << 5 | j << 10 | (31-j) << 15
// (the third field is the shift of the k mask, k > j; the fourth brings bit j
// to the sign bit).  A slot past the last pair, or a negative one, gets
// i = 0, j = N-1: no position lies after N-1, so its k mask is empty.
TD_HD uint32_t td_pair_code(int N, int q) {
    const int NP = N < 3 ? 0 : (N - 1) * (N - 2) / 2;
    if (q < 0 || q >= NP) {
        const uint32_t jj = N >= 2 ? (uint32_t)(N - 1) : 0u;
        return (jj << 5) | (jj << 10) | ((31u - jj) << 15);
    }
    int rank = NP - 1 - q;  // lexicographic rank of the pair
    int i = 0;
    while (rank >= N - 2 - i) {  // pairs with first element i: j = i+1 .. N-2
        rank -= N - 2 - i;
        ++i;
    }
    const int j = i + 1 + rank;
    return (uint32_t)i | ((uint32_t)j << 5) | ((uint32_t)j << 10) | ((uint32_t)(31 - j) << 15);
}

// Key of a pinned state in the tables of explored states: L with its nibbles
// from N-1 on cleared.  The first 14 nibbles and whether nibble 14 exceeds
// nibble 15 determine it (the two are the values left over by a permutation
// of 0..15; for N <= 16 nibble 15 is cleared), so it fits in 57 bits.
TD_HD uint64_t td_tt_key(uint64_t L) {
    const uint64_t order = ((L >> 56) & 15u) > ((L >> 60) & 15u) ? 1ull : 0ull;
    return (L & 0x00ffffffffffffffull) | (order << 56);
}

// ---- restarts of the free order ----------------------------------------------
//
// The free-order search has a heavy tail: on near-reverse S_16 the median
// search takes ~30 expansions and a few take tens of thousands, because an
// early wrong turn leads into a large subtree without a witness.  A search
// therefore restarts with another child order after a budget of expansions;
// the budgets follow the Luby sequence (base x 1, 1, 2, 1, 1, 2, 4, ...), and
// the attempt after TD_RESTARTS ends is unbounded, so a search without a
// witness still completes.  Restarting never changes a verdict: every attempt
// explores a subtree order of the same tree, and the last one all of it.

// With 32 budgeted attempts the unbounded one (attempt 32) runs in the plain
// order: 7 x 32 and 11 x level x 32 are 0 mod 32 and bits 5-6 of 32 are 0.
// The plain order is the best single order on the long searches that reach
// it; in the host emulation 32 attempts cut the mean near-reverse S_16 search
// by 10-15% against 24, whose last order is a rotated one.
#define TD_RESTARTS 32  // attempts with a budget; the next one runs to the end

// The i-th term (i >= 1) of the Luby sequence 1, 1, 2, 1, 1, 2, 4, 1, 1, ...
TD_HD uint32_t td_luby(uint32_t i) {
    for (;;) {
        uint32_t k = 1;
        while (((1u << k) - 1u) < i) ++k;
        if (i == (1u << k) - 1u) return 1u << (k - 1);
        i -= (1u << (k - 1)) - 1u;
    }
}

// Expansion budget of attempt a (0-based) for a base budget; ~0u = unbounded.
TD_HD uint32_t td_attempt_budget(uint32_t base, int a) {
    if (base == 0 || a >= TD_RESTARTS) return ~0u;
    const uint64_t b = (uint64_t)base * td_luby((uint32_t)a + 1u);
    return b >= 0xffffffffull ? ~0u : (uint32_t)b;
}

// Child order of attempt a: bits 0-4 rotate the lane priority, bit 5 takes
// the lowest pair round of a lane first, bit 6 the largest k first.  Attempt 0
// is the plain free order.
TD_HD uint32_t td_order_variant(int a) {
    if (a == 0) return 0u;
    return ((uint32_t)(7 * a) & 31u) | (((uint32_t)a & 1u) << 5) | ((((uint32_t)a >> 1) & 1u) << 6);
}

// The order at DFS level `level` of attempt a: the rotation also moves by
// 11 x level x a, so that the levels of one attempt do not all favour the
// same lanes (in the host emulation this halved the mean expansions of
// near-reverse S_16 searches against one rotation per attempt).
TD_HD uint32_t td_level_order(uint32_t ord, int a, int level) {
    if (a == 0) return 0u;
    return (ord & ~31u) | ((ord + 11u * (uint32_t)level * (uint32_t)a) & 31u);
}

// Per-position cycle descriptor: leader (smallest pinned position of the
// cycle), dist (omega steps to the leader), len (cycle length).
TD_HD uint32_t td_pair_entry(int leader_p, int dist_p, int len_p, int leader_q,
                             int dist_q) {
    const int S = leader_p == leader_q;
    int P = 0, G;
    if (S) {
        int w = dist_p - dist_q;
        if (w < 0) w += len_p;
        P = w & 1;
        G = dist_p > dist_q;
    } else {
        G = len_p == 1;
    }
    return (uint32_t)(S | (P << 1) | (G << 2) | ((len_p & 1) << 3));
}

// ---- acceptance and pruning masks ------------------------------------------
//
// satisfies_rate and can_still_reach (sorting_search.cu:336-373) depend only on
// (oddCycles, depth); for each depth they become a bitmask over oddCycles.
// The f32 operations are the reference's, in the same order.

TD_HD int td_accepts(int N, int init, float min_rate, int full, int odd, int depth) {
    if (depth <= 0) return 0;
    if (full && odd != N) return 0;
    const int gained = odd - init;
    const float ratio = (float)gained / (float)depth;
    return gained > 0 && ratio >= min_rate;
}

// Odd-length cycles of omega for the pinned state (L, off) over N symbols,
// and a bit per caller position whose symbol omega fixes.  Beta reads B = (0,
// L[0]+1, ..., L[N-2]+1) from pinned position 0, caller position c sits at
// pinned position (c + off) mod N, and omega(B[p]) = B[p-1] + 1 (mod N).
TD_HD int td_pinned_cycles(uint64_t L, int off, int N, uint32_t *fixed_at_caller) {
    uint8_t B[TD_MAX_N], om[TD_MAX_N];
    for (int p = 0; p < N; ++p) B[p] = p ? (uint8_t)(td_nib(L, p - 1) + 1) : 0;
    uint32_t fixed = 0;
    for (int p = 0; p < N; ++p) {
        const int prev = B[p == 0 ? N - 1 : p - 1] + 1;
        om[B[p]] = (uint8_t)(prev == N ? 0 : prev);
        if (om[B[p]] == B[p]) {
            int c = p - off;
            c += c < 0 ? N : 0;
            fixed |= 1u << c;
        }
    }
    uint32_t seen = 0;
    int odd = 0;
    for (int x = 0; x < N; ++x) {
        if ((seen >> x) & 1u) continue;
        int len = 0;
        for (int y = x; !((seen >> y) & 1u); y = om[y]) {
            seen |= 1u << y;
            ++len;
        }
        odd += len & 1;
    }
    *fixed_at_caller = fixed;
    return odd;
}

TD_HD int td_can_reach(int N, int init, float min_rate, int max_depth, int full,
                       int odd, int depth) {
    const int missing = N - odd;
    if (full) return depth + (missing + 1) / 2 <= max_depth;
    const int gained = odd - init;
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

// Replay of a witness: every move is an in-range position triple i<j<k,
// there are at most max_moves of them, and the node they reach passes the
// instance's acceptance test (satisfies_rate, sorting_search.cu:336-346; with
// full sorting, omega = id).  With full sorting this is CertificateValidator's
// replay (CertificateValidator.java:14-50) in pinned form plus the rate test;
// with partial sorting it is the same test on the odd-cycle count reached.
// (The search never returns a path whose earlier nodes pass the test, so a
// witness cut short fails it.)
TD_HD int td_witness_ok(const td_instance &x, const td_result &r) {
    const int N = x.n_symbols;
    if (!(r.status == TD_FOUND && r.depth >= 1 && r.depth <= x.max_moves && N >= 3 && N <= TD_MAX_N)) return 0;
    uint64_t L = x.perm;
    int off = x.offset;
    for (int d = 0; d < r.depth; ++d) {
        const int m = r.moves[d];
        const int i = m & 31, j = (m >> 5) & 31, k = (m >> 10) & 31;
        if (!(i < j && j < k && k < N)) return 0;
        uint64_t nL;
        int noff;
        td_apply_move(L, off, N, i, j, k, &nL, &noff);
        L = nL;
        off = noff;
    }
    int odd;
    if (td_inst_full(x)) {
        // omega = id  <=>  beta = rho  <=>  L = 0, 1, ..., N-2
        uint64_t ident = 0;
        for (int m = 0; m < 16; ++m) ident |= (uint64_t)m << (4 * m);
        const uint64_t mask = N - 1 >= 16 ? ~0ull : ((1ull << (4 * (N - 1))) - 1ull);
        odd = ((L ^ ident) & mask) == 0 ? N : 0;
    } else {
        uint32_t fixed;
        odd = td_pinned_cycles(L, off, N, &fixed);
    }
    return td_accepts(N, td_inst_init(x), x.min_rate, td_inst_full(x), odd, r.depth);
}

// ---- the inverse instance (free order, full sorting) ------------------------
//
// A permutation and its inverse are the same number of transpositions from
// the identity, and a witness for one gives one for the other.  Searches of
// the two often differ by orders of magnitude in expansions, so the batch
// engine races them (td_steal_kernel).  In pinned form the inverse of the
// state (L, off) is L^-1 (nibble L[m] holds m) with the caller's array
// starting at pinned position 0; its odd-cycle count equals that of (L, off),
// so the acceptance and pruning masks of full sorting carry over unchanged.

TD_HD uint64_t td_inverse_pinned(uint64_t L, int N) {
    uint64_t R = 0;
    for (int m = 0; m < 16; ++m) R |= (uint64_t)m << (4 * (m < N - 1 ? (int)td_nib(L, m) : m));
    return R;
}

// The caller's array of the pinned state (L, off): the label at each caller
// position (pinned position c + off mod N holds B[p] = p ? L[p-1]+1 : 0).
TD_HD void td_caller_array(uint64_t L, int off, int N, uint8_t *A) {
    for (int c = 0; c < N; ++c) {
        int p = c + off;
        p -= p >= N ? N : 0;
        A[c] = p ? (uint8_t)(td_nib(L, p - 1) + 1u) : (uint8_t)0;
    }
}

// The caller-position move (i, j, k) on an array: blocks [i, j) and [j, k)
// change places.
TD_HD void td_swap_blocks(uint8_t *A, int i, int j, int k) {
    uint8_t t[TD_MAX_N];
    for (int m = i; m < k; ++m) t[m] = A[m];
    for (int m = i; m < k; ++m) A[m] = m < i + (k - j) ? t[m + (j - i)] : t[m - (k - j)];
}

// A witness of the inverse instance (td_inverse_pinned(L, N), offset 0):
// inv[0..k-1] in its caller positions -> the witness of (L, off) in the
// caller's positions, out[0..k-1].  Returns 0 if the moves do not fit.
//
// With A the caller's array and B the inverse's, B = R_off . A^-1 (R_s: the
// rotation c -> c + s).  If B . s_1 ... s_k is sorted (a rotation), then
// A = (s_1 ... s_k) . R_u for some u, and the answer A . t_1 ... t_k passes,
// up to a rotation of positions, through the arrays S_m = s_1 ... s_m (the
// identity array after the moves s_1..s_m) for m = k, k-1, ..., 0.  The step
// from S_m to S_{m-1} is the block swap s_m^-1 = (i, i + k - j, k).  A block
// swap of a cyclic array is fixed by its three cut points, so t is the block
// swap of the caller's current array at the cuts between the same two
// neighbouring labels.
TD_HD int td_witness_from_inverse(uint64_t L, int off, int N, const uint16_t *inv, int k, uint16_t *out) {
    uint8_t X[TD_MAX_N], S[TD_MAX_N];
    td_caller_array(L, off, N, X);
    for (int m = k; m >= 1; --m) {
        for (int p = 0; p < N; ++p) S[p] = (uint8_t)p;
        for (int q = 0; q < m; ++q) td_swap_blocks(S, inv[q] & 31, (inv[q] >> 5) & 31, (inv[q] >> 10) & 31);
        const int i = inv[m - 1] & 31, j = (inv[m - 1] >> 5) & 31, kk = (inv[m - 1] >> 10) & 31;
        if (!(i < j && j < kk && kk < N)) return 0;
        const int g[3] = {i, i + kk - j, kk};
        int c3[3];
        for (int t = 0; t < 3; ++t) {
            const uint8_t u = S[g[t] == 0 ? N - 1 : g[t] - 1], v = S[g[t]];
            c3[t] = -1;
            for (int c = 0; c < N; ++c)
                if (X[c == 0 ? N - 1 : c - 1] == u && X[c] == v) { c3[t] = c; break; }
            if (c3[t] < 0) return 0;
        }
        // ascending order
        if (c3[0] > c3[1]) { const int w = c3[0]; c3[0] = c3[1]; c3[1] = w; }
        if (c3[1] > c3[2]) { const int w = c3[1]; c3[1] = c3[2]; c3[2] = w; }
        if (c3[0] > c3[1]) { const int w = c3[0]; c3[0] = c3[1]; c3[1] = w; }
        if (!(c3[0] < c3[1] && c3[1] < c3[2])) return 0;
        out[k - m] = td_pack_move(c3[0], c3[1], c3[2]);
        td_swap_blocks(X, c3[0], c3[1], c3[2]);
    }
    return 1;
}

// ---- instance preparation (host side) --------------------------------------

// Odd-length cycles of omega, fixed points included (sorting_search.cu:211-226).
TD_HD int td_count_odd_cycles(const uint8_t *omega, int N) {
    uint32_t seen = 0;
    int odd = 0;
    for (int s = 0; s < N; ++s) {
        if (seen & (1u << s)) continue;
        int len = 0, x = s;
        do { seen |= 1u << x; ++len; x = omega[x]; } while (x != s);
        odd += len & 1;
    }
    return odd;
}

// Caller pair (beta array, omega one-line) -> pinned instance.  Returns 0, or
// TD_ERR_ARG when the sizes are out of range, an array is not a permutation of
// 0..N-1, or rho = omega . beta is not an N-cycle (the reference's callers only
// pass pairs whose product is an N-cycle, CyclicTargetPair.java:39-45).
TD_HD int td_prepare_pair(const uint8_t *beta, const uint8_t *omega, int N, int init,
                          float min_rate, int max_moves, int full, td_instance *out) {
    if (N < 0 || N > TD_MAX_N) return TD_ERR_ARG;
    if (max_moves <= 0 || max_moves > TD_MAX_DEPTH) return TD_ERR_ARG;
    if (init < 0 || init > 31) return TD_ERR_ARG;
    uint64_t L = 0;
    for (int m = 0; m < 16; ++m) L |= (uint64_t)m << (4 * m);
    if (N >= 1) {
        uint32_t seen_b = 0, seen_o = 0;
        for (int x = 0; x < N; ++x) {
            if (beta[x] >= N || omega[x] >= N) return TD_ERR_ARG;
            seen_b |= 1u << beta[x];
            seen_o |= 1u << omega[x];
        }
        const uint32_t all = (N == 32) ? ~0u : ((1u << N) - 1u);
        if (seen_b != all || seen_o != all) return TD_ERR_ARG;
        uint8_t next_of[TD_MAX_N], rho[TD_MAX_N], sigma[TD_MAX_N];
        for (int x = 0; x < N; ++x) next_of[beta[x]] = beta[(x + 1) % N];
        for (int x = 0; x < N; ++x) rho[x] = omega[next_of[x]];
        int r = beta[0];
        for (int m = 0; m < N; ++m) { sigma[r] = (uint8_t)m; r = rho[r]; }
        if (r != beta[0]) return TD_ERR_ARG;
        for (int x = 0; x < N; ++x) {  // rho must visit every symbol once
            int steps = 0, y = x;
            do { y = rho[y]; ++steps; } while (y != x && steps <= N);
            if (steps != N) return TD_ERR_ARG;
        }
        L = 0;
        for (int m = 0; m < 16; ++m) {
            const uint64_t v = (m < N - 1) ? (uint64_t)(sigma[beta[m + 1]] - 1) : (uint64_t)m;
            L |= v << (4 * m);
        }
    }
    out->perm = L;
    out->min_rate = min_rate;
    out->n_symbols = (uint8_t)N;
    out->offset = 0;
    out->max_moves = (uint8_t)max_moves;
    out->packed = (uint8_t)((init & 31) | (full ? 0x80 : 0));
    return 0;
}

// S_n permutation pi (values 0..n-1) -> the reference pair over N = n+1
// symbols: beta = (0 1 ... n), rho = (0, pi0+1, ..., pi_{n-1}+1),
// omega = rho . beta^-1, initialEvenCycles = odd cycles of omega.
TD_HD void td_perm_to_pair(const int8_t *pi, int n, uint8_t *beta, uint8_t *omega, int *init) {
    const int N = n + 1;
    uint8_t seq[TD_MAX_N], rho[TD_MAX_N];
    seq[0] = 0;
    for (int m = 0; m < n; ++m) seq[m + 1] = (uint8_t)(pi[m] + 1);
    for (int m = 0; m < N; ++m) rho[seq[m]] = seq[(m + 1) % N];
    for (int x = 0; x < N; ++x) {
        beta[x] = (uint8_t)x;
        omega[x] = rho[(x + N - 1) % N];
    }
    *init = td_count_odd_cycles(omega, N);
}
