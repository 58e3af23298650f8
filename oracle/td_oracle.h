/*
 * td_oracle.h -- CPU oracle for the td16 witness search.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * search (emitter/src/native/backtracking/sorting_search.cu) run with a single
 * work queue, of the witness replay (emitter/src/main/java/br/unb/cic/tdp/base/
 * CertificateValidator.java) and of the certificate byte format
 * (CertificateCodec.java).  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark may load it.  The product path never calls it.
 *
 * Parity pins: the reference's known-answer tests (GPUSortingSearchSmokeTest,
 * CertificateCodecTest, CommonOperationsTest, PermutationGroupsTest,
 * OddLengthOrientedCyclesTest, CommonOperations.d(n)) and fixtures produced
 * by the compiled reference kernel itself (tests/golden/).
 */
#ifndef TD_ORACLE_H
#define TD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDO_MAX_N 17     /* emitter/src/native/core/common.cuh:14-16 */
#define TDO_MAX_DEPTH 9  /* emitter/src/native/core/common.cuh:10-12 */

/* search outcome */
#define TDO_NOT_FOUND 0
#define TDO_FOUND 1
#define TDO_EINVAL (-1)
#define TDO_BUDGET (-2)  /* the expansion budget ran out before a verdict */

typedef struct {
    uint64_t expansions; /* nodes whose children were evaluated */
    uint64_t pops;       /* nodes taken off the work stack */
    uint64_t triples;    /* triple evaluations performed */
} tdo_stats;

int tdo_triple_count(int n);
uint16_t tdo_pack_move(int i, int j, int k);
void tdo_unpack_move(uint16_t m, int *i, int *j, int *k);

/* number of odd-length cycles of omega, fixed points included */
int tdo_count_odd_cycles(const uint8_t *omega, int n);
/* change of that count under omega <- omega . (a b c)^-1; TDO_DELTA_SKIP when
 * a, b, c lie in three different cycles */
#define TDO_DELTA_SKIP (-1000)
int tdo_delta_odd_cycles(const uint8_t *omega, int a, int b, int c);

/* acceptance / pruning predicates (f32 arithmetic as in the reference) */
int tdo_accepts(int n, int init_odd, float min_rate, int full, int odd, int depth);
int tdo_can_reach(int n, int init_odd, float min_rate, int max_depth, int full, int odd, int depth);

/*
 * One search with the reference's single-queue move order.  Inputs are the
 * current beta array and omega one-line (N symbols each).  On TDO_FOUND,
 * out_moves[0..*out_depth) receive the position triples packed 5 bits each
 * (i | j<<5 | k<<10), exactly the reference's PackedMove.
 */
int tdo_search(const uint8_t *beta, const uint8_t *omega, int n, int init_odd,
               float min_rate, int max_depth, int full,
               uint16_t *out_moves, int *out_depth, tdo_stats *stats);

/* Expansion budget of every later search (0, the default, = none): a search
 * that would expand more nodes returns TDO_BUDGET.  For screening candidate
 * test cases only. */
void tdo_set_expansion_budget(uint64_t max_expansions);

/* Batch of independent searches on `threads` host threads (one instance per
 * thread at a time).  Records are laid out with strides of TDO_MAX_N bytes
 * (beta, omega) and TDO_MAX_DEPTH moves.  Returns 0 or TDO_EINVAL. */
int tdo_search_batch(int count, const uint8_t *beta, const uint8_t *omega,
                     const uint8_t *n, const int32_t *init_odd,
                     const float *min_rate, const int32_t *max_depth,
                     const uint8_t *full, int32_t *out_status,
                     int32_t *out_depth, uint16_t *out_moves,
                     uint64_t *out_expansions, int threads);

/* S_n instance (pi over 0..n-1) -> reference pair over N = n+1 symbols */
void tdo_perm_to_pair(const int8_t *pi, int n, uint8_t *beta, uint8_t *omega,
                      int *init_odd);

/* The benchmark's seeded instances (int8 stride 16), generated without the
 * engine library: instance i draws from splitmix64 seeded seed ^ i; n
 * uniform in [n_min, n_max]; with probability hard_pct/100 the reverse
 * permutation composed with hard_min..hard_max uniform block transpositions,
 * else a Fisher-Yates uniform permutation.  Same output as the engine's
 * td_synth_perms. */
int tdo_synth_perms(uint64_t seed, int count, int n_min, int n_max, int hard_pct,
                    int hard_min, int hard_max, int8_t *perms, uint8_t *n_out);

/* position triples -> symbol triples, evolving a copy of beta
 * (GPUSortingSearch.java:229-238) */
void tdo_positions_to_symbols(const uint8_t *beta, int n, const uint16_t *moves,
                              int count, uint8_t *out_abc);

/* witness replay; 0 when accepted, else a negative code with a message */
int tdo_validate(const uint8_t *beta, const uint8_t *omega, int n,
                 const uint8_t *abc, int count, int max_moves, char *err,
                 size_t errlen);

/* certificate byte format */
int tdo_codec_key(const uint8_t *omega, int n, uint8_t *out, int cap);
int tdo_codec_value(const uint8_t *abc, int count, uint8_t *out, int cap);
int tdo_codec_decode_key(const uint8_t *in, int len, int n, uint8_t *omega);
int tdo_codec_decode_value(const uint8_t *in, int len, uint8_t *abc, int cap);

/* permutation algebra used by the replay (one-line arrays over n symbols) */
/* CommonOperations.applyTranspositionOptimized: block swap at the sorted
 * positions of a, b, c in the cycle's symbol array */
void tdo_apply_transposition(const uint8_t *cycle, int n, int a, int b, int c,
                             uint8_t *out);
/* out = p . q, i.e. out[x] = p[q[x]] (PermutationGroups.computeProduct) */
void tdo_compose(const uint8_t *p, const uint8_t *q, int n, uint8_t *out);
/* one-line form of the cycle (cyc[0] cyc[1] ... cyc[len-1]) on n symbols */
void tdo_cycle_oneline(const uint8_t *cyc, int len, int n, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
