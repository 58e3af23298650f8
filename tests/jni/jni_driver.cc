// jni_driver.cc -- runs the JNI shim (td16_b200/csrc/td_jni.cc) without a JVM.
//
// TEST INFRASTRUCTURE ONLY.  Supplies a fake JNIEnv (tests/jni/jni.h) whose
// arrays, classes and pending exception live in this process, calls the
// shim's natives the way GPUSortingSearch.java does, and checks the results:
//   fake      built with -DTD_FAKE_ENGINE: the td_* entry points below stand
//             in for the engine and return each status in turn, so that the
//             mapping of every status to a RuntimeException and the int[][]
//             shapes are checked without a GPU
//   real-cpu  linked to libtd16b200.so on a machine without a GPU: argument
//             checks and initialisation failures
//   real-gpu  linked to libtd16b200.so with a B200: real searches, every
//             witness replayed, batch, per-call and pair-consumer natives
//             agreeing
// Prints one line per failed check and "jni ok <checks>" at the end; exits 1
// on any failure.
#include <jni.h>

#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "td16_b200.h"

extern "C" {
JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(JNIEnv *, jclass, jint, jintArray, jlong);
JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(
    JNIEnv *, jclass, jbyteArray, jbyteArray, jint, jfloat, jint, jboolean, jint);
JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeqBatch(
    JNIEnv *, jclass, jobjectArray, jobjectArray, jintArray, jfloatArray, jintArray, jbooleanArray, jint);
JNIEXPORT jlong JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_openPairConsumer(JNIEnv *, jclass, jint, jint, jint,
                                                                                   jdouble, jint, jstring);
JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_acceptPair(JNIEnv *, jclass, jlong, jlong, jbyteArray,
                                                                            jbyteArray, jint, jfloat, jint, jboolean);
JNIEXPORT jlongArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(JNIEnv *, jclass, jlong);
}

namespace {

// ---- the fake JVM side --------------------------------------------------------

struct Obj {
    enum Kind { CLASS, BYTES, INTS, FLOATS, BOOLS, OBJECTS, STRING, LONGS } kind;
    std::string name;  // class name, the element class of an object array, or a string's text
    std::vector<jbyte> b;
    std::vector<jint> i;
    std::vector<jfloat> f;
    std::vector<jboolean> z;
    std::vector<jobject> o;
    std::vector<jlong> l;
};

std::vector<Obj *> g_heap;
bool g_pending = false;
std::string g_exc_class, g_exc_msg;
int g_local_refs = 0;

template <class H>
H make(Obj *o) {
    g_heap.push_back(o);
    ++g_local_refs;
    return reinterpret_cast<H>(o);
}
Obj *get(const void *h) { return reinterpret_cast<Obj *>(const_cast<void *>(h)); }

void raise(const char *cls, const char *msg) {
    g_pending = true;
    g_exc_class = cls;
    g_exc_msg = msg;
}

template <class T>
bool in_range(const std::vector<T> &v, jsize start, jsize len) {
    if (start < 0 || len < 0 || (size_t)start + (size_t)len > v.size()) {
        raise("java/lang/ArrayIndexOutOfBoundsException", "region out of bounds");
        return false;
    }
    return true;
}

jboolean f_exception_check(JNIEnv *) { return g_pending; }
void f_exception_clear(JNIEnv *) { g_pending = false; }
jclass f_find_class(JNIEnv *, const char *name) { return make<jclass>(new Obj{Obj::CLASS, name}); }
jint f_throw_new(JNIEnv *, jclass cls, const char *msg) {
    raise(get(cls)->name.c_str(), msg);
    return 0;
}
void f_delete_local_ref(JNIEnv *, jobject) { --g_local_refs; }
jsize f_array_length(JNIEnv *, jarray a) {
    Obj *o = get(a);
    switch (o->kind) {
        case Obj::BYTES: return (jsize)o->b.size();
        case Obj::INTS: return (jsize)o->i.size();
        case Obj::FLOATS: return (jsize)o->f.size();
        case Obj::BOOLS: return (jsize)o->z.size();
        case Obj::OBJECTS: return (jsize)o->o.size();
        case Obj::LONGS: return (jsize)o->l.size();
        default: return 0;
    }
}
void f_get_bytes(JNIEnv *, jbyteArray a, jsize s, jsize l, jbyte *out) {
    if (in_range(get(a)->b, s, l)) std::memcpy(out, get(a)->b.data() + s, (size_t)l);
}
void f_get_ints(JNIEnv *, jintArray a, jsize s, jsize l, jint *out) {
    if (in_range(get(a)->i, s, l)) std::memcpy(out, get(a)->i.data() + s, sizeof(jint) * l);
}
void f_get_floats(JNIEnv *, jfloatArray a, jsize s, jsize l, jfloat *out) {
    if (in_range(get(a)->f, s, l)) std::memcpy(out, get(a)->f.data() + s, sizeof(jfloat) * l);
}
void f_get_bools(JNIEnv *, jbooleanArray a, jsize s, jsize l, jboolean *out) {
    if (in_range(get(a)->z, s, l)) std::memcpy(out, get(a)->z.data() + s, (size_t)l);
}
jobjectArray f_new_object_array(JNIEnv *, jsize n, jclass cls, jobject init) {
    Obj *o = new Obj{Obj::OBJECTS, get(cls)->name};
    o->o.assign(n, init);
    return make<jobjectArray>(o);
}
jintArray f_new_int_array(JNIEnv *, jsize n) {
    Obj *o = new Obj{Obj::INTS, "[I"};
    o->i.assign(n, 0);
    return make<jintArray>(o);
}
void f_set_ints(JNIEnv *, jintArray a, jsize s, jsize l, const jint *in) {
    if (in_range(get(a)->i, s, l)) std::memcpy(get(a)->i.data() + s, in, sizeof(jint) * l);
}
jobject f_get_element(JNIEnv *, jobjectArray a, jsize i) {
    if (!in_range(get(a)->o, i, 1)) return nullptr;
    ++g_local_refs;
    return get(a)->o[i];
}
void f_set_element(JNIEnv *, jobjectArray a, jsize i, jobject v) {
    if (in_range(get(a)->o, i, 1)) get(a)->o[i] = v;
}
int g_strings_held = 0;
const char *f_get_string_utf(JNIEnv *, jstring str, jboolean *copy) {
    if (copy) *copy = 0;
    ++g_strings_held;
    return get(str)->name.c_str();
}
void f_release_string_utf(JNIEnv *, jstring, const char *) { --g_strings_held; }
jlongArray f_new_long_array(JNIEnv *, jsize n) {
    Obj *o = new Obj{Obj::LONGS, "[J"};
    o->l.assign(n, 0);
    return make<jlongArray>(o);
}
void f_set_longs(JNIEnv *, jlongArray a, jsize s, jsize l, const jlong *in) {
    if (in_range(get(a)->l, s, l)) std::memcpy(get(a)->l.data() + s, in, sizeof(jlong) * l);
}

const TestJniFunctions kFunctions = {f_exception_check, f_exception_clear, f_find_class,   f_throw_new,
                                     f_delete_local_ref, f_array_length,  f_get_bytes,    f_get_ints,
                                     f_get_floats,      f_get_bools,      f_new_object_array, f_new_int_array,
                                     f_set_ints,        f_get_element,    f_set_element,
                                     f_get_string_utf,  f_release_string_utf, f_new_long_array, f_set_longs};
JNIEnv g_env{&kFunctions};

jbyteArray bytes(std::vector<int> v) {
    Obj *o = new Obj{Obj::BYTES, "[B"};
    for (int x : v) o->b.push_back((jbyte)x);
    return make<jbyteArray>(o);
}
jintArray ints(std::vector<jint> v) {
    Obj *o = new Obj{Obj::INTS, "[I"};
    o->i = v;
    return make<jintArray>(o);
}
jfloatArray floats(std::vector<jfloat> v) {
    Obj *o = new Obj{Obj::FLOATS, "[F"};
    o->f = v;
    return make<jfloatArray>(o);
}
jbooleanArray bools(std::vector<jboolean> v) {
    Obj *o = new Obj{Obj::BOOLS, "[Z"};
    o->z = v;
    return make<jbooleanArray>(o);
}
jstring jstr(const std::string &text) { return make<jstring>(new Obj{Obj::STRING, text}); }
std::vector<jlong> longs_of(jlongArray a) { return get(a)->l; }
jobjectArray byte_rows(const std::vector<std::vector<int>> &rows) {
    Obj *o = new Obj{Obj::OBJECTS, "[B"};
    for (auto &r : rows) o->o.push_back(reinterpret_cast<jobject>(bytes(r)));
    return make<jobjectArray>(o);
}

// int[][] -> rows of three
std::vector<std::vector<int>> moves_of(jobjectArray a) {
    std::vector<std::vector<int>> out;
    for (jobject row : get(a)->o) out.push_back(std::vector<int>(get(row)->i.begin(), get(row)->i.end()));
    return out;
}

int g_checks = 0, g_failures = 0;
void check(bool ok, const std::string &what) {
    ++g_checks;
    if (!ok) {
        ++g_failures;
        std::printf("FAIL %s\n", what.c_str());
    }
}
bool threw(const char *msg) {
    const bool ok = g_pending && g_exc_class == "java/lang/RuntimeException" && g_exc_msg == msg;
    if (!ok) std::printf("  (pending %d class '%s' message '%s')\n", (int)g_pending, g_exc_class.c_str(),
                         g_exc_msg.c_str());
    g_pending = false;
    return ok;
}
[[maybe_unused]] bool threw_any() {
    const bool ok = g_pending && g_exc_class == "java/lang/RuntimeException" && !g_exc_msg.empty();
    g_pending = false;
    return ok;
}

jobjectArray search(std::vector<int> beta, std::vector<int> omega, int init, float rate, int maxd, bool full,
                    int slot) {
    return Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(&g_env, nullptr, bytes(beta),
                                                                         bytes(omega), init, rate, maxd, full, slot);
}

// the reference pair of a permutation pi of 0..n-1 (beta = 0..n, rho the
// n+1-cycle (0, pi0+1, ..., pi_{n-1}+1), omega(x) = rho((x-1) mod N))
[[maybe_unused]] void pair_of(const std::vector<int> &pi, std::vector<int> &beta, std::vector<int> &omega, int &init) {
    const int N = (int)pi.size() + 1;
    std::vector<int> seq(N), rho(N);
    seq[0] = 0;
    for (int m = 0; m + 1 < N; ++m) seq[m + 1] = pi[m] + 1;
    for (int m = 0; m < N; ++m) rho[seq[m]] = seq[(m + 1) % N];
    beta.assign(N, 0);
    omega.assign(N, 0);
    for (int x = 0; x < N; ++x) {
        beta[x] = x;
        omega[x] = rho[(x + N - 1) % N];
    }
    std::vector<int> seen(N, 0);
    init = 0;
    for (int s = 0; s < N; ++s) {
        if (seen[s]) continue;
        int len = 0;
        for (int x = s; !seen[x]; x = omega[x]) seen[x] = 1, ++len;
        init += len & 1;
    }
}

// replays position triples on (beta, omega): each move must be i<j<k in
// range, and the end state must have omega = identity
[[maybe_unused]] bool replays(std::vector<int> beta, std::vector<int> omega, const std::vector<std::vector<int>> &moves, int maxd) {
    const int N = (int)beta.size();
    if ((int)moves.size() > maxd || moves.empty()) return false;
    for (auto &m : moves) {
        if (m.size() != 3 || !(0 <= m[0] && m[0] < m[1] && m[1] < m[2] && m[2] < N)) return false;
        const int a = beta[m[0]], b = beta[m[1]], c = beta[m[2]];
        std::vector<int> om = omega;
        om[a] = omega[c];
        om[b] = omega[a];
        om[c] = omega[b];
        omega = om;
        std::vector<int> nb;
        for (int q = 0; q < m[0]; ++q) nb.push_back(beta[q]);
        for (int q = m[1]; q < m[2]; ++q) nb.push_back(beta[q]);
        for (int q = m[0]; q < m[1]; ++q) nb.push_back(beta[q]);
        for (int q = m[2]; q < N; ++q) nb.push_back(beta[q]);
        beta = nb;
    }
    for (int x = 0; x < N; ++x)
        if (omega[x] != x) return false;
    return true;
}

}  // namespace

#ifdef TD_FAKE_ENGINE
// ---- a stand-in engine: returns the scripted status and records the call ----
static int g_next_rc = TD_OK;
static std::string g_next_msg;
static std::vector<int16_t> g_next_moves;
static std::vector<int> g_seen_devices, g_seen_beta;
static int g_seen_total = 0, g_seen_n = 0, g_seen_maxd = 0, g_seen_full = -1, g_seen_slot = -1;
static float g_seen_rate = 0;
static uint64_t g_seen_budget = 0;
static std::vector<int32_t> g_pair_status;

extern "C" int td_init_slots(int total, const int *devs, int ndev, uint64_t budget, char *err, size_t errlen) {
    g_seen_total = total;
    g_seen_devices.assign(devs, devs + ndev);
    g_seen_budget = budget;
    if (g_next_rc != TD_OK) std::snprintf(err, errlen, "%s", g_next_msg.c_str());
    return g_next_rc;
}
extern "C" int td_search(int slot, const uint8_t *beta, const uint8_t *, int n, int, float rate, int maxd, int full,
                         int16_t *out, int *depth, char *err, size_t errlen) {
    g_seen_slot = slot;
    g_seen_n = n;
    g_seen_beta.assign(beta, beta + n);
    g_seen_rate = rate;
    g_seen_maxd = maxd;
    g_seen_full = full;
    *depth = 0;
    if (g_next_rc == TD_OK) {
        *depth = (int)g_next_moves.size() / 3;
        std::memcpy(out, g_next_moves.data(), g_next_moves.size() * sizeof(int16_t));
    } else if (g_next_rc != TD_NOT_FOUND) {
        std::snprintf(err, errlen, "%s", g_next_msg.c_str());
    }
    return g_next_rc;
}
extern "C" int td_search_pairs(int slot, int count, const uint8_t *, const uint8_t *, const uint8_t *n,
                               const int32_t *, const float *, const int32_t *, const uint8_t *, unsigned,
                               int32_t *status, int32_t *depth, int16_t *ijk, char *err, size_t errlen) {
    g_seen_slot = slot;
    g_seen_n = count ? n[count - 1] : -1;
    if (g_next_rc != TD_OK) {
        std::snprintf(err, errlen, "%s", g_next_msg.c_str());
        return g_next_rc;
    }
    for (int p = 0; p < count; ++p) {
        status[p] = g_pair_status[p];
        depth[p] = status[p] == TD_OK ? (int)g_next_moves.size() / 3 : 0;
        for (int q = 0; q < 27; ++q) ijk[27 * p + q] = q < (int)g_next_moves.size() ? g_next_moves[q] : 0;
    }
    return TD_OK;
}

// the pair consumer and certificate writer, recorded
static int g_open_rc = TD_OK, g_accept_rc = TD_OK, g_close_rc = TD_OK;
static std::string g_open_msg, g_close_msg, g_seen_path;
static int g_seen_open[5];
static double g_seen_delay = 0;
static void *g_seen_writer = nullptr;
static bool g_writer_null = false, g_writer_closed = false, g_batcher_closed = false;
static long long g_writer_written = 0;
static uint64_t g_seen_tag = 0;
static td_batcher_stats g_next_stats{};
static int g_writer_token, g_batcher_token;

extern "C" void *td_cert_writer_open(const char *path, double) {
    g_seen_path = path;
    g_writer_closed = false;
    return g_writer_null ? nullptr : &g_writer_token;
}
extern "C" long long td_cert_writer_close(void *w) {
    g_writer_closed = w == &g_writer_token;
    return g_writer_written;
}
extern "C" int td_batcher_open(int first_slot, int slots, int batch, double delay, int pending, unsigned,
                               td_batcher_search_fn, void *writer, td_batcher_done_fn, void *, void **h, char *err,
                               size_t errlen) {
    const int seen[5] = {first_slot, slots, batch, pending, 0};
    std::memcpy(g_seen_open, seen, sizeof seen);
    g_seen_delay = delay;
    g_seen_writer = writer;
    g_batcher_closed = false;
    if (g_open_rc != TD_OK) {
        std::snprintf(err, errlen, "%s", g_open_msg.c_str());
        return g_open_rc;
    }
    *h = &g_batcher_token;
    return TD_OK;
}
extern "C" int td_batcher_accept(void *h, uint64_t tag, const uint8_t *beta, const uint8_t *, int n, int,
                                 float rate, int maxd, int full) {
    if (h != &g_batcher_token) return TD_INVALID_ARG;
    g_seen_tag = tag;
    g_seen_n = n;
    g_seen_beta.assign(beta, beta + n);
    g_seen_rate = rate;
    g_seen_maxd = maxd;
    g_seen_full = full;
    return g_accept_rc;
}
extern "C" int td_batcher_close(void *h, td_batcher_stats *st, char *err, size_t errlen) {
    g_batcher_closed = h == &g_batcher_token;
    *st = g_next_stats;
    if (g_close_rc != TD_OK) std::snprintf(err, errlen, "%s", g_close_msg.c_str());
    return g_close_rc;
}

static void run_fake_consumer() {
    auto open = [](jstring path) {
        return Java_br_unb_cic_tdp_base_GPUSortingSearch_openPairConsumer(&g_env, nullptr, 2, 3, 128, 0.25, 5, path);
    };
    auto accept = [](jlong h, std::vector<int> beta, std::vector<int> omega) {
        Java_br_unb_cic_tdp_base_GPUSortingSearch_acceptPair(&g_env, nullptr, h, 41, beta.empty() ? nullptr : bytes(beta),
                                                             bytes(omega), 1, 1.7777778f, 8, false);
    };
    jlong h = open(nullptr);
    check(h != 0 && !g_pending && g_seen_open[0] == 2 && g_seen_open[1] == 3 && g_seen_open[2] == 128 &&
              g_seen_open[3] == 5 && g_seen_delay == 0.25 && g_seen_writer == nullptr,
          "openPairConsumer passes its settings through, no writer without a path");
    accept(h, {0, 200, 2}, {1, 2, 0});
    check(!g_pending && g_seen_tag == 41 && g_seen_n == 3 && g_seen_beta[1] == 200 && g_seen_rate == 1.7777778f &&
              g_seen_maxd == 8 && g_seen_full == 0,
          "acceptPair passes tag, bytes unsigned, rate, depth and fullSorting");
    accept(0, {0, 1, 2}, {1, 2, 0});
    check(threw("the pair consumer is not open"), "acceptPair(0)");
    accept(h, {}, {1, 2, 0});
    check(threw("beta and omega must not be null"), "acceptPair(null beta)");
    accept(h, {0, 1, 2}, {1, 2});
    check(threw("beta and omega must have equal lengths"), "acceptPair(unequal lengths)");
    accept(h, std::vector<int>(18, 0), std::vector<int>(18, 0));
    check(threw("performGpuSortingSearch: n exceeds MAX_N"), "acceptPair(n > 17)");
    g_accept_rc = TD_INVALID_ARG;
    accept(h, {0, 1, 2}, {1, 2, 0});
    check(threw("the pair consumer rejected the pair"), "acceptPair rejected");
    g_accept_rc = TD_OK;
    g_next_stats = td_batcher_stats{10, 2, 6, 3, 1, 6, 0.5};
    jlongArray st = Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, h);
    check(st && !g_pending && g_batcher_closed && longs_of(st) == std::vector<jlong>({10, 2, 6, 3, 1, 0}),
          "closePairConsumer: long[6], no certificates without a writer");
    check(Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, 0) == nullptr &&
              threw("the pair consumer is not open"),
          "closePairConsumer(0)");

    h = open(jstr("/tmp/certs.bin"));
    check(h != 0 && g_seen_path == "/tmp/certs.bin" && g_seen_writer == &g_writer_token && g_strings_held == 0,
          "openPairConsumer with a path opens the certificate writer and releases the string");
    g_writer_written = 6;
    st = Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, h);
    check(st && g_writer_closed && longs_of(st)[5] == 6, "closePairConsumer closes the writer and counts its records");
    g_writer_written = 0;

    g_writer_null = true;
    check(open(jstr("/nonexistent/x")) == 0 && threw("cannot open the certificate file"), "unwritable path");
    g_writer_null = false;
    g_open_rc = TD_INVALID_ARG;
    g_open_msg = "td_batcher_open: needs slots";
    check(open(jstr("/tmp/c2.bin")) == 0 && threw("td_batcher_open: needs slots") && g_writer_closed,
          "open failure raises and closes the writer");
    g_open_rc = TD_OK;
    h = open(nullptr);
    g_close_rc = TD_CUDA_ERROR;
    g_close_msg = "CUDA error";
    check(Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, h) == nullptr &&
              threw("CUDA error") && g_batcher_closed,
          "a failed batch call raises at close");
    g_close_rc = TD_OK;
}

static void run_fake() {
    auto init = [](jintArray devs, jlong budget) {
        Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(&g_env, nullptr, 4, devs, budget);
    };
    init(nullptr, 1 << 20);
    check(threw("devices must not be null"), "initSlots(null devices)");
    init(ints({0}), 0);
    check(threw("queueBytesBudget must be positive"), "initSlots(budget 0)");
    g_next_rc = TD_OK;
    init(ints({0, 3}), 1ll << 33);
    check(!g_pending && g_seen_total == 4 && g_seen_devices == std::vector<int>({0, 3}) &&
              g_seen_budget == (1ull << 33),
          "initSlots passes its arguments through");
    g_next_rc = TD_INVALID_ARG;
    g_next_msg = "devices must contain distinct CUDA device ordinals";
    init(ints({1, 1}), 1 << 20);
    check(threw("devices must contain distinct CUDA device ordinals"), "initSlots error message");

    check(Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(&g_env, nullptr, nullptr, bytes({1}), 0, 0,
                                                                       1, true, 0) == nullptr &&
              threw("beta and omega must not be null"),
          "search(null beta)");
    check(search({0, 1, 2}, {1, 2}, 1, 0, 1, true, 0) == nullptr && threw("beta and omega must have equal lengths"),
          "search(unequal lengths)");
    g_next_rc = TD_OK;
    g_next_moves = {0, 1, 2, 1, 3, 4};
    jobjectArray r = search({0, 200, 2, 3, 4}, {1, 2, 3, 4, 0}, 1, 1.7777778f, 9, false, 5);
    check(r && !g_pending && get(r)->name == "[I" &&
              moves_of(r) == std::vector<std::vector<int>>({{0, 1, 2}, {1, 3, 4}}),
          "found: int[2][3]");
    check(g_seen_slot == 5 && g_seen_n == 5 && g_seen_beta[1] == 200 && g_seen_rate == 1.7777778f &&
              g_seen_maxd == 9 && g_seen_full == 0,
          "search passes bytes unsigned, rate, depth, fullSorting and slot");
    g_next_rc = TD_NOT_FOUND;
    r = search({0, 1, 2}, {1, 2, 0}, 1, 0, 1, true, 0);
    check(r && !g_pending && get(r)->o.empty(), "not found: empty int[0][], not null");
    const struct {
        int rc;
        const char *msg;
    } errors[] = {{TD_OVERFLOW, "GPU sorting search queue overflow"},
                  {TD_TIMEOUT, "GPU sorting search deadline reached"},
                  {TD_CUDA_ERROR, "td_engine.cu:1: CUDA error cudaErrorLaunchFailure (unspecified launch failure)"},
                  {TD_INVALID_ARG, "invalid GPU sorting slot"}};
    for (auto &e : errors) {
        g_next_rc = e.rc;
        g_next_msg = e.msg;
        raise("java/lang/IllegalStateException", "left pending by an earlier call");
        check(search({0, 1, 2}, {1, 2, 0}, 1, 0, 1, true, 0) == nullptr && threw(e.msg),
              std::string("status ") + std::to_string(e.rc) + " -> RuntimeException(message)");
    }

    auto batch = [](jobjectArray b, jobjectArray o, int count) {
        std::vector<jint> init(count, 1), maxd(count, 9);
        return Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeqBatch(
            &g_env, nullptr, b, o, ints(init), floats(std::vector<jfloat>(count, 0.f)), ints(maxd),
            bools(std::vector<jboolean>(count, 1)), 2);
    };
    check(batch(nullptr, byte_rows({{1}}), 1) == nullptr && threw("batch arrays must not be null"),
          "batch(null)");
    check(batch(byte_rows({{0, 1, 2}}), byte_rows({{1, 2, 0}, {1, 2, 0}}), 1) == nullptr &&
              threw("batch arrays must have equal lengths"),
          "batch(unequal counts)");
    check(batch(byte_rows({std::vector<int>(18, 0)}), byte_rows({std::vector<int>(18, 0)}), 1) == nullptr &&
              threw("pair 0: performGpuSortingSearch: n exceeds MAX_N"),
          "batch(n > 17)");
    g_next_rc = TD_OK;
    g_next_moves = {0, 1, 2};
    g_pair_status = {TD_OK, TD_NOT_FOUND, TD_OK};
    r = batch(byte_rows({{0, 1, 2}, {0, 1, 2, 3}, {0, 1, 2}}), byte_rows({{1, 2, 0}, {0, 1, 2, 3}, {1, 2, 0}}), 3);
    check(r && !g_pending && get(r)->name == "[[I" && get(r)->o.size() == 3 && g_seen_slot == 2 && g_seen_n == 3,
          "batch: int[3][][]");
    if (r && get(r)->o.size() == 3) {
        check(moves_of(reinterpret_cast<jobjectArray>(get(r)->o[0])) == std::vector<std::vector<int>>({{0, 1, 2}}),
              "batch pair 0 witness");
        check(get(get(r)->o[1])->o.empty(), "batch pair 1 empty");
    }
    g_pair_status = {TD_OK, TD_OVERFLOW};
    check(batch(byte_rows({{0, 1, 2}, {0, 1, 2}}), byte_rows({{1, 2, 0}, {1, 2, 0}}), 2) == nullptr &&
              threw("pair 1: GPU sorting search queue overflow"),
          "batch overflow -> RuntimeException");
    g_next_rc = TD_CUDA_ERROR;
    g_next_msg = "CUDA error";
    check(batch(byte_rows({{0, 1, 2}}), byte_rows({{1, 2, 0}}), 1) == nullptr && threw("CUDA error"),
          "batch call error -> RuntimeException");
    run_fake_consumer();
}
#else
static void run_real(bool gpu) {
    if (!gpu) {
        Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(&g_env, nullptr, 2, ints({0}), 1 << 20);
        check(threw_any(), "initSlots without a GPU raises");
        check(search({0, 1, 2}, {1, 2, 0}, 1, 2.0f, 1, true, 0) == nullptr && threw("invalid GPU sorting slot"),
              "search on an uninitialised slot");
        const jlong h = Java_br_unb_cic_tdp_base_GPUSortingSearch_openPairConsumer(&g_env, nullptr, 0, 1, 8, 0.001, 0,
                                                                                   nullptr);
        check(h != 0 && !g_pending, "openPairConsumer without a GPU");
        Java_br_unb_cic_tdp_base_GPUSortingSearch_acceptPair(&g_env, nullptr, h, 0, bytes({0, 1, 2}), bytes({1, 2, 0}),
                                                             1, 2.0f, 1, true);
        check(!g_pending, "acceptPair without a GPU");
        check(Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, h) == nullptr && threw_any(),
              "a batch on an uninitialised slot raises at close");
        return;
    }
    Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(&g_env, nullptr, 2, ints({0}), 32 << 20);
    check(!g_pending, "initSlots(2, [0], 32 MiB)");
    jobjectArray r = search({0, 1, 2}, {1, 2, 0}, 1, 2.0f, 1, true, 0);
    check(r && moves_of(r) == std::vector<std::vector<int>>({{0, 1, 2}}), "smoke: [[0,1,2]]");
    r = search({0, 1}, {1, 0}, 0, 0.f, 1, true, 1);
    check(r && get(r)->o.empty() && !g_pending, "N < 3: int[0][]");
    check(search({0, 1, 2}, {1, 2, 0}, 1, 2.0f, 10, true, 0) == nullptr &&
              threw("performGpuSortingSearch: invalid maximumDepth"),
          "maxMoves 10");
    check(search({0, 1, 2}, {1, 2, 0}, 1, 2.0f, 1, true, 2) == nullptr && threw("invalid GPU sorting slot"),
          "slot out of range");
    // 96 seeded S_10 pairs: per call and batched, every witness replays and
    // the verdicts agree
    std::mt19937 rng(7);
    std::vector<std::vector<int>> betas, omegas;
    std::vector<jint> inits, maxds;
    for (int c = 0; c < 96; ++c) {
        std::vector<int> pi(10);
        for (int m = 0; m < 10; ++m) pi[m] = m;
        std::shuffle(pi.begin(), pi.end(), rng);
        std::vector<int> beta, omega;
        int init;
        pair_of(pi, beta, omega, init);
        betas.push_back(beta);
        omegas.push_back(omega);
        inits.push_back(init);
        maxds.push_back(c % 2 ? 5 : 6);
    }
    std::vector<int> single(96);
    for (int c = 0; c < 96; ++c) {
        r = search(betas[c], omegas[c], inits[c], 0.f, maxds[c], true, c % 2);
        check(r && !g_pending, "per-call search " + std::to_string(c));
        single[c] = r && !get(r)->o.empty();
        if (single[c]) check(replays(betas[c], omegas[c], moves_of(r), maxds[c]), "per-call replay " + std::to_string(c));
    }
    r = Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeqBatch(
        &g_env, nullptr, byte_rows(betas), byte_rows(omegas), ints(inits), floats(std::vector<jfloat>(96, 0.f)),
        ints(maxds), bools(std::vector<jboolean>(96, 1)), 1);
    check(r && !g_pending && get(r)->o.size() == 96, "batch of 96");
    int found = 0;
    for (int c = 0; r && c < 96; ++c) {
        jobjectArray row = reinterpret_cast<jobjectArray>(get(r)->o[c]);
        const bool f = !get(row)->o.empty();
        found += f;
        check(f == (bool)single[c], "batch verdict " + std::to_string(c));
        if (f) check(replays(betas[c], omegas[c], moves_of(row), maxds[c]), "batch replay " + std::to_string(c));
    }
    check(found > 0 && found < 96, "both verdicts occur");
    // the same pairs through the native consumer, witnesses to a certificate file
    char path[] = "/tmp/td_jni_certsXXXXXX";
    const int fd = mkstemp(path);
    check(fd >= 0, "temporary certificate file");
    if (fd >= 0) close(fd);
    const jlong h = Java_br_unb_cic_tdp_base_GPUSortingSearch_openPairConsumer(&g_env, nullptr, 0, 2, 32, 0.002, 0,
                                                                               jstr(path));
    check(h != 0 && !g_pending, "openPairConsumer(2 slots, batches of 32)");
    for (int c = 0; h && c < 96; ++c)
        Java_br_unb_cic_tdp_base_GPUSortingSearch_acceptPair(&g_env, nullptr, h, c, bytes(betas[c]), bytes(omegas[c]),
                                                             inits[c], 0.f, maxds[c], true);
    check(!g_pending, "acceptPair x 96");
    jlongArray st = h ? Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(&g_env, nullptr, h) : nullptr;
    check(st && !g_pending &&
              longs_of(st) == std::vector<jlong>({96, longs_of(st)[1], found, 96 - found, 0, found}) &&
              longs_of(st)[1] >= 3,
          "consumer: every pair searched, the batch verdicts, one certificate per witness");
    unlink(path);
    td_destroy();
}
#endif

int main(int argc, char **argv) {
    const std::string mode = argc > 1 ? argv[1] : "";
#ifdef TD_FAKE_ENGINE
    if (mode != "fake") return 2;
    run_fake();
#else
    if (mode != "real-cpu" && mode != "real-gpu") return 2;
    run_real(mode == "real-gpu");
#endif
    std::printf("jni %s %d checks, %d failed\n", g_failures ? "FAILED" : "ok", g_checks, g_failures);
    for (Obj *o : g_heap) delete o;
    return g_failures ? 1 : 0;
}
