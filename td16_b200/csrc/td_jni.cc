// td_jni.cc -- JNI shim: class br.unb.cic.tdp.base.GPUSortingSearch binds
// these natives from library td16_jni; each forwards to the C ABI of
// libtd16b200.so.
//   initSlots, searchForSortingSeq   the reference's two natives
//                                    (GPUSortingSearch.java:115-117,
//                                    emitter/src/native/jni/jni_sorter.cu:24-117)
//   searchForSortingSeqBatch         an addition for a case producer that
//                                    hands over pairs in groups
//   openPairConsumer, acceptPair,    an addition for the enumerator's
//   closePairConsumer                Consumer<CyclicTargetPair>: pairs handed
//                                    over one per call, searched in batches by
//                                    the native consumer (td_batcher_*), found
//                                    witnesses written as certificates
// A non-OK status becomes a java.lang.RuntimeException carrying the engine's
// message, as jni_sorter.cu:15-22,111-115 does for every C++ exception.  Built
// only where a JDK's jni.h exists (td16_b200/build.py); the tests compile it
// against a minimal hand-written jni.h and a fake JNIEnv (tests/jni/).
#include <jni.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "td16_b200.h"

static void throw_runtime(JNIEnv *env, const char *message) {
    if (env->ExceptionCheck()) env->ExceptionClear();
    jclass cls = env->FindClass("java/lang/RuntimeException");
    if (cls) {
        env->ThrowNew(cls, message);
        env->DeleteLocalRef(cls);
    }
}

extern "C" JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(
    JNIEnv *env, jclass, jint total_slots, jintArray devices, jlong budget) {
    if (devices == nullptr) {
        throw_runtime(env, "devices must not be null");
        return;
    }
    if (budget <= 0) {
        throw_runtime(env, "queueBytesBudget must be positive");
        return;
    }
    const jsize count = env->GetArrayLength(devices);
    std::vector<jint> devs(count > 0 ? count : 1);
    if (count > 0) env->GetIntArrayRegion(devices, 0, count, devs.data());
    std::vector<int> ints(devs.begin(), devs.begin() + count);
    char err[512] = {0};
    const int rc = td_init_slots((int)total_slots, ints.data(), (int)count, (uint64_t)budget, err, sizeof err);
    if (rc != TD_OK) throw_runtime(env, err[0] ? err : "initSlots failed");
}

// int[depth][3] of position triples (empty, not null, without a witness)
static jobjectArray moves_array(JNIEnv *env, const int16_t *ijk, int depth) {
    jclass int_array = env->FindClass("[I");
    jobjectArray outer = env->NewObjectArray(depth, int_array, nullptr);
    for (int d = 0; d < depth; ++d) {
        const jint move[3] = {ijk[3 * d], ijk[3 * d + 1], ijk[3 * d + 2]};
        jintArray inner = env->NewIntArray(3);
        env->SetIntArrayRegion(inner, 0, 3, move);
        env->SetObjectArrayElement(outer, d, inner);
        env->DeleteLocalRef(inner);
    }
    env->DeleteLocalRef(int_array);
    return outer;
}

extern "C" JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(
    JNIEnv *env, jclass, jbyteArray beta, jbyteArray omega, jint initial_even_cycles, jfloat min_rate,
    jint max_moves, jboolean full_sorting, jint slot) {
    if (beta == nullptr || omega == nullptr) {
        throw_runtime(env, "beta and omega must not be null");
        return nullptr;
    }
    const jsize n = env->GetArrayLength(beta);
    if (env->GetArrayLength(omega) != n) {
        throw_runtime(env, "beta and omega must have equal lengths");
        return nullptr;
    }
    std::vector<uint8_t> b(n > 0 ? n : 1), o(n > 0 ? n : 1);
    if (n > 0) {
        env->GetByteArrayRegion(beta, 0, n, reinterpret_cast<jbyte *>(b.data()));
        env->GetByteArrayRegion(omega, 0, n, reinterpret_cast<jbyte *>(o.data()));
    }
    int16_t ijk[27];
    int depth = 0;
    char err[512] = {0};
    const int rc = td_search((int)slot, b.data(), o.data(), (int)n, (int)initial_even_cycles, (float)min_rate,
                             (int)max_moves, full_sorting ? 1 : 0, ijk, &depth, err, sizeof err);
    if (rc != TD_OK && rc != TD_NOT_FOUND) {
        throw_runtime(env, err[0] ? err : "GPU sorting search failed");
        return nullptr;
    }
    return moves_array(env, ijk, rc == TD_OK ? depth : 0);
}

// The batch form: pair p is (betas[p], omegas[p], initialEvenCycles[p],
// minRates[p], maxMoves[p], fullSorting[p]); returns int[count][][3], entry p
// as searchForSortingSeq would return it.  A pair that searchForSortingSeq
// would reject raises the same RuntimeException class, prefixed with the
// pair's index, and the call returns null.
extern "C" JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeqBatch(
    JNIEnv *env, jclass, jobjectArray betas, jobjectArray omegas, jintArray initial_even_cycles,
    jfloatArray min_rates, jintArray max_moves, jbooleanArray full_sorting, jint slot) {
    if (!betas || !omegas || !initial_even_cycles || !min_rates || !max_moves || !full_sorting) {
        throw_runtime(env, "batch arrays must not be null");
        return nullptr;
    }
    const jsize count = env->GetArrayLength(betas);
    if (env->GetArrayLength(omegas) != count || env->GetArrayLength(initial_even_cycles) != count ||
        env->GetArrayLength(min_rates) != count || env->GetArrayLength(max_moves) != count ||
        env->GetArrayLength(full_sorting) != count) {
        throw_runtime(env, "batch arrays must have equal lengths");
        return nullptr;
    }
    const size_t c = count > 0 ? (size_t)count : 1;
    std::vector<uint8_t> b(17 * c, 0), o(17 * c, 0), n(c, 0), full(c, 0);
    std::vector<int32_t> init(c, 0), maxd(c, 0), status(c, 0), depth(c, 0);
    std::vector<float> rate(c, 0.f);
    std::vector<int16_t> ijk(27 * c, 0);
    for (jsize p = 0; p < count; ++p) {
        jbyteArray bp = (jbyteArray)env->GetObjectArrayElement(betas, p);
        jbyteArray op = (jbyteArray)env->GetObjectArrayElement(omegas, p);
        if (!bp || !op) {
            char msg[96];
            std::snprintf(msg, sizeof msg, "pair %d: beta and omega must not be null", (int)p);
            throw_runtime(env, msg);
            return nullptr;
        }
        const jsize len = env->GetArrayLength(bp);
        if (env->GetArrayLength(op) != len || len > 17) {
            char msg[96];
            std::snprintf(msg, sizeof msg, "pair %d: %s", (int)p,
                          len > 17 ? "performGpuSortingSearch: n exceeds MAX_N"
                                   : "beta and omega must have equal lengths");
            throw_runtime(env, msg);
            return nullptr;
        }
        if (len > 0) {
            env->GetByteArrayRegion(bp, 0, len, reinterpret_cast<jbyte *>(&b[17 * (size_t)p]));
            env->GetByteArrayRegion(op, 0, len, reinterpret_cast<jbyte *>(&o[17 * (size_t)p]));
        }
        n[p] = (uint8_t)len;
        env->DeleteLocalRef(bp);
        env->DeleteLocalRef(op);
    }
    if (count > 0) {
        std::vector<jint> ji(c), jm(c);
        std::vector<jboolean> jf(c);
        env->GetIntArrayRegion(initial_even_cycles, 0, count, ji.data());
        env->GetFloatArrayRegion(min_rates, 0, count, rate.data());
        env->GetIntArrayRegion(max_moves, 0, count, jm.data());
        env->GetBooleanArrayRegion(full_sorting, 0, count, jf.data());
        for (size_t p = 0; p < (size_t)count; ++p) {
            init[p] = ji[p];
            maxd[p] = jm[p];
            full[p] = jf[p] ? 1 : 0;
        }
    }
    char err[512] = {0};
    const int rc = td_search_pairs((int)slot, (int)count, b.data(), o.data(), n.data(), init.data(), rate.data(),
                                   maxd.data(), full.data(), 0u, status.data(), depth.data(), ijk.data(), err,
                                   sizeof err);
    if (rc != TD_OK) {
        throw_runtime(env, err[0] ? err : "GPU sorting search failed");
        return nullptr;
    }
    for (jsize p = 0; p < count; ++p) {
        const char *what = nullptr;
        if (status[p] == TD_OVERFLOW) what = "GPU sorting search queue overflow";
        else if (status[p] == TD_TIMEOUT) what = "GPU sorting search deadline reached";
        else if (status[p] == TD_INVALID_ARG) what = "performGpuSortingSearch: invalid input";
        else if (status[p] != TD_OK && status[p] != TD_NOT_FOUND) what = "GPU sorting search failed";
        if (what) {
            char msg[160];
            std::snprintf(msg, sizeof msg, "pair %d: %s", (int)p, what);
            throw_runtime(env, msg);
            return nullptr;
        }
    }
    jclass moves_class = env->FindClass("[[I");
    jobjectArray outer = env->NewObjectArray(count, moves_class, nullptr);
    for (jsize p = 0; p < count; ++p) {
        jobjectArray inner = moves_array(env, &ijk[27 * (size_t)p], status[p] == TD_OK ? depth[p] : 0);
        env->SetObjectArrayElement(outer, p, inner);
        env->DeleteLocalRef(inner);
    }
    env->DeleteLocalRef(moves_class);
    return outer;
}

// ---- the native pair consumer ---------------------------------------------

namespace {
struct JniPairConsumer {
    void *batcher;
    void *writer;  // certificate file, or null
};
}  // namespace

// Opens a consumer whose `slots` workers (slots firstSlot ..) search batches
// of batchSize pairs (or what has waited maxDelaySeconds); at most maxPending
// full batches wait (0: twice the slots) before acceptPair blocks.  With a
// certificatePath, found witnesses are written there as certificate records
// (the codec's bytes).  Returns the handle for acceptPair / closePairConsumer.
extern "C" JNIEXPORT jlong JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_openPairConsumer(
    JNIEnv *env, jclass, jint first_slot, jint slots, jint batch_size, jdouble max_delay_s, jint max_pending,
    jstring certificate_path) {
    void *writer = nullptr;
    if (certificate_path != nullptr) {
        const char *path = env->GetStringUTFChars(certificate_path, nullptr);
        if (path == nullptr) return 0;  // the JVM has raised OutOfMemoryError
        writer = td_cert_writer_open(path, 5.0);
        env->ReleaseStringUTFChars(certificate_path, path);
        if (writer == nullptr) {
            throw_runtime(env, "cannot open the certificate file");
            return 0;
        }
    }
    void *h = nullptr;
    char err[512] = {0};
    const int rc = td_batcher_open((int)first_slot, (int)slots, (int)batch_size, (double)max_delay_s,
                                   (int)max_pending, 0u, nullptr, writer, nullptr, nullptr, &h, err, sizeof err);
    if (rc != TD_OK) {
        if (writer) td_cert_writer_close(writer);
        throw_runtime(env, err[0] ? err : "openPairConsumer failed");
        return 0;
    }
    return reinterpret_cast<jlong>(new JniPairConsumer{h, writer});
}

// Hands one pair to the consumer (blocks while its queue is full).  `tag`
// identifies the pair in the consumer's statistics and callbacks.
extern "C" JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_acceptPair(
    JNIEnv *env, jclass, jlong handle, jlong tag, jbyteArray beta, jbyteArray omega, jint initial_even_cycles,
    jfloat min_rate, jint max_moves, jboolean full_sorting) {
    auto *c = reinterpret_cast<JniPairConsumer *>(handle);
    if (c == nullptr) {
        throw_runtime(env, "the pair consumer is not open");
        return;
    }
    if (beta == nullptr || omega == nullptr) {
        throw_runtime(env, "beta and omega must not be null");
        return;
    }
    const jsize n = env->GetArrayLength(beta);
    if (env->GetArrayLength(omega) != n) {
        throw_runtime(env, "beta and omega must have equal lengths");
        return;
    }
    if (n > 17) {
        throw_runtime(env, "performGpuSortingSearch: n exceeds MAX_N");
        return;
    }
    uint8_t b[17], o[17];
    if (n > 0) {
        env->GetByteArrayRegion(beta, 0, n, reinterpret_cast<jbyte *>(b));
        env->GetByteArrayRegion(omega, 0, n, reinterpret_cast<jbyte *>(o));
    }
    const int rc = td_batcher_accept(c->batcher, (uint64_t)tag, b, o, (int)n, (int)initial_even_cycles,
                                     (float)min_rate, (int)max_moves, full_sorting ? 1 : 0);
    if (rc != TD_OK) throw_runtime(env, "the pair consumer rejected the pair");
}

// Searches what is left, closes the certificate file and frees the consumer.
// Returns long[6]: pairs, batches, found, not found, errors (per-pair error
// statuses), certificates written.  A batch call that failed (a CUDA error,
// an invalid slot) raises RuntimeException with its message instead.
extern "C" JNIEXPORT jlongArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_closePairConsumer(
    JNIEnv *env, jclass, jlong handle) {
    auto *c = reinterpret_cast<JniPairConsumer *>(handle);
    if (c == nullptr) {
        throw_runtime(env, "the pair consumer is not open");
        return nullptr;
    }
    td_batcher_stats st{};
    char err[512] = {0};
    const int rc = td_batcher_close(c->batcher, &st, err, sizeof err);
    const long long written = c->writer ? td_cert_writer_close(c->writer) : 0;
    delete c;
    if (rc != TD_OK) {
        throw_runtime(env, err[0] ? err : "GPU sorting search failed");
        return nullptr;
    }
    if (written < 0) {
        throw_runtime(env, "writing the certificate file failed");
        return nullptr;
    }
    const jlong out[6] = {(jlong)st.pairs, (jlong)st.batches, (jlong)st.found, (jlong)st.not_found,
                          (jlong)st.errors, (jlong)written};
    jlongArray arr = env->NewLongArray(6);
    env->SetLongArrayRegion(arr, 0, 6, out);
    return arr;
}
