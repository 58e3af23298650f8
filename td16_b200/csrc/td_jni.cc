// td_jni.cc -- JNI shim: class br.unb.cic.tdp.base.GPUSortingSearch binds these
// two natives (GPUSortingSearch.java:115-117) from library td16_jni; both
// forward to the C ABI of libtd16b200.so.  A non-OK status becomes a
// java.lang.RuntimeException carrying the engine's message, as in
// emitter/src/native/jni/jni_sorter.cu:15-22, 111-115.  Built only where a
// JDK's jni.h exists (td16_b200/build.py).
#include <jni.h>

#include <cstdint>
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
