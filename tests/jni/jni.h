/*
 * jni.h -- a minimal stand-in for the JDK's JNI header, for testing the JNI
 * shim (td16_b200/csrc/td_jni.cc) where no JDK is installed.
 *
 * TEST INFRASTRUCTURE ONLY.  It declares just the types and JNIEnv calls the
 * shim uses, with the same names and argument types as the JNI
 * specification, so that the shim compiles unchanged against either header.
 * The function table here is this file's own (it is not the JDK's table
 * layout): a shim built against it only runs with the fake environment of
 * tests/jni/jni_driver.cc, never inside a JVM.
 */
#ifndef TD16_TEST_JNI_H
#define TD16_TEST_JNI_H

#include <stdint.h>

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_ABORT 2

typedef int32_t jint;
typedef int64_t jlong;
typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

class _jobject {};
class _jclass : public _jobject {};
class _jthrowable : public _jobject {};
class _jarray : public _jobject {};
class _jobjectArray : public _jarray {};
class _jbyteArray : public _jarray {};
class _jintArray : public _jarray {};
class _jfloatArray : public _jarray {};
class _jbooleanArray : public _jarray {};
class _jlongArray : public _jarray {};
class _jstring : public _jobject {};

typedef _jobject *jobject;
typedef _jclass *jclass;
typedef _jthrowable *jthrowable;
typedef _jarray *jarray;
typedef _jobjectArray *jobjectArray;
typedef _jbyteArray *jbyteArray;
typedef _jintArray *jintArray;
typedef _jfloatArray *jfloatArray;
typedef _jbooleanArray *jbooleanArray;
typedef _jlongArray *jlongArray;
typedef _jstring *jstring;

struct JNIEnv_;

/* the calls the shim makes, one pointer each */
struct TestJniFunctions {
    jboolean (*ExceptionCheck)(JNIEnv_ *);
    void (*ExceptionClear)(JNIEnv_ *);
    jclass (*FindClass)(JNIEnv_ *, const char *);
    jint (*ThrowNew)(JNIEnv_ *, jclass, const char *);
    void (*DeleteLocalRef)(JNIEnv_ *, jobject);
    jsize (*GetArrayLength)(JNIEnv_ *, jarray);
    void (*GetByteArrayRegion)(JNIEnv_ *, jbyteArray, jsize, jsize, jbyte *);
    void (*GetIntArrayRegion)(JNIEnv_ *, jintArray, jsize, jsize, jint *);
    void (*GetFloatArrayRegion)(JNIEnv_ *, jfloatArray, jsize, jsize, jfloat *);
    void (*GetBooleanArrayRegion)(JNIEnv_ *, jbooleanArray, jsize, jsize, jboolean *);
    jobjectArray (*NewObjectArray)(JNIEnv_ *, jsize, jclass, jobject);
    jintArray (*NewIntArray)(JNIEnv_ *, jsize);
    void (*SetIntArrayRegion)(JNIEnv_ *, jintArray, jsize, jsize, const jint *);
    jobject (*GetObjectArrayElement)(JNIEnv_ *, jobjectArray, jsize);
    void (*SetObjectArrayElement)(JNIEnv_ *, jobjectArray, jsize, jobject);
    const char *(*GetStringUTFChars)(JNIEnv_ *, jstring, jboolean *);
    void (*ReleaseStringUTFChars)(JNIEnv_ *, jstring, const char *);
    jlongArray (*NewLongArray)(JNIEnv_ *, jsize);
    void (*SetLongArrayRegion)(JNIEnv_ *, jlongArray, jsize, jsize, const jlong *);
};

struct JNIEnv_ {
    const TestJniFunctions *functions;
    jboolean ExceptionCheck() { return functions->ExceptionCheck(this); }
    void ExceptionClear() { functions->ExceptionClear(this); }
    jclass FindClass(const char *name) { return functions->FindClass(this, name); }
    jint ThrowNew(jclass cls, const char *msg) { return functions->ThrowNew(this, cls, msg); }
    void DeleteLocalRef(jobject obj) { functions->DeleteLocalRef(this, obj); }
    jsize GetArrayLength(jarray a) { return functions->GetArrayLength(this, a); }
    void GetByteArrayRegion(jbyteArray a, jsize s, jsize l, jbyte *b) { functions->GetByteArrayRegion(this, a, s, l, b); }
    void GetIntArrayRegion(jintArray a, jsize s, jsize l, jint *b) { functions->GetIntArrayRegion(this, a, s, l, b); }
    void GetFloatArrayRegion(jfloatArray a, jsize s, jsize l, jfloat *b) { functions->GetFloatArrayRegion(this, a, s, l, b); }
    void GetBooleanArrayRegion(jbooleanArray a, jsize s, jsize l, jboolean *b) {
        functions->GetBooleanArrayRegion(this, a, s, l, b);
    }
    jobjectArray NewObjectArray(jsize n, jclass cls, jobject init) { return functions->NewObjectArray(this, n, cls, init); }
    jintArray NewIntArray(jsize n) { return functions->NewIntArray(this, n); }
    void SetIntArrayRegion(jintArray a, jsize s, jsize l, const jint *b) { functions->SetIntArrayRegion(this, a, s, l, b); }
    jobject GetObjectArrayElement(jobjectArray a, jsize i) { return functions->GetObjectArrayElement(this, a, i); }
    void SetObjectArrayElement(jobjectArray a, jsize i, jobject v) { functions->SetObjectArrayElement(this, a, i, v); }
    const char *GetStringUTFChars(jstring s, jboolean *copy) { return functions->GetStringUTFChars(this, s, copy); }
    void ReleaseStringUTFChars(jstring s, const char *c) { functions->ReleaseStringUTFChars(this, s, c); }
    jlongArray NewLongArray(jsize n) { return functions->NewLongArray(this, n); }
    void SetLongArrayRegion(jlongArray a, jsize s, jsize l, const jlong *b) { functions->SetLongArrayRegion(this, a, s, l, b); }
};
typedef JNIEnv_ JNIEnv;

#endif
