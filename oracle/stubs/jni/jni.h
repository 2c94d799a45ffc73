/* ORACLE / TEST INFRASTRUCTURE: a minimal stand-in for the JDK's <jni.h>,
 * enough to compile the reference's JNI glue
 * (src/jni/dr_inference_hawkes_NativeHPHSingleton.cpp) without a JDK and to
 * call it from a test process.  Only the names and signatures the glue uses
 * are kept.  A jdoubleArray here is a plain {length, data} pair that the test
 * builds itself, and JNIEnv's three array methods act on it directly: there
 * is no Java virtual machine behind them. */
#ifndef HPHC_STUB_JNI_H
#define HPHC_STUB_JNI_H

#include <stdint.h>

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_ABORT 2

typedef int32_t jint;
typedef int64_t jlong;
typedef double jdouble;
typedef uint8_t jboolean;
typedef jint jsize;
typedef void* jobject;

struct HphcStubDoubleArray {
    jsize length;
    jdouble* data;
};
typedef struct HphcStubDoubleArray* jdoubleArray;

#ifdef __cplusplus
struct JNIEnv {
    jsize GetArrayLength(jdoubleArray a) { return a->length; }
    jdouble* GetDoubleArrayElements(jdoubleArray a, jboolean*) { return a->data; }
    void ReleaseDoubleArrayElements(jdoubleArray, jdouble*, jint) {}
};
#else
typedef struct JNIEnv JNIEnv;
#endif

#endif
