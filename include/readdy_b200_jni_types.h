/*
 * readdy_b200_jni_types.h -- the subset of the JNI types and of the JNIEnv
 * function table that the JNI entry point uses, laid out as the Java Native
 * Interface specification's "JNI Functions" table (slot numbers below are the
 * table indices the specification gives).  It exists because this build
 * environment has no JDK; building against a JDK defines RDGPU_USE_SYSTEM_JNI
 * and uses <jni.h> instead, with no source change.
 */
#ifndef READDY_B200_JNI_TYPES_H
#define READDY_B200_JNI_TYPES_H
#include <stdint.h>

typedef uint8_t jboolean;
typedef int8_t jbyte;
typedef uint16_t jchar;
typedef int16_t jshort;
typedef int32_t jint;
typedef int64_t jlong;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

struct _jobject;
typedef struct _jobject* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jfloatArray;
typedef jobject jthrowable;
struct _jfieldID;
typedef struct _jfieldID* jfieldID;
struct _jmethodID;
typedef struct _jmethodID* jmethodID;

typedef union jvalue {
    jboolean z; jbyte b; jchar c; jshort s; jint i; jlong j; jfloat f; jdouble d; jobject l;
} jvalue;

#define JNI_FALSE 0
#define JNI_TRUE 1
#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL

/* table slots used here */
#define RDGPU_JNI_DeleteLocalRef                23
#define RDGPU_JNI_GetObjectClass                31
#define RDGPU_JNI_GetMethodID                   33
#define RDGPU_JNI_CallBooleanMethodA            39
#define RDGPU_JNI_GetFieldID                    94
#define RDGPU_JNI_GetObjectField                95
#define RDGPU_JNI_GetStringUTFChars            169
#define RDGPU_JNI_ReleaseStringUTFChars        170
#define RDGPU_JNI_GetArrayLength               171
#define RDGPU_JNI_NewFloatArray                181
#define RDGPU_JNI_GetPrimitiveArrayCritical    222
#define RDGPU_JNI_ReleasePrimitiveArrayCritical 223
#define RDGPU_JNI_ExceptionCheck               228
#define RDGPU_JNI_TABLE_SIZE                   233

struct JNINativeInterface_ {
    void* slot[RDGPU_JNI_TABLE_SIZE];
};

#ifdef __cplusplus
struct JNIEnv_;
typedef JNIEnv_ JNIEnv;
struct JNIEnv_ {
    const struct JNINativeInterface_* functions;
#define RDGPU_JNI_FN(T, i) reinterpret_cast<T>(functions->slot[i])
    void DeleteLocalRef(jobject o)
    { RDGPU_JNI_FN(void (*)(JNIEnv*, jobject), RDGPU_JNI_DeleteLocalRef)(this, o); }
    jclass GetObjectClass(jobject o)
    { return RDGPU_JNI_FN(jclass (*)(JNIEnv*, jobject), RDGPU_JNI_GetObjectClass)(this, o); }
    jmethodID GetMethodID(jclass c, const char* n, const char* s)
    { return RDGPU_JNI_FN(jmethodID (*)(JNIEnv*, jclass, const char*, const char*), RDGPU_JNI_GetMethodID)(this, c, n, s); }
    jboolean CallBooleanMethodA(jobject o, jmethodID m, const jvalue* a)
    { return RDGPU_JNI_FN(jboolean (*)(JNIEnv*, jobject, jmethodID, const jvalue*), RDGPU_JNI_CallBooleanMethodA)(this, o, m, a); }
    jfieldID GetFieldID(jclass c, const char* n, const char* s)
    { return RDGPU_JNI_FN(jfieldID (*)(JNIEnv*, jclass, const char*, const char*), RDGPU_JNI_GetFieldID)(this, c, n, s); }
    jobject GetObjectField(jobject o, jfieldID f)
    { return RDGPU_JNI_FN(jobject (*)(JNIEnv*, jobject, jfieldID), RDGPU_JNI_GetObjectField)(this, o, f); }
    const char* GetStringUTFChars(jstring s, jboolean* c)
    { return RDGPU_JNI_FN(const char* (*)(JNIEnv*, jstring, jboolean*), RDGPU_JNI_GetStringUTFChars)(this, s, c); }
    void ReleaseStringUTFChars(jstring s, const char* u)
    { RDGPU_JNI_FN(void (*)(JNIEnv*, jstring, const char*), RDGPU_JNI_ReleaseStringUTFChars)(this, s, u); }
    jsize GetArrayLength(jarray a)
    { return RDGPU_JNI_FN(jsize (*)(JNIEnv*, jarray), RDGPU_JNI_GetArrayLength)(this, a); }
    jfloatArray NewFloatArray(jsize n)
    { return RDGPU_JNI_FN(jfloatArray (*)(JNIEnv*, jsize), RDGPU_JNI_NewFloatArray)(this, n); }
    void* GetPrimitiveArrayCritical(jarray a, jboolean* c)
    { return RDGPU_JNI_FN(void* (*)(JNIEnv*, jarray, jboolean*), RDGPU_JNI_GetPrimitiveArrayCritical)(this, a, c); }
    void ReleasePrimitiveArrayCritical(jarray a, void* p, jint mode)
    { RDGPU_JNI_FN(void (*)(JNIEnv*, jarray, void*, jint), RDGPU_JNI_ReleasePrimitiveArrayCritical)(this, a, p, mode); }
    jboolean ExceptionCheck()
    { return RDGPU_JNI_FN(jboolean (*)(JNIEnv*), RDGPU_JNI_ExceptionCheck)(this); }
#undef RDGPU_JNI_FN
};
#else
typedef const struct JNINativeInterface_* JNIEnv;
#endif

#endif
