/*
 * readdy_b200_jni.h -- the JNI entry point of the native GPU core, exported
 * by libCReaDDyGPU.so (loaded by System.loadLibrary("CReaDDyGPU"),
 * src/readdy/impl/sim/top/TopGPU.java:485).
 *
 * Same symbol and signature as the reference's lib/simulationGPU.h:15-16
 * (Java method readdy.impl.sim.top.TopGPU.cCreateSimulation, signature
 * (ZLjava/lang/String;Ljava/lang/String;Ljava/lang/String;Ljava/lang/String;
 * Ljava/lang/String;Ljava/lang/String;)V), implemented on the C ABI of
 * readdy_b200.h.  Protocol as lib/ReaDDyGPU.cpp:31-503: per frame of
 * stepsPerFrame steps it calls boolean frameCallback(int, float[]) with
 * [N, (x, y, z, gpuIndex, readdyId) x N] and then applies the edits in the
 * field float[] cReactions = [count, (readdyId, newType, x, y, z, gpuIndex) x
 * count]; a false return ends the run.  Errors are printed and end the call
 * (the function is void, as in the reference).
 */
#ifndef READDY_B200_JNI_H
#define READDY_B200_JNI_H
#ifdef RDGPU_USE_SYSTEM_JNI
#include <jni.h>
#else
#include "readdy_b200_jni_types.h"
#endif
#ifdef __cplusplus
extern "C" {
#endif

JNIEXPORT void JNICALL Java_readdy_impl_sim_top_TopGPU_cCreateSimulation(
    JNIEnv* env, jobject self, jboolean testmode, jstring paramParticles, jstring tplgyPotentials,
    jstring paramGroups, jstring tplgyCoord, jstring tplgyGroups, jstring paramGlobal);

#ifdef __cplusplus
}
#endif
#endif
