// jni_shim.cpp -- Java_readdy_impl_sim_top_TopGPU_cCreateSimulation on the
// C ABI (the reference's lib/ReaDDyGPU.cpp:31-503 protocol).
//
// Per frame: rdgpu_step(stepsPerFrame), download positions, call
// boolean frameCallback(int frame, float[] [N, (x,y,z,gpuIndex,readdyId) x N])
// (ReaDDyGPU.cpp:264-300), then read float[] cReactions
// [count, (readdyId, newType, x, y, z, gpuIndex) x count] (ReaDDyGPU.cpp:307-417):
// gpuIndex != -1 deletes that slot, newType != -1 appends a particle, then the
// survivors are compacted in order, the appended ones follow, and the state is
// re-uploaded and re-binned (rdgpu_set_particles).
//
// Environment (no reference counterpart): READDY_GPU_PRECISION=f32c selects
// the FP32-compensated engine (default: the plain FP64 drop-in);
// READDY_GPU_SEED sets the Philox seed (default 0; the reference seeds cuRAND
// with time(NULL), CudaSimulation.cu:773).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "readdy_b200.h"
#include "readdy_b200_inputs.h"
#include "readdy_b200_jni.h"

namespace {

std::string jstr(JNIEnv* env, jstring s)
{
    if (!s) return std::string();
    const char* c = env->GetStringUTFChars(s, nullptr);
    std::string r = c ? c : "";
    if (c) env->ReleaseStringUTFChars(s, c);
    return r;
}

bool file_has(const std::string& path, const char* tag)
{
    if (path.empty()) return false;
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    std::string s;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, n);
    fclose(f);
    return s.find(tag) != std::string::npos;
}

}  // namespace

extern "C" JNIEXPORT void JNICALL Java_readdy_impl_sim_top_TopGPU_cCreateSimulation(
    JNIEnv* env, jobject obj, jboolean testmode, jstring paramParticles, jstring tplgyPotentials,
    jstring paramGroups, jstring tplgyCoord, jstring tplgyGroups, jstring paramGlobal)
{
    const std::string pp = jstr(env, paramParticles), tp = jstr(env, tplgyPotentials);
    const std::string pgr = jstr(env, paramGroups), tc = jstr(env, tplgyCoord);
    const std::string tgr = jstr(env, tplgyGroups), pg = jstr(env, paramGlobal);

    // maxCutoff = 10 nm as the reference's JNI path hard-codes it (ReaDDyGPU.cpp:101);
    // used only for harmonic attractive/spring pairs, which have no own cutoff
    rdgpu_inputs_handle in = nullptr;
    if (rdgpu_inputs_read(pp.c_str(), tp.c_str(), pg.c_str(), tc.c_str(), 10.0, &in) != RDGPU_OK) {
        printf("error while reading input files: %s\n", rdgpu_inputs_error(nullptr));
        fflush(stdout);
        return;
    }
    rdgpu_system_desc desc;
    rdgpu_run_params run;
    rdgpu_inputs_desc(in, &desc, &run);
    int64_t n = rdgpu_inputs_count(in);
    std::vector<double> xyz(3 * n);
    std::vector<float> xyzf;
    std::vector<int32_t> types(n), ids(n);
    rdgpu_inputs_particles(in, xyz.data(), types.data(), ids.data());
    // particle groups -> bonded pairs (the reference's groups kernel,
    // CudaSimulation.cu:1829-1836, fed by GroupReader.cpp:13-40)
    std::vector<int32_t> bond_ij, bond_pot;
    std::vector<rdgpu_pair_pot> bond_pots;
    if (file_has(tgr, "<g ")) {
        if (rdgpu_inputs_read_groups(in, pgr.c_str(), tgr.c_str()) != RDGPU_OK) {
            printf("error while reading groups: %s\n", rdgpu_inputs_error(in));
            rdgpu_inputs_free(in);
            fflush(stdout);
            return;
        }
        int64_t nb = 0;
        int32_t np = 0, nu = 0;
        rdgpu_inputs_bond_counts(in, &nb, &np, &nu);
        bond_ij.resize(2 * nb);
        bond_pot.resize(nb);
        bond_pots.resize(np);
        rdgpu_inputs_bonds(in, bond_ij.data(), bond_pot.data(), bond_pots.data());
        if (nu > 0) printf("note: %d group potential(s) not handled by this core were skipped\n", nu);
    }
    rdgpu_inputs_free(in);
    const bool verbose = testmode || run.testmode;
    if (run.n_unsupported > 0)
        printf("note: %d potential(s) not handled by this core were skipped\n", run.n_unsupported);

    rdgpu_options opt;
    memset(&opt, 0, sizeof(opt));
    opt.device = run.device;
    const char* prec = getenv("READDY_GPU_PRECISION");
    opt.precision = (prec && strcmp(prec, "f32c") == 0) ? RDGPU_PREC_F32C : RDGPU_PREC_F64;
    const char* seed = getenv("READDY_GPU_SEED");
    opt.seed = seed ? strtoull(seed, nullptr, 10) : 0;
    rdgpu_handle h = nullptr;
    if (rdgpu_create(&desc, &opt, &h) != RDGPU_OK) {
        printf("error during initialization: %s\n", rdgpu_last_error(nullptr));
        fflush(stdout);
        return;
    }
    if (rdgpu_set_particles(h, nullptr, n, xyz.data(), types.data()) != RDGPU_OK ||
        (!bond_pot.empty() && rdgpu_set_bonds(h, (int64_t)bond_pot.size(), bond_ij.data(), bond_pot.data(),
                                              (int32_t)bond_pots.size(), bond_pots.data()) != RDGPU_OK)) {
        printf("error during initialization: %s\n", rdgpu_last_error(h));
        rdgpu_destroy(h);
        fflush(stdout);
        return;
    }
    // choose the neighbour search and capture the step graphs once, before
    // the frames (otherwise a handle tunes only on a call of >= 400 steps)
    if (rdgpu_autotune(h) != RDGPU_OK) {
        printf("error during initialization: %s\n", rdgpu_last_error(h));
        rdgpu_destroy(h);
        fflush(stdout);
        return;
    }
    jclass cls = env->GetObjectClass(obj);
    jmethodID mid = env->GetMethodID(cls, "frameCallback", "(I[F)Z");
    if (!mid) {
        printf("method frameCallback(I[F)Z not found\n");
        rdgpu_destroy(h);
        fflush(stdout);
        return;
    }
    jfieldID fid = env->GetFieldID(cls, "cReactions", "[F");
    printf("%lld frames with each %lld steps\n", (long long)run.n_frames, (long long)run.steps_per_frame);

    for (int64_t frame = 0; frame < run.n_frames; ++frame) {
        if (rdgpu_step(h, run.steps_per_frame) != RDGPU_OK) {
            printf("error: %s\n", rdgpu_last_error(h));
            break;
        }
        // the frame is float[] (ReaDDyGPU.cpp:264-292): download FP32 directly
        xyzf.resize(3 * n);
        if (rdgpu_get_particles_f32(h, xyzf.data(), types.data()) != RDGPU_OK) {
            printf("error while copying positions from device: %s\n", rdgpu_last_error(h));
            break;
        }
        if (verbose) printf("frame: %lld (step %lld)\n", (long long)frame, (long long)(frame * run.steps_per_frame));

        // positions to Java: [N, (x, y, z, gpuIndex, readdyId) x N]
        jfloatArray arr = env->NewFloatArray((jsize)(5 * n + 1));
        if (!arr) { printf("cant allocate the position array\n"); break; }
        jfloat* P = (jfloat*)env->GetPrimitiveArrayCritical(arr, nullptr);
        if (!P) { printf("cant get array pointer\n"); break; }
        P[0] = (jfloat)n;
        for (int64_t j = 0; j < n; ++j) {
            P[1 + 5 * j + 0] = xyzf[3 * j + 0];
            P[1 + 5 * j + 1] = xyzf[3 * j + 1];
            P[1 + 5 * j + 2] = xyzf[3 * j + 2];
            P[1 + 5 * j + 3] = (jfloat)j;
            P[1 + 5 * j + 4] = (jfloat)ids[j];
        }
        env->ReleasePrimitiveArrayCritical(arr, P, 0);
        jvalue args[2];
        args[0].i = (jint)frame;
        args[1].l = arr;
        jboolean ok = env->CallBooleanMethodA(obj, mid, args);
        env->DeleteLocalRef(arr);
        if (!ok || env->ExceptionCheck()) {
            printf("error in java\n");
            break;
        }
        if (!fid) continue;

        // reactions from Java
        jobject robj = env->GetObjectField(obj, fid);
        if (!robj) continue;
        jsize len = env->GetArrayLength(robj);
        std::vector<float> R(len > 0 ? len : 0);
        if (len > 0) {
            jfloat* rp = (jfloat*)env->GetPrimitiveArrayCritical(robj, nullptr);
            if (rp) {
                memcpy(R.data(), rp, len * sizeof(float));
                env->ReleasePrimitiveArrayCritical(robj, rp, 0);
            } else {
                R.clear();
            }
        }
        env->DeleteLocalRef(robj);
        if (R.empty() || R[0] <= 0) continue;
        int64_t count = (int64_t)R[0];
        if (1 + 6 * count > (int64_t)R.size()) {
            printf("error: cReactions holds %lld entries but announces %lld reactions\n", (long long)R.size(),
                   (long long)count);
            break;
        }
        // the readdy ids follow the edits on the host; the particles are edited
        // on the device (rdgpu_apply_edits), nothing is re-uploaded
        std::vector<char> gone(n, 0);
        std::vector<int32_t> added;
        bool bad = false;
        for (int64_t r = 0; r < count; ++r) {
            const float* e = &R[1 + 6 * r];
            int id = (int)e[0], newType = (int)e[1], index = (int)e[5];
            if (index != -1) {
                if (index < 0 || index >= n || gone[index]) { bad = true; break; }
                gone[index] = 1;
            }
            if (newType != -1) {
                if (newType < 0 || newType >= desc.n_types) { bad = true; break; }
                added.push_back(id);
            }
        }
        if (bad) {
            printf("error: invalid reaction entry in cReactions\n");
            break;
        }
        if (rdgpu_apply_edits(h, &R[1], count) != RDGPU_OK) {
            printf("error while applying reactions: %s\n", rdgpu_last_error(h));
            break;
        }
        std::vector<int32_t> nids;
        nids.reserve(ids.size() + added.size());
        for (int64_t i = 0; i < n; ++i)
            if (!gone[i]) nids.push_back(ids[i]);
        for (int32_t id : added) nids.push_back(id);
        ids.swap(nids);
        n = (int64_t)ids.size();
        xyz.resize(3 * n);
        types.resize(n);
    }
    rdgpu_destroy(h);
    printf("END\n");
    fflush(stdout);
}
