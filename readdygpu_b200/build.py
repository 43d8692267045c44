"""Builds the in-tree shared libraries.

    python readdygpu_b200/build.py [--force]

(run by path, not with -m: importing the package would load the library that
is about to be rebuilt)

  readdygpu_b200/libreaddy_b200.so   engine: hand-written CUDA for sm_100a + C ABI
  readdygpu_b200/libreaddy_workloads.so  seeded synthetic benchmark inputs
  readdygpu_b200/libCReaDDyGPU.so    the JNI entry point of the reference's
                                     native core on top of the C ABI, the input
                                     reader and the output writers
Every CUDA source is compiled with -gencode arch=compute_100a,code=sm_100a.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_engine(force=False):
    out = os.path.join(HERE, "libreaddy_b200.so")
    deps = [os.path.join(CSRC, f) for f in ("engine.cu", "engine_kernels.cuh", "engine_device.cuh", "rdf_noalloc.cu")]
    deps.append(os.path.join(ROOT, "include", "readdy_b200.h"))
    if force or _stale(out, deps):
        _run([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                              os.path.join(CSRC, "engine.cu"), os.path.join(CSRC, "rdf_noalloc.cu"), "-o", out])
    return out


def build_jni(force=False):
    srcs = [os.path.join(CSRC, f) for f in ("jni_shim.cpp", "xml_input.cpp", "output.cpp")]
    if not all(os.path.exists(s) for s in srcs):
        return None
    out = os.path.join(HERE, "libCReaDDyGPU.so")
    deps = srcs + [os.path.join(CSRC, "xml_input.h")] + [
        os.path.join(ROOT, "include", h) for h in ("readdy_b200.h", "readdy_b200_jni.h",
                                                    "readdy_b200_jni_types.h", "readdy_b200_inputs.h",
                                                    "readdy_b200_output.h")] + [
        os.path.join(HERE, "libreaddy_b200.so")]
    if force or _stale(out, [d for d in deps if os.path.exists(d)]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall"] + srcs +
             ["-I", os.path.join(ROOT, "include"), "-L", HERE, "-lreaddy_b200",
              "-Wl,-rpath,$ORIGIN", "-o", out])
    return out


def build_workloads(force=False):
    src = os.path.join(CSRC, "workloads.cpp")
    out = os.path.join(HERE, "libreaddy_workloads.so")
    if force or _stale(out, [src, os.path.join(ROOT, "include", "readdy_b200_workloads.h")]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", src,
              "-I", os.path.join(ROOT, "include"), "-o", out])
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    build_engine(force)
    build_workloads(force)
    build_jni(force)


if __name__ == "__main__":
    main()
