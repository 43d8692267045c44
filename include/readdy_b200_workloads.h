/*
 * readdy_b200_workloads.h -- synthetic input generation for the benchmark
 * workloads (no counterpart in the reference, which reads coordinates from
 * tplgy_coordinates.xml, lib/ReaDDyGPU_Cpp/XMLHandler/CoordReader.cpp:16-65).
 */
#ifndef READDY_B200_WORKLOADS_H
#define READDY_B200_WORKLOADS_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Random sequential insertion of n spheres of diameter `diam` into the
   periodic box [0,L)^3 without overlap (centre distance >= diam), using a
   SplitMix64 stream seeded with `seed`.  Writes xyz (3n doubles).  Returns the
   number placed (< n when max_attempts proposals were exhausted).           */
int64_t rdgpu_rsa_spheres(int64_t n, double L, double diam, uint64_t seed,
                          int64_t max_attempts, double* xyz);

#ifdef __cplusplus
}
#endif
#endif
