/*
 * readdy_b200_inputs.h -- reader for the ReaDDy input files the native GPU
 * core consumes, without Xerces-C.  Replaces the Xerces handlers of lib/ReaDDyGPU_Cpp/XMLHandler
 * (XMLReader.cpp:19-67, GlobalParametersHandler.cpp:54-146,
 * ParticleParametersHandler.cpp:111-160, PotentialParametersHandler.cpp:51-79,
 * CoordReader.cpp:16-65) and the parse step Simulation::parse
 * (Simulation.cpp:206-280).
 */
#ifndef READDY_B200_INPUTS_H
#define READDY_B200_INPUTS_H
#include <stdint.h>
#include "readdy_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct rdgpu_inputs* rdgpu_inputs_handle;

typedef struct {
    int64_t n_frames;         /* <nSimulationSteps> (ReaDDyGPU.cpp:209 frame loop)           */
    int64_t steps_per_frame;  /* round(<dt> / <dtOpenMM>) (XMLReader.cpp:67)                 */
    double  dt_frame;         /* <dt>: reaction / frame interval [s]                          */
    int32_t device;           /* <cudaDeviceIndex> or <cudaDevice>                            */
    int32_t testmode;         /* <testmode>                                                   */
    int32_t n_unsupported;    /* potentials skipped (unknown type, id-bound pairs)            */
    int32_t reserved;
} rdgpu_run_params;

/* Parse the input files (groups: rdgpu_inputs_read_groups).  Returns
   RDGPU_OK or RDGPU_ERR_ARG with a message in rdgpu_inputs_error(NULL).      */
int rdgpu_inputs_read(const char* param_particles, const char* tplgy_potentials,
                      const char* param_global, const char* tplgy_coordinates,
                      double max_cutoff, rdgpu_inputs_handle* out);
int rdgpu_inputs_desc(rdgpu_inputs_handle h, rdgpu_system_desc* desc, rdgpu_run_params* run);
int64_t rdgpu_inputs_count(rdgpu_inputs_handle h);
/* xyz: 3n doubles, types: n, ids: n (the ReaDDy particle ids)               */
int rdgpu_inputs_particles(rdgpu_inputs_handle h, double* xyz, int32_t* types, int32_t* ids);
/* Particle groups (param_groups.xml, tplgy_groups.xml) as bonded pairs for
   rdgpu_set_bonds: the k-th <particleGroup> is group type k; each of its
   HARMONIC / WEAK_INTERACTION_PIECEWISE_HARMONIC potentials acts on the
   internal-id pairs of its affectedInternalIdPairs; each <g type="k"
   internalAndParticleId="[[u,id];...]"> instance maps internal ids to the
   ReaDDy particle ids of tplgy_coordinates.  Replaces GroupParametersHandler
   (GroupParametersHandler.cpp:41-190) and GroupReader (GroupReader.cpp:13-40).
   Other group potential types are counted in n_unsupported and skipped.     */
int rdgpu_inputs_read_groups(rdgpu_inputs_handle h, const char* param_groups, const char* tplgy_groups);
int rdgpu_inputs_bond_counts(rdgpu_inputs_handle h, int64_t* n_bonds, int32_t* n_pots, int32_t* n_unsupported);
/* ij: 2 x n_bonds gpu indices (positions in tplgy_coordinates), pot: n_bonds,
   pots: n_pots                                                               */
int rdgpu_inputs_bonds(rdgpu_inputs_handle h, int32_t* ij, int32_t* pot, rdgpu_pair_pot* pots);
const char* rdgpu_inputs_error(rdgpu_inputs_handle h);
void rdgpu_inputs_free(rdgpu_inputs_handle h);

#ifdef __cplusplus
}
#endif
#endif
