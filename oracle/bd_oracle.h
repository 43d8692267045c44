/*
 * bd_oracle.h -- CPU oracle for the ReaDDy Brownian-dynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * CPU semantics (the Java core: src/readdy/impl/sim/core/pot/potentials/P*.java,
 * bd/PotentialDisplacementComputer.java, bd/DiffusionEngine.java) plus the
 * GPU path's periodic minimum image and Euler-Maruyama update
 * (lib/ReaDDyGPU_Cpp/CudaKernels/CudaSimulation.cu:996-1002,1838-1919).
 * It is used by the tests (as the checker), by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg.  The product (readdygpu_b200) never links it.
 *
 * Parity is pinned against the reference's own JUnit known-answer tests
 * (test/readdy/impl/sim/core/pot/potentials/P2_HarmonicTest.java:135-176,
 * P1_DiskTest.java:136-251, bd/PotentialDisplacementComputerTest.java:155-306),
 * whose numbers are in tests/golden/reference_kats.json.
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H

#include <stdint.h>
#include "../include/readdy_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- single potentials, Java semantics (absolute coordinates) --------- */

/* gradient as the Java classes return it: -dV/dx1 (the force on particle 1).
   r0_pair is the collision radius sum of the pair (used when p->r0 < 0).
   Returns 0, or -1 for an unknown kind/subtype.                             */
int orc_pair_gradient(const rdgpu_pair_pot* p, double r0_pair,
                      const double x1[3], const double x2[3], double dist,
                      double grad[3], double* energy);

/* external potential force (-dV/dx) and energy at x for a particle of
   radius p_radius.                                                          */
int orc_ext_gradient(const rdgpu_ext_pot* p, double p_radius, const double x[3],
                     double grad[3], double* energy);

/* cutoff of potential p on a pair with collision radius sum r0_pair */
double orc_pair_cutoff(const rdgpu_pair_pot* p, double r0_pair, double max_cutoff);

/* ---- whole-system evaluation ------------------------------------------ */

/* Box-relative FP64 state exactly as the FP64 engine stores it:
   xrel = x - lo, wrapped into [0, L) on periodic axes.                      */
void orc_to_rel_f64(const rdgpu_system_desc* d, int64_t n, const double* xabs,
                    double* xrel);
/* FP32 state as the compensated engine stores it: hi = (float)xrel and the
   compensation c = hi - xrel (true position = hi - c).                       */
void orc_to_rel_f32(const rdgpu_system_desc* d, int64_t n, const double* xabs,
                    float* hi, float* comp);

/* Forces (-grad V, pair + external) and total energy at box-relative FP64
   positions; all forces from x(t).  n_threads <= 1: serial.                  */
int orc_forces_f64(const rdgpu_system_desc* d, int64_t n, const double* xrel,
                   const int32_t* types, double* forces, double* energy,
                   int n_threads);

/* Neighbour digest (count, wrapping sum of splitmix64(j)) with the FP64 or
   the FP32 predicate r^2 < rc^2, evaluated with the same non-fused
   arithmetic as the engine.  Brute force O(N^2): small systems only.        */
void orc_neighbor_digest_f64(const rdgpu_system_desc* d, int64_t n,
                             const double* xrel, const int32_t* types,
                             int32_t* counts, uint64_t* hashes);
void orc_neighbor_digest_f32(const rdgpu_system_desc* d, int64_t n,
                             const float* xrel, const int32_t* types,
                             int32_t* counts, uint64_t* hashes);

/* The same digests from a cell list, OpenMP over n_threads threads: for
   large systems (the benchmark configurations at their full sizes).         */
void orc_neighbor_digest_cells_f64(const rdgpu_system_desc* d, int64_t n,
                                   const double* xrel, const int32_t* types,
                                   int32_t* counts, uint64_t* hashes, int n_threads);
void orc_neighbor_digest_cells_f32(const rdgpu_system_desc* d, int64_t n,
                                   const float* xrel, const int32_t* types,
                                   int32_t* counts, uint64_t* hashes, int n_threads);

/* One Euler-Maruyama step with injected noise (3 per particle):
   x <- x + D dt/(kB T) F + sqrt(2 D dt) xi, then periodic wrap.
   Returns 0, or RDGPU_ERR_JUMP if a particle moved more than a box length.  */
/* Adds the forces and energy of bonded pairs (particle groups).           */
int orc_bond_forces_f64(const rdgpu_system_desc* d, int64_t n, const double* x, const int32_t* types,
                        int64_t nb, const int32_t* ij, const int32_t* pot, int32_t npots,
                        const rdgpu_pair_pot* pots, double* forces, double* energy);

int orc_step_f64(const rdgpu_system_desc* d, int64_t n, double* xrel,
                 const int32_t* types, const double* noise, int n_threads);

/* RDF counts with the FP64 bin predicate on stored positions (double or
   float), all ordered pairs i != j.  counts has n_types^2 * nbins entries and
   is ADDED to.                                                               */
void orc_rdf_counts_f64(const rdgpu_system_desc* d, int64_t n, const double* xrel,
                        const int32_t* types, int32_t nbins, double rmax,
                        uint64_t* counts);
void orc_rdf_counts_f32(const rdgpu_system_desc* d, int64_t n, const float* xrel,
                        const int32_t* types, int32_t nbins, double rmax,
                        uint64_t* counts);
/* squared bin edges (nbins+1 values) used by both sides */
void orc_rdf_edges2(int32_t nbins, double rmax, double* edges2);

/* ---- random numbers ---------------------------------------------------- */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* the three N(0,1) draws of particle `index` at step `step` (Box-Muller on
   the four Philox words), FP64                                              */
void orc_bd_normals(uint64_t seed, int64_t step, int64_t index, double out[3]);

uint64_t orc_splitmix64(uint64_t x);

/* ---- CPU baseline: cell-list BD steps with Philox noise ---------------- */

/* Runs nsteps steps on box-relative FP64 positions, OpenMP over particles
   with n_threads threads.  Returns 0 or a negative RDGPU_ERR_* code.          */
int orc_run_steps_f64(const rdgpu_system_desc* d, int64_t n, double* xrel,
                      const int32_t* types, uint64_t seed, int64_t first_step,
                      int64_t nsteps, int n_threads);

int orc_max_threads(void);

/* Config-3 input for the benchmark's reference arm: random sequential
   insertion of n spheres of diameter diam into the periodic box [0,L)^3,
   SplitMix64 proposals from `seed`; returns the number placed.              */
int64_t orc_rsa_spheres(int64_t n, double L, double diam, uint64_t seed, int64_t max_attempts, double* xyz);

#ifdef __cplusplus
}
#endif
#endif
