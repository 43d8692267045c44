/*
 * readdy_b200.h -- C ABI of the B200-native ReaDDy Brownian-dynamics engine.
 *
 * This is the boundary that replaces the reference's native GPU core
 * (lib/ReaDDyGPU_Cpp/CudaKernels/CudaSimulation.cuh:39-116, class CudaSimulation,
 * driven by lib/ReaDDyGPU.cpp:31 through JNI).  The JNI entry point itself
 * (Java_readdy_impl_sim_top_TopGPU_cCreateSimulation, lib/simulationGPU.h:15-16)
 * is declared in readdy_b200_jni.h and is built on top of these functions.
 *
 * Conventions
 *   - Plain C types only; every pointer argument is a HOST pointer unless its
 *     name ends in _dev.  The library owns all device memory of a handle.
 *   - Every function returns an int status: RDGPU_OK (0) or a negative
 *     RDGPU_ERR_* code (the reference's CudaSimulation methods return 0 = ok,
 *     1 = error, CudaSimulation.cu:138-455).  rdgpu_last_error() gives the text.
 *   - Units follow ReaDDy: nm, s, kJ/mol, K; D in nm^2/s.
 *   - Particles are addressed by their index in the arrays handed to
 *     rdgpu_set_particles (the reference's "gpuIndex", ReaDDyGPU.cpp:288).
 *     All per-particle outputs come back in that order.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     call fails with RDGPU_ERR_CUDA.
 */
#ifndef READDY_B200_H
#define READDY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RDGPU_ABI_VERSION 1

#define RDGPU_MAX_TYPES          16
#define RDGPU_MAX_PAIR_POTS      32
#define RDGPU_MAX_EXT_POTS       16
#define RDGPU_MAX_POTS_PER_PAIR  4

/* status codes */
#define RDGPU_OK              0
#define RDGPU_ERR_ARG        -1   /* invalid argument / description          */
#define RDGPU_ERR_CUDA       -2   /* CUDA runtime error or no device          */
#define RDGPU_ERR_OVERFLOW   -3   /* reserved; not returned                   */
#define RDGPU_ERR_NONFINITE  -4   /* a particle position became NaN/Inf       */
#define RDGPU_ERR_STATE      -5   /* call out of order (e.g. no particles)    */
#define RDGPU_ERR_NOMEM      -6   /* device allocation failed                 */
#define RDGPU_ERR_JUMP       -7   /* a particle moved more than a box length  */

/* precision of a handle */
#define RDGPU_PREC_F64   0   /* plain FP64 positions and forces (the drop-in)      */
#define RDGPU_PREC_F32C  1   /* FP32 forces, Kahan-compensated FP32 positions      */

/* pair (order-two) potential kinds */
#define RDGPU_P2_HARMONIC        1  /* P2_Harmonic.java:144-234                          */
#define RDGPU_P2_WEAK_PIECEWISE  2  /* P2_WeakInteractionPiecewiseHarmonic.java:114-206 */

/* external (order-one) potential kinds */
#define RDGPU_P1_DISK      1   /* P1_Disk.java:112-320      */
#define RDGPU_P1_CYLINDER  2   /* P1_Cylinder.java:109-340  */
#define RDGPU_P1_SPHERE    3   /* P1_Sphere.java:119-340    */
#define RDGPU_P1_CUBE      4   /* P1_Cube.java (box wall)   */

/* subtypes (the reference's subtype ids, Simulation.cpp:102-205) */
#define RDGPU_SUB_ATTRACTIVE  1
#define RDGPU_SUB_REPULSIVE   2
#define RDGPU_SUB_SPRING      3   /* harmonic only  */
#define RDGPU_SUB_MEMBRANE    4   /* sphere only    */

typedef struct {
    int32_t kind;                 /* RDGPU_P2_*                                       */
    int32_t subtype;              /* RDGPU_SUB_* (ignored for WEAK_PIECEWISE)          */
    double  k;                    /* forceConst [kJ/mol/nm^2]                          */
    double  r0;                   /* < 0: use the pair's collision radius sum
                                     (P2_Harmonic.java:124-128); >= 0: explicit r0   */
    double  length;               /* WEAK_PIECEWISE: well width l                      */
    double  depth;                /* WEAK_PIECEWISE: well depth d [kJ/mol]             */
    uint8_t pairs[RDGPU_MAX_TYPES * RDGPU_MAX_TYPES]; /* 1: acts on (t1,t2); symmetric */
} rdgpu_pair_pot;

typedef struct {
    int32_t kind;                 /* RDGPU_P1_*                                       */
    int32_t subtype;              /* RDGPU_SUB_*                                      */
    double  k;                    /* forceConst                                        */
    double  center[3];            /* DISK, CYLINDER, SPHERE                            */
    double  normal[3];            /* DISK, CYLINDER (normalised by the library)        */
    double  radius;               /* DISK, CYLINDER, SPHERE                            */
    double  height;               /* CYLINDER                                          */
    double  origin[3];            /* CUBE                                              */
    double  extension[3];         /* CUBE                                              */
    int32_t consider_radius;      /* SPHERE/CUBE: use the particle radius (default 1)  */
    uint8_t types[RDGPU_MAX_TYPES]; /* 1: acts on particles of that type               */
} rdgpu_ext_pot;

typedef struct {
    int32_t n_types;
    double  D[RDGPU_MAX_TYPES];                 /* diffusion constant [nm^2/s]      */
    /* coll_radius[i*RDGPU_MAX_TYPES+j]: radius of type i when in contact with j.
       Pair r0 = coll_radius[i][j] + coll_radius[j][i]
       (ParticleParametersFactory.java:167-170).                                     */
    double  coll_radius[RDGPU_MAX_TYPES * RDGPU_MAX_TYPES];
    /* default collision radius of a type, the pRadius handed to external
       potentials (DiffusionEngine.java:105, defaultCollRadiusMap).                  */
    double  p_radius[RDGPU_MAX_TYPES];
    int32_t n_pair;
    rdgpu_pair_pot pair[RDGPU_MAX_PAIR_POTS];
    int32_t n_ext;
    rdgpu_ext_pot ext[RDGPU_MAX_EXT_POTS];
    double  kB;                                 /* kJ/(mol K)                       */
    double  T;                                  /* K                                */
    double  dt;                                 /* BD time step [s]                 */
    double  lo[3], hi[3];                       /* lattice bounds [nm]              */
    int32_t periodic[3];                        /* 1: periodic along that axis      */
    /* cutoff used for harmonic attractive/spring pairs, which have no natural
       cutoff (the reference uses maxCutoff, ReaDDyGPU.cpp:101).  0: none allowed. */
    double  max_cutoff;
    /* cell edge; 0 = the largest pair cutoff.  Must be >= that cutoff.             */
    double  cell_size;
} rdgpu_system_desc;

/* one system of a batch: its own box and Philox seed */
typedef struct {
    double   lo[3], hi[3];
    int32_t  periodic[3];
    uint64_t seed;
} rdgpu_box;

/* Neighbour search of the step.  CELLS walks the 27-cell neighbourhood of
   every particle in every step.  LIST evaluates a pair list of radius
   rc + skin per type pair that is rebuilt (with a re-sort by cell) when a
   pair closer than its cutoff is missing from it, or a particle has moved
   more than about skin since the last build; after every step the particles
   that moved more than about skin/2 have their current neighbourhood
   checked against the list.  The pair set and the FP32 forces are identical
   to CELLS.  AUTO starts with CELLS and, at the first rdgpu_step of >= 4 x
   graph_steps steps, times CELLS and LIST at skins of 0.1 .. 0.5 x rc_max on
   the handle's particles and keeps the fastest.  Every energy, force, digest
   or RDF evaluation in LIST mode re-sorts and rebuilds the list (one build in
   list_builds).                                                                */
#define RDGPU_NB_AUTO  0
#define RDGPU_NB_CELLS 1
#define RDGPU_NB_LIST  2

typedef struct {
    int32_t  precision;           /* RDGPU_PREC_*                                      */
    int32_t  device;              /* CUDA device ordinal                               */
    int32_t  neighbour_mode;      /* RDGPU_NB_*                                        */
    int32_t  graph_steps;         /* steps captured per CUDA graph; 0 = 100, <0 = off  */
    double   skin;                /* pair-list skin [nm] for RDGPU_NB_LIST; 0 = 0.25 x
                                     the largest pair cutoff                           */
    uint64_t seed;                /* Philox seed of a single-system handle             */
} rdgpu_options;

typedef struct {
    double   energy;                    /* total potential energy [kJ/mol], FP64     */
    double   msd[RDGPU_MAX_TYPES];      /* mean squared displacement per type [nm^2] */
    int64_t  count[RDGPU_MAX_TYPES];    /* particles per type                        */
    int64_t  step;                      /* steps done since rdgpu_set_particles      */
    int32_t  neighbour_mode;            /* RDGPU_NB_CELLS or RDGPU_NB_LIST in effect */
    int32_t  list_builds;               /* pair-list builds so far (before this call's
                                           energy evaluation, which adds one)          */
    double   skin;                      /* pair-list skin in effect [nm], 0: cells   */
    int32_t  list_capacity;             /* pair-list slots per particle              */
    int32_t  list_entry_bytes;          /* 2: partners as 16-bit offsets, 4: as 32-bit
                                           indices (an offset did not fit 16 bits);
                                           0 with the cell walk                       */
} rdgpu_metrics;

typedef struct rdgpu_engine* rdgpu_handle;

/* ---- lifetime ---------------------------------------------------------- */

/* Single system; box from desc->lo/hi/periodic.  Replaces
   CudaSimulation::CudaSimulation + initialize (CudaSimulation.cu:138-455).       */
int rdgpu_create(const rdgpu_system_desc* desc, const rdgpu_options* opt,
                 rdgpu_handle* out);

/* A batch of independent replicate systems that share the particle types and
   potentials of desc but each have their own box and seed.  All systems step
   together in one persistent launch per step.  No reference counterpart (the
   reference runs one system per process).                                     */
int rdgpu_create_batch(const rdgpu_system_desc* desc, int32_t n_systems,
                       const rdgpu_box* boxes, const rdgpu_options* opt,
                       rdgpu_handle* out);

int rdgpu_destroy(rdgpu_handle h);

/* Text of the last error on this handle (or of the last failed create when
   h is NULL).  Valid until the next call on the handle.                       */
const char* rdgpu_last_error(rdgpu_handle h);

/* ---- state ------------------------------------------------------------- */

/* Upload particles (absolute coordinates, xyz interleaved) and bin them.
   offsets: n_systems+1 prefix offsets into the arrays (NULL for a single
   system).  Resets the step counter, the MSD origin and the RDF accumulator.
   Replaces copyPosToDevice + copyTypesToDevice + createNeighborList +
   copyNeighborListToDevice (CudaSimulation.cu:562-626, ReaDDyGPU.cpp:421-442). */
int rdgpu_set_particles(rdgpu_handle h, const int64_t* offsets, int64_t n_total,
                        const double* xyz, const int32_t* types);

/* Download positions (absolute, xyz interleaved) and types in particle-index
   order.  Replaces copyPosFromDevice (CudaSimulation.cu:2309 ff).             */
int rdgpu_get_particles(rdgpu_handle h, double* xyz, int32_t* types);

/* The same with FP32 coordinates, as the reference moves them
   (copyPosToDevice / copyPosFromDevice take float, CudaSimulation.cu:562-626,
   and the JNI frame is float[], ReaDDyGPU.cpp:264-292): half the bytes over
   PCIe.  Upload is exact into either precision (an FP32C handle starts with
   zero compensation); download rounds each coordinate to FP32.              */
int rdgpu_set_particles_f32(rdgpu_handle h, const int64_t* offsets, int64_t n_total,
                            const float* xyz, const int32_t* types);
int rdgpu_get_particles_f32(rdgpu_handle h, float* xyz, int32_t* types);

int rdgpu_num_particles(rdgpu_handle h, int64_t* n_total);

/* Bonded pairs of particle groups (ReaDDy group potentials): each bond
   applies one pair potential to two particles at any distance (minimum
   image).  ij: 2 x n_bonds particle indices; pot: n_bonds indices into
   pots[n_pots] (kind HARMONIC or WEAK_INTERACTION_PIECEWISE_HARMONIC; r0 < 0
   takes the collision-radius sum of the two types; `pairs` is not used).
   Replaces the reference's groups kernel (CudaSimulation.cu:1829-1836,
   launched at :2454) with the Java group semantics: every listed pair with
   its own potential and each particle's own type (the reference passes
   particle 1's type twice and applies potential 0 to every pair).  The
   bonds replace any earlier ones; rdgpu_set_particles clears them;
   rdgpu_apply_edits drops the bonds of deleted particles and renumbers the
   rest.  Single-system handles only.                                          */
int rdgpu_set_bonds(rdgpu_handle h, int64_t n_bonds, const int32_t* ij, const int32_t* pot, int32_t n_pots,
                    const rdgpu_pair_pot* pots);

/* Applies one frame's reaction edits on the device, in the layout of ReaDDy's
   cReactions field: count entries of (readdyId, newType, x, y, z, gpuIndex).
   gpuIndex != -1 deletes that particle; newType != -1 appends a particle of
   that type at (x, y, z), absolute.  Survivors keep their order, appended
   particles follow, and particle indices become 0 .. n-1 in that order.
   Survivors keep their state (FP32 compensation, image counters, MSD
   origin); appended particles start their MSD at their position; the step
   count and the RDF accumulator continue.  Invalid entries (index out of
   range or repeated, type out of range, non-integer type or index) leave the
   state unchanged and return RDGPU_ERR_ARG.  Single-system handles only.
   Replaces the host-side edit, compaction and re-upload of the reference
   (ReaDDyGPU.cpp:303-461), which moved every particle through host memory.   */
int rdgpu_apply_edits(rdgpu_handle h, const float* edits, int64_t count);

/* ---- dynamics ---------------------------------------------------------- */

/* Advance every system by nsteps Brownian-dynamics steps (Philox noise keyed
   by (seed, step, particle index)).  Replaces the per-step launch sequence
   orderOne/warpOrderTwo/groups/update (CudaSimulation.cu:2309-2476).          */
int rdgpu_step(rdgpu_handle h, int64_t nsteps);

/* One step that takes its Gaussian noise from the host array noise
   (3 per particle, particle-index order) instead of Philox.  For parity
   testing against the CPU path with identical noise.                         */
int rdgpu_step_with_noise(rdgpu_handle h, const double* noise);

/* Philox seed of system `sys` (single system: 0). */
int rdgpu_set_seed(rdgpu_handle h, int32_t sys, uint64_t seed);

/* ---- diagnostics and observables -------------------------------------- */

/* Forces F = -grad V (pair + external) at the current positions, particle-index
   order, 3 per particle, and the total energy.  Uses the same device code as
   the step kernel.                                                            */
int rdgpu_forces(rdgpu_handle h, double* forces, double* energy);

/* Per particle: number of neighbours j != i with r_ij^2 < rc(ti,tj)^2 and the
   wrapping sum of splitmix64(index_j) over them (order independent).          */
int rdgpu_neighbor_digest(rdgpu_handle h, int32_t* counts, uint64_t* hashes);

/* The Gaussian noise rdgpu_step would draw at step `step` (3 per particle). */
int rdgpu_debug_noise(rdgpu_handle h, int64_t step, double* noise);

/* RDF pair counts: for every ordered pair (i,j), i != j, in the same system
   with r < rmax, counts[(ti*n_types+tj)*nbins + bin] += 1 where bin is the k
   with (k*w)^2 <= r^2 < ((k+1)*w)^2, w = rmax/nbins (FP64 predicate on the
   stored positions).  Equivalent to the reference's per-unordered-pair
   increment of [ti][tj] and [tj][ti] (CudaSimulation.cu:1815-1818).
   accumulate != 0 adds to the device accumulator (one "frame"); the host
   array then receives the accumulated counts; accumulate == 0 returns only
   this frame's counts and leaves the accumulator alone.  The frame sorts
   copies of the particles into a grid of its own (cells of edge >= rmax)
   and leaves the simulation's state and lists as they are; when a periodic
   box edge holds fewer than 3 such cells it re-sorts the simulation's
   particles on their own cells instead (a list build in pair-list mode).    */
int rdgpu_rdf(rdgpu_handle h, int32_t nbins, double rmax, int32_t accumulate,
              uint64_t* counts, int64_t* frames);

/* g(r) of the accumulator, normalised in FP64:
   g[ti][tj][k] = counts / (frames * N_ti * (N_tj - [ti==tj]) / V * shell_k),
   shell_k = 4/3 pi ((k+1)^3 - k^3) w^3, V the box volume (single system).     */
int rdgpu_rdf_normalized(rdgpu_handle h, double* g);

int rdgpu_metrics_get(rdgpu_handle h, rdgpu_metrics* m);

/* ---- RDF counts without device allocation ------------------------------ */

/* Limits of rdgpu_rdf_counts_noalloc (its scratch is a fixed static array). */
#define RDGPU_NOALLOC_MAX_PARTICLES  65536
#define RDGPU_NOALLOC_MAX_CELLS      131072
#define RDGPU_NOALLOC_MAX_BINS       4096

/* RDF pair counts of one periodic/non-periodic box for callers that cannot
   allocate device memory: a host runtime that owns the device memory pool
   (a JVM handing out direct buffers, a plug-in that must not change the
   device footprint after start-up).  No counterpart in the reference.
   xyz_dev (3n doubles, absolute coordinates) and types_dev (n ints) are
   device pointers the caller owns; counts_dev (n_types^2 * nbins uint64) is
   the device output, overwritten with this call's counts -- the same counts
   rdgpu_rdf(accumulate = 0) gives for these particles in an FP64 handle with
   the same box.  Scratch: a static device array of about 3.7 MB held by every
   GPU that loads the library; the first call on a device resolves its
   address (make that call before any stream capture).  Calls on the same
   device share the scratch: calls that overlap on the GPU race.  Runs on
   `stream` (a cudaStream_t, NULL = default) and synchronises it before
   returning.  Rejects n > RDGPU_NOALLOC_MAX_PARTICLES, nbins >
   RDGPU_NOALLOC_MAX_BINS and boxes needing more than RDGPU_NOALLOC_MAX_CELLS
   cells with RDGPU_ERR_ARG; rdgpu_last_error(NULL) gives the reason.         */
int rdgpu_rdf_counts_noalloc(const double* xyz_dev, const int32_t* types_dev, int64_t n,
                             int32_t n_types, const double lo[3], const double hi[3],
                             const int32_t periodic[3], int32_t nbins, double rmax,
                             uint64_t* counts_dev, void* stream);

/* ---- device-resident access for benchmarks ----------------------------- */

/* The cudaStream_t the handle launches on (as void*). */
void* rdgpu_stream(rdgpu_handle h);

/* Kernels launched by this handle so far (for launch accounting). */
int64_t rdgpu_launch_count(rdgpu_handle h);

/* Runs nsteps steps one launch at a time (no CUDA graph) with CUDA events on
   the handle's stream around the step kernel and around what follows it in
   the step: the counting sort (scan + scatter) of the cell walk, or the
   list check, re-sort and list build of the pair list (no-ops in steps that
   need no rebuild).  Steps are queued in batches of 16 without a
   synchronisation in between, so each event pair brackets a kernel that was
   already queued; the first step of a batch (queued on an idle stream) is not
   counted.  Returns the mean durations per step in milliseconds.  The state
   advances exactly as with rdgpu_step.  No reference counterpart
   (measurement hook).                                                        */
int rdgpu_step_profile(rdgpu_handle h, int64_t nsteps, double* step_kernel_ms, double* sort_ms);

/* Runs the neighbour-search autotuner of an RDGPU_NB_AUTO handle now, on its
   current particles, instead of at its first long rdgpu_step (once per
   handle), then captures the CUDA graph of the mode in effect, so that the
   next rdgpu_step pays neither.  The state and step count are unchanged.  No
   reference counterpart.                                                     */
int rdgpu_autotune(rdgpu_handle h);

#ifdef __cplusplus
}
#endif
#endif /* READDY_B200_H */
