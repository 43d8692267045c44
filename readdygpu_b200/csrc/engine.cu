// engine.cu -- host side of the B200 Brownian-dynamics engine and the C ABI
// declared in include/readdy_b200.h.
//
// Replaces the reference's CudaSimulation host wrapper
// (lib/ReaDDyGPU_Cpp/CudaKernels/CudaSimulation.cu:138-626, 2309-2476):
// device state, cell binning, per-step launches.  One stream per handle; the
// steps of rdgpu_step are replayed from a captured CUDA graph of
// step_kernel -> scan_tiles -> scan_apply -> scatter per step.
#include <algorithm>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/readdy_b200.h"
#include "engine_kernels.cuh"

using namespace rdgpu;

namespace {
thread_local std::string g_create_error;
constexpr int kStepBlock = 128;    // cell-walk step kernel
constexpr int kListBlock = 128;    // pair-list step kernel
// internal: do_steps_list stopped early so that do_steps re-tunes (never returned by the ABI)
constexpr int RDGPU_OK_CONTINUE = 1;
// hot particles (moved more than about skin/2 since the build) the list check
// looks at after a step, at most (fewer for small handles); with more, the
// step rebuilds the list instead
constexpr int kHotMax = 8192;
// hot_max = npart / kHotDiv (at least 8, at most kHotMax)
constexpr long long kHotDiv = 300;
// the list check: blocks of 8 warps, one warp per hot particle at a time, at
// most 512 blocks (two hot particles per warp at the cap of 8192; grids of
// 128, 256 and 1019 blocks measured slower per step on config 4)
constexpr int kCheckBlock = 256;
constexpr int kCheckBlocks = 512;
}  // namespace

std::string& rdgpu_global_error() { return g_create_error; }

// the opaque handle type of the C ABI
struct rdgpu_engine {
    int prec = RDGPU_PREC_F64;
    int device = 0;
    cudaStream_t stream = nullptr;
    rdgpu_system_desc desc{};
    rdgpu_options opt{};
    int nsys = 0;
    bool value_image = false;            // some periodic axis has fewer than 3 cells
    bool hrep = false;                   // only single harmonic-repulsion pair terms
    std::vector<rdgpu_box> boxes;
    std::vector<SysDev> sys_h;
    SysDev* sys_d = nullptr;
    void* tab_d = nullptr;
    void* ext_d = nullptr;
    int n_ext = 0;
    // cells
    long long ncells_tot = 0;
    int ntiles = 0;
    int* start = nullptr;                // ncells_tot + 1
    int* counts = nullptr;               // ncells_tot
    int* tile_sum = nullptr;             // ntiles
    // particles
    long long npart_tot = 0, cap_particles = 0;
    std::vector<long long> part_off;     // n_sys + 1
    std::vector<int> types_h;            // by global index (host copy, see sync_types)
    bool types_h_valid = false;          // types_h matches the device state
    void* bufA[2] = {nullptr, nullptr};  // two state buffers; FP32: pos, FP64: records
    void* bufB[2] = {nullptr, nullptr};  // FP32: aux
    int cur = 0;                         // the buffer that holds the current state
    int* tcell = nullptr;
    int* tslot = nullptr;
    unsigned short* sys_of = nullptr;
    double* x0_d = nullptr;              // MSD origin, box-relative unwrapped
    double* vec_d = nullptr;             // 3N doubles scratch
    double* val_d = nullptr;             // N doubles scratch
    int* ityp_d = nullptr;               // N ints scratch
    unsigned long long* u64_d = nullptr; // N scratch
    int* ed_flag = nullptr;              // reaction edits: deleted flag, keep flag, new id by old id
    int* ed_keep = nullptr;
    int* ed_newid = nullptr;
    int* ed_tile = nullptr;              // tile sums of the id scan
    void* ed_buf = nullptr;              // deleted indices and appended particles of one frame
    size_t ed_buf_bytes = 0;
    // bonded pairs (particle groups)
    int* inv = nullptr;                  // sorted index of each particle id
    long long nbonds = 0;
    int* bstart = nullptr;               // CSR by particle id
    int* bpart = nullptr;
    int* bterm = nullptr;
    void* btab = nullptr;                // PairTerm<R> per (potential, type pair) in use
    std::vector<int> bond_ij_h;          // 2 per bond
    std::vector<int> bond_pot_h;
    std::vector<rdgpu_pair_pot> bond_pots_h;
    // control
    int* err = nullptr;
    long long* err_step = nullptr;
    long long* step_d = nullptr;
    double* red_d = nullptr;
    long long* redc_d = nullptr;
    double* part_d = nullptr;            // partial sums of the typed reductions
    long long* off_d = nullptr;          // particle offsets of the systems (n_systems + 1)
    long long* pcnt_d = nullptr;
    int* pinned_err = nullptr;
    long long* pinned_step = nullptr;
    long long step_h = 0;
    // RDF accumulator
    unsigned long long* rdf_acc = nullptr;
    unsigned long long* rdf_tmp = nullptr;
    double* rdf_e2 = nullptr;
    int rdf_nbins = 0;
    double rdf_rmax = 0.0;
    long long rdf_frames = 0;
    // RDF coarse grid (cells of edge >= rmax): grids per system, counting
    // sort arrays, particles sorted by coarse cell
    RdfGrid* rdf_grid_d = nullptr;
    int rdf_grid_n = 0;
    int* rdf_cnt = nullptr;
    int* rdf_start = nullptr;
    int* rdf_tsum = nullptr;
    long long rdf_cells_cap = 0;
    void* rdf_rec = nullptr;
    long long rdf_rec_cap = 0;
    // neighbour search
    int nb_req = RDGPU_NB_AUTO;          // requested mode
    int nb_mode = RDGPU_NB_CELLS;        // mode in effect
    double skin_req = 0.0;               // requested pair-list skin (0: automatic)
    double skin = 0.0;                   // pair-list skin in effect
    double max_rc = 0.0;                 // largest pair cutoff
    double cell_cut = 0.0;               // lower bound of the cell edge of the current grid
    bool tuned = false;
    bool tuning = false;                 // inside tune(): its trials do not re-tune
    bool retune = false;                 // the lists outgrew their capacity: tune again
    ListCtl* ctl = nullptr;
    ListCtl* pinned_ctl = nullptr;
    int nbuild_h = 0;
    int4* nbr = nullptr;                 // pair-list entry groups (narrow: 8 offsets, wide: 4 indices)
    uint2* head = nullptr;               // list heads: build position on a 16-bit lattice, list length
    bool list_wide = false;              // 32-bit entries (a partner's offset did not fit 16 bits)
    int* hot = nullptr;                  // particles that moved more than about skin/2 since the build
    cudaStream_t stream2 = nullptr;      // captures the re-sort into conditional graph nodes
    bool capturing = false;
    long long list_stride = 0;
    int list_cap = 0;
    std::vector<double> rc_h;            // pair cutoff per type pair (0: no potential)
    void* rl2_d = nullptr;               // squared list radius per type pair, in the state precision
    // captured step graphs by step count, cell walk and pair list: graph_steps
    // steps and every power of two below it.  A call of n steps replays
    // n / graph_steps full graphs and the rest as a sum of powers of two, so
    // short calls run graphed too.
    std::map<int, cudaGraphExec_t> cgraphs;
    std::map<int, cudaGraphExec_t> lgraphs;
    int graph_steps = 100;
    long long launches = 0;
    std::string last_error;
};

namespace {

using Engine = rdgpu_engine;

template <class R> int sync_types(Engine* E);

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            E->last_error = std::string(#call) + ": " + cudaGetErrorString(e_);   \
            return (e_ == cudaErrorMemoryAllocation) ? RDGPU_ERR_NOMEM : RDGPU_ERR_CUDA; \
        }                                                                          \
    } while (0)

int fail(Engine* E, int code, const std::string& msg)
{
    E->last_error = msg;
    return code;
}

template <class T> void dfree(T*& p)
{
    if (p) cudaFree((void*)p);
    p = nullptr;
}



// ---------------------------------------------------------------------------
// parameter tables
// ---------------------------------------------------------------------------
double pair_cutoff(const rdgpu_pair_pot& p, double r0pair, double maxc)
{
    double r0 = p.r0 >= 0.0 ? p.r0 : r0pair;
    if (p.kind == RDGPU_P2_HARMONIC) return p.subtype == RDGPU_SUB_REPULSIVE ? r0 : maxc;
    if (p.kind == RDGPU_P2_WEAK_PIECEWISE) return r0 + p.length;
    return 0.0;
}

int validate(const rdgpu_system_desc& d, std::string& why)
{
    if (d.n_types < 1 || d.n_types > RDGPU_MAX_TYPES) { why = "n_types out of range"; return -1; }
    if (d.n_pair < 0 || d.n_pair > RDGPU_MAX_PAIR_POTS) { why = "n_pair out of range"; return -1; }
    if (d.n_ext < 0 || d.n_ext > RDGPU_MAX_EXT_POTS) { why = "n_ext out of range"; return -1; }
    if (!(d.kB > 0 && d.T > 0 && d.dt > 0)) { why = "kB, T and dt must be positive"; return -1; }
    for (int t = 0; t < d.n_types; ++t)
        if (!(d.D[t] >= 0 && std::isfinite(d.D[t]))) { why = "diffusion constants must be finite and >= 0"; return -1; }
    for (int p = 0; p < d.n_pair; ++p) {
        const rdgpu_pair_pot& q = d.pair[p];
        if (q.kind == RDGPU_P2_HARMONIC) {
            if (q.subtype < 1 || q.subtype > 3) { why = "harmonic subtype must be attractive, repulsive or spring"; return -1; }
            if (q.subtype != RDGPU_SUB_REPULSIVE && !(d.max_cutoff > 0)) {
                why = "harmonic attractive/spring potentials need max_cutoff > 0";
                return -1;
            }
        } else if (q.kind == RDGPU_P2_WEAK_PIECEWISE) {
            if (!(q.length > 0)) { why = "weak interaction needs length > 0"; return -1; }
        } else {
            why = "unknown pair potential kind";
            return -1;
        }
    }
    for (int p = 0; p < d.n_ext; ++p) {
        const rdgpu_ext_pot& q = d.ext[p];
        if (q.kind < 1 || q.kind > 4) { why = "unknown external potential kind"; return -1; }
        bool ok = (q.subtype == 1 || q.subtype == 2) || (q.kind == RDGPU_P1_SPHERE && q.subtype == 4);
        if (!ok) { why = "invalid external potential subtype"; return -1; }
        if (q.kind == 1 || q.kind == 2) {
            double nn = std::sqrt(q.normal[0] * q.normal[0] + q.normal[1] * q.normal[1] + q.normal[2] * q.normal[2]);
            if (!(nn > 0)) { why = "disk/cylinder normal must be non-zero"; return -1; }
        }
    }
    return 0;
}

template <class R> void build_tab(const rdgpu_system_desc& d, TypeTab<R>& t, double& max_rc, std::string& why, int& bad)
{
    memset(&t, 0, sizeof(t));
    t.S = d.n_types;
    t.n_ext = d.n_ext;
    max_rc = 0.0;
    bad = 0;
    const int M = RDGPU_MAX_TYPES;
    for (int i = 0; i < d.n_types; ++i) {
        t.a[i] = (R)(d.D[i] * d.dt / (d.kB * d.T));
        t.b[i] = (R)std::sqrt(2.0 * d.D[i] * d.dt);
        t.prad[i] = (R)d.p_radius[i];
        for (int j = 0; j < d.n_types; ++j) {
            double r0pair = d.coll_radius[i * M + j] + d.coll_radius[j * M + i];
            double rc = 0.0;
            int nt = 0;
            for (int p = 0; p < d.n_pair; ++p) {
                const rdgpu_pair_pot& q = d.pair[p];
                if (!q.pairs[i * M + j] && !q.pairs[j * M + i]) continue;
                double c = pair_cutoff(q, r0pair, d.max_cutoff);
                if (c > rc) rc = c;
                if (nt >= MAX_TERMS) { bad = 1; why = "more than 4 pair potentials on one type pair"; return; }
                PairTerm<R>& pt = t.term[(i * MAXT + j) * MAX_TERMS + nt];
                pt.kind = q.kind;
                pt.sub = q.subtype;
                pt.k = (R)q.k;
                pt.r0 = (R)(q.r0 >= 0.0 ? q.r0 : r0pair);
                pt.l = (R)q.length;
                pt.d = (R)q.depth;
                double qq = q.length > 0 ? (1.0 / (0.5 * q.length)) * (1.0 / (0.5 * q.length)) : 0.0;
                pt.q = (R)qq;
                ++nt;
            }
            t.nterm[i * MAXT + j] = nt;
            t.rc2[i * MAXT + j] = (R)(rc * rc);
            if (rc > max_rc) max_rc = rc;
        }
    }
}

template <class R> void build_ext(const rdgpu_system_desc& d, const rdgpu_box& b, ExtTerm<R>* out)
{
    for (int p = 0; p < d.n_ext; ++p) {
        const rdgpu_ext_pot& q = d.ext[p];
        ExtTerm<R> e;
        memset(&e, 0, sizeof(e));
        e.kind = q.kind;
        e.sub = q.subtype;
        e.k = (R)q.k;
        double nn = std::sqrt(q.normal[0] * q.normal[0] + q.normal[1] * q.normal[1] + q.normal[2] * q.normal[2]);
        for (int a = 0; a < 3; ++a) {
            e.c[a] = (R)(q.center[a] - b.lo[a]);
            e.nrm[a] = nn > 0 ? (R)(q.normal[a] / nn) : R(0);
            double lo = q.origin[a], hi = q.origin[a] + q.extension[a];
            if (!(lo < hi)) std::swap(lo, hi);
            e.blo[a] = (R)(lo - b.lo[a]);
            e.bhi[a] = (R)(hi - b.lo[a]);
        }
        e.rad = (R)q.radius;
        {
            const double r2 = q.radius * q.radius;
            e.rad2h = (R)r2;
            e.rad2l = (R)(r2 - (double)e.rad2h);
        }
        e.h = (R)q.height;
        e.consider = q.consider_radius;
        e.tmask = 0;
        for (int t = 0; t < d.n_types; ++t)
            if (q.types[t]) e.tmask |= (1u << t);
        out[p] = e;
    }
}

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------


// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------
void drop_graph_map(std::map<int, cudaGraphExec_t>& m)
{
    for (auto& kv : m) cudaGraphExecDestroy(kv.second);
    m.clear();
}

void drop_graphs(Engine* E)
{
    drop_graph_map(E->cgraphs);
    drop_graph_map(E->lgraphs);
}

// the current state moved to buffer c; the cell-walk graphs captured the old one
void set_cur(Engine* E, int c)
{
    if (c != E->cur) drop_graph_map(E->cgraphs);
    E->cur = c;
}

// The graph sizes a call of `remaining` steps replays, largest first: full
// graphs of graph_steps steps, then the bits of the remainder.
template <class F> int for_each_graph(const Engine* E, long long remaining, F&& f)
{
    const long long G = E->graph_steps;
    for (long long g = 0; g < remaining / G; ++g) {
        const int rc = f((int)G);
        if (rc) return rc;
    }
    const long long r = remaining % G;
    for (long long p = 1LL << 30; p >= 1; p >>= 1)
        if (r & p) {
            const int rc = f((int)p);
            if (rc) return rc;
        }
    return RDGPU_OK;
}

void free_particles(Engine* E)
{
    for (int b = 0; b < 2; ++b) { dfree(E->bufA[b]); dfree(E->bufB[b]); }
    dfree(E->tcell); dfree(E->tslot);
    dfree(E->nbr); dfree(E->head); dfree(E->hot);
    E->list_stride = 0;
    E->list_cap = 0;
    dfree(E->sys_of); dfree(E->x0_d); dfree(E->vec_d); dfree(E->val_d); dfree(E->ityp_d); dfree(E->u64_d);
    dfree(E->ed_flag); dfree(E->ed_keep); dfree(E->ed_newid); dfree(E->ed_tile); dfree(E->inv);
    E->cap_particles = 0;
}

// grow-only per-particle buffers
int ensure_particle_buffers(Engine* E, long long ntot)
{
    const long long N = std::max<long long>(ntot, 1);
    if (N <= E->cap_particles) return RDGPU_OK;
    drop_graphs(E);
    free_particles(E);
    const long long M = N + N / 4;      // headroom for reactions adding particles
    const size_t rec = E->prec == RDGPU_PREC_F32C ? 16 : 32;
    for (int b = 0; b < 2; ++b) {
        CK(cudaMalloc(&E->bufA[b], M * rec));
        if (E->prec == RDGPU_PREC_F32C) CK(cudaMalloc(&E->bufB[b], M * 16));
    }
    E->cur = 0;
    CK(cudaMalloc(&E->tcell, M * sizeof(int)));
    CK(cudaMalloc(&E->tslot, M * sizeof(int)));
    CK(cudaMalloc(&E->sys_of, M * sizeof(unsigned short)));
    CK(cudaMalloc(&E->x0_d, M * 3 * sizeof(double)));
    CK(cudaMalloc(&E->vec_d, M * 3 * sizeof(double)));
    CK(cudaMalloc(&E->val_d, M * sizeof(double)));
    CK(cudaMalloc(&E->ityp_d, M * sizeof(int)));
    CK(cudaMalloc(&E->u64_d, M * sizeof(unsigned long long)));
    CK(cudaMalloc(&E->ed_flag, (M + 1) * sizeof(int)));
    CK(cudaMalloc(&E->ed_keep, (M + 1) * sizeof(int)));
    CK(cudaMalloc(&E->ed_newid, (M + 1) * sizeof(int)));
    CK(cudaMalloc(&E->ed_tile, ((M + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(int)));
    CK(cudaMalloc(&E->inv, M * sizeof(int)));
    E->cap_particles = M;
    return RDGPU_OK;
}

template <class R> State<R> state(void* A, void* B)
{
    State<R> s;
    if constexpr (sizeof(R) == 4) { s.pos = (float4*)A; s.aux = (float4*)B; }
    else s.rec = (Rec64*)A;
    return s;
}

template <class R> State<R> cur_state(Engine* E) { return state<R>(E->bufA[E->cur], E->bufB[E->cur]); }
template <class R> State<R> stg_state(Engine* E) { return state<R>(E->bufA[E->cur ^ 1], E->bufB[E->cur ^ 1]); }

template <class R> Args<R> make_args(Engine* E)
{
    Args<R> a;
    memset(&a, 0, sizeof(a));
    a.sys = E->sys_d;
    a.sys_of = E->sys_of;
    a.ntot = E->npart_tot;
    a.nsys = E->nsys;
    a.n_ext = E->n_ext;
    a.tab = (const TypeTab<R>*)E->tab_d;
    a.ext = (const ExtTerm<R>*)E->ext_d;
    a.cur = cur_state<R>(E);
    a.stg = stg_state<R>(E);
    a.start = E->start;
    a.counts = E->counts;
    a.tcell = E->tcell;
    a.tslot = E->tslot;
    a.err = E->err;
    a.err_step = E->err_step;
    a.step_ptr = E->step_d;
    if (E->nbonds > 0) {
        a.bstart = E->bstart;
        a.bpart = E->bpart;
        a.bterm = E->bterm;
        a.btab = (const PairTerm<R>*)E->btab;
        a.inv = E->inv;
    }
    return a;
}

int grid_for(long long n, int block = 256)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

// scan + scatter of the staging arrays (tcell/tslot/counts filled)
template <class R> void launch_sort(Engine* E)
{
    scan_tiles_kernel<<<E->ntiles, SCAN_BLOCK, 0, E->stream>>>(E->counts, E->ncells_tot, E->tile_sum, E->err,
                                                               nullptr);
    scan_apply_kernel<<<E->ntiles, SCAN_BLOCK, 0, E->stream>>>(E->counts, E->ncells_tot, E->tile_sum, E->ntiles,
                                                               E->start, E->err, nullptr);
    if (E->npart_tot > 0)
        scatter_kernel<R><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(
            stg_state<R>(E), cur_state<R>(E), E->tcell, E->tslot, E->start, E->npart_tot, E->err,
            E->nbonds > 0 ? E->inv : nullptr);
    E->launches += (E->npart_tot > 0) ? 3 : 2;
}

int reset_counters(Engine* E, long long t)
{
    CK(cudaMemsetAsync(E->err, 0, sizeof(int), E->stream));
    const long long big = 0x7fffffffffffffffLL;
    CK(cudaMemcpyAsync(E->err_step, &big, sizeof(long long), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemcpyAsync(E->step_d, &t, sizeof(long long), cudaMemcpyHostToDevice, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    E->step_h = t;
    return RDGPU_OK;
}

// the sorted state of step t is in cur/start; the counts must be zero
int prepare_step_state(Engine* E, long long t)
{
    CK(cudaMemsetAsync(E->counts, 0, std::max<long long>(E->ncells_tot, 1) * sizeof(int), E->stream));
    return reset_counters(E, t);
}

template <class R> void launch_step_kernel(Engine* E, Args<R>& a)
{
    const int grid = (int)((E->npart_tot + kStepBlock - 1) / kStepBlock);
    if (E->value_image)
        step_kernel<R, true, false, kStepBlock><<<grid, kStepBlock, 0, E->stream>>>(a);
    else if (E->hrep)
        step_kernel<R, false, true, kStepBlock><<<grid, kStepBlock, 0, E->stream>>>(a);
    else
        step_kernel<R, false, false, kStepBlock><<<grid, kStepBlock, 0, E->stream>>>(a);
    ++E->launches;
}

template <class R> int launch_steps(Engine* E, int n, const double* noise_d)
{
    Args<R> a = make_args<R>(E);
    a.noise = noise_d;
    for (int k = 0; k < n; ++k) {
        a.step_off = k;
        launch_step_kernel<R>(E, a);
        launch_sort<R>(E);
    }
    advance_kernel<<<1, 32, 0, E->stream>>>(E->step_d, E->err, n);
    ++E->launches;
    CK(cudaGetLastError());
    return RDGPU_OK;
}

// the cell-walk graph of n steps (captured on first use)
template <class R> int capture_graph(Engine* E, int n, cudaGraphExec_t* out)
{
    const auto it = E->cgraphs.find(n);
    if (it != E->cgraphs.end()) { *out = it->second; return RDGPU_OK; }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
    long long l0 = E->launches;
    int rc = launch_steps<R>(E, n, nullptr);
    cudaError_t ce = cudaStreamEndCapture(E->stream, &g);
    E->launches = l0;
    if (rc) return rc;
    CK(ce);
    cudaGraphExec_t x = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    E->cgraphs[n] = x;
    *out = x;
    return RDGPU_OK;
}

template <class R> int do_steps_cells(Engine* E, long long nsteps, const double* noise_d)
{
    const long long target = E->step_h + nsteps;
    long long remaining = nsteps;
    if (E->graph_steps > 0 && !noise_d) {
        int rc = for_each_graph(E, remaining, [&](int n) -> int {
            cudaGraphExec_t x;
            const int r = capture_graph<R>(E, n, &x);
            if (r) return r;
            CK(cudaGraphLaunch(x, E->stream));
            E->launches += (long long)n * ((E->npart_tot > 0) ? 4 : 3) + 1;
            return RDGPU_OK;
        });
        if (rc) return rc;
        remaining = 0;
    }
    while (remaining > 0) {
        const int n = (int)std::min<long long>(remaining, 1000);
        int rc = launch_steps<R>(E, n, noise_d);
        if (rc) return rc;
        remaining -= n;
    }
    CK(cudaMemcpyAsync(E->pinned_err, E->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaMemcpyAsync(E->pinned_step, E->err_step, sizeof(long long), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    const int ef = *E->pinned_err;
    if (ef == 0) {
        E->step_h = target;
        return RDGPU_OK;
    }
    // the failing step's input is the current sorted state (its sort was skipped)
    const long long tf = *E->pinned_step;
    int rc = prepare_step_state(E, tf);
    if (rc) return rc;
    if (ef & EF_NONFINITE)
        return fail(E, RDGPU_ERR_NONFINITE, "a particle position became non-finite at step " + std::to_string(tf));
    return fail(E, RDGPU_ERR_JUMP, "a particle moved more than a box length at step " + std::to_string(tf));
}

// box edge as the engine stores it
double edge(const Engine* E, int s, int a)
{
    return E->prec == RDGPU_PREC_F32C ? (double)E->sys_h[s].Lf[a] : E->sys_h[s].L[a];
}

int cells_along(double Lp, double cut)
{
    if (!(cut > 0.0)) return 1;
    double q = std::floor(Lp / (cut * (1.0 + 1e-5)));
    return (int)std::max(1.0, std::min(q, 2048.0));
}

// (Re)builds the cell grids of all systems with cell edges >= cut; the
// particles must be re-sorted afterwards.
int configure_cells(Engine* E, double cut, std::string& why)
{
    long long cb = 0;
    bool vi = false;
    for (int s = 0; s < E->nsys; ++s) {
        SysDev& v = E->sys_h[s];
        long long nc = 1;
        for (int a = 0; a < 3; ++a) {
            const double Lp = edge(E, s, a);
            const int n = cells_along(Lp, cut);
            v.n[a] = n;
            v.invcf[a] = (float)((double)n / (double)v.Lf[a]);
            v.invc[a] = (double)n / Lp;
            nc *= n;
            if (v.per[a] && n < 3) vi = true;
        }
        if (nc > (1LL << 26)) { why = "too many cells in one system (box / cutoff too large)"; return RDGPU_ERR_ARG; }
        v.ncells = (int)nc;
        v.cell_base = cb;
        cb += nc;
    }
    if (cb >= 0x7fffffffLL) { why = "too many cells in the batch"; return RDGPU_ERR_ARG; }
    drop_graphs(E);
    const int ntiles = (int)((cb + SCAN_TILE - 1) / SCAN_TILE);
    if (cb > E->ncells_tot || !E->start) {
        dfree(E->start); dfree(E->counts); dfree(E->tile_sum);
        if (cudaMalloc(&E->start, (cb + 1) * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&E->counts, std::max<long long>(cb, 1) * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&E->tile_sum, std::max(ntiles, 1) * sizeof(int)) != cudaSuccess) {
            why = "device allocation failed";
            return RDGPU_ERR_NOMEM;
        }
    }
    E->ncells_tot = cb;
    E->ntiles = ntiles;
    E->value_image = vi;
    E->cell_cut = cut;
    cudaMemsetAsync(E->start, 0, (cb + 1) * sizeof(int), E->stream);
    cudaMemsetAsync(E->counts, 0, std::max<long long>(cb, 1) * sizeof(int), E->stream);
    cudaMemcpyAsync(E->sys_d, E->sys_h.data(), E->nsys * sizeof(SysDev), cudaMemcpyHostToDevice, E->stream);
    if (cudaStreamSynchronize(E->stream) != cudaSuccess) { why = "cell grid upload failed"; return RDGPU_ERR_CUDA; }
    return RDGPU_OK;
}

// ---------------------------------------------------------------------------
// pair-list mode (list_step_kernel and the re-sort chain; see the kernels)
// ---------------------------------------------------------------------------
double largest_edge(const Engine* E)
{
    double lmax = 0.0;
    for (int s = 0; s < E->nsys; ++s)
        for (int a = 0; a < 3; ++a) lmax = std::max(lmax, E->sys_h[s].L[a]);
    return lmax;
}

// the hot-particle threshold th: skin/2 less the FP32 rounding of positions
// and squared distances
double list_threshold(const Engine* E, double skin)
{
    return 0.5 * skin * (1.0 - 2e-3) - 4.0 * largest_edge(E) * std::ldexp(1.0, -20);
}

// error bound of the lattice estimate of a displacement (2 bins per axis)
double list_lattice_error(const Engine* E)
{
    return std::sqrt(3.0) * 2.0 * largest_edge(E) * std::ldexp(1.0, -16) * (1.0 + 1e-3);
}

template <class R> ListArgs<R> make_list_args(Engine* E, bool with_list)
{
    ListArgs<R> v;
    memset(&v, 0, sizeof(v));
    v.b0 = state<R>(E->bufA[0], E->bufB[0]);
    v.b1 = state<R>(E->bufA[1], E->bufB[1]);
    v.ctl = E->ctl;
    v.nbr = with_list ? E->nbr : nullptr;
    v.head = E->head;
    v.hot = E->hot;
    v.stride = E->list_stride;
    v.cap = E->list_cap;
    v.narrow = E->list_wide ? 0 : 1;
    // list radius and displacement thresholds.  A pair missing from the list
    // that is closer than its cutoff at a later step has moved by more than
    // 2 th together, th being kept below skin/2 by a margin for the FP32
    // rounding of positions (a few ulp of the largest box edge) and of the
    // squared distances: one of the two moved more than th (list_check_kernel
    // looks at those).  Beyond 2 th the check's cell walk may miss partners,
    // and the step kernel asks for a rebuild outright.  The step kernel
    // estimates a displacement on the 16-bit lattice of the list heads, to
    // within dq = 2 bins per axis (head_disp2), so it compares the estimate
    // with th - sqrt(3) dq and 2 th - sqrt(3) dq.
    v.rl2t = (const R*)E->rl2_d;
    const double rl = E->max_rc + E->skin;
    v.rl2max = (R)(rl * rl * (1.0 + 1e-6));
    const double th = list_threshold(E, E->skin);
    const double dq = list_lattice_error(E);
    v.thr2 = (float)(th - dq > 0 ? (th - dq) * (th - dq) : 0.0);
    v.cap2 = (float)(th - dq > 0 ? (2.0 * th - dq) * (2.0 * th - dq) : 0.0);
    // a larger cap stretches the intervals between rebuilds, but the check
    // costs more per step and the sorted order decays for longer (on config
    // 4, caps of 2048 to 32768 measured best at 8192)
    v.hot_max = (int)std::min<long long>(kHotMax, std::max<long long>(8, E->npart_tot / kHotDiv));
    return v;
}

// the skin is usable: the hot-particle threshold keeps half of skin/2 after
// its margins, and >= 3 cells of edge >= rc_max + skin on every periodic
// axis of every system
bool list_eligible(Engine* E, double skin)
{
    if (!(skin > 0.0) || !(E->max_rc > 0.0)) return false;
    if (list_threshold(E, skin) - list_lattice_error(E) < 0.25 * skin) return false;
    const double cut = std::max(E->desc.cell_size, E->max_rc + skin);
    for (int s = 0; s < E->nsys; ++s)
        for (int a = 0; a < 3; ++a)
            if (E->sys_h[s].per[a] && cells_along(edge(E, s, a), cut) < 3) return false;
    return true;
}

// list storage for cap entries per particle (wide: 32-bit entries)
int ensure_list(Engine* E, int cap, bool wide)
{
    const long long stride = std::max<long long>(E->cap_particles, 1);
    if (cap <= E->list_cap && stride == E->list_stride && wide == E->list_wide && E->nbr) return RDGPU_OK;
    // whole groups of 8 entries (one int4 narrow, two wide): the step kernel
    // requests the first 8 entries before it knows the list length; at most
    // 2^16 - 1 (the list head's count field)
    cap = std::min((std::max(std::max(cap, E->list_cap), 8) + 7) & ~7, 65528);
    drop_graph_map(E->lgraphs);
    dfree(E->nbr); dfree(E->head); dfree(E->hot);
    E->list_cap = 0;
    E->list_stride = 0;
    const long long groups = wide ? cap / 4 : cap / 8;
    CK(cudaMalloc(&E->nbr, (size_t)groups * stride * sizeof(int4)));
    CK(cudaMalloc(&E->head, stride * sizeof(uint2)));
    CK(cudaMalloc(&E->hot, kHotMax * sizeof(int)));
    E->list_cap = cap;
    E->list_stride = stride;
    E->list_wide = wide;
    return RDGPU_OK;
}


// capacity after an overflowing build: twice the longest list met, so that a
// system that keeps clustering (attractive interactions) overflows a few
// times at most; each overflow costs a re-sort and a new step graph
int list_regrow_cap(Engine* E)
{
    const long long c = 2LL * E->pinned_ctl->maxcnt + 8;
    return (int)std::min<long long>(c, 1 << 20);
}

// storage after a build that failed with flags ef (EF_LISTOVF: a list longer
// than the capacity; EF_LISTWIDE: an offset beyond 16 bits)
int ensure_list_after(Engine* E, int ef)
{
    const int cap = (ef & EF_LISTOVF) ? list_regrow_cap(E) : E->list_cap;
    return ensure_list(E, cap, E->list_wide || (ef & EF_LISTWIDE) != 0);
}

// list capacity from the densest system, x2 for fluctuations and clusters
int list_cap_estimate(Engine* E)
{
    const double rl = E->max_rc + E->skin;
    double best = 0.0;
    for (int s = 0; s < E->nsys; ++s) {
        double vol = 1.0;
        for (int a = 0; a < 3; ++a) vol *= edge(E, s, a);
        const double rho = (double)E->sys_h[s].npart / vol;
        best = std::max(best, rho * 4.0 / 3.0 * 3.14159265358979 * rl * rl * rl);
    }
    return (int)std::min(4096.0, std::ceil(2.0 * best) + 16.0);
}

template <class R> void launch_chain(Engine* E, const Args<R>& a, const ListArgs<R>& v, long long off,
                                     cudaStream_t st)
{
    const long long N = E->npart_tot;
    list_count_kernel<R><<<grid_for(N), 256, 0, st>>>(a, v, off);
    scan_tiles_kernel<<<E->ntiles, SCAN_BLOCK, 0, st>>>(E->counts, E->ncells_tot, E->tile_sum, E->err,
                                                        &E->ctl->need);
    scan_apply_kernel<<<E->ntiles, SCAN_BLOCK, 0, st>>>(E->counts, E->ncells_tot, E->tile_sum, E->ntiles,
                                                        E->start, E->err, &E->ctl->need);
    list_scatter_kernel<R><<<grid_for(N), 256, 0, st>>>(a, v, off);
    if (v.nbr)
        list_build_kernel<R, 128><<<(int)((N + 127) / 128), 128, 0, st>>>(a, v, off);
    list_finish_kernel<<<1, 32, 0, st>>>(E->ctl, E->err);
}

// the list check after a step (list_check_kernel): a warp per hot particle
// up to hot_max (kCheckBlocks blocks at most); the blocks that the step's hot
// particles do not fill exit at once
template <class R> void launch_check(Engine* E, const Args<R>& a, const ListArgs<R>& v, long long off,
                                     cudaGraphConditionalHandle h, int set_cond, cudaStream_t st)
{
    constexpr int wpb = kCheckBlock / 32;
    const int grid = std::max(1, std::min(kCheckBlocks, (v.hot_max + wpb - 1) / wpb));
    list_check_kernel<R, kCheckBlock><<<grid, kCheckBlock, 0, st>>>(a, v, off, h, set_cond);
}

// Inside a stream capture: the re-sort of a step becomes a conditional graph
// node whose body (the chain above) runs only when the step raised the
// rebuild flag, so steps without a rebuild launch two kernels, not eight.
template <class R> int add_conditional_chain(Engine* E, const Args<R>& a, const ListArgs<R>& v, long long off)
{
    cudaStreamCaptureStatus st;
    unsigned long long id;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t nd;
    CK(cudaStreamGetCaptureInfo(E->stream, &st, &id, &g, &deps, &nd));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    launch_check<R>(E, a, v, off, h, 1, E->stream);
    CK(cudaGetLastError());
    CK(cudaStreamGetCaptureInfo(E->stream, &st, &id, &g, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
    CK(cudaStreamUpdateCaptureDependencies(E->stream, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(E->stream2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_chain<R>(E, a, v, off, E->stream2);
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(E->stream2, &out));
    return RDGPU_OK;
}

template <class R, bool NARROW>
void launch_list_step_kernel_w(Engine* E, const Args<R>& a, const ListArgs<R>& v, int grid, bool allper)
{
    if (E->hrep && allper)
        list_step_kernel<R, true, true, kListBlock, NARROW><<<grid, kListBlock, 0, E->stream>>>(a, v);
    else if (E->hrep)
        list_step_kernel<R, true, false, kListBlock, NARROW><<<grid, kListBlock, 0, E->stream>>>(a, v);
    else if (allper)
        list_step_kernel<R, false, true, kListBlock, NARROW><<<grid, kListBlock, 0, E->stream>>>(a, v);
    else
        list_step_kernel<R, false, false, kListBlock, NARROW><<<grid, kListBlock, 0, E->stream>>>(a, v);
}

template <class R> void launch_list_step_kernel(Engine* E, const Args<R>& a, const ListArgs<R>& v)
{
    const int grid = (int)((E->npart_tot + kListBlock - 1) / kListBlock);
    bool allper = true;
    for (int s = 0; s < E->nsys; ++s)
        for (int q = 0; q < 3; ++q) allper = allper && E->sys_h[s].per[q];
    if (v.narrow)
        launch_list_step_kernel_w<R, true>(E, a, v, grid, allper);
    else
        launch_list_step_kernel_w<R, false>(E, a, v, grid, allper);
    ++E->launches;
}

template <class R> int launch_list_steps(Engine* E, int n, const double* noise_d)
{
    Args<R> a = make_args<R>(E);
    a.noise = noise_d;
    const ListArgs<R> v = make_list_args<R>(E, true);
    for (int k = 0; k < n; ++k) {
        a.step_off = k;
        launch_list_step_kernel<R>(E, a, v);
        if (E->capturing) {
            int rc = add_conditional_chain<R>(E, a, v, k + 1);
            if (rc) return rc;
            ++E->launches;
        } else {
            launch_check<R>(E, a, v, k + 1, 0, 0, E->stream);
            launch_chain<R>(E, a, v, k + 1, E->stream);
            E->launches += v.nbr ? 7 : 6;
        }
    }
    advance_kernel<<<1, 32, 0, E->stream>>>(E->step_d, E->err, n);
    ++E->launches;
    CK(cudaGetLastError());
    return RDGPU_OK;
}

// device control block and counters for the input of step step_h in buffer cur
int write_ctl(Engine* E, int need)
{
    ListCtl c;
    c.need = need;
    c.nreb = (int)((E->cur ^ (int)(E->step_h & 1)) & 1);
    c.maxcnt = 0;
    c.nbuild = E->nbuild_h;
    c.nhot = 0;
    c.done = 0;
    CK(cudaMemcpyAsync(E->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, E->stream));
    return reset_counters(E, E->step_h);
}

int read_back(Engine* E)
{
    CK(cudaMemcpyAsync(E->pinned_err, E->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaMemcpyAsync(E->pinned_step, E->err_step, sizeof(long long), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaMemcpyAsync(E->pinned_ctl, E->ctl, sizeof(ListCtl), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    E->nbuild_h = E->pinned_ctl->nbuild;
    return RDGPU_OK;
}

// Re-sorts the current state (the input of step step_h) by cell into the
// other buffer and, with_list, builds the pair lists; an overflowing build
// grows the lists and is redone.
template <class R> int resort(Engine* E, bool with_list)
{
    if (E->npart_tot == 0) return RDGPU_OK;
    for (int attempt = 0; attempt < 16; ++attempt) {
        int rc = write_ctl(E, 1);
        if (rc) return rc;
        Args<R> a = make_args<R>(E);
        const ListArgs<R> v = make_list_args<R>(E, with_list);
        launch_chain<R>(E, a, v, 0, E->stream);
        E->launches += v.nbr ? 6 : 5;
        CK(cudaGetLastError());
        rc = read_back(E);
        if (rc) return rc;
        const int ef = *E->pinned_err;
        if (ef == 0) {
            set_cur(E, E->cur ^ 1);
            return reset_counters(E, E->step_h);
        }
        if (ef & ~(EF_LISTOVF | EF_LISTWIDE)) return fail(E, RDGPU_ERR_CUDA, "re-sort failed");
        // the scan cleared the counts; the current state is untouched
        rc = ensure_list_after(E, ef);
        if (rc) return rc;
    }
    return fail(E, RDGPU_ERR_CUDA, "pair-list build did not converge");
}

// switch to the pair list with the given skin (the particles, if any, are
// re-sorted on the list's cell grid and the lists built)
template <class R> int enter_list(Engine* E, double skin)
{
    std::string why;
    const double cut = std::max(E->desc.cell_size, E->max_rc + skin);
    if (E->cell_cut != cut) {
        int rc = configure_cells(E, cut, why);
        if (rc) return fail(E, rc, why);
    }
    if (E->skin != skin) drop_graph_map(E->lgraphs);
    E->skin = skin;
    E->nb_mode = RDGPU_NB_LIST;
    {
        // list radius per type pair: its own cutoff + skin (the same margin as rl2max)
        std::vector<double> t(MAXT * MAXT, 0.0);
        for (int q = 0; q < MAXT * MAXT; ++q)
            if (E->rc_h[q] > 0.0) t[q] = (E->rc_h[q] + skin) * (E->rc_h[q] + skin) * (1.0 + 1e-6);
        const size_t rs = E->prec == RDGPU_PREC_F32C ? sizeof(float) : sizeof(double);
        if (!E->rl2_d) CK(cudaMalloc(&E->rl2_d, MAXT * MAXT * rs));
        if (E->prec == RDGPU_PREC_F32C) {
            std::vector<float> f(t.begin(), t.end());
            CK(cudaMemcpy(E->rl2_d, f.data(), MAXT * MAXT * rs, cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(E->rl2_d, t.data(), MAXT * MAXT * rs, cudaMemcpyHostToDevice));
        }
    }
    if (E->part_off.empty() || E->npart_tot == 0) return RDGPU_OK;
    int rc = ensure_list(E, list_cap_estimate(E), E->list_wide);
    if (rc) return rc;
    return resort<R>(E, true);
}

// switch to the cell walk (particles re-sorted on its grid)
template <class R> int enter_cells(Engine* E)
{
    std::string why;
    const double cut = std::max(E->desc.cell_size, E->max_rc);
    const bool regrid = E->cell_cut != cut;
    if (regrid) {
        int rc = configure_cells(E, cut, why);
        if (rc) return fail(E, rc, why);
    }
    const bool was_list = E->nb_mode == RDGPU_NB_LIST;
    E->nb_mode = RDGPU_NB_CELLS;
    if (E->part_off.empty() || E->npart_tot == 0) return RDGPU_OK;
    if (regrid || was_list) return resort<R>(E, false);
    return RDGPU_OK;
}

// the pair-list graph of n steps (captured on first use)
template <class R> int capture_list_graph(Engine* E, int n, cudaGraphExec_t* out)
{
    const auto it = E->lgraphs.find(n);
    if (it != E->lgraphs.end()) { *out = it->second; return RDGPU_OK; }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
    long long l0 = E->launches;
    E->capturing = true;
    int rc = launch_list_steps<R>(E, n, nullptr);
    E->capturing = false;
    cudaError_t ce = cudaStreamEndCapture(E->stream, &g);
    E->launches = l0;
    if (rc) return rc;
    CK(ce);
    cudaGraphExec_t x = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    E->lgraphs[n] = x;
    *out = x;
    return RDGPU_OK;
}

template <class R> int do_steps_list(Engine* E, long long nsteps, const double* noise_d)
{
    const long long target = E->step_h + nsteps;
    while (E->step_h < target) {
        long long remaining = target - E->step_h;
        int rc = write_ctl(E, 0);
        if (rc) return rc;
        const int nb0 = E->nbuild_h;
        const bool graphed = E->graph_steps > 0 && !noise_d;
        if (graphed) {
            rc = for_each_graph(E, remaining, [&](int n) -> int {
                cudaGraphExec_t x;
                const int r = capture_list_graph<R>(E, n, &x);
                if (r) return r;
                CK(cudaGraphLaunch(x, E->stream));
                E->launches += 2LL * n + 1;
                return RDGPU_OK;
            });
            if (rc) return rc;
            remaining = 0;
        }
        // without graphs (injected noise, or graphs off): kernel by kernel
        // (the step counter and parity carry over on the device)
        while (remaining > 0) {
            const int n = (int)std::min<long long>(remaining, 1000);
            rc = launch_list_steps<R>(E, n, noise_d);
            if (rc) return rc;
            remaining -= n;
        }
        rc = read_back(E);
        if (rc) return rc;
        // the re-sorts that ran inside the graphs (six kernels each)
        if (graphed) E->launches += 6LL * std::max(0, E->nbuild_h - nb0);
        const int ef = *E->pinned_err;
        const int nreb = E->pinned_ctl->nreb;
        if (ef == 0) {
            E->step_h = target;
            set_cur(E, (int)((target + nreb) & 1));
            return RDGPU_OK;
        }
        // the input of step tf is intact in buffer (tf + nreb) & 1
        const long long tf = *E->pinned_step;
        E->step_h = tf;
        set_cur(E, (int)((tf + nreb) & 1));
        if ((ef & ~(EF_LISTOVF | EF_LISTWIDE)) == 0) {
            rc = ensure_list_after(E, ef);
            if (rc) return rc;
            rc = resort<R>(E, true);
            if (rc) return rc;
            // the particles gathered into denser clusters than the tuner saw:
            // an AUTO handle times its options again on the new state
            if ((ef & EF_LISTOVF) && E->nb_req == RDGPU_NB_AUTO && !E->tuning && !noise_d) {
                E->retune = true;
                return RDGPU_OK_CONTINUE;
            }
            continue;
        }
        rc = prepare_step_state(E, tf);
        if (rc) return rc;
        if (ef & EF_NONFINITE)
            return fail(E, RDGPU_ERR_NONFINITE, "a particle position became non-finite at step " + std::to_string(tf));
        return fail(E, RDGPU_ERR_JUMP, "a particle moved more than a box length at step " + std::to_string(tf));
    }
    return RDGPU_OK;
}

template <class R> int do_steps_mode(Engine* E, long long nsteps, const double* noise_d)
{
    return E->nb_mode == RDGPU_NB_LIST ? do_steps_list<R>(E, nsteps, noise_d) : do_steps_cells<R>(E, nsteps, noise_d);
}

// The autotuner: times the cell walk and the pair list at a few skins on the
// handle's own particles (graph_steps steps each after as many warm-up
// steps, from a snapshot of the state that is restored afterwards) and keeps
// the fastest.  The trajectory does not depend on the choice: the noise is
// keyed by the step, and the FP32 forces are identical in both modes.
template <class R> int tune(Engine* E)
{
    E->tuned = true;
    E->tuning = true;
    struct Done { Engine* e; ~Done() { e->tuning = false; } } done_{E};
    const long long N = E->npart_tot;
    if (N == 0 || E->graph_steps <= 0) return RDGPU_OK;
    // the trials' launches and list builds are not the run's
    const long long launches0 = E->launches;
    const int nbuild0 = E->nbuild_h;
    const size_t recA = sizeof(R) == 4 ? 16 : 32;
    void* snapA = nullptr;
    void* snapB = nullptr;
    CK(cudaMalloc(&snapA, N * recA));
    if (sizeof(R) == 4) CK(cudaMalloc(&snapB, N * 16));
    const long long step0 = E->step_h;
    auto snap = [&](bool save) -> int {
        void* a = E->bufA[E->cur];
        void* b = E->bufB[E->cur];
        CK(cudaMemcpyAsync(save ? snapA : a, save ? a : snapA, N * recA, cudaMemcpyDeviceToDevice, E->stream));
        if (sizeof(R) == 4) CK(cudaMemcpyAsync(save ? snapB : b, save ? b : snapB, N * 16, cudaMemcpyDeviceToDevice, E->stream));
        CK(cudaStreamSynchronize(E->stream));
        return RDGPU_OK;
    };
    int rc = snap(true);
    std::vector<double> skins = {0.0};
    for (double f : {0.1, 0.2, 0.275, 0.35, 0.425, 0.5})
        if (list_eligible(E, f * E->max_rc)) skins.push_back(f * E->max_rc);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best_ms = 1e300, best_skin = 0.0;
    for (size_t c = 0; c < skins.size() && rc == RDGPU_OK; ++c) {
        // restore the snapshot as the input of step step0, sorted for the candidate
        rc = snap(false);
        if (rc) break;
        E->step_h = step0;
        rc = prepare_step_state(E, step0);
        if (rc) break;
        // the snapshot is sorted for the grid it was taken on; re-sort on the candidate's
        rc = skins[c] > 0.0 ? enter_list<R>(E, skins[c]) : (E->nb_mode = RDGPU_NB_LIST, enter_cells<R>(E));
        if (rc) break;
        // a trial that fails (the dynamics itself, e.g. a particle leaving the
        // box) disqualifies the candidate; the real run reports the failure
        if (do_steps_mode<R>(E, E->graph_steps, nullptr) != RDGPU_OK) continue;
        // three graphs: several rebuild intervals of the larger skins
        cudaEventRecord(e0, E->stream);
        const int trial = do_steps_mode<R>(E, 3LL * E->graph_steps, nullptr);
        cudaEventRecord(e1, E->stream);
        cudaEventSynchronize(e1);
        if (trial != RDGPU_OK) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best_skin = skins[c]; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rs = snap(false);
    if (rc == RDGPU_OK) rc = rs;
    cudaFree(snapA);
    if (snapB) cudaFree(snapB);
    if (rc) return rc;
    E->step_h = step0;
    E->launches = launches0;
    E->nbuild_h = nbuild0;
    rc = prepare_step_state(E, step0);
    if (rc) return rc;
    return best_skin > 0.0 ? enter_list<R>(E, best_skin) : (E->nb_mode = RDGPU_NB_LIST, enter_cells<R>(E));
}

// captures the step graphs of the mode in effect, graph_steps steps and the
// powers of two below it, so that no later call captures (nothing runs)
template <class R> int prepare_graph(Engine* E)
{
    if (E->graph_steps <= 0) return RDGPU_OK;
    std::vector<int> sizes = {E->graph_steps};
    for (int p = 1; p < E->graph_steps; p <<= 1) sizes.push_back(p);
    for (int n : sizes) {
        cudaGraphExec_t x;
        const int rc = E->nb_mode == RDGPU_NB_LIST ? capture_list_graph<R>(E, n, &x) : capture_graph<R>(E, n, &x);
        if (rc) return rc;
    }
    return RDGPU_OK;
}

template <class R> int do_steps(Engine* E, long long nsteps, const double* noise_d)
{
    const long long target = E->step_h + nsteps;
    for (;;) {
        const long long left = target - E->step_h;
        if (left <= 0) return RDGPU_OK;
        if (E->nb_req == RDGPU_NB_AUTO && (!E->tuned || E->retune) && !noise_d &&
            left >= 4LL * std::max(E->graph_steps, 1)) {
            E->retune = false;
            int rc = tune<R>(E);
            if (rc) return rc;
        }
        const int rc = do_steps_mode<R>(E, left, noise_d);
        if (rc != RDGPU_OK_CONTINUE) return rc;
    }
}

int setup_systems(Engine* E, std::string& why)
{
    const rdgpu_system_desc& d = E->desc;
    double max_rc = 0.0;
    int bad = 0;
    size_t tabsz;
    std::vector<char> tabbuf;
    if (E->prec == RDGPU_PREC_F32C) {
        tabsz = sizeof(TypeTab<float>);
        tabbuf.resize(tabsz);
        build_tab<float>(d, *(TypeTab<float>*)tabbuf.data(), max_rc, why, bad);
    } else {
        tabsz = sizeof(TypeTab<double>);
        tabbuf.resize(tabsz);
        build_tab<double>(d, *(TypeTab<double>*)tabbuf.data(), max_rc, why, bad);
    }
    if (bad) return -1;
    E->max_rc = max_rc;
    E->rc_h.assign(MAXT * MAXT, 0.0);
    for (int q = 0; q < MAXT * MAXT; ++q) {
        const double r2 = E->prec == RDGPU_PREC_F32C ? (double)((TypeTab<float>*)tabbuf.data())->rc2[q]
                                                     : ((TypeTab<double>*)tabbuf.data())->rc2[q];
        E->rc_h[q] = std::sqrt(r2) * (1.0 + 1e-7);   // at least the cutoff the kernels test against
    }
    if (d.cell_size > 0.0 && d.cell_size < max_rc) { why = "cell_size is smaller than the largest pair cutoff"; return -1; }
    E->sys_h.assign(E->nsys, SysDev{});
    for (int s = 0; s < E->nsys; ++s) {
        const rdgpu_box& b = E->boxes[s];
        SysDev& v = E->sys_h[s];
        memset(&v, 0, sizeof(v));
        for (int a = 0; a < 3; ++a) {
            double L = b.hi[a] - b.lo[a];
            if (!(L > 0)) { why = "box bounds must satisfy hi > lo"; return -1; }
            float Lf = (float)L;
            double Lp = (E->prec == RDGPU_PREC_F32C) ? (double)Lf : L;
            if (b.periodic[a] && max_rc > 0.0 && Lp < 2.0 * max_rc) {
                why = "periodic box edge shorter than twice the pair cutoff (minimum image)";
                return -1;
            }
            v.per[a] = b.periodic[a] ? 1 : 0;
            v.Lf[a] = Lf;
            v.qs[a] = (float)(65536.0 / Lp);
            v.iqs[a] = (float)(Lp / 65536.0);
            v.halff[a] = 0.5f * Lf;
            v.ilf[a] = b.periodic[a] ? 1.0f / Lf : 0.0f;
            v.il[a] = b.periodic[a] ? 1.0 / L : 0.0;
            v.L[a] = L;
            v.half[a] = 0.5 * L;
            v.lo[a] = b.lo[a];
        }
        v.seed = b.seed;
    }
    if (cudaMalloc(&E->tab_d, tabsz) != cudaSuccess) { why = "cudaMalloc failed"; return -2; }
    cudaMemcpy(E->tab_d, tabbuf.data(), tabsz, cudaMemcpyHostToDevice);
    E->n_ext = d.n_ext;
    size_t esz = (E->prec == RDGPU_PREC_F32C ? sizeof(ExtTerm<float>) : sizeof(ExtTerm<double>)) *
                 std::max(1, E->nsys * d.n_ext);
    std::vector<char> ebuf(esz);
    for (int s = 0; s < E->nsys; ++s) {
        if (E->prec == RDGPU_PREC_F32C) build_ext<float>(d, E->boxes[s], (ExtTerm<float>*)ebuf.data() + s * d.n_ext);
        else build_ext<double>(d, E->boxes[s], (ExtTerm<double>*)ebuf.data() + s * d.n_ext);
    }
    if (cudaMalloc(&E->ext_d, esz) != cudaSuccess) { why = "cudaMalloc failed"; return -2; }
    cudaMemcpy(E->ext_d, ebuf.data(), esz, cudaMemcpyHostToDevice);
    return 0;
}

// Event timing of the step kernel and of what follows it in a step.  Steps
// go out in batches of kProfBatch without a synchronisation in between, so
// that while the GPU runs one step the host has queued the next: an event
// pair then brackets the kernel alone.  The first step of each batch starts
// on an idle stream (its first event would also time the host's launch) and
// is not counted.
constexpr int kProfBatch = 16;

struct ProfEvents {
    cudaEvent_t ev[3 * kProfBatch] = {};
    int made = 0;
    ~ProfEvents()
    {
        for (int k = 0; k < made; ++k) cudaEventDestroy(ev[k]);
    }
    cudaError_t create()
    {
        for (; made < 3 * kProfBatch; ++made) {
            const cudaError_t e = cudaEventCreate(&ev[made]);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // adds the batch's kernel and follower times (steps 1 .. nb-1)
    void add(int nb, double& tk, double& ts, long long& counted) const
    {
        for (int k = 1; k < nb; ++k) {
            float m1 = 0.f, m2 = 0.f;
            cudaEventElapsedTime(&m1, ev[3 * k], ev[3 * k + 1]);
            cudaEventElapsedTime(&m2, ev[3 * k + 1], ev[3 * k + 2]);
            tk += m1;
            ts += m2;
            ++counted;
        }
    }
};

template <class R> int profile_list(Engine* E, long long nsteps, double* kms, double* sms)
{
    ProfEvents pe;
    CK(pe.create());
    double tk = 0.0, ts = 0.0;
    long long counted = 0;
    const long long target = E->step_h + nsteps;
    int rc = RDGPU_OK;
    while (E->step_h < target) {
        rc = write_ctl(E, 0);
        if (rc) break;
        Args<R> a = make_args<R>(E);
        const ListArgs<R> v = make_list_args<R>(E, true);
        const int nb = (int)std::min<long long>(kProfBatch, target - E->step_h);
        for (int k = 0; k < nb; ++k) {
            a.step_off = k;
            CK(cudaEventRecord(pe.ev[3 * k], E->stream));
            launch_list_step_kernel<R>(E, a, v);
            CK(cudaEventRecord(pe.ev[3 * k + 1], E->stream));
            launch_check<R>(E, a, v, k + 1, 0, 0, E->stream);
            launch_chain<R>(E, a, v, k + 1, E->stream);
            E->launches += 7;
            CK(cudaEventRecord(pe.ev[3 * k + 2], E->stream));
        }
        advance_kernel<<<1, 32, 0, E->stream>>>(E->step_d, E->err, nb);
        ++E->launches;
        CK(cudaGetLastError());
        rc = read_back(E);
        if (rc) break;
        const int ef = *E->pinned_err;
        const int nreb = E->pinned_ctl->nreb;
        if (ef == 0) {
            pe.add(nb, tk, ts, counted);
            E->step_h += nb;
            set_cur(E, (int)((E->step_h + nreb) & 1));
            continue;
        }
        // a failed step (the step kernel, or the re-sort for the next one):
        // the input of the failing step tf is intact; a list overflow grows
        // the lists and re-sorts (the batch is not timed), anything else is
        // reported
        E->step_h = *E->pinned_step;
        set_cur(E, (int)((E->step_h + nreb) & 1));
        if (ef & ~(EF_LISTOVF | EF_LISTWIDE)) {
            rc = prepare_step_state(E, E->step_h);
            if (!rc) rc = fail(E, (ef & EF_NONFINITE) ? RDGPU_ERR_NONFINITE : RDGPU_ERR_JUMP,
                               "a step failed during profiling at step " + std::to_string(E->step_h));
            break;
        }
        rc = ensure_list_after(E, ef);
        if (!rc) rc = resort<R>(E, true);
        if (rc) break;
    }
    if (rc) return rc;
    if (kms) *kms = counted > 0 ? tk / counted : 0.0;
    if (sms) *sms = counted > 0 ? ts / counted : 0.0;
    return RDGPU_OK;
}

template <class R> int profile_impl(Engine* E, long long nsteps, double* kms, double* sms)
{
    if (E->nb_mode == RDGPU_NB_LIST) return profile_list<R>(E, nsteps, kms, sms);
    ProfEvents pe;
    CK(pe.create());
    double tk = 0.0, ts = 0.0;
    long long counted = 0;
    for (long long done = 0; done < nsteps;) {
        const int nb = (int)std::min<long long>(kProfBatch, nsteps - done);
        Args<R> a = make_args<R>(E);
        for (int k = 0; k < nb; ++k) {
            a.step_off = k;
            CK(cudaEventRecord(pe.ev[3 * k], E->stream));
            launch_step_kernel<R>(E, a);
            CK(cudaEventRecord(pe.ev[3 * k + 1], E->stream));
            launch_sort<R>(E);
            CK(cudaEventRecord(pe.ev[3 * k + 2], E->stream));
        }
        advance_kernel<<<1, 32, 0, E->stream>>>(E->step_d, E->err, nb);
        ++E->launches;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(E->pinned_err, E->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
        CK(cudaMemcpyAsync(E->pinned_step, E->err_step, sizeof(long long), cudaMemcpyDeviceToHost, E->stream));
        CK(cudaStreamSynchronize(E->stream));
        if (*E->pinned_err) {
            // the failing step's input is the current sorted state (its sort was skipped)
            const long long tf = *E->pinned_step;
            const int rc = prepare_step_state(E, tf);
            if (rc) return rc;
            return fail(E, RDGPU_ERR_JUMP, "a step failed during profiling at step " + std::to_string(tf));
        }
        pe.add(nb, tk, ts, counted);
        E->step_h += nb;
        done += nb;
    }
    if (kms) *kms = counted > 0 ? tk / counted : 0.0;
    if (sms) *sms = counted > 0 ? ts / counted : 0.0;
    return RDGPU_OK;
}

// ---------------------------------------------------------------------------
// bonded pairs (particle groups)
// ---------------------------------------------------------------------------
void free_bonds(Engine* E)
{
    dfree(E->bstart); dfree(E->bpart); dfree(E->bterm); dfree(E->btab);
    if (E->nbonds > 0) drop_graphs(E);   // kernel arguments change
    E->nbonds = 0;
}

void clear_bonds(Engine* E)
{
    free_bonds(E);
    E->bond_ij_h.clear();
    E->bond_pot_h.clear();
    E->bond_pots_h.clear();
}

// the bonds of bond_ij_h / bond_pot_h to the device: a list per particle id
// (each bond in both of its particles' lists) with its potential resolved for
// the two types, and the sorted index of every id
template <class R> int upload_bonds(Engine* E)
{
    free_bonds(E);
    const long long nb = (long long)E->bond_pot_h.size();
    if (nb == 0 || E->npart_tot == 0) return RDGPU_OK;
    {
        const int rc = sync_types<R>(E);
        if (rc) return rc;
    }
    const long long N = E->npart_tot;
    const int M = RDGPU_MAX_TYPES;
    std::vector<int> start(N + 1, 0), part(2 * nb), term(2 * nb);
    for (long long b = 0; b < nb; ++b) { start[E->bond_ij_h[2 * b] + 1]++; start[E->bond_ij_h[2 * b + 1] + 1]++; }
    for (long long i = 0; i < N; ++i) start[i + 1] += start[i];
    std::vector<int> fill(start.begin(), start.end() - 1);
    std::vector<PairTerm<R>> tab;
    std::map<long long, int> key_to_term;
    auto term_of = [&](int p, int ta, int tb) {
        const long long key = ((long long)p * M + ta) * M + tb;
        auto it = key_to_term.find(key);
        if (it != key_to_term.end()) return it->second;
        const rdgpu_pair_pot& q = E->bond_pots_h[p];
        const double r0pair = E->desc.coll_radius[ta * M + tb] + E->desc.coll_radius[tb * M + ta];
        PairTerm<R> t;
        memset(&t, 0, sizeof(t));
        t.kind = q.kind;
        t.sub = q.subtype;
        t.k = (R)q.k;
        t.r0 = (R)(q.r0 >= 0.0 ? q.r0 : r0pair);
        t.l = (R)q.length;
        t.d = (R)q.depth;
        t.q = (R)(q.length > 0 ? (1.0 / (0.5 * q.length)) * (1.0 / (0.5 * q.length)) : 0.0);
        tab.push_back(t);
        key_to_term[key] = (int)tab.size() - 1;
        return (int)tab.size() - 1;
    };
    for (long long b = 0; b < nb; ++b) {
        const int i = E->bond_ij_h[2 * b], j = E->bond_ij_h[2 * b + 1], p = E->bond_pot_h[b];
        const int ti = E->types_h[i], tj = E->types_h[j];
        const int ki = fill[i]++, kj = fill[j]++;
        part[ki] = j;
        term[ki] = term_of(p, ti, tj);
        part[kj] = i;
        term[kj] = term_of(p, tj, ti);
    }
    CK(cudaMalloc(&E->bstart, (N + 1) * sizeof(int)));
    CK(cudaMalloc(&E->bpart, 2 * nb * sizeof(int)));
    CK(cudaMalloc(&E->bterm, 2 * nb * sizeof(int)));
    CK(cudaMalloc(&E->btab, tab.size() * sizeof(PairTerm<R>)));
    CK(cudaMemcpyAsync(E->bstart, start.data(), (N + 1) * sizeof(int), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemcpyAsync(E->bpart, part.data(), 2 * nb * sizeof(int), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemcpyAsync(E->bterm, term.data(), 2 * nb * sizeof(int), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemcpyAsync(E->btab, tab.data(), tab.size() * sizeof(PairTerm<R>), cudaMemcpyHostToDevice, E->stream));
    inv_kernel<R><<<grid_for(N), 256, 0, E->stream>>>(cur_state<R>(E), N, E->inv);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(E->stream));
    E->nbonds = nb;
    drop_graphs(E);
    return RDGPU_OK;
}

template <class R> int set_bonds_impl(Engine* E, long long nb, const int* ij, const int* pot, int npots,
                                      const rdgpu_pair_pot* pots)
{
    const long long N = E->npart_tot;
    for (int p = 0; p < npots; ++p) {
        const rdgpu_pair_pot& q = pots[p];
        if (q.kind == RDGPU_P2_HARMONIC) {
            if (q.subtype < 1 || q.subtype > 3) return fail(E, RDGPU_ERR_ARG, "bond potential: invalid harmonic subtype");
        } else if (q.kind == RDGPU_P2_WEAK_PIECEWISE) {
            if (!(q.length > 0)) return fail(E, RDGPU_ERR_ARG, "bond potential: weak interaction needs length > 0");
        } else {
            return fail(E, RDGPU_ERR_ARG, "bond potential: unknown kind");
        }
    }
    for (long long b = 0; b < nb; ++b) {
        const long long i = ij[2 * b], j = ij[2 * b + 1];
        if (i < 0 || j < 0 || i >= N || j >= N || i == j)
            return fail(E, RDGPU_ERR_ARG, "bond " + std::to_string(b) + ": particle index out of range or self bond");
        if (pot[b] < 0 || pot[b] >= npots) return fail(E, RDGPU_ERR_ARG, "bond " + std::to_string(b) + ": potential index out of range");
    }
    clear_bonds(E);
    E->bond_ij_h.assign(ij, ij + 2 * nb);
    E->bond_pot_h.assign(pot, pot + nb);
    E->bond_pots_h.assign(pots, pots + npots);
    int rc = upload_bonds<R>(E);
    if (rc) clear_bonds(E);
    return rc;
}

template <class R, class In> int set_particles_impl(Engine* E, const long long* offsets, long long ntot,
                                                    const In* xyz, const int* types)
{
    // validate the layout before touching the handle's state
    std::vector<long long> off;
    if (E->nsys == 1) {
        off = {0, ntot};
    } else {
        if (!offsets) return fail(E, RDGPU_ERR_ARG, "offsets required for a batch");
        off.assign(offsets, offsets + E->nsys + 1);
        if (off[0] != 0 || off[E->nsys] != ntot)
            return fail(E, RDGPU_ERR_ARG, "offsets must start at 0 and end at n_total");
    }
    for (int s = 0; s < E->nsys; ++s) {
        long long n = off[s + 1] - off[s];
        if (n < 0 || n > 0x7fffffff) return fail(E, RDGPU_ERR_ARG, "invalid particle count");
    }
    if (ntot > 0x7fffffff) return fail(E, RDGPU_ERR_ARG, "at most 2^31-1 particles per handle");
    E->part_off.clear();   // no valid state until this call completes
    clear_bonds(E);        // bonds name particles of the previous upload
    if (ntot != E->npart_tot) drop_graphs(E);   // launch shapes depend on the particle count
    int rc = ensure_particle_buffers(E, ntot);
    if (rc) return rc;
    for (int s = 0; s < E->nsys; ++s) {
        E->sys_h[s].part_base = off[s];
        E->sys_h[s].npart = (int)(off[s + 1] - off[s]);
    }
    E->npart_tot = ntot;
    CK(cudaMemcpyAsync(E->sys_d, E->sys_h.data(), E->nsys * sizeof(SysDev), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemsetAsync(E->err, 0, sizeof(int), E->stream));
    CK(cudaMemsetAsync(E->counts, 0, std::max<long long>(E->ncells_tot, 1) * sizeof(int), E->stream));
    if (ntot > 0) {
        CK(cudaMemcpyAsync(E->off_d, off.data(), (E->nsys + 1) * sizeof(long long), cudaMemcpyHostToDevice, E->stream));
        sys_of_kernel<<<grid_for(ntot), 256, 0, E->stream>>>(E->off_d, E->nsys, ntot, E->sys_of);
        // (the FP64 staging buffer holds FP32 coordinates in its first half)
        CK(cudaMemcpyAsync(E->vec_d, xyz, ntot * 3 * sizeof(In), cudaMemcpyHostToDevice, E->stream));
        CK(cudaMemcpyAsync(E->ityp_d, types, ntot * sizeof(int), cudaMemcpyHostToDevice, E->stream));
        ingest_kernel<R, In><<<grid_for(ntot), 256, 0, E->stream>>>(E->sys_d, E->sys_of, ntot, (const In*)E->vec_d, E->ityp_d,
                                                                E->desc.n_types, stg_state<R>(E),
                                                                E->tcell, E->tslot, E->counts, E->x0_d, E->err);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(E->pinned_err, E->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
        CK(cudaStreamSynchronize(E->stream));
        if (*E->pinned_err & EF_BADINPUT)
            return fail(E, RDGPU_ERR_ARG, "particle type out of range, non-finite coordinate, or a coordinate "
                                          "more than 64 box lengths outside the box");
    }
    // the host copy of the types is downloaded when needed (sync_types)
    E->types_h_valid = false;
    const bool list_mode = E->nb_mode == RDGPU_NB_LIST && ntot > 0;
    if (list_mode) {
        // the list re-sort below sorts the ingested particles itself: the
        // staging buffer becomes the current state (its counts are cleared
        // by prepare_step_state)
        set_cur(E, E->cur ^ 1);
    } else {
        launch_sort<R>(E);
    }
    CK(cudaGetLastError());
    E->rdf_frames = 0;
    if (E->rdf_acc && E->rdf_nbins > 0) {
        const int S = E->desc.n_types;
        CK(cudaMemsetAsync(E->rdf_acc, 0, (size_t)S * S * E->rdf_nbins * sizeof(unsigned long long), E->stream));
    }
    rc = prepare_step_state(E, 0);
    if (rc) return rc;
    E->part_off = off;
    if (list_mode) {
        rc = ensure_list(E, list_cap_estimate(E), E->list_wide);
        if (!rc) rc = resort<R>(E, true);
        if (rc) { E->part_off.clear(); return rc; }
    }
    return RDGPU_OK;
}

// grows the per-particle buffers to hold n particles, keeping the current
// state and the MSD origins of the first npart_tot particles
template <class R> int grow_preserving(Engine* E, long long n)
{
    if (n <= E->cap_particles) return RDGPU_OK;
    const long long nold = E->npart_tot;
    const size_t recA = sizeof(R) == 4 ? 16 : 32;
    void* keepA = E->bufA[E->cur];
    void* keepB = E->bufB[E->cur];
    double* keepX0 = E->x0_d;
    E->bufA[E->cur] = nullptr;
    E->bufB[E->cur] = nullptr;
    E->x0_d = nullptr;
    int rc = ensure_particle_buffers(E, n);    // new buffers, current state in buffer 0
    if (rc == RDGPU_OK && nold > 0) {
        cudaError_t e = cudaMemcpyAsync(E->bufA[0], keepA, nold * recA, cudaMemcpyDeviceToDevice, E->stream);
        if (e == cudaSuccess && keepB)
            e = cudaMemcpyAsync(E->bufB[0], keepB, nold * 16, cudaMemcpyDeviceToDevice, E->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(E->x0_d, keepX0, nold * 3 * sizeof(double), cudaMemcpyDeviceToDevice, E->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
        if (e != cudaSuccess) rc = fail(E, RDGPU_ERR_CUDA, std::string("buffer growth: ") + cudaGetErrorString(e));
    }
    cudaFree(keepA);
    if (keepB) cudaFree(keepB);
    cudaFree(keepX0);
    return rc;
}

// Reaction edits of one frame on the device (ReaDDyGPU.cpp:303-461 semantics):
// delete by gpu index, append new particles, survivors keep their order and
// the appended ones follow; ids are renumbered 0 .. n-1 in that order.
template <class R> int apply_edits_impl(Engine* E, const float* ed, long long count)
{
    {
        const int rc = sync_types<R>(E);
        if (rc) return rc;
    }
    const long long N = E->npart_tot;
    const int S = E->desc.n_types;
    std::vector<char> gone(std::max<long long>(N, 1), 0);
    std::vector<int> del;
    std::vector<double> axyz;
    std::vector<int> atype;
    for (long long r = 0; r < count; ++r) {
        const float* e = ed + 6 * r;
        const double ft = e[1], fi = e[5];
        if (!(std::isfinite(ft) && std::isfinite(fi)) || ft != std::floor(ft) || fi != std::floor(fi))
            return fail(E, RDGPU_ERR_ARG, "reaction entry " + std::to_string(r) + ": type and index must be integers");
        const long long index = (long long)fi;
        const int newType = (int)ft;
        if (index != -1) {
            if (index < 0 || index >= N || gone[index])
                return fail(E, RDGPU_ERR_ARG, "reaction entry " + std::to_string(r) + ": invalid or repeated gpu index");
            gone[index] = 1;
            del.push_back((int)index);
        }
        if (newType != -1) {
            if (newType < 0 || newType >= S)
                return fail(E, RDGPU_ERR_ARG, "reaction entry " + std::to_string(r) + ": type out of range");
            axyz.push_back(e[2]);
            axyz.push_back(e[3]);
            axyz.push_back(e[4]);
            atype.push_back(newType);
        }
    }
    const long long nd = (long long)del.size(), na = (long long)atype.size();
    if (nd == 0 && na == 0) return RDGPU_OK;
    const long long nkeep = N - nd, N2 = nkeep + na;
    if (N2 > 0x7fffffff) return fail(E, RDGPU_ERR_ARG, "at most 2^31-1 particles per handle");
    int rc = grow_preserving<R>(E, N2);
    if (rc) { E->part_off.clear(); return rc; }
    drop_graphs(E);   // launch shapes depend on the particle count
    auto bad = [&](const char* what) { E->part_off.clear(); return fail(E, RDGPU_ERR_CUDA, what); };
    // the frame's edits on the device: appended coordinates, types, deleted indices
    const size_t need = (size_t)na * 3 * sizeof(double) + (size_t)(na + nd) * sizeof(int);
    if (need > E->ed_buf_bytes) {
        dfree(E->ed_buf);
        E->ed_buf_bytes = 0;
        if (cudaMalloc(&E->ed_buf, need) != cudaSuccess) return bad("device allocation failed");
        E->ed_buf_bytes = need;
    }
    double* axyz_d = (double*)E->ed_buf;
    int* atype_d = (int*)(axyz_d + 3 * na);
    int* del_d = atype_d + na;
    if (nd) CK(cudaMemcpyAsync(del_d, del.data(), nd * sizeof(int), cudaMemcpyHostToDevice, E->stream));
    if (na) {
        CK(cudaMemcpyAsync(axyz_d, axyz.data(), 3 * na * sizeof(double), cudaMemcpyHostToDevice, E->stream));
        CK(cudaMemcpyAsync(atype_d, atype.data(), na * sizeof(int), cudaMemcpyHostToDevice, E->stream));
    }
    CK(cudaMemsetAsync(E->ed_flag, 0, (N + 1) * sizeof(int), E->stream));
    CK(cudaMemsetAsync(E->err, 0, sizeof(int), E->stream));
    if (nd) edit_mark_kernel<<<grid_for(nd), 256, 0, E->stream>>>(del_d, nd, E->ed_flag);
    if (N > 0) {
        const int nt = (int)((N + SCAN_TILE - 1) / SCAN_TILE);
        edit_keep_kernel<<<grid_for(N), 256, 0, E->stream>>>(E->ed_flag, N, E->ed_keep);
        scan_tiles_kernel<<<nt, SCAN_BLOCK, 0, E->stream>>>(E->ed_keep, N, E->ed_tile, E->err, nullptr);
        scan_apply_kernel<<<nt, SCAN_BLOCK, 0, E->stream>>>(E->ed_keep, N, E->ed_tile, nt, E->ed_newid, E->err,
                                                            nullptr);
        // survivors and appended particles at their new ids in the staging buffer
        edit_restage_kernel<R><<<grid_for(N), 256, 0, E->stream>>>(E->sys_d, N, cur_state<R>(E), stg_state<R>(E),
                                                                    E->ed_flag, E->ed_newid, E->tcell, E->tslot,
                                                                    E->counts, E->x0_d, E->vec_d);
    }
    if (na)
        edit_append_kernel<R><<<grid_for(na), 256, 0, E->stream>>>(E->sys_d, nkeep, na, axyz_d, atype_d, S,
                                                                   stg_state<R>(E), E->tcell, E->tslot, E->counts,
                                                                   E->vec_d, E->err);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(E->pinned_err, E->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    if (*E->pinned_err & EF_BADINPUT) {
        // the staging buffer is rejected; the current state is untouched, but
        // the counts hold the staged particles: clear them
        CK(cudaMemsetAsync(E->counts, 0, std::max<long long>(E->ncells_tot, 1) * sizeof(int), E->stream));
        CK(cudaMemsetAsync(E->err, 0, sizeof(int), E->stream));
        CK(cudaStreamSynchronize(E->stream));
        return fail(E, RDGPU_ERR_ARG, "appended particle with a non-finite coordinate or far outside the box");
    }
    // the new MSD origins and particle count, then the counting sort staging -> current
    if (N2 > 0) CK(cudaMemcpyAsync(E->x0_d, E->vec_d, N2 * 3 * sizeof(double), cudaMemcpyDeviceToDevice, E->stream));
    E->npart_tot = N2;
    E->sys_h[0].npart = (int)N2;
    E->part_off = {0, N2};
    CK(cudaMemsetAsync(E->sys_of, 0, std::max<long long>(N2, 1) * sizeof(unsigned short), E->stream));
    CK(cudaMemcpyAsync(E->sys_d, E->sys_h.data(), sizeof(SysDev), cudaMemcpyHostToDevice, E->stream));
    launch_sort<R>(E);
    CK(cudaGetLastError());
    // host copy of the types by id
    std::vector<int> nt;
    nt.reserve(N2);
    for (long long i = 0; i < N; ++i)
        if (!gone[i]) nt.push_back(E->types_h[i]);
    for (int t : atype) nt.push_back(t);
    E->types_h.swap(nt);
    E->types_h_valid = true;
    // bonds: those of deleted particles go, the rest follow the new ids
    if (!E->bond_pot_h.empty()) {
        std::vector<int> nid(std::max<long long>(N, 1), -1);
        long long c = 0;
        for (long long i = 0; i < N; ++i)
            if (!gone[i]) nid[i] = (int)c++;
        std::vector<int> ij, pot;
        for (size_t b = 0; b < E->bond_pot_h.size(); ++b) {
            const int i = nid[E->bond_ij_h[2 * b]], j = nid[E->bond_ij_h[2 * b + 1]];
            if (i < 0 || j < 0) continue;
            ij.push_back(i);
            ij.push_back(j);
            pot.push_back(E->bond_pot_h[b]);
        }
        E->bond_ij_h.swap(ij);
        E->bond_pot_h.swap(pot);
        rc = upload_bonds<R>(E);
        if (rc) { E->part_off.clear(); return rc; }
    }
    rc = reset_counters(E, E->step_h);
    if (rc) return rc;
    if (E->nb_mode == RDGPU_NB_LIST && N2 > 0) {
        rc = ensure_list(E, list_cap_estimate(E), E->list_wide);
        if (!rc) rc = resort<R>(E, true);
        if (rc) { E->part_off.clear(); return rc; }
    }
    return RDGPU_OK;
}

template <class R, class Out> int get_particles_impl(Engine* E, Out* xyz, int* types)
{
    const long long N = E->npart_tot;
    if (N == 0) return RDGPU_OK;
    emit_kernel<R, Out><<<grid_for(N), 256, 0, E->stream>>>(E->sys_d, E->sys_of, N, cur_state<R>(E), (Out*)E->vec_d,
                                                            E->ityp_d);
    CK(cudaGetLastError());
    if (xyz) CK(cudaMemcpyAsync(xyz, E->vec_d, N * 3 * sizeof(Out), cudaMemcpyDeviceToHost, E->stream));
    if (types) CK(cudaMemcpyAsync(types, E->ityp_d, N * sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    return RDGPU_OK;
}

// the host copy of the types by global index, downloaded after an upload
// (bonds, reaction edits and the RDF normalisation read it)
template <class R> int sync_types(Engine* E)
{
    if (E->types_h_valid) return RDGPU_OK;
    E->types_h.resize(E->npart_tot);
    if (E->npart_tot > 0) {
        const int rc = get_particles_impl<R, double>(E, nullptr, E->types_h.data());
        if (rc) return rc;
    }
    E->types_h_valid = true;
    return RDGPU_OK;
}

template <class R, int MODE> void launch_diag(Engine* E, double* f, double* e, int* c, unsigned long long* h)
{
    Args<R> a = make_args<R>(E);
    if (E->value_image)
        diag_kernel<R, MODE, true><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(a, f, e, c, h);
    else
        diag_kernel<R, MODE, false><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(a, f, e, c, h);
}

// the diagnostics walk the cells: in pair-list mode re-sort first (the
// particles have moved since the last build)
template <class R> int fresh_cells(Engine* E)
{
    return E->nb_mode == RDGPU_NB_LIST ? resort<R>(E, true) : RDGPU_OK;
}

// sums of v by type into red_d/redc_d: wants 0..nwant-1, type S meaning all
constexpr int kSumParts = 148 * 4;
void launch_typed_sums(Engine* E, const double* v, const int* types, int S, int nwant)
{
    const long long n = E->npart_tot;
    const long long chunk = std::max<long long>(1, (n + kSumParts - 1) / kSumParts);
    typed_partial_kernel<<<dim3(kSumParts, nwant), TSUM_BLOCK, 0, E->stream>>>(v, types, n, S, chunk, E->part_d,
                                                                              E->pcnt_d);
    typed_final_kernel<<<nwant, TSUM_BLOCK, 0, E->stream>>>(E->part_d, E->pcnt_d, kSumParts, E->red_d, E->redc_d);
}

template <class R> int forces_impl(Engine* E, double* forces, double* energy)
{
    int rc = fresh_cells<R>(E);
    if (rc) return rc;
    launch_diag<R, 1>(E, E->vec_d, E->val_d, nullptr, nullptr);
    CK(cudaGetLastError());
    if (forces) CK(cudaMemcpyAsync(forces, E->vec_d, E->npart_tot * 3 * sizeof(double), cudaMemcpyDeviceToHost, E->stream));
    if (energy) {
        launch_typed_sums(E, E->val_d, E->ityp_d, 0, 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(energy, E->red_d, sizeof(double), cudaMemcpyDeviceToHost, E->stream));
    }
    CK(cudaStreamSynchronize(E->stream));
    return RDGPU_OK;
}

template <class R> int digest_impl(Engine* E, int* counts, unsigned long long* hashes)
{
    int rc = fresh_cells<R>(E);
    if (rc) return rc;
    launch_diag<R, 2>(E, nullptr, nullptr, E->ityp_d, E->u64_d);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(counts, E->ityp_d, E->npart_tot * sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaMemcpyAsync(hashes, E->u64_d, E->npart_tot * sizeof(unsigned long long), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    return RDGPU_OK;
}

__global__ void add_u64_kernel(unsigned long long* acc, const unsigned long long* v, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) acc[i] += v[i];
}

// FP64 RDF normalisation on the device
__global__ void rdf_norm_kernel(const unsigned long long* c, int S, int nbins, double w, double frames,
                                double vol, const long long* nper, double* g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S * S * nbins) return;
    int k = i % nbins, tj = (i / nbins) % S, ti = i / (nbins * S);
    const double pi = 3.14159265358979323846;
    double r0 = k * w, r1 = (k + 1) * w;
    double shell = 4.0 / 3.0 * pi * (r1 * r1 * r1 - r0 * r0 * r0);
    double pairs = (double)nper[ti] * (double)(nper[tj] - (ti == tj ? 1 : 0));
    double denom = frames * pairs / vol * shell;
    g[i] = denom > 0 ? (double)c[i] / denom : 0.0;
}

// The RDF frame on the simulation's own cell grid (rdf_kernel): for boxes
// whose coarse grid would have fewer than 3 cells along a periodic axis.
template <class R> int rdf_fine(Engine* E, int nbins, double rmax)
{
    const int S = E->desc.n_types;
    const int H = S * S * nbins;
    int rc = fresh_cells<R>(E);
    if (rc) return rc;
    // the block's histogram and the bin edges in shared memory when they fit
    const size_t smem = (size_t)((H + 1) & ~1) * 4 + (size_t)(nbins + 1) * 8;
    const int use_smem = smem <= 48 * 1024 ? 1 : 0;
    // one particle per thread: the per-particle work varies little
    const int grid = (int)((E->npart_tot + 127) / 128);
    rdf_kernel<R><<<grid, 128, use_smem ? smem : 0, E->stream>>>(
        E->sys_d, E->sys_of, E->npart_tot, cur_state<R>(E), E->start, S, nbins, E->rdf_e2,
        rmax / (double)nbins, use_smem, E->rdf_tmp);
    CK(cudaGetLastError());
    return RDGPU_OK;
}

// The RDF frame on a grid of its own (rdf_rows_kernel), from the current
// state in any order (no re-sort of the simulation's cells): cells of edge
// >= rmax/2, at least 5 and at most 500 along every axis.  Returns
// RDGPU_OK_CONTINUE (rdf_fine then takes the frame) when some system has
// fewer than 5 along a periodic axis (a box shorter than 2.5 rmax), the
// grid has 2^27 cells or more, or the bin edges do not fit shared memory
// (more than 4095 bins).
template <class R> int rdf_tiled(Engine* E, int nbins, double rmax)
{
    const int S = E->desc.n_types;
    const int H = S * S * nbins;
    std::vector<RdfGrid> gh(E->nsys);
    long long nc = 0;
    double lmax = 0.0;
    for (int s = 0; s < E->nsys; ++s) {
        RdfGrid& g = gh[s];
        memset(&g, 0, sizeof(g));
        long long m = 1;
        for (int a = 0; a < 3; ++a) {
            const double Lp = edge(E, s, a);
            const int n = std::min(cells_along(Lp, 0.5 * rmax), 500);
            if (E->sys_h[s].per[a] && n < 5) return RDGPU_OK_CONTINUE;
            g.n[a] = n;
            g.per[a] = E->sys_h[s].per[a];
            g.L[a] = Lp;
            g.invc[a] = (double)n / Lp;
            lmax = std::max(lmax, Lp);
            m *= n;
        }
        g.base = nc;
        nc += m;
    }
    if (nc >= (1LL << 27)) return RDGPU_OK_CONTINUE;
    if ((size_t)(nbins + 1) * sizeof(float2) > 32 * 1024) return RDGPU_OK_CONTINUE;
    const long long N = E->npart_tot;
    const size_t recsz = sizeof(RdfRec<R>);
    if (E->rdf_grid_n < E->nsys) {
        dfree(E->rdf_grid_d);
        CK(cudaMalloc(&E->rdf_grid_d, E->nsys * sizeof(RdfGrid)));
        E->rdf_grid_n = E->nsys;
    }
    const int ntiles = (int)((nc + SCAN_TILE - 1) / SCAN_TILE);
    if (nc > E->rdf_cells_cap) {
        dfree(E->rdf_cnt); dfree(E->rdf_start); dfree(E->rdf_tsum);
        CK(cudaMalloc(&E->rdf_cnt, nc * sizeof(int)));
        CK(cudaMalloc(&E->rdf_start, (nc + 1) * sizeof(int)));
        CK(cudaMalloc(&E->rdf_tsum, std::max(ntiles, 1) * sizeof(int)));
        E->rdf_cells_cap = nc;
    }
    if (N * (long long)recsz > E->rdf_rec_cap) {
        dfree(E->rdf_rec);
        CK(cudaMalloc(&E->rdf_rec, E->cap_particles * recsz));
        E->rdf_rec_cap = E->cap_particles * (long long)recsz;
    }
    CK(cudaMemcpyAsync(E->rdf_grid_d, gh.data(), E->nsys * sizeof(RdfGrid), cudaMemcpyHostToDevice, E->stream));
    CK(cudaMemsetAsync(E->rdf_cnt, 0, nc * sizeof(int), E->stream));
    const State<R> cur = cur_state<R>(E);
    RdfRec<R>* rec = (RdfRec<R>*)E->rdf_rec;
    // tcell / tslot are staging arrays of a step's sort, free between steps
    rdf_count_kernel<R><<<grid_for(N), 256, 0, E->stream>>>(E->sys_of, N, cur, E->rdf_grid_d, E->tcell, E->tslot,
                                                            E->rdf_cnt);
    scan_tiles_kernel<<<ntiles, SCAN_BLOCK, 0, E->stream>>>(E->rdf_cnt, nc, E->rdf_tsum, E->err, nullptr);
    scan_apply_kernel<<<ntiles, SCAN_BLOCK, 0, E->stream>>>(E->rdf_cnt, nc, E->rdf_tsum, ntiles, E->rdf_start,
                                                            E->err, nullptr);
    rdf_scatter_kernel<R><<<grid_for(N), 256, 0, E->stream>>>(N, cur, E->tcell, E->tslot, E->rdf_start, rec);
    // FP32 pre-selection radius: rmax widened by the FP32 rounding of the
    // coordinates (within a box length of the box) and of the distance
    const double rpre = rmax + 64.0 * std::ldexp(1.0, -24) * lmax;
    const float r2pre = (float)(rpre * rpre * (1.0 + 1e-5));
    // Bound on |FP32 r^2 - FP64 r^2| of a pair closer than the pre-selection
    // radius (rdf_rows_kernel): each FP32 displacement is within eps of the
    // exact one (the FP32 conversion of the two coordinates of an FP64 state, the
    // shifted candidate and the difference, each within 2^-24 of values below
    // 2 lmax + rmax), so r^2 within 2 sqrt(3) rmax eps + 3 eps^2; the FP32
    // squares and sums, the FP32 bin edges and the comparisons round by
    // 2^-24 rmax^2 each (8 allowed), the FP64 distance by 2^-53 rmax^2 each.
    const double eps = std::ldexp(1.0, -24) * (3.0 * lmax + 4.0 * rmax) * 1.01;
    const double rr = rpre;
    const float dlt = (float)((2.0 * std::sqrt(3.0) * rr * eps + 3.0 * eps * eps +
                               8.0 * std::ldexp(1.0, -24) * rr * rr + 8.0 * std::ldexp(1.0, -53) * rr * rr) *
                              (1.0 + 1e-3));
    // dynamic shared memory: the edge pairs, then the block's histogram
    const size_t epairs = (size_t)(nbins + 1) * sizeof(float2);
    const int use_smem = epairs + (size_t)H * 4 <= 32 * 1024 ? 1 : 0;
    const size_t smem = epairs + (use_smem ? (size_t)H * 4 : 0);
    const int grid = (int)std::min<long long>((nc + RDR_WARPS - 1) / RDR_WARPS, 148LL * 8);
    const double w = rmax / (double)nbins;
    // the warps' queues take about 40 KB of static shared memory, so the
    // dynamic part (up to 32 KB) needs the opt-in above 48 KB per block
    auto go = [&](auto kernel) {
        if (smem > 8 * 1024)
            CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kernel<<<grid, RDR_WARPS * 32, smem, E->stream>>>(E->rdf_grid_d, E->nsys, nc, E->rdf_start, rec, S, nbins,
                                                         E->rdf_e2, w, r2pre, dlt, E->rdf_tmp);
        return RDGPU_OK;
    };
    int lrc;
    if (S == 1) lrc = use_smem ? go(rdf_rows_kernel<R, false, true>) : go(rdf_rows_kernel<R, false, false>);
    else lrc = use_smem ? go(rdf_rows_kernel<R, true, true>) : go(rdf_rows_kernel<R, true, false>);
    if (lrc) return lrc;
    CK(cudaGetLastError());
    return RDGPU_OK;
}

template <class R> int rdf_impl(Engine* E, int nbins, double rmax, int accumulate, unsigned long long* out, long long* frames)
{
    const int S = E->desc.n_types;
    const int H = S * S * nbins;
    int rc = RDGPU_OK;
    if (E->rdf_nbins != nbins || E->rdf_rmax != rmax) {
        dfree(E->rdf_acc); dfree(E->rdf_tmp); dfree(E->rdf_e2);
        CK(cudaMalloc(&E->rdf_acc, H * sizeof(unsigned long long)));
        CK(cudaMalloc(&E->rdf_tmp, H * sizeof(unsigned long long)));
        CK(cudaMalloc(&E->rdf_e2, (nbins + 1) * sizeof(double)));
        CK(cudaMemsetAsync(E->rdf_acc, 0, H * sizeof(unsigned long long), E->stream));
        std::vector<double> e2(nbins + 1);
        const double w = rmax / (double)nbins;
        for (int k = 0; k <= nbins; ++k) { double e = (double)k * w; e2[k] = e * e; }
        CK(cudaMemcpyAsync(E->rdf_e2, e2.data(), (nbins + 1) * sizeof(double), cudaMemcpyHostToDevice, E->stream));
        CK(cudaStreamSynchronize(E->stream));
        E->rdf_nbins = nbins;
        E->rdf_rmax = rmax;
        E->rdf_frames = 0;
    }
    CK(cudaMemsetAsync(E->rdf_tmp, 0, H * sizeof(unsigned long long), E->stream));
    if (E->npart_tot > 0) {
        rc = rdf_tiled<R>(E, nbins, rmax);
        if (rc != RDGPU_OK_CONTINUE) {
            if (rc) return rc;
        } else {
            rc = rdf_fine<R>(E, nbins, rmax);
            if (rc) return rc;
        }
    }
    if (accumulate) {
        add_u64_kernel<<<(H + 255) / 256, 256, 0, E->stream>>>(E->rdf_acc, E->rdf_tmp, H);
        CK(cudaGetLastError());
        E->rdf_frames++;
        if (out) CK(cudaMemcpyAsync(out, E->rdf_acc, H * sizeof(unsigned long long), cudaMemcpyDeviceToHost, E->stream));
    } else if (out) {
        CK(cudaMemcpyAsync(out, E->rdf_tmp, H * sizeof(unsigned long long), cudaMemcpyDeviceToHost, E->stream));
    }
    CK(cudaStreamSynchronize(E->stream));
    if (frames) *frames = E->rdf_frames;
    return RDGPU_OK;
}

template <class R> int msd_impl(Engine* E, rdgpu_metrics* m)
{
    const int S = E->desc.n_types;
    msd_kernel<R><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(E->sys_d, E->sys_of, E->npart_tot,
                                                                   cur_state<R>(E), E->x0_d, E->val_d,
                                                                   E->ityp_d);
    CK(cudaGetLastError());
    launch_typed_sums(E, E->val_d, E->ityp_d, S, S);
    CK(cudaGetLastError());
    std::vector<double> sums(S);
    std::vector<long long> cnts(S);
    CK(cudaMemcpyAsync(sums.data(), E->red_d, S * sizeof(double), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaMemcpyAsync(cnts.data(), E->redc_d, S * sizeof(long long), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    for (int i = 0; i < S; ++i) {
        m->count[i] = cnts[i];
        m->msd[i] = cnts[i] > 0 ? sums[i] / (double)cnts[i] : 0.0;
    }
    return RDGPU_OK;
}

int create_impl(const rdgpu_system_desc* desc, int nsys, const rdgpu_box* boxes, const rdgpu_options* opt,
                rdgpu_handle* out)
{
    if (!desc || !out || nsys < 1 || (nsys > 1 && !boxes)) {
        g_create_error = "null argument or no systems";
        return RDGPU_ERR_ARG;
    }
    if (nsys > 65535) {
        g_create_error = "at most 65535 systems per batch";
        return RDGPU_ERR_ARG;
    }
    std::string why;
    if (validate(*desc, why)) {
        g_create_error = why;
        return RDGPU_ERR_ARG;
    }
    rdgpu_options o{};
    if (opt) o = *opt;
    if (o.precision != RDGPU_PREC_F64 && o.precision != RDGPU_PREC_F32C) {
        g_create_error = "unknown precision";
        return RDGPU_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        g_create_error = "no CUDA device (this library has no CPU fallback)";
        return RDGPU_ERR_CUDA;
    }
    if (o.device < 0 || o.device >= ndev) {
        g_create_error = "device ordinal out of range";
        return RDGPU_ERR_ARG;
    }
    if (cudaSetDevice(o.device) != cudaSuccess) {
        g_create_error = "cudaSetDevice failed";
        return RDGPU_ERR_CUDA;
    }
    Engine* E = new Engine();
    E->prec = o.precision;
    E->device = o.device;
    E->desc = *desc;
    E->opt = o;
    E->nsys = nsys;
    if (nsys == 1 && !boxes) {
        rdgpu_box b{};
        for (int a = 0; a < 3; ++a) { b.lo[a] = desc->lo[a]; b.hi[a] = desc->hi[a]; b.periodic[a] = desc->periodic[a]; }
        b.seed = o.seed;
        E->boxes.assign(1, b);
    } else {
        E->boxes.assign(boxes, boxes + nsys);
    }
    E->graph_steps = o.graph_steps == 0 ? 100 : (o.graph_steps < 0 ? 0 : o.graph_steps);
    if (o.neighbour_mode < RDGPU_NB_AUTO || o.neighbour_mode > RDGPU_NB_LIST || !(o.skin >= 0.0)) {
        g_create_error = "invalid neighbour_mode or skin";
        delete E;
        return RDGPU_ERR_ARG;
    }
    E->nb_req = o.neighbour_mode;
    E->skin_req = o.skin;
    auto bail = [&](int code, const std::string& msg) {
        g_create_error = msg;
        rdgpu_destroy(E);
        return code;
    };
    if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&E->stream2, cudaStreamNonBlocking) != cudaSuccess)
        return bail(RDGPU_ERR_CUDA, "cudaStreamCreate failed");
    if (cudaMalloc(&E->sys_d, nsys * sizeof(SysDev)) != cudaSuccess ||
        cudaMalloc(&E->err, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&E->err_step, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&E->step_d, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&E->red_d, (RDGPU_MAX_TYPES + 1) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&E->redc_d, (RDGPU_MAX_TYPES + 1) * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&E->part_d, (RDGPU_MAX_TYPES + 1) * kSumParts * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&E->off_d, (nsys + 1) * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&E->pcnt_d, (RDGPU_MAX_TYPES + 1) * kSumParts * sizeof(long long)) != cudaSuccess ||
        cudaMallocHost(&E->pinned_err, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&E->pinned_step, sizeof(long long)) != cudaSuccess)
        return bail(RDGPU_ERR_NOMEM, "device allocation failed");
    int rc = setup_systems(E, why);
    if (rc) return bail(rc == -2 ? RDGPU_ERR_NOMEM : RDGPU_ERR_ARG, why);
    // the harmonic-repulsion-only fast path applies when every pair potential is
    // a harmonic repulsion and no type pair carries more than one of them
    {
        bool h = true;
        for (int p = 0; p < desc->n_pair; ++p)
            if (!(desc->pair[p].kind == RDGPU_P2_HARMONIC && desc->pair[p].subtype == RDGPU_SUB_REPULSIVE)) h = false;
        const int M = RDGPU_MAX_TYPES;
        for (int i = 0; i < desc->n_types && h; ++i)
            for (int j = 0; j < desc->n_types && h; ++j) {
                int n = 0;
                for (int p = 0; p < desc->n_pair; ++p) n += (desc->pair[p].pairs[i * M + j] || desc->pair[p].pairs[j * M + i]);
                if (n > 1) h = false;
            }
        E->hrep = h;
    }
    // cells of all systems, for the cell walk
    rc = configure_cells(E, std::max(desc->cell_size, E->max_rc), why);
    if (rc) return bail(rc, why);
    if (cudaMalloc(&E->ctl, sizeof(ListCtl)) != cudaSuccess ||
        cudaMallocHost(&E->pinned_ctl, sizeof(ListCtl)) != cudaSuccess)
        return bail(RDGPU_ERR_NOMEM, "device allocation failed");
    cudaMemsetAsync(E->ctl, 0, sizeof(ListCtl), E->stream);
    if (cudaStreamSynchronize(E->stream) != cudaSuccess) return bail(RDGPU_ERR_CUDA, "initialisation failed");
    if (E->nb_req == RDGPU_NB_LIST) {
        // a requested pair list that the boxes cannot hold falls back to the cell walk
        const double skin = E->skin_req > 0.0 ? E->skin_req : 0.25 * E->max_rc;
        if (list_eligible(E, skin)) {
            rc = E->prec == RDGPU_PREC_F32C ? enter_list<float>(E, skin) : enter_list<double>(E, skin);
            if (rc) return bail(rc, E->last_error);
        }
    }
    *out = E;
    return RDGPU_OK;
}

}  // namespace

extern "C" {

int rdgpu_create(const rdgpu_system_desc* desc, const rdgpu_options* opt, rdgpu_handle* out)
{
    return create_impl(desc, 1, nullptr, opt, out);
}

int rdgpu_create_batch(const rdgpu_system_desc* desc, int32_t n_systems, const rdgpu_box* boxes,
                       const rdgpu_options* opt, rdgpu_handle* out)
{
    return create_impl(desc, n_systems, boxes, opt, out);
}

int rdgpu_destroy(rdgpu_handle h)
{
    Engine* E = (Engine*)h;
    if (!E) return RDGPU_ERR_ARG;
    cudaSetDevice(E->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    drop_graphs(E);
    free_particles(E);
    dfree(E->sys_d); dfree(E->tab_d); dfree(E->ext_d); dfree(E->start); dfree(E->counts); dfree(E->tile_sum);
    dfree(E->err); dfree(E->err_step); dfree(E->step_d); dfree(E->ctl); dfree(E->rl2_d);
    if (E->pinned_ctl) cudaFreeHost(E->pinned_ctl);
    dfree(E->red_d); dfree(E->redc_d); dfree(E->part_d); dfree(E->pcnt_d); dfree(E->ed_buf); dfree(E->off_d); dfree(E->rdf_acc); dfree(E->rdf_tmp); dfree(E->rdf_e2);
    dfree(E->rdf_grid_d); dfree(E->rdf_cnt); dfree(E->rdf_start); dfree(E->rdf_tsum); dfree(E->rdf_rec);
    if (E->pinned_err) cudaFreeHost(E->pinned_err);
    if (E->pinned_step) cudaFreeHost(E->pinned_step);
    if (E->stream) cudaStreamDestroy(E->stream);
    if (E->stream2) cudaStreamDestroy(E->stream2);
    delete E;
    return RDGPU_OK;
}

const char* rdgpu_last_error(rdgpu_handle h)
{
    if (!h) return g_create_error.c_str();
    return ((Engine*)h)->last_error.c_str();
}

#define DISPATCH(E, fn, ...) \
    ((E)->prec == RDGPU_PREC_F32C ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

#define GUARD(E)                                                          \
    if (!(E)) return RDGPU_ERR_ARG;                                       \
    if (cudaSetDevice((E)->device) != cudaSuccess) return fail((E), RDGPU_ERR_CUDA, "cudaSetDevice failed")

#define NEED_PARTICLES(E) \
    if ((E)->part_off.empty()) return fail((E), RDGPU_ERR_STATE, "no particles set")

int rdgpu_set_particles(rdgpu_handle h, const int64_t* offsets, int64_t n_total, const double* xyz,
                        const int32_t* types)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    if (n_total < 0 || (n_total > 0 && (!xyz || !types))) return fail(E, RDGPU_ERR_ARG, "invalid particle arrays");
    return DISPATCH(E, set_particles_impl, E, (const long long*)offsets, (long long)n_total, xyz, (const int*)types);
}

int rdgpu_apply_edits(rdgpu_handle h, const float* edits, int64_t count)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (E->nsys != 1) return fail(E, RDGPU_ERR_ARG, "reaction edits are defined for a single system");
    if (count < 0 || (count > 0 && !edits)) return fail(E, RDGPU_ERR_ARG, "invalid edit array");
    return DISPATCH(E, apply_edits_impl, E, edits, (long long)count);
}

int rdgpu_set_bonds(rdgpu_handle h, int64_t n_bonds, const int32_t* ij, const int32_t* pot, int32_t n_pots,
                    const rdgpu_pair_pot* pots)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (E->nsys != 1) return fail(E, RDGPU_ERR_ARG, "bonds are defined for a single system");
    if (n_bonds < 0 || n_pots < 0 || (n_bonds > 0 && (!ij || !pot || !pots || n_pots < 1)))
        return fail(E, RDGPU_ERR_ARG, "invalid bond arrays");
    if (n_bonds > 0x3fffffff) return fail(E, RDGPU_ERR_ARG, "too many bonds");
    return DISPATCH(E, set_bonds_impl, E, (long long)n_bonds, (const int*)ij, (const int*)pot, (int)n_pots, pots);
}

int rdgpu_get_particles(rdgpu_handle h, double* xyz, int32_t* types)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    return DISPATCH(E, get_particles_impl, E, xyz, (int*)types);
}

int rdgpu_set_particles_f32(rdgpu_handle h, const int64_t* offsets, int64_t n_total, const float* xyz,
                            const int32_t* types)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    if (n_total < 0 || (n_total > 0 && (!xyz || !types))) return fail(E, RDGPU_ERR_ARG, "invalid particle arrays");
    return DISPATCH(E, set_particles_impl, E, (const long long*)offsets, (long long)n_total, xyz, (const int*)types);
}

int rdgpu_get_particles_f32(rdgpu_handle h, float* xyz, int32_t* types)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    return DISPATCH(E, get_particles_impl, E, xyz, (int*)types);
}

int rdgpu_num_particles(rdgpu_handle h, int64_t* n)
{
    Engine* E = (Engine*)h;
    if (!E || !n) return RDGPU_ERR_ARG;
    *n = E->npart_tot;
    return RDGPU_OK;
}

int rdgpu_step(rdgpu_handle h, int64_t nsteps)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (nsteps < 0) return fail(E, RDGPU_ERR_ARG, "nsteps < 0");
    if (nsteps == 0 || E->npart_tot == 0) { E->step_h += nsteps; return prepare_step_state(E, E->step_h); }
    return DISPATCH(E, do_steps, E, (long long)nsteps, (const double*)nullptr);
}

int rdgpu_step_with_noise(rdgpu_handle h, const double* noise)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (!noise) return fail(E, RDGPU_ERR_ARG, "noise is null");
    if (E->npart_tot == 0) return RDGPU_OK;
    CK(cudaMemcpyAsync(E->vec_d, noise, E->npart_tot * 3 * sizeof(double), cudaMemcpyHostToDevice, E->stream));
    return DISPATCH(E, do_steps, E, 1LL, (const double*)E->vec_d);
}

int rdgpu_set_seed(rdgpu_handle h, int32_t sys, uint64_t seed)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    if (sys < 0 || sys >= E->nsys) return fail(E, RDGPU_ERR_ARG, "system index out of range");
    E->sys_h[sys].seed = seed;
    E->boxes[sys].seed = seed;
    CK(cudaMemcpyAsync(E->sys_d + sys, &E->sys_h[sys], sizeof(SysDev), cudaMemcpyHostToDevice, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    return RDGPU_OK;
}

int rdgpu_forces(rdgpu_handle h, double* forces, double* energy)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (E->npart_tot == 0) { if (energy) *energy = 0.0; return RDGPU_OK; }
    return DISPATCH(E, forces_impl, E, forces, energy);
}

int rdgpu_neighbor_digest(rdgpu_handle h, int32_t* counts, uint64_t* hashes)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (!counts || !hashes) return fail(E, RDGPU_ERR_ARG, "null output");
    if (E->npart_tot == 0) return RDGPU_OK;
    return DISPATCH(E, digest_impl, E, (int*)counts, (unsigned long long*)hashes);
}

int rdgpu_debug_noise(rdgpu_handle h, int64_t step, double* noise)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (!noise) return fail(E, RDGPU_ERR_ARG, "null output");
    if (E->npart_tot == 0) return RDGPU_OK;
    if (E->prec == RDGPU_PREC_F32C)
        noise_kernel<float><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(E->sys_d, E->sys_of, E->npart_tot, step, E->vec_d);
    else
        noise_kernel<double><<<grid_for(E->npart_tot), 256, 0, E->stream>>>(E->sys_d, E->sys_of, E->npart_tot, step, E->vec_d);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(noise, E->vec_d, E->npart_tot * 3 * sizeof(double), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    return RDGPU_OK;
}

int rdgpu_rdf(rdgpu_handle h, int32_t nbins, double rmax, int32_t accumulate, uint64_t* counts, int64_t* frames)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (nbins < 1 || nbins > 100000 || !(rmax > 0)) return fail(E, RDGPU_ERR_ARG, "invalid RDF bins/range");
    return DISPATCH(E, rdf_impl, E, (int)nbins, rmax, (int)accumulate, (unsigned long long*)counts, (long long*)frames);
}

int rdgpu_rdf_normalized(rdgpu_handle h, double* g)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (!E->rdf_acc || E->rdf_frames == 0) return fail(E, RDGPU_ERR_STATE, "no accumulated RDF frames");
    if (E->nsys != 1) return fail(E, RDGPU_ERR_ARG, "normalised RDF is defined for a single system");
    const int S = E->desc.n_types, H = S * S * E->rdf_nbins;
    std::vector<long long> nper(S, 0);
    int rc = DISPATCH(E, sync_types, E);
    if (rc) return rc;
    for (int t : E->types_h) nper[t]++;
    double vol = 1.0;
    for (int a = 0; a < 3; ++a)
        vol *= (E->prec == RDGPU_PREC_F32C) ? (double)E->sys_h[0].Lf[a] : E->sys_h[0].L[a];
    long long* nper_d = nullptr;
    double* g_d = nullptr;
    CK(cudaMalloc(&nper_d, S * sizeof(long long)));
    CK(cudaMalloc(&g_d, H * sizeof(double)));
    CK(cudaMemcpyAsync(nper_d, nper.data(), S * sizeof(long long), cudaMemcpyHostToDevice, E->stream));
    rdf_norm_kernel<<<(H + 255) / 256, 256, 0, E->stream>>>(E->rdf_acc, S, E->rdf_nbins, E->rdf_rmax / E->rdf_nbins,
                                                            (double)E->rdf_frames, vol, nper_d, g_d);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(g, g_d, H * sizeof(double), cudaMemcpyDeviceToHost, E->stream));
    CK(cudaStreamSynchronize(E->stream));
    cudaFree(nper_d);
    cudaFree(g_d);
    return RDGPU_OK;
}

int rdgpu_metrics_get(rdgpu_handle h, rdgpu_metrics* m)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (!m) return fail(E, RDGPU_ERR_ARG, "null output");
    memset(m, 0, sizeof(*m));
    m->step = E->step_h;
    m->neighbour_mode = E->nb_mode;
    m->list_builds = E->nbuild_h;
    m->skin = E->nb_mode == RDGPU_NB_LIST ? E->skin : 0.0;
    m->list_capacity = E->nb_mode == RDGPU_NB_LIST ? E->list_cap : 0;
    m->list_entry_bytes = E->nb_mode == RDGPU_NB_LIST ? (E->list_wide ? 4 : 2) : 0;
    if (E->npart_tot == 0) return RDGPU_OK;
    int rc = rdgpu_forces(h, nullptr, &m->energy);
    if (rc) return rc;
    return DISPATCH(E, msd_impl, E, m);
}

void* rdgpu_stream(rdgpu_handle h)
{
    Engine* E = (Engine*)h;
    return E ? (void*)E->stream : nullptr;
}

int rdgpu_step_profile(rdgpu_handle h, int64_t nsteps, double* step_kernel_ms, double* sort_ms)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (nsteps < 1 || E->npart_tot == 0) return fail(E, RDGPU_ERR_ARG, "nsteps >= 1 and particles needed");
    return DISPATCH(E, profile_impl, E, (long long)nsteps, step_kernel_ms, sort_ms);
}

int rdgpu_autotune(rdgpu_handle h)
{
    Engine* E = (Engine*)h;
    GUARD(E);
    NEED_PARTICLES(E);
    if (E->npart_tot == 0) return RDGPU_OK;
    if (E->nb_req == RDGPU_NB_AUTO && !E->tuned) {
        int rc = DISPATCH(E, tune, E);
        if (rc) return rc;
    }
    return DISPATCH(E, prepare_graph, E);
}

int64_t rdgpu_launch_count(rdgpu_handle h)
{
    Engine* E = (Engine*)h;
    return E ? E->launches : 0;
}

}  // extern "C"
