// rdf_noalloc.cu -- RDF pair counts for callers that cannot allocate device
// memory.
//
// Some hosts of this library cannot call cudaMalloc: a JVM or another
// runtime that hands out device buffers from its own pool, or a plug-in that
// must not change the device's memory footprint after start-up.  rdgpu_rdf_counts_noalloc computes the
// same counts as rdgpu_rdf, on positions and types the caller already has on
// the device, and writes them to a caller-provided device buffer.  Its scratch
// memory (cell binning) is the file-scope array below, which every GPU that
// loads the library holds until the process exits.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/readdy_b200.h"
#include "engine_device.cuh"

namespace {

using namespace rdgpu;

constexpr int NA_MAX_PARTICLES = RDGPU_NOALLOC_MAX_PARTICLES;
constexpr int NA_MAX_CELLS = RDGPU_NOALLOC_MAX_CELLS;
constexpr int NA_MAX_BINS = RDGPU_NOALLOC_MAX_BINS;

struct alignas(32) NaRec {
    double x, y, z;
    int type;
    int cell;
};

struct NaScratch {
    NaRec rec[NA_MAX_PARTICLES];        // particles sorted by cell
    int cnt[NA_MAX_CELLS];              // particles per cell
    int off[NA_MAX_CELLS + 1];          // exclusive prefix of cnt
    int cursor[NA_MAX_CELLS];           // scatter cursors
    double e2[NA_MAX_BINS + 1];         // squared bin edges
    int flags;                          // input errors
};

// The scratch of every call (about 3.8 MB on each device that loads the
// library).  Host code must not use this name as an address: it is resolved
// per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_na_scratch[sizeof(NaScratch)];

std::mutex g_na_mutex;
void* g_na_ptr[64] = {nullptr};          // resolved scratch address per device

struct NaBox {
    double L[3], half[3], lo[3];
    int n[3], per[3];
    double invc[3];
};

__device__ __forceinline__ bool na_wrap(double& x, double L, int per)
{
    if (!per) return true;
    for (int k = 0; k < 64 && x >= L; ++k) x -= L;
    for (int k = 0; k < 64 && x < 0.0; ++k) x += L;
    if (x >= L || x < 0.0) {
        if (x >= L && x - L < L) x = 0.0;
        else return false;
    }
    return true;
}

// box-relative position (the FP64 engine's stored representation) and cell
__device__ __forceinline__ bool na_locate(const double* xyz, long long i, const NaBox& b, double r[3], int& cell)
{
    bool ok = true;
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double x = __dsub_rn(xyz[3 * i + a], b.lo[a]);
        ok = ok && isfinite(x) && na_wrap(x, b.L[a], b.per[a]);
        r[a] = x;
        int k = (int)(x * b.invc[a]);
        c[a] = k < 0 ? 0 : (k >= b.n[a] ? b.n[a] - 1 : k);
    }
    cell = (c[2] * b.n[1] + c[1]) * b.n[0] + c[0];
    return ok;
}

__global__ void na_clear(NaScratch* s, int ncells, int nbins, double w)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncells; i += gridDim.x * blockDim.x) s->cnt[i] = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= nbins; k += gridDim.x * blockDim.x) {
        const double e = (double)k * w;
        s->e2[k] = e * e;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) s->flags = 0;
}

__global__ void na_count(NaScratch* s, const double* xyz, const int* types, long long n, int ntypes, NaBox b)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double r[3];
        int cell;
        const bool ok = na_locate(xyz, i, b, r, cell) && types[i] >= 0 && types[i] < ntypes;
        if (!ok) { atomicOr(&s->flags, 1); continue; }
        atomicAdd(&s->cnt[cell], 1);
    }
}

// exclusive scan of the cell counts, one block
__global__ void na_scan(NaScratch* s, int ncells)
{
    __shared__ int warp_tot[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, B = blockDim.x;
    const int per = (ncells + B - 1) / B;
    const int b0 = tid * per;
    int sum = 0;
    for (int k = 0; k < per; ++k)
        if (b0 + k < ncells) sum += s->cnt[b0 + k];
    int incl = warp_incl_scan(sum, lane);
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int v = lane < B / 32 ? warp_tot[lane] : 0;
        int vi = warp_incl_scan(v, lane);
        if (lane < B / 32) warp_tot[lane] = vi - v;
    }
    __syncthreads();
    int run = warp_tot[wid] + incl - sum;
    for (int k = 0; k < per; ++k) {
        if (b0 + k < ncells) {
            s->off[b0 + k] = run;
            s->cursor[b0 + k] = run;
            run += s->cnt[b0 + k];
        }
    }
    if (tid == B - 1) s->off[ncells] = run;
}

__global__ void na_scatter(NaScratch* s, const double* xyz, const int* types, long long n, NaBox b)
{
    if (s->flags) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double r[3];
        int cell;
        na_locate(xyz, i, b, r, cell);
        const int slot = atomicAdd(&s->cursor[cell], 1);
        NaRec q;
        q.x = r[0]; q.y = r[1]; q.z = r[2];
        q.type = types[i];
        q.cell = cell;
        s->rec[slot] = q;
    }
}

// ordered pairs i != j with r < rmax: the FP64 predicate and bin rule of the
// engine's rdf_kernel
__global__ void na_rdf(const NaScratch* __restrict__ s, long long n, int S, int nbins, double w, NaBox b,
                       int use_smem, unsigned long long* hist)
{
    extern __shared__ unsigned int sh[];
    const int H = S * S * nbins;
    if (use_smem) {
        for (int i = threadIdx.x; i < H; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    if (!s->flags) {
        const double rmax2 = s->e2[nbins];
        const double rmax = w * nbins;
        int lo3[3], cntax[3];
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
             i += (long long)gridDim.x * blockDim.x) {
            const NaRec p = s->rec[i];
            const int cc[3] = {p.cell % b.n[0], (p.cell / b.n[0]) % b.n[1], p.cell / (b.n[0] * b.n[1])};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                // half-width in cells; the margin keeps the outer layer when
                // rmax / cell edge rounds onto an integer (the cell edge
                // L / floor(L / rmax) can round to a hair below rmax)
                int r = (int)ceil(rmax * b.invc[a] * (1.0 + 1e-12));
                if (r < 1) r = 1;
                if (b.per[a]) {
                    if (2 * r + 1 >= b.n[a]) { lo3[a] = 0; cntax[a] = b.n[a]; }
                    else { lo3[a] = cc[a] - r; cntax[a] = 2 * r + 1; }
                } else {
                    const int l = max(0, cc[a] - r), h = min(b.n[a] - 1, cc[a] + r);
                    lo3[a] = l;
                    cntax[a] = h - l + 1;
                }
            }
            for (int iz = 0; iz < cntax[2]; ++iz) {
                int z = lo3[2] + iz;
                if (b.per[2]) z = (z % b.n[2] + b.n[2]) % b.n[2];
                for (int iy = 0; iy < cntax[1]; ++iy) {
                    int y = lo3[1] + iy;
                    if (b.per[1]) y = (y % b.n[1] + b.n[1]) % b.n[1];
                    for (int ix = 0; ix < cntax[0]; ++ix) {
                        int x = lo3[0] + ix;
                        if (b.per[0]) x = (x % b.n[0] + b.n[0]) % b.n[0];
                        const int nc = (z * b.n[1] + y) * b.n[0] + x;
                        for (int j = s->off[nc]; j < s->off[nc + 1]; ++j) {
                            if (j == i) continue;
                            const NaRec q = s->rec[j];
                            const double dx = mimg_sym(p.x, q.x, b.L[0], b.half[0], b.per[0]);
                            const double dy = mimg_sym(p.y, q.y, b.L[1], b.half[1], b.per[1]);
                            const double dz = mimg_sym(p.z, q.z, b.L[2], b.half[2], b.per[2]);
                            const double r2 = dist2(dx, dy, dz);
                            if (!(r2 < rmax2)) continue;
                            int k = (int)(sqrt(r2) / w);
                            k = min(max(k, 0), nbins - 1);
                            while (k > 0 && s->e2[k] > r2) --k;
                            while (k < nbins - 1 && s->e2[k + 1] <= r2) ++k;
                            const int hidx = (p.type * S + q.type) * nbins + k;
                            if (use_smem) atomicAdd(sh + hidx, 1u);
                            else atomicAdd(hist + hidx, 1ull);
                        }
                    }
                }
            }
        }
    }
    if (use_smem) {
        __syncthreads();
        for (int i = threadIdx.x; i < H; i += blockDim.x)
            if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
    }
}

}  // namespace

// the text rdgpu_last_error(NULL) returns (engine.cu)
std::string& rdgpu_global_error();

namespace {
int na_fail(int code, const std::string& msg)
{
    rdgpu_global_error() = msg;
    return code;
}
}  // namespace

extern "C" int rdgpu_rdf_counts_noalloc(const double* xyz_dev, const int32_t* types_dev, int64_t n,
                                        int32_t n_types, const double lo[3], const double hi[3],
                                        const int32_t periodic[3], int32_t nbins, double rmax,
                                        uint64_t* counts_dev, void* stream)
{
    if (!lo || !hi || !periodic || !counts_dev || (n > 0 && (!xyz_dev || !types_dev)))
        return na_fail(RDGPU_ERR_ARG, "null argument");
    if (n < 0 || n > NA_MAX_PARTICLES)
        return na_fail(RDGPU_ERR_ARG, "rdgpu_rdf_counts_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                                          std::to_string(NA_MAX_PARTICLES) + " particles");
    if (n_types < 1 || n_types > RDGPU_MAX_TYPES) return na_fail(RDGPU_ERR_ARG, "n_types out of range");
    if (nbins < 1 || nbins > NA_MAX_BINS)
        return na_fail(RDGPU_ERR_ARG, "rdgpu_rdf_counts_noalloc: nbins exceeds the maximum of " +
                                          std::to_string(NA_MAX_BINS));
    if (!(rmax > 0)) return na_fail(RDGPU_ERR_ARG, "rmax must be positive");
    NaBox b;
    long long ncells = 1;
    for (int a = 0; a < 3; ++a) {
        const double L = hi[a] - lo[a];
        if (!(L > 0)) return na_fail(RDGPU_ERR_ARG, "box bounds must satisfy hi > lo");
        b.L[a] = L;
        b.half[a] = 0.5 * L;
        b.lo[a] = lo[a];
        b.per[a] = periodic[a] ? 1 : 0;
        int k = (int)std::floor(L / rmax);
        if (k < 1) k = 1;
        if (k > 50) k = 50;          // 50^3 cells fit RDGPU_NOALLOC_MAX_CELLS
        b.n[a] = k;
        b.invc[a] = (double)k / L;
        ncells *= k;
    }
    if (ncells > NA_MAX_CELLS) return na_fail(RDGPU_ERR_ARG, "too many cells");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return na_fail(RDGPU_ERR_CUDA, "no CUDA device");
    // set-up, once per device, with that device current: resolve the address
    // of the static scratch (first call on a device; make it before any
    // stream capture)
    NaScratch* s;
    {
        std::lock_guard<std::mutex> g(g_na_mutex);
        if (!g_na_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
            if (e != cudaSuccess || !p)
                return na_fail(RDGPU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_na_ptr[dev] = p;
        }
        s = (NaScratch*)g_na_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int S = n_types, H = S * S * nbins;
    const double w = rmax / (double)nbins;
    if (cudaMemsetAsync(counts_dev, 0, (size_t)H * sizeof(unsigned long long), st) != cudaSuccess)
        return na_fail(RDGPU_ERR_CUDA, "cudaMemsetAsync failed");
    const int blocks = 148 * 4;
    na_clear<<<blocks, 256, 0, st>>>(s, (int)ncells, nbins, w);
    if (n > 0) {
        na_count<<<blocks, 256, 0, st>>>(s, xyz_dev, types_dev, n, n_types, b);
        na_scan<<<1, 1024, 0, st>>>(s, (int)ncells);
        na_scatter<<<blocks, 256, 0, st>>>(s, xyz_dev, types_dev, n, b);
        const int use_smem = (H * 4 <= 48 * 1024) ? 1 : 0;
        na_rdf<<<blocks, 128, use_smem ? H * 4 : 0, st>>>(s, n, S, nbins, w, b, use_smem,
                                                          (unsigned long long*)counts_dev);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(RDGPU_ERR_CUDA, cudaGetErrorString(e));
    int flags = 0;
    if (cudaMemcpyAsync(&flags, &s->flags, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return na_fail(RDGPU_ERR_CUDA, "synchronisation failed");
    if (flags) return na_fail(RDGPU_ERR_ARG, "particle type out of range, non-finite coordinate, or a coordinate "
                                             "more than 64 box lengths outside the box");
    return RDGPU_OK;
}
