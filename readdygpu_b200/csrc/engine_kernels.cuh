// engine_kernels.cuh -- __global__ kernels of the Brownian-dynamics engine.
//
// State layout (all systems of a batch share the arrays; a system's
// particles are a contiguous range of the sorted arrays):
//   FP32C: pos[i] = float4(x, y, z, bits(type | image counters))
//          aux[i] = float4(cx, cy, cz, bits(id)); true position = pos - aux
//   FP64:  rec[i] = Rec64{x, y, z, w = type | images, id}
//   sorted by cell: particles of cell c are [start[c], start[c+1]), cells of
//   system s are numbered from cell_base[s], cell id = (z*n1 + y)*n0 + x.
//
// One Brownian-dynamics step = four launches captured in a CUDA graph:
//   step_kernel     forces over the 27-cell neighbourhood (9 contiguous row
//                   ranges of the sorted arrays), external forces,
//                   Euler-Maruyama with Philox noise, wrap; writes the new
//                   state to the staging arrays with its new cell and its
//                   slot in that cell (atomicAdd on the cell counts)
//   scan_tiles      tile sums of the cell counts
//   scan_apply      cell starts (exclusive prefix), counts cleared
//   scatter_kernel  staging -> sorted arrays at start[cell] + slot
// With the pair list (list_step_kernel, list_check_kernel and the re-sort
// chain further down) a step is the step kernel, the check of the particles
// that moved more than about skin/2 since the last build and, only when the
// check or the step asks for it, the re-sort and list build.
// This replaces the reference's orderOne / warpOrderTwo / update launches and
// its linked-list relinking under spin locks
// (lib/ReaDDyGPU_Cpp/CudaKernels/CudaSimulation.cu:1034-1236, 1402-1782,
// 1838-1919).
#pragma once
#include <type_traits>
#include "engine_device.cuh"

namespace rdgpu {

constexpr int EF_BADINPUT = 8;
constexpr int SCAN_TILE = 4096;     // cells per scan tile
constexpr int SCAN_BLOCK = 256;

template <class R> struct State;
template <> struct State<float> {
    float4* pos;
    float4* aux;
};
template <> struct State<double> {
    Rec64* rec;
};

template <class R> struct Args {
    const SysDev* sys;
    const unsigned short* sys_of;   // system of each particle index (static)
    long long ntot;
    int nsys;
    int n_ext;
    const TypeTab<R>* tab;
    const ExtTerm<R>* ext;          // [sys * n_ext + e]
    State<R> cur;                   // sorted state
    State<R> stg;                   // staging (new state by sorted index)
    const int* start;               // cell starts, ncells_tot + 1
    int* counts;                    // per cell, zero before a step
    int* tcell;                     // new global cell per particle
    int* tslot;                     // slot in the new cell
    int* err;
    long long* err_step;
    const long long* step_ptr;
    int step_off;
    const double* noise;            // injected noise (3 per global index) or null
    // bonded pairs of particle groups (single system; null: none)
    const int* bstart;              // bonds of particle id: bstart[id] .. bstart[id+1]
    const int* bpart;               // partner id of each bond entry
    const int* bterm;               // its potential term
    const PairTerm<R>* btab;        // resolved bond potential terms
    int* inv;                       // sorted index of each particle id (kept by the scatters)
};

// force accumulators: FP32 sums pair forces in 2^-32 fixed point (exact,
// order independent), FP64 sums in double.
template <class R> struct Acc;
template <> struct Acc<float> {
    long long fx, fy, fz;
    float e;
    __device__ __forceinline__ void zero() { fx = fy = fz = 0; e = 0.f; }
    __device__ __forceinline__ void add(float pre, float dx, float dy, float dz)
    {
        // scaling by 2^32 is exact, so (-pre 2^32) d == ((-pre) d) 2^32
        const float q = -pre * FX_SCALE;
        fx += __float2ll_rn(q * dx);
        fy += __float2ll_rn(q * dy);
        fz += __float2ll_rn(q * dz);
    }
    __device__ __forceinline__ void force(float F[3]) const
    {
        F[0] = __ll2float_rn(fx) * FX_INV;
        F[1] = __ll2float_rn(fy) * FX_INV;
        F[2] = __ll2float_rn(fz) * FX_INV;
    }
};
template <> struct Acc<double> {
    double fx, fy, fz, e;
    __device__ __forceinline__ void zero() { fx = fy = fz = e = 0.0; }
    __device__ __forceinline__ void add(double pre, double dx, double dy, double dz)
    {
        fx -= pre * dx;
        fy -= pre * dy;
        fz -= pre * dz;
    }
    __device__ __forceinline__ void force(double F[3]) const { F[0] = fx; F[1] = fy; F[2] = fz; }
};

// ---------------------------------------------------------------------------
// state access
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_pos(const State<float>& s, long long i, float x[3], int& w)
{
    const float4 p = __ldg(s.pos + i);
    x[0] = p.x; x[1] = p.y; x[2] = p.z;
    w = __float_as_int(p.w);
}
__device__ __forceinline__ void load_pos(const State<double>& s, long long i, double x[3], int& w)
{
    const double2* p = reinterpret_cast<const double2*>(s.rec + i);
    const double2 a = __ldg(p), b = __ldg(p + 1);
    x[0] = a.x; x[1] = a.y; x[2] = b.x;
    w = __double2loint(b.y);
}
__device__ __forceinline__ int load_id(const State<float>& s, long long i) { return __float_as_int(__ldg(&s.aux[i].w)); }
__device__ __forceinline__ int load_id(const State<double>& s, long long i) { return __ldg(&s.rec[i].id); }

template <class R>
__device__ __forceinline__ void cell_coords(const SysDev& s, const R x[3], int c[3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        R inv;
        if constexpr (sizeof(R) == 4) inv = s.invcf[a]; else inv = s.invc[a];
        int k = (int)(x[a] * inv);
        c[a] = k < 0 ? 0 : (k >= s.n[a] ? s.n[a] - 1 : k);
    }
}

// ---------------------------------------------------------------------------
// Pair sum over the 27-cell neighbourhood: 9 rows (dy, dz), each one or two
// contiguous ranges of the sorted arrays.  MODE 0: forces; 1: forces +
// energy; 2: neighbour digest.  VALUE_IMAGE: minimum image chosen per
// candidate (systems with fewer than 3 cells on a periodic axis, where each
// neighbour cell is visited once); otherwise the image is the cell wrap of
// the range, which for >= 3 cells gives the same displacement xi - (xj + kL)
// for every pair inside the cutoff.
// ---------------------------------------------------------------------------
// Harmonic-repulsion-only fast path: every type pair has at most the one
// term k (r - r0)/r for r < r0 (P2_Harmonic.java:167-178 with rc = r0), with
// k and r0 in shared memory; the general path walks the term table.
template <class R> struct FastTab {
    R k[MAXT * MAXT];
    R r0[MAXT * MAXT];
};

template <class R, int MODE, bool VALUE_IMAGE, bool SHIFT, bool HREP>
__device__ __forceinline__ void range_pairs(const State<R>& st, int j0, int j1, int self, const R xi[3], int ti,
                                            R sx, R sy, R sz, const R* __restrict__ rc2, const FastTab<R>* __restrict__ ft,
                                            const Box<R>& bx, const SysDev& s, const TypeTab<R>* __restrict__ tab,
                                            Acc<R>& acc, int& ncount, unsigned long long& hash)
{
    for (int j = j0; j < j1; ++j) {
        R xj[3];
        int wj;
        load_pos(st, j, xj, wj);
        R dx, dy, dz;
        if (VALUE_IMAGE) {
            dx = mimg(xi[0], xj[0], bx.L[0], bx.half[0], s.per[0]);
            dy = mimg(xi[1], xj[1], bx.L[1], bx.half[1], s.per[1]);
            dz = mimg(xi[2], xj[2], bx.L[2], bx.half[2], s.per[2]);
        } else if (SHIFT) {
            dx = sub_rn(xi[0], add_rn(xj[0], sx));
            dy = sub_rn(xi[1], add_rn(xj[1], sy));
            dz = sub_rn(xi[2], add_rn(xj[2], sz));
        } else {
            dx = sub_rn(xi[0], xj[0]);
            dy = sub_rn(xi[1], xj[1]);
            dz = sub_rn(xi[2], xj[2]);
        }
        const R r2 = dist2(dx, dy, dz);
        const int pidx = ti * MAXT + (wj & 0xff);
        if (r2 < rc2[pidx] && j != self) {
            if (MODE == 2) {
                ncount++;
                hash += splitmix64((unsigned long long)load_id(st, j));
                continue;
            }
            if (HREP && MODE == 0) {
                // force only: pre = k (r - r0) / r; r == 0 has no direction
                if (r2 > R(0)) {
                    R pre;
                    if constexpr (sizeof(R) == 4) pre = ft->k[pidx] * (1.0f - ft->r0[pidx] * rsqrtf(r2));
                    else { const R r = sqrt(r2); pre = ft->k[pidx] * (r - ft->r0[pidx]) / r; }
                    acc.add(pre, dx, dy, dz);
                }
                continue;
            }
            const R r = sqrt(r2);
            const int nt = tab->nterm[pidx];
            for (int m = 0; m < nt; ++m) {
                R pre, e;
                pair_term(tab->term[pidx * MAX_TERMS + m], r, pre, e);
                acc.add(pre, dx, dy, dz);
                if (MODE == 1) acc.e += R(0.5) * e;
            }
        }
    }
}

// squared gap between coordinate x (cell-local offset f in [0, c)) and the
// neighbour cell at offset d: 0 for d == 0, f^2 below, (c - f)^2 above
template <class R>
__device__ __forceinline__ R gap2(int d, R f, R c)
{
    const R g = d < 0 ? f : (d > 0 ? c - f : R(0));
    return g * g;
}

// Pair sum over the 27-cell neighbourhood.  Cells whose nearest point is
// farther than the particle's largest cutoff (with a relative margin of 1e-4,
// far above rounding) are skipped: they cannot hold a neighbour, so the
// neighbour set is unchanged.
template <class R, int MODE, bool VALUE_IMAGE, bool HREP>
__device__ __forceinline__ void neighbourhood(const State<R>& st, const int* __restrict__ start, const SysDev& s,
                                              const int c[3], int self, const R xi[3], int ti,
                                              const R* __restrict__ rc2, const FastTab<R>* __restrict__ ft,
                                              const TypeTab<R>* __restrict__ tab, Acc<R>& acc, int& ncount,
                                              unsigned long long& hash, R rmax2)
{
    Box<R> bx;
    bx.load(s);
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    R cw[3], f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if constexpr (sizeof(R) == 4) cw[a] = R(1) / s.invcf[a]; else cw[a] = R(1) / s.invc[a];
        f[a] = xi[a] - (R)c[a] * cw[a];
        // a periodic axis with fewer than 3 cells reaches each cell from
        // either side: no pruning along it (zero gaps)
        if (VALUE_IMAGE && s.per[a] && s.n[a] < 3) { f[a] = R(0); cw[a] = R(0); }
    }
    const R lim = rmax2 * R(1.0001);
    for (int dz = -1; dz <= 1; ++dz) {
        const R gz = gap2(dz, f[2], cw[2]);
        if (gz >= lim) continue;
        int z = c[2] + dz;
        R sz = R(0);
        if (z < 0 || z >= n2) {
            if (!s.per[2]) continue;
            if (VALUE_IMAGE && n2 < 3) continue;       // each cell once: only in-range offsets
            sz = z < 0 ? -bx.L[2] : bx.L[2];
            z = z < 0 ? z + n2 : z - n2;
        }
        for (int dy = -1; dy <= 1; ++dy) {
            const R gyz = gz + gap2(dy, f[1], cw[1]);
            if (gyz >= lim) continue;
            int y = c[1] + dy;
            R sy = R(0);
            if (y < 0 || y >= n1) {
                if (!s.per[1]) continue;
                if (VALUE_IMAGE && n1 < 3) continue;
                sy = y < 0 ? -bx.L[1] : bx.L[1];
                y = y < 0 ? y + n1 : y - n1;
            }
            const int row = (int)s.cell_base + (z * n1 + y) * n0;
            const bool shifted = (sy != R(0)) || (sz != R(0));
            // x cells of the row within reach
            int xa = (gyz + f[0] * f[0] < lim) ? c[0] - 1 : c[0];
            int xb = (gyz + (cw[0] - f[0]) * (cw[0] - f[0]) < lim) ? c[0] + 1 : c[0];
            if (VALUE_IMAGE) {
                if (!s.per[0] || n0 < 3) { xa = max(xa, 0); xb = min(xb, n0 - 1); }
                else {
                    // ranges with the x wrap: the image is chosen per candidate
                    if (xa < 0) {
                        range_pairs<R, MODE, true, false, HREP>(st, start[row + n0 - 1], start[row + n0], self, xi, ti,
                                                                R(0), R(0), R(0), rc2, ft, bx, s, tab, acc, ncount, hash);
                        xa = 0;
                    }
                    if (xb >= n0) {
                        range_pairs<R, MODE, true, false, HREP>(st, start[row], start[row + 1], self, xi, ti, R(0),
                                                                R(0), R(0), rc2, ft, bx, s, tab, acc, ncount, hash);
                        xb = n0 - 1;
                    }
                }
                range_pairs<R, MODE, true, false, HREP>(st, start[row + xa], start[row + xb + 1], self, xi, ti, R(0),
                                                        R(0), R(0), rc2, ft, bx, s, tab, acc, ncount, hash);
                continue;
            }
            if (!s.per[0]) {
                xa = max(xa, 0);
                xb = min(xb, n0 - 1);
            } else {
                if (xa < 0) {
                    range_pairs<R, MODE, false, true, HREP>(st, start[row + n0 - 1], start[row + n0], self, xi, ti,
                                                            -bx.L[0], sy, sz, rc2, ft, bx, s, tab, acc, ncount, hash);
                    xa = 0;
                }
                if (xb >= n0) {
                    range_pairs<R, MODE, false, true, HREP>(st, start[row], start[row + 1], self, xi, ti, bx.L[0], sy,
                                                            sz, rc2, ft, bx, s, tab, acc, ncount, hash);
                    xb = n0 - 1;
                }
            }
            if (shifted)
                range_pairs<R, MODE, false, true, HREP>(st, start[row + xa], start[row + xb + 1], self, xi, ti, R(0),
                                                        sy, sz, rc2, ft, bx, s, tab, acc, ncount, hash);
            else
                range_pairs<R, MODE, false, false, HREP>(st, start[row + xa], start[row + xb + 1], self, xi, ti, R(0),
                                                         R(0), R(0), rc2, ft, bx, s, tab, acc, ncount, hash);
        }
    }
}

// ---------------------------------------------------------------------------
// Flattened force walk for systems with >= 3 cells on every periodic axis.
//
// The per-row loops of neighbourhood() make a warp iterate, for every one of
// the 9 rows, as often as its longest lane needs, and run the accepted-pair
// block in nearly every iteration for the few lanes that accept.  Here each
// thread walks its 9 row ranges as ONE sequence of candidates (the warp
// iterates max over lanes of the candidate total), and accepted pairs go to a
// short per-thread list in shared memory that is evaluated in bulk.  Row
// bounds are loaded up front, all 18 loads in flight together, and kept in
// shared memory.  The periodic x wrap of boundary cells is a second, rare
// pass.  Rows, images, pruning and the pair set are those of neighbourhood();
// forces of FP32 states are bit-identical (fixed-point accumulation).
// ---------------------------------------------------------------------------
template <class R> struct PairRec;
template <> struct __align__(16) PairRec<float> { float dx, dy, dz; int pidx; };
template <> struct __align__(16) PairRec<double> { double dx, dy, dz; long long pidx; };

template <class R, bool HREP, int BLOCK>
__device__ __forceinline__ void flush_pairs(const PairRec<R>* __restrict__ l, int cnt,
                                            const FastTab<R>* __restrict__ ft,
                                            const TypeTab<R>* __restrict__ tab, Acc<R>& acc)
{
    for (int m = 0; m < cnt; ++m) {
        const PairRec<R> p = l[m * BLOCK];
        const int pidx = (int)p.pidx;
        const R r2 = dist2(p.dx, p.dy, p.dz);
        if (HREP) {
            // pre = k (r - r0) / r; r == 0 has no direction
            if (r2 > R(0)) {
                R pre;
                if constexpr (sizeof(R) == 4) pre = ft->k[pidx] * (1.0f - ft->r0[pidx] * rsqrtf(r2));
                else { const R r = sqrt(r2); pre = ft->k[pidx] * (r - ft->r0[pidx]) / r; }
                acc.add(pre, p.dx, p.dy, p.dz);
            }
        } else {
            const R r = sqrt(r2);
            const int nt = tab->nterm[pidx];
            for (int q = 0; q < nt; ++q) {
                R pre, e;
                pair_term(tab->term[pidx * MAX_TERMS + q], r, pre, e);
                acc.add(pre, p.dx, p.dy, p.dz);
            }
        }
    }
}

// shift code of one axis: 0 none, 1 minus L, 2 plus L
template <class R> __device__ __forceinline__ R shift_of(unsigned code, R L)
{
    return (code & 1u) ? -L : ((code & 2u) ? L : R(0));
}

template <class R, bool HREP, int BLOCK, int CAP>
__device__ __forceinline__ void neighbourhood_flat(const State<R>& st, const int* __restrict__ start,
                                                   const SysDev& s, const int c[3], int self, const R xi[3], int ti,
                                                   const R* __restrict__ rc2, const FastTab<R>* __restrict__ ft,
                                                   const TypeTab<R>* __restrict__ tab, Acc<R>& acc, R rmax2,
                                                   int* __restrict__ s_j0, int* __restrict__ s_j1,
                                                   PairRec<R>* __restrict__ s_list)
{
    const int tid = threadIdx.x;
    Box<R> bx;
    bx.load(s);
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    R cw[3], f[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        if constexpr (sizeof(R) == 4) cw[q] = R(1) / s.invcf[q]; else cw[q] = R(1) / s.invc[q];
        f[q] = xi[q] - (R)c[q] * cw[q];
    }
    const R lim = rmax2 * R(1.0001);
    const R fx2 = f[0] * f[0], gx2 = (cw[0] - f[0]) * (cw[0] - f[0]);
    // rows r = 3 (dz + 1) + (dy + 1): bounds to shared memory, image shift
    // codes of y and z packed 2 bits per row, x-wrap rows as a bit mask
    unsigned ycode = 0, zcode = 0, wrap = 0;
    int rowpos[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        int z = c[2] + dz, y = c[1] + dy;
        bool v = true;
        unsigned zc = 0, yc = 0;
        if (z < 0) { if (s.per[2]) { z += n2; zc = 1; } else v = false; }
        else if (z >= n2) { if (s.per[2]) { z -= n2; zc = 2; } else v = false; }
        if (y < 0) { if (s.per[1]) { y += n1; yc = 1; } else v = false; }
        else if (y >= n1) { if (s.per[1]) { y -= n1; yc = 2; } else v = false; }
        const R gyz = gap2(dz, f[2], cw[2]) + gap2(dy, f[1], cw[1]);
        v = v && gyz < lim;
        const int row = (int)s.cell_base + (z * n1 + y) * n0;
        int xa = (gyz + fx2 < lim) ? c[0] - 1 : c[0];
        int xb = (gyz + gx2 < lim) ? c[0] + 1 : c[0];
        if (v && s.per[0] && (xa < 0 || xb >= n0)) wrap |= 1u << r;
        xa = max(xa, 0);
        xb = min(xb, n0 - 1);
        ycode |= yc << (2 * r);
        zcode |= zc << (2 * r);
        rowpos[r] = row;
        s_j0[r * BLOCK + tid] = v ? __ldg(start + row + xa) : 0;
        s_j1[r * BLOCK + tid] = v ? __ldg(start + row + xb + 1) : 0;
    }
    int cnt = 0;
    R sx = R(0);
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            if (!wrap) break;
            // the wrapped-around boundary cell of each wrap row, shifted by -L
            // (cell n0 - 1 seen from cell 0) or +L (cell 0 seen from n0 - 1)
            const bool lo = c[0] == 0;
            sx = lo ? -bx.L[0] : bx.L[0];
#pragma unroll
            for (int r = 0; r < 9; ++r) {
                const bool w = (wrap >> r) & 1u;
                const int cx = rowpos[r] + (lo ? n0 - 1 : 0);
                s_j0[r * BLOCK + tid] = w ? __ldg(start + cx) : 0;
                s_j1[r * BLOCK + tid] = w ? __ldg(start + cx + 1) : 0;
            }
        }
        int r = -1, j = 0, e = 0;
        R sy = R(0), sz = R(0);
        for (;;) {
            if (j >= e) {
                do {
                    if (++r == 9) break;
                    j = s_j0[r * BLOCK + tid];
                    e = s_j1[r * BLOCK + tid];
                } while (j >= e);
                if (r == 9) break;
                sy = shift_of<R>(ycode >> (2 * r), bx.L[1]);
                sz = shift_of<R>(zcode >> (2 * r), bx.L[2]);
            }
            R xj[3];
            int wj;
            load_pos(st, j, xj, wj);
            const R dx = sub_rn(xi[0], add_rn(xj[0], sx));
            const R dy = sub_rn(xi[1], add_rn(xj[1], sy));
            const R dz = sub_rn(xi[2], add_rn(xj[2], sz));
            const R r2 = dist2(dx, dy, dz);
            const int pidx = ti * MAXT + (wj & 0xff);
            if (r2 < rc2[pidx] && j != self) {
                PairRec<R> p;
                p.dx = dx; p.dy = dy; p.dz = dz; p.pidx = pidx;
                s_list[cnt * BLOCK + tid] = p;
                if (++cnt == CAP) {
                    flush_pairs<R, HREP, BLOCK>(s_list + tid, cnt, ft, tab, acc);
                    cnt = 0;
                }
            }
            ++j;
        }
    }
    flush_pairs<R, HREP, BLOCK>(s_list + tid, cnt, ft, tab, acc);
}

// ---------------------------------------------------------------------------
// Euler-Maruyama update + wrap (CudaSimulation.cu:1852-1858 with the Java
// mobility D dt/(kB T), ParticleParametersFactory.java:152-155)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int img_add(int w, int axis, int delta)
{
    const int sh = 8 + 8 * axis;
    int v = ((w >> sh) + delta) & 0xff;
    return (w & ~(0xff << sh)) | (v << sh);
}

// FP32 with Kahan compensation: true position = x - c.  ALLPER: every axis
// of the system is periodic (known to the caller; spares the per-axis test)
template <bool ALLPER = false>
__device__ __forceinline__ int em_update(float x[3], float c[3], int& w, const float F[3], const float xi[3], float A,
                                         float B, const SysDev& s)
{
    int ef = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float inc = A * F[a] + B * xi[a];
        float y = inc - c[a];
        float t = x[a] + y;
        c[a] = (t - x[a]) - y;
        x[a] = t;
        if (ALLPER || s.per[a]) {
            const float L = s.Lf[a];
            if (x[a] >= L) {
                x[a] = x[a] - L;                // exact (Sterbenz)
                w = img_add(w, a, 1);
            } else if (x[a] < 0.0f) {
                float sum = x[a] + L;           // Fast2Sum: sum + e == x + L
                float e = x[a] - (sum - L);
                c[a] = c[a] - e;
                x[a] = sum;
                w = img_add(w, a, -1);
                if (x[a] >= L) { x[a] = x[a] - L; w = img_add(w, a, 1); }
            }
            if (!(x[a] >= 0.0f && x[a] < L)) ef |= EF_JUMP;
        }
        if (!isfinite(x[a])) ef |= EF_NONFINITE;
    }
    return ef;
}

template <bool ALLPER = false>
__device__ __forceinline__ int em_update(double x[3], double* /*c*/, int& w, const double F[3], const double xi[3],
                                         double A, double B, const SysDev& s)
{
    int ef = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = x[a] + (A * F[a] + B * xi[a]);
        if (ALLPER || s.per[a]) {
            const double L = s.L[a];
            if (v >= L) { v -= L; w = img_add(w, a, 1); }
            else if (v < 0.0) { v += L; w = img_add(w, a, -1); }
            if (v >= L) { v = 0.0; w = img_add(w, a, 1); }
            if (!(v >= 0.0 && v < L)) ef |= EF_JUMP;
        }
        if (!isfinite(v)) ef |= EF_NONFINITE;
        x[a] = v;
    }
    return ef;
}

// ---------------------------------------------------------------------------
// The step kernel: one thread per particle of the sorted arrays
// ---------------------------------------------------------------------------
// forces (and, for MODE 1, half energies) of the bonds of particle id: one
// pair potential each, at any distance, minimum image (the groups of
// ReaDDy; CudaSimulation.cu:1829-1836 with each particle's own type)
template <class R, int MODE>
__device__ __forceinline__ void bond_forces(const Args<R>& a, const State<R>& st, int id, const R xi[3],
                                            const SysDev& s, Acc<R>& acc)
{
    Box<R> bx;
    bx.load(s);
    for (int b = a.bstart[id]; b < a.bstart[id + 1]; ++b) {
        const int j = a.inv[a.bpart[b]];
        R xj[3];
        int wj;
        load_pos(st, j, xj, wj);
        const R dx = mimg_sel(xi[0], xj[0], bx.L[0], bx.half[0], s.per[0]);
        const R dy = mimg_sel(xi[1], xj[1], bx.L[1], bx.half[1], s.per[1]);
        const R dz = mimg_sel(xi[2], xj[2], bx.L[2], bx.half[2], s.per[2]);
        const R r = sqrt(dist2(dx, dy, dz));
        R pre, e;
        pair_term(a.btab[a.bterm[b]], r, pre, e);
        acc.add(pre, dx, dy, dz);
        if (MODE == 1) acc.e += R(0.5) * e;
    }
}

// sorted index of every particle id
template <class R>
__global__ void inv_kernel(State<R> cur, long long ntot, int* __restrict__ inv)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x)
        inv[load_id(cur, i)] = (int)i;
}

template <class R, bool VALUE_IMAGE, bool HREP, int BLOCK>
__global__ void __launch_bounds__(BLOCK, (sizeof(R) == 4 ? 1024 : 768) / BLOCK) step_kernel(Args<R> a)
{
    __shared__ R s_rc2[MAXT * MAXT];
    __shared__ R s_rmax2[MAXT];
    __shared__ FastTab<R> s_ft;
    constexpr int CAP = 4;
    constexpr bool FLAT = !VALUE_IMAGE && sizeof(R) == 8;
    __shared__ int s_j0[FLAT ? 9 * BLOCK : 1], s_j1[FLAT ? 9 * BLOCK : 1];
    __shared__ PairRec<R> s_list[FLAT ? CAP * BLOCK : 1];
    if (*((volatile int*)a.err)) return;   // an earlier step failed: keep its input intact
    // rows of the S types in use (entries (ti, tj) with ti >= S are never read)
    for (int k = threadIdx.x; k < MAXT * a.tab->S; k += BLOCK) {
        s_rc2[k] = a.tab->rc2[k];
        if (HREP) {
            s_ft.k[k] = a.tab->nterm[k] ? a.tab->term[k * MAX_TERMS].k : R(0);
            s_ft.r0[k] = a.tab->nterm[k] ? a.tab->term[k * MAX_TERMS].r0 : R(0);
        }
    }
    for (int k = threadIdx.x; k < MAXT; k += BLOCK) {
        R m = R(0);
        for (int j = 0; j < MAXT; ++j) m = max(m, a.tab->rc2[k * MAXT + j]);
        s_rmax2[k] = m;
    }
    __syncthreads();
    const long long t = (a.step_ptr ? *a.step_ptr : 0LL) + a.step_off;
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    if (i >= a.ntot) return;
    const int si = a.sys_of[i];
    const SysDev& s = a.sys[si];
    R xi[3];
    int wi;
    load_pos(a.cur, i, xi, wi);
    const int ti = wi & 0xff;
    R c[3] = {R(0), R(0), R(0)};
    int id;
    if constexpr (sizeof(R) == 4) {
        const float4 q = __ldg(a.cur.aux + i);
        c[0] = q.x; c[1] = q.y; c[2] = q.z;
        id = __float_as_int(q.w);
    } else {
        id = __ldg(&a.cur.rec[i].id);
    }
    int cc[3];
    cell_coords(s, xi, cc);
    Acc<R> acc;
    acc.zero();
    int nc = 0;
    unsigned long long hh = 0;
    // FP64 states take the flattened walk (faster there); FP32 states the
    // per-row walk, which measured slightly faster for them
    if (VALUE_IMAGE || sizeof(R) == 4)
        neighbourhood<R, 0, VALUE_IMAGE, HREP>(a.cur, a.start, s, cc, i, xi, ti, s_rc2, &s_ft, a.tab, acc, nc, hh,
                                               s_rmax2[ti]);
    else
        neighbourhood_flat<R, HREP, BLOCK, CAP>(a.cur, a.start, s, cc, i, xi, ti, s_rc2, &s_ft, a.tab, acc,
                                                s_rmax2[ti], s_j0, s_j1, s_list);
    if (a.bstart) bond_forces<R, 0>(a, a.cur, id, xi, s, acc);
    R F[3];
    acc.force(F);
    if (a.n_ext > 0) {
        const ExtTerm<R>* ep = a.ext + (long long)si * a.n_ext;
        R ee = R(0);
        for (int e = 0; e < a.n_ext; ++e)
            if ((ep[e].tmask >> ti) & 1u) ext_force(ep[e], a.tab->prad[ti], xi, F, ee);
    }
    R xn[3];
    if (a.noise) {
        const double* nz = a.noise + 3 * (s.part_base + id);
        xn[0] = (R)nz[0]; xn[1] = (R)nz[1]; xn[2] = (R)nz[2];
    } else {
        bd_normals(s.seed, t, (long long)id, xn);
    }
    int ef = em_update(xi, c, wi, F, xn, a.tab->a[ti], a.tab->b[ti], s);
    int nc3[3];
    cell_coords(s, xi, nc3);
    const long long ncell = s.cell_base + ((long long)nc3[2] * s.n[1] + nc3[1]) * s.n[0] + nc3[0];
    a.tslot[i] = atomicAdd(a.counts + ncell, 1);
    a.tcell[i] = (int)ncell;
    if constexpr (sizeof(R) == 4) {
        a.stg.pos[i] = make_float4(xi[0], xi[1], xi[2], __int_as_float(wi));
        a.stg.aux[i] = make_float4(c[0], c[1], c[2], __int_as_float(id));
    } else {
        Rec64 r;
        r.x = xi[0]; r.y = xi[1]; r.z = xi[2]; r.w = wi; r.id = id;
        a.stg.rec[i] = r;
    }
    if (ef) {
        atomicOr(a.err, ef);
        atomicMin((unsigned long long*)a.err_step, (unsigned long long)t);
    }
}

// ---------------------------------------------------------------------------
// counting sort: tile sums, exclusive prefix, scatter
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SCAN_BLOCK) scan_tiles_kernel(const int* __restrict__ counts, long long ncells,
                                                                int* __restrict__ tile_sum, const int* err,
                                                                const int* gate)
{
    __shared__ int red[SCAN_BLOCK / 32];
    if (*((volatile const int*)err)) return;
    if (gate && !*((volatile const int*)gate)) return;
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    int sum = 0;
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_BLOCK) {
        const long long c = base + k;
        if (c < ncells) sum += counts[c];
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < SCAN_BLOCK / 32; ++w) tot += red[w];
        tile_sum[blockIdx.x] = tot;
    }
}

// start[c] = exclusive prefix of counts; counts cleared for the next step;
// start[ncells] = total.  The tile goes through shared memory so that every
// global access is coalesced.
__global__ void __launch_bounds__(SCAN_BLOCK) scan_apply_kernel(int* __restrict__ counts, long long ncells,
                                                                const int* __restrict__ tile_sum, int ntiles,
                                                                int* __restrict__ start, const int* err,
                                                                const int* gate)
{
    constexpr int PER = SCAN_TILE / SCAN_BLOCK;
    __shared__ int s_t[SCAN_TILE + SCAN_TILE / 32];   // padded against bank conflicts
    __shared__ int s_w[SCAN_BLOCK / 32];
    __shared__ int s_base;
    if (*((volatile const int*)err)) return;
    if (gate && !*((volatile const int*)gate)) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long long base_c = (long long)blockIdx.x * SCAN_TILE;
    // base of this tile: sum of the preceding tile sums
    int b = 0;
    for (int k = tid; k < (int)blockIdx.x; k += SCAN_BLOCK) b += tile_sum[k];
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(FULL, b, o);
    if (lane == 0) s_w[wid] = b;
    // coalesced load of the tile; the counts are cleared for the next step
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = k * SCAN_BLOCK + tid;
        const long long c = base_c + e;
        int v = 0;
        if (c < ncells) {
            v = counts[c];
            counts[c] = 0;
        }
        s_t[e + (e >> 5)] = v;
    }
    __syncthreads();
    if (tid == 0) {
        int tot = 0;
        for (int w = 0; w < SCAN_BLOCK / 32; ++w) tot += s_w[w];
        s_base = tot;
    }
    // each thread scans PER contiguous elements
    int v[PER];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = tid * PER + k;
        v[k] = s_t[e + (e >> 5)];
        sum += v[k];
    }
    const int incl = warp_incl_scan(sum, lane);
    __syncthreads();
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int x = lane < SCAN_BLOCK / 32 ? s_w[lane] : 0;
        const int xs = warp_incl_scan(x, lane);
        if (lane < SCAN_BLOCK / 32) s_w[lane] = xs - x;
    }
    __syncthreads();
    int run = s_base + s_w[wid] + incl - sum;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = tid * PER + k;
        s_t[e + (e >> 5)] = run;
        run += v[k];
    }
    if (blockIdx.x == ntiles - 1 && tid == SCAN_BLOCK - 1) start[ncells] = run;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = k * SCAN_BLOCK + tid;
        const long long c = base_c + e;
        if (c < ncells) start[c] = s_t[e + (e >> 5)];
    }
}

template <class R>
__global__ void scatter_kernel(State<R> stg, State<R> dst, const int* __restrict__ tcell, const int* __restrict__ tslot,
                               const int* __restrict__ start, long long ntot, const int* err, int* __restrict__ inv)
{
    if (*((volatile const int*)err)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const long long d = start[tcell[i]] + tslot[i];
        if constexpr (sizeof(R) == 4) {
            const float4 q = stg.aux[i];
            dst.pos[d] = stg.pos[i];
            dst.aux[d] = q;
            if (inv) inv[__float_as_int(q.w)] = (int)d;
        } else {
            const Rec64 r = stg.rec[i];
            dst.rec[d] = r;
            if (inv) inv[r.id] = (int)d;
        }
    }
}

// advances the device step counter after a captured run of n steps, unless a
// step failed (the host then resumes from the failing step)
__global__ void advance_kernel(long long* step, const int* err, int n)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && *err == 0) *step += n;
}

// ---------------------------------------------------------------------------
// input / output
// ---------------------------------------------------------------------------
// absolute coordinates -> the stored representation (the oracle's
// orc_to_rel_f64 / orc_to_rel_f32: the same IEEE double operations), with
// validation of types and coordinates.  The wrap loop is bounded: a
// coordinate more than 64 box lengths outside the box is rejected.
__device__ __forceinline__ bool wrap_rel_dev(double& x, double L, int per)
{
    if (!per) return true;
    for (int k = 0; k < 64 && x >= L; ++k) x -= L;
    for (int k = 0; k < 64 && x < 0.0; ++k) x += L;
    if (x >= L || x < 0.0) {
        if (x >= L && x - L < L) x = 0.0;   // x == L after rounding
        else return false;
    }
    return true;
}

// system of every particle from the prefix offsets (off[0] = 0, off[nsys] = ntot)
__global__ void sys_of_kernel(const long long* __restrict__ off, int nsys, long long ntot,
                              unsigned short* __restrict__ so)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nsys;            // off[lo] <= g < off[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (off[mid] <= g) lo = mid; else hi = mid;
        }
        so[g] = (unsigned short)lo;
    }
}

// one particle from absolute coordinates into staging slot g with the given
// id: box-relative FP64 (or FP32 + compensation) coordinates, its cell and
// slot, and its MSD origin
template <class R>
__device__ __forceinline__ void ingest_one(const SysDev& s, long long g, int id, const double* __restrict__ x3, int t,
                                           int ntypes, State<R> stg, int* __restrict__ tcell,
                                           int* __restrict__ tslot, int* __restrict__ counts,
                                           double* __restrict__ x0, int* err)
{
    bool ok = t >= 0 && t < ntypes;
    R xs[3];
    if constexpr (sizeof(R) == 4) {
        float h[3], c[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float Lf = s.Lf[a];
            double xr = __dsub_rn(x3[a], s.lo[a]);
            ok = ok && isfinite(xr) && wrap_rel_dev(xr, (double)Lf, s.per[a]);
            float hh = __double2float_rn(xr);
            if (s.per[a] && hh >= Lf) { hh = 0.0f; xr = __dsub_rn(xr, (double)Lf); }
            h[a] = hh;
            c[a] = __double2float_rn(__dsub_rn((double)hh, xr));
            x0[3 * g + a] = xr;
            xs[a] = hh;
        }
        stg.pos[g] = make_float4(h[0], h[1], h[2], __int_as_float(t));
        stg.aux[g] = make_float4(c[0], c[1], c[2], __int_as_float(id));
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double xr = __dsub_rn(x3[a], s.lo[a]);
            ok = ok && isfinite(xr) && wrap_rel_dev(xr, s.L[a], s.per[a]);
            xs[a] = xr;
            x0[3 * g + a] = xr;
        }
        Rec64 r;
        r.x = xs[0]; r.y = xs[1]; r.z = xs[2]; r.w = t; r.id = id;
        stg.rec[g] = r;
    }
    if (!ok) {
        atomicOr(err, EF_BADINPUT);
        xs[0] = xs[1] = xs[2] = R(0);
    }
    int cc[3];
    cell_coords(s, xs, cc);
    const long long cell = s.cell_base + ((long long)cc[2] * s.n[1] + cc[1]) * s.n[0] + cc[0];
    tcell[g] = (int)cell;
    tslot[g] = atomicAdd(counts + cell, 1);
}

// writes the particles (input order; FP64 or FP32 coordinates) into the
// staging arrays with their cell and slot, ready for scan + scatter
template <class R, class In>
__global__ void ingest_kernel(const SysDev* __restrict__ sys, const unsigned short* __restrict__ sys_of, long long ntot,
                              const In* __restrict__ xyz, const int* __restrict__ types, int ntypes, State<R> stg,
                              int* __restrict__ tcell, int* __restrict__ tslot, int* __restrict__ counts,
                              double* __restrict__ x0, int* err)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = sys[sys_of[g]];
        const double xd[3] = {(double)xyz[3 * g], (double)xyz[3 * g + 1], (double)xyz[3 * g + 2]};
        ingest_one<R>(s, g, (int)(g - s.part_base), xd, types[g], ntypes, stg, tcell, tslot, counts, x0, err);
    }
}

// ---------------------------------------------------------------------------
// Reaction edits on the device (one system): the deleted ids are flagged,
// the survivors get new ids by an exclusive scan of the keep flags over the
// old ids (their order is kept), and survivors and appended particles are
// staged at their new ids for the counting sort.
// ---------------------------------------------------------------------------
__global__ void edit_mark_kernel(const int* __restrict__ del, long long nd, int* __restrict__ flag)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nd; k += (long long)gridDim.x * blockDim.x)
        flag[del[k]] = 1;
}

__global__ void edit_keep_kernel(const int* __restrict__ flag, long long n, int* __restrict__ keep)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        keep[i] = 1 - flag[i];
}

template <class R>
__global__ void edit_restage_kernel(const SysDev* __restrict__ sys, long long n, State<R> cur, State<R> stg,
                                    const int* __restrict__ flag, const int* __restrict__ newid,
                                    int* __restrict__ tcell, int* __restrict__ tslot, int* __restrict__ counts,
                                    const double* __restrict__ x0, double* __restrict__ x0n)
{
    const SysDev& s = sys[0];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int id = load_id(cur, i);
        if (flag[id]) continue;
        const int nid = newid[id];
        R x[3];
        if constexpr (sizeof(R) == 4) {
            const float4 p = cur.pos[i];
            float4 q = cur.aux[i];
            q.w = __int_as_float(nid);
            stg.pos[nid] = p;
            stg.aux[nid] = q;
            x[0] = p.x; x[1] = p.y; x[2] = p.z;
        } else {
            Rec64 r = cur.rec[i];
            r.id = nid;
            stg.rec[nid] = r;
            x[0] = r.x; x[1] = r.y; x[2] = r.z;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) x0n[3 * (long long)nid + a] = x0[3 * (long long)id + a];
        int cc[3];
        cell_coords(s, x, cc);
        const long long cell = s.cell_base + ((long long)cc[2] * s.n[1] + cc[1]) * s.n[0] + cc[0];
        tcell[nid] = (int)cell;
        tslot[nid] = atomicAdd(counts + cell, 1);
    }
}

template <class R>
__global__ void edit_append_kernel(const SysDev* __restrict__ sys, long long base, long long na,
                                   const double* __restrict__ xyz, const int* __restrict__ types, int ntypes,
                                   State<R> stg, int* __restrict__ tcell, int* __restrict__ tslot,
                                   int* __restrict__ counts, double* __restrict__ x0n, int* err)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < na; k += (long long)gridDim.x * blockDim.x)
        ingest_one<R>(sys[0], base + k, (int)(base + k), xyz + 3 * k, types[k], ntypes, stg, tcell, tslot, counts,
                      x0n, err);
}

// sorted arrays -> absolute coordinates (FP64, or rounded to FP32) and types
// by global index
template <class R, class Out>
__global__ void emit_kernel(const SysDev* __restrict__ sys, const unsigned short* __restrict__ sys_of, long long ntot,
                            State<R> cur, Out* __restrict__ xyz, int* __restrict__ types)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = sys[sys_of[i]];
        if constexpr (sizeof(R) == 4) {
            const float4 p = cur.pos[i], c = cur.aux[i];
            const long long g = s.part_base + __float_as_int(c.w);
            xyz[3 * g + 0] = (Out)__dadd_rn(__dsub_rn((double)p.x, (double)c.x), s.lo[0]);
            xyz[3 * g + 1] = (Out)__dadd_rn(__dsub_rn((double)p.y, (double)c.y), s.lo[1]);
            xyz[3 * g + 2] = (Out)__dadd_rn(__dsub_rn((double)p.z, (double)c.z), s.lo[2]);
            types[g] = __float_as_int(p.w) & 0xff;
        } else {
            const Rec64 r = cur.rec[i];
            const long long g = s.part_base + r.id;
            xyz[3 * g + 0] = (Out)__dadd_rn(r.x, s.lo[0]);
            xyz[3 * g + 1] = (Out)__dadd_rn(r.y, s.lo[1]);
            xyz[3 * g + 2] = (Out)__dadd_rn(r.z, s.lo[2]);
            types[g] = r.w & 0xff;
        }
    }
}

// ---------------------------------------------------------------------------
// diagnostics: forces + energy, neighbour digest (the step kernel's pair code)
// ---------------------------------------------------------------------------
template <class R, int MODE, bool VALUE_IMAGE>
__global__ void diag_kernel(Args<R> a, double* forces, double* energy, int* ncount, unsigned long long* hashes)
{
    __shared__ R s_rc2[MAXT * MAXT];
    __shared__ R s_rmax2[MAXT];
    for (int k = threadIdx.x; k < MAXT * MAXT; k += blockDim.x) s_rc2[k] = a.tab->rc2[k];
    for (int k = threadIdx.x; k < MAXT; k += blockDim.x) {
        R m = R(0);
        for (int j = 0; j < MAXT; ++j) m = max(m, a.tab->rc2[k * MAXT + j]);
        s_rmax2[k] = m;
    }
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const int si = a.sys_of[i];
        const SysDev& s = a.sys[si];
        R xi[3];
        int wi;
        load_pos(a.cur, i, xi, wi);
        const int ti = wi & 0xff;
        const long long g = s.part_base + load_id(a.cur, i);
        int cc[3];
        cell_coords(s, xi, cc);
        Acc<R> acc;
        acc.zero();
        int nc = 0;
        unsigned long long hh = 0;
        neighbourhood<R, MODE, VALUE_IMAGE, false>(a.cur, a.start, s, cc, (int)i, xi, ti, s_rc2, nullptr, a.tab,
                                                   acc, nc, hh, s_rmax2[ti]);
        if (MODE == 1 && a.bstart) bond_forces<R, 1>(a, a.cur, load_id(a.cur, i), xi, s, acc);
        if (MODE == 2) {
            ncount[g] = nc;
            hashes[g] = hh;
            continue;
        }
        R F[3];
        acc.force(F);
        R ee = R(0);
        const ExtTerm<R>* ep = a.ext + (long long)si * a.n_ext;
        for (int e = 0; e < a.n_ext; ++e)
            if ((ep[e].tmask >> ti) & 1u) ext_force(ep[e], a.tab->prad[ti], xi, F, ee);
        forces[3 * g + 0] = (double)F[0];
        forces[3 * g + 1] = (double)F[1];
        forces[3 * g + 2] = (double)F[2];
        energy[g] = (double)acc.e + (double)ee;
    }
}

// Gaussian draws of step t by global particle index
template <class R>
__global__ void noise_kernel(const SysDev* sys, const unsigned short* sys_of, long long ntot, long long t, double* out)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = sys[sys_of[g]];
        R xn[3];
        bd_normals(s.seed, t, g - s.part_base, xn);
        out[3 * g] = xn[0];
        out[3 * g + 1] = xn[1];
        out[3 * g + 2] = xn[2];
    }
}

// ---------------------------------------------------------------------------
// RDF: counts of ordered pairs by (ti, tj, bin), FP64 predicate on the stored
// positions.  As in the reference (CudaSimulation.cu:1784-1827), each pair is
// evaluated once, from its lower sorted index, and counted for both (ti, tj)
// and (tj, ti); the displacement is symmetric in i and j (mimg_sym), so this
// equals counting both orientations separately.
//
// The cells within rmax of particle i are walked as rows of x-adjacent cells
// (one contiguous range of sorted particles each, split where the row wraps):
// rows whose (y, z) gap to i is beyond rmax are skipped and each row's x range
// is cut to the cells that can hold a partner; within a range only partners
// after i are taken.  An axis whose stencil would wrap onto itself (2R + 1 >=
// n cells) is walked once, whole, with the minimum image taken per candidate;
// otherwise the image is the cell wrap of the row, which for pairs within
// rmax < L/2 is the minimum image.  Either way dx = (xi - xj) - k L with the
// same IEEE operations as the oracle.
// ---------------------------------------------------------------------------
struct RdfAxis {
    int lo, cnt;        // cells lo .. lo + cnt - 1 (before wrapping)
    bool whole;         // the whole axis once, image per candidate
};

// 8 blocks of 128 per SM (64 registers, a few spilled) measured fastest
template <class R>
__global__ void __launch_bounds__(128, 8) rdf_kernel(const SysDev* __restrict__ sys, const unsigned short* __restrict__ sys_of, long long ntot,
                           State<R> cur, const int* __restrict__ start, int S, int nbins,
                           const double* __restrict__ e2, double w, int use_smem, unsigned long long* hist)
{
    // shared memory (use_smem): the block's histogram, then the squared bin
    // edges; otherwise neither
    extern __shared__ unsigned int sh[];
    const int H = S * S * nbins;
    const double* e2s = e2;
    if (use_smem) {
        double* se2 = reinterpret_cast<double*>(sh + ((H + 1) & ~1));
        for (int i = threadIdx.x; i < H; i += blockDim.x) sh[i] = 0;
        for (int i = threadIdx.x; i <= nbins; i += blockDim.x) se2[i] = e2[i];
        e2s = se2;
        __syncthreads();
    }
    const double rmax2 = e2[nbins];
    const double rmax = w * nbins;
    const float inv_wf = (float)(1.0 / w);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = sys[sys_of[i]];
        R xr[3];
        int wi;
        load_pos(cur, i, xr, wi);
        const int ti = wi & 0xff;
        const double xi[3] = {(double)xr[0], (double)xr[1], (double)xr[2]};
        double L[3], half[3], cw[3], f[3];
        int cc[3];
        RdfAxis ax[3];
        cell_coords(s, xr, cc);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if constexpr (sizeof(R) == 4) L[a] = (double)s.Lf[a]; else L[a] = s.L[a];
            half[a] = 0.5 * L[a];
            cw[a] = L[a] / s.n[a];
            f[a] = xi[a] - cc[a] * cw[a];
            // cells per side that can hold a partner; the margin keeps a
            // quotient that rounds down onto an integer from dropping a layer
            int r = (int)ceil(rmax / cw[a] * (1.0 + 1e-12));
            if (r < 1) r = 1;
            if (s.per[a] && 2 * r + 1 >= s.n[a]) {
                ax[a].lo = 0; ax[a].cnt = s.n[a]; ax[a].whole = true;
            } else if (s.per[a]) {
                ax[a].lo = cc[a] - r; ax[a].cnt = 2 * r + 1; ax[a].whole = false;
            } else {
                const int l = max(0, cc[a] - r), h = min(s.n[a] - 1, cc[a] + r);
                ax[a].lo = l; ax[a].cnt = h - l + 1; ax[a].whole = false;
            }
        }
        // squared distance from i to the cell slab at offset d along an axis
        // (0 inside its own cell and for whole axes), shrunk by a margin that
        // covers the rounding of the cell geometry
        const double eps = 1e-9 * (rmax + cw[0] + cw[1] + cw[2]);
        auto gap2a = [&](int a, int q) -> double {
            if (ax[a].whole || q == cc[a]) return 0.0;
            const double g = q > cc[a] ? (q - cc[a] - 1) * cw[a] + (cw[a] - f[a]) : (cc[a] - q - 1) * cw[a] + f[a];
            const double gg = g - eps;
            return gg > 0.0 ? gg * gg : 0.0;
        };
        for (int iz = 0; iz < ax[2].cnt; ++iz) {
            const int zq = ax[2].lo + iz;
            const double gz = gap2a(2, zq);
            if (gz >= rmax2) continue;
            int z = zq;
            double sz = 0.0;
            if (z < 0) { z += s.n[2]; sz = -L[2]; }
            else if (z >= s.n[2]) { z -= s.n[2]; sz = L[2]; }
            for (int iy = 0; iy < ax[1].cnt; ++iy) {
                const int yq = ax[1].lo + iy;
                const double gyz = gz + gap2a(1, yq);
                if (gyz >= rmax2) continue;
                int y = yq;
                double sy = 0.0;
                if (y < 0) { y += s.n[1]; sy = -L[1]; }
                else if (y >= s.n[1]) { y -= s.n[1]; sy = L[1]; }
                const long long row = s.cell_base + ((long long)z * s.n[1] + y) * s.n[0];
                // x cells of this row that can hold a partner
                int xa = ax[0].lo, xb = ax[0].lo + ax[0].cnt - 1;
                if (!ax[0].whole) {
                    while (xa < cc[0] && gyz + gap2a(0, xa) >= rmax2) ++xa;
                    while (xb > cc[0] && gyz + gap2a(0, xb) >= rmax2) --xb;
                }
                // up to three contiguous ranges: wrapped left, inside, wrapped right
                for (int part = 0; part < 3; ++part) {
                    int c0, c1;
                    double sx = 0.0;
                    if (part == 0) { c0 = xa; c1 = min(xb, -1); sx = -L[0]; }
                    else if (part == 1) { c0 = max(xa, 0); c1 = min(xb, s.n[0] - 1); }
                    else { c0 = max(xa, s.n[0]); c1 = xb; sx = L[0]; }
                    if (c0 > c1) continue;
                    const int off = part == 0 ? s.n[0] : (part == 2 ? -s.n[0] : 0);
                    const int j1 = start[row + c1 + off + 1];
                    const int j0 = max(start[row + c0 + off], (int)i + 1);
                    for (int j = j0; j < j1; ++j) {
                        R xq[3];
                        int wj;
                        load_pos(cur, j, xq, wj);
                        const double dx = ax[0].whole ? mimg_sym(xi[0], (double)xq[0], L[0], half[0], 1)
                                                      : sub_rn(sub_rn(xi[0], (double)xq[0]), sx);
                        const double dy = ax[1].whole ? mimg_sym(xi[1], (double)xq[1], L[1], half[1], 1)
                                                      : sub_rn(sub_rn(xi[1], (double)xq[1]), sy);
                        const double dz = ax[2].whole ? mimg_sym(xi[2], (double)xq[2], L[2], half[2], 1)
                                                      : sub_rn(sub_rn(xi[2], (double)xq[2]), sz);
                        const double r2 = dist2(dx, dy, dz);
                        if (!(r2 < rmax2)) continue;
                        // the bin: an FP32 estimate, then the exact FP64 edges decide
                        const float r2f = (float)r2;
                        int k = r2f > 0.0f ? (int)(r2f * rsqrtf(r2f) * inv_wf) : 0;
                        k = min(max(k, 0), nbins - 1);
                        while (k > 0 && e2s[k] > r2) --k;
                        while (k < nbins - 1 && e2s[k + 1] <= r2) ++k;
                        const int tj = wj & 0xff;
                        const int h1 = (ti * S + tj) * nbins + k, h2 = (tj * S + ti) * nbins + k;
                        if (use_smem) {
                            if (h1 == h2) atomicAdd(sh + h1, 2u);
                            else { atomicAdd(sh + h1, 1u); atomicAdd(sh + h2, 1u); }
                        } else {
                            if (h1 == h2) atomicAdd(hist + h1, 2ull);
                            else { atomicAdd(hist + h1, 1ull); atomicAdd(hist + h2, 1ull); }
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

// ---------------------------------------------------------------------------
// RDF on a grid of its own (rdf_rows_kernel below and its counting sort):
// the particles sorted by the cell of that grid, as RdfRec records.
struct RdfGrid {
    int n[3];
    int per[3];
    long long base;      // first coarse cell of the system
    double L[3];         // the engine's period per axis
    double invc[3];      // n / L
};

template <class R> struct RdfRec;
template <> struct RdfRec<float> { float4 p; };                                   // x, y, z, bits(type)
template <> struct __align__(32) RdfRec<double> { double x, y, z; int t, pad; };

template <class R>
__device__ __forceinline__ long long rdf_cell_of(const RdfGrid& g, const R x[3])
{
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double q = floor((double)x[a] * g.invc[a]);
        c[a] = q < 0.0 ? 0 : (q >= (double)g.n[a] ? g.n[a] - 1 : (int)q);
    }
    return g.base + ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
}

template <class R>
__global__ void rdf_count_kernel(const unsigned short* __restrict__ sys_of, long long ntot, State<R> cur,
                                 const RdfGrid* __restrict__ grids, int* __restrict__ tcell, int* __restrict__ tslot,
                                 int* __restrict__ counts)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        R x[3];
        int w;
        load_pos(cur, i, x, w);
        const long long c = rdf_cell_of(grids[sys_of[i]], x);
        tslot[i] = atomicAdd(counts + c, 1);
        tcell[i] = (int)c;
    }
}

template <class R>
__global__ void rdf_scatter_kernel(long long ntot, State<R> cur, const int* __restrict__ tcell,
                                   const int* __restrict__ tslot, const int* __restrict__ start,
                                   RdfRec<R>* __restrict__ rec)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        R x[3];
        int w;
        load_pos(cur, i, x, w);
        const long long d = start[tcell[i]] + tslot[i];
        RdfRec<R> r;
        if constexpr (sizeof(R) == 4) {
            r.p = make_float4(x[0], x[1], x[2], __int_as_float(w & 0xff));
        } else {
            r.x = x[0]; r.y = x[1]; r.z = x[2]; r.t = w & 0xff; r.pad = 0;
        }
        rec[d] = r;
    }
}

template <class R>
__device__ __forceinline__ void rdf_count(int ti, int tj, int k, int S, int nbins, int use_smem,
                                          unsigned* __restrict__ sh, unsigned long long* __restrict__ hist)
{
    const int h1 = (ti * S + tj) * nbins + k, h2 = (tj * S + ti) * nbins + k;
    if (use_smem) {
        if (h1 == h2) atomicAdd(sh + h1, 2u);
        else { atomicAdd(sh + h1, 1u); atomicAdd(sh + h2, 1u); }
    } else {
        if (h1 == h2) atomicAdd(hist + h1, 2ull);
        else { atomicAdd(hist + h1, 1ull); atomicAdd(hist + h2, 1ull); }
    }
}

// ---------------------------------------------------------------------------
// RDF on a grid of cells of edge >= rmax/2 (rdf_rows_kernel).  Every
// periodic axis has at least 5 of them, so a pair closer than rmax sits in
// two cells at most 2 apart along every axis, and each unordered pair of
// such cells is met exactly once among a cell's 62 forward offsets (dz > 0;
// dz == 0, dy > 0; dz == dy == 0, dx > 0): two offsets in [-2, 2] never
// reach the same cell, and d, -d never both.  A warp takes one cell (the own
// cell): its particles, up to RDR_OWN at a time, go to per-warp shared memory
// as packed FP32 pairs.  The candidates are the 13 forward rows of the
// stencil (a row: the cells x-2 .. x+2 at one (dy, dz); the row dy = dz = 0
// holds x+1 and x+2 only) and the own cell itself (partners of higher index),
// as up to 27 contiguous ranges of sorted particles (a row splits in two
// where it wraps around a periodic x bound).  They are fetched 32 at a time,
// one per lane, and moved to their periodic image next to the own cell; a
// candidate farther from the own particles' bounding box than the FP32 test
// radius is dropped (about a third of them: the stencil's corners), the
// others are queued per warp in order.  The queue is worked off in chunks of
// 64, two candidates per lane, each tested against two own particles per
// step with packed f32x2 arithmetic: dx = own - candidate image, r^2 =
// fma(dz, dz, fma(dy, dy, dx dx)), over-accepting through r2pre (the bound
// and dlt are derived with rdf_tiled on the host).  An accepted pair is
// binned at once: by the FP32 distance when r^2 is farther than dlt from
// both edges of its bin, else by the exact FP64 rule of rdf_kernel
// (rdr_exact).  Each pair is counted for both orientations.
// ---------------------------------------------------------------------------
constexpr int RDR_WARPS = 8;
constexpr int RDR_OWN = 64;        // own particles per pass of a cell (32 packed pairs)
constexpr int RDR_SELF = 26;       // range slot of the own cell (slots 2q, 2q+1: row q, parts A and B)
constexpr int RDR_CPL = 2;         // candidates per lane and chunk
constexpr int RDR_QUEUE = 32 * RDR_CPL + 32;   // candidate queue of a warp: a chunk and one batch more

struct RdrWarp {
    ulonglong2 oxy[RDR_OWN / 2];            // packed (x0, x1), (y0, y1) of own pair p
    unsigned long long oz[RDR_OWN / 2];     // packed (z0, z1)
    int2 ot[RDR_OWN / 2];                   // their types
    int rbase[32];                          // first sorted index of range slot r
    int rlen[32];                           // its length
    int rpre[32];                           // exclusive prefix of the lengths; INT_MAX past slot 27
    float4 rsh[32];                         // FP32 image shift of its candidates; w: bits(shift code)
    float4 cq[RDR_QUEUE];                   // queued candidates: image x, y, z; w: bits(type)
    int4 ci[RDR_QUEUE];                     // their sorted index, own bound (RDR_OWN: none), shift code
    float box[6];                           // bounding box of the own particles: low x, y, z, high x, y, z
};

// row q of the forward half of the stencil: offsets (dy, dz) and the x range
__device__ __forceinline__ void rdr_row(int q, int& dy, int& dz, int& dxlo, int& dxhi)
{
    if (q < 10) { dz = 1 + q / 5; dy = q % 5 - 2; dxlo = -2; dxhi = 2; }
    else if (q < 12) { dz = 0; dy = q - 9; dxlo = -2; dxhi = 2; }
    else if (q == 12) { dz = 0; dy = 0; dxlo = 1; dxhi = 2; }
    else { dz = 0; dy = 0; dxlo = 0; dxhi = 0; }      // q == 13: the own cell
}

template <bool MULTI>
__device__ __forceinline__ void rdr_count(int ti, int tj, int k, int S, int nbins, int use_smem,
                                          unsigned* __restrict__ sh, unsigned long long* __restrict__ hist)
{
    if (!MULTI) {
        if (use_smem) atomicAdd(sh + k, 2u);
        else atomicAdd(hist + k, 2ull);
    } else {
        rdf_count<float>(ti, tj, k, S, nbins, use_smem, sh, hist);
    }
}

// The exact rule for a pair the FP32 distance cannot bin: own particle i,
// candidate j of a range with shift code `code`; dx = (xi - xj) - sx with
// sx the candidate's image shift, r^2 and the bin as in rdf_kernel.
template <class R, bool MULTI>
__device__ __forceinline__ void rdr_exact(const RdfRec<R>* __restrict__ rec, int i, int j, int code, int ti, int tj,
                                       const RdfGrid* __restrict__ g, int S, int nbins, double rmax2, double w,
                                       const double* __restrict__ e2, int use_smem, unsigned* sh,
                                       unsigned long long* __restrict__ hist)
{
    double xi[3], xj[3];
    if constexpr (sizeof(R) == 4) {
        const float4 a = __ldg(&rec[i].p), b = __ldg(&rec[j].p);
        xi[0] = a.x; xi[1] = a.y; xi[2] = a.z;
        xj[0] = b.x; xj[1] = b.y; xj[2] = b.z;
    } else {
        const RdfRec<double> a = rec[i], b = rec[j];
        xi[0] = a.x; xi[1] = a.y; xi[2] = a.z;
        xj[0] = b.x; xj[1] = b.y; xj[2] = b.z;
    }
    double d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int sc = (code >> (2 * a)) & 3;
        const double sx = sc == 1 ? g->L[a] : (sc == 2 ? -g->L[a] : 0.0);
        d[a] = sub_rn(sub_rn(xi[a], xj[a]), sx);
    }
    const double r2 = dist2(d[0], d[1], d[2]);
    if (!(r2 < rmax2)) return;
    int k = (int)(sqrt(r2) / w);
    k = min(max(k, 0), nbins - 1);
    while (k > 0 && __ldg(e2 + k) > r2) --k;
    while (k < nbins - 1 && __ldg(e2 + k + 1) <= r2) ++k;
    rdr_count<MULTI>(ti, tj, k, S, nbins, use_smem, sh, hist);
}

// stand-ins for a missing own particle or candidate: their squared distance
// to anything (each other included) overflows, never accepted
constexpr float RDR_FAR_OWN = 3e30f, RDR_FAR_CAND = -3e30f;

// a candidate as packed pairs against two own particles
struct RdrCand {
    f32x2 X, Y, Z;
    int j, tj, omax, code;
};

// Candidate t of the cell's ranges (t >= C: none) at its image next to the
// own cell: x, y, z and bits(type) in c, (sorted index, own bound, shift
// code) in m.  r: the lane's range slot for its previous candidate (0 at
// the start), advanced to the last slot with rpre <= t (empty slots are
// passed over; a lane's candidates only move forward).
template <class R>
__device__ __forceinline__ void rdr_fetch(const RdrWarp& W, const RdfRec<R>* __restrict__ rec, int t, int C, int ob,
                                          int& r, float4& c, int4& m)
{
    while (W.rpre[r + 1] <= t) ++r;
    c = make_float4(RDR_FAR_CAND, RDR_FAR_CAND, RDR_FAR_CAND, 0.f);
    m = make_int4(0, RDR_OWN, 0, 0);
    if (t < C) {
        const int j = W.rbase[r] + (t - W.rpre[r]);
        const float4 s4 = W.rsh[r];
        float4 p;
        if constexpr (sizeof(R) == 4) {
            p = __ldg(&rec[j].p);
        } else {
            const RdfRec<double> d = rec[j];
            p = make_float4((float)d.x, (float)d.y, (float)d.z, __int_as_float(d.t));
        }
        c = make_float4(p.x + s4.x, p.y + s4.y, p.z + s4.z, p.w);
        // own o pairs with a candidate of the own cell only when ob + o < j
        m = make_int4(j, r == RDR_SELF ? j - ob : RDR_OWN, __float_as_int(s4.w), 0);
    }
}

__device__ __forceinline__ RdrCand rdr_cand(const float4& c, const int4& m)
{
    RdrCand q;
    q.X = f2_pack(c.x, c.x); q.Y = f2_pack(c.y, c.y); q.Z = f2_pack(c.z, c.z);
    q.j = m.x; q.tj = __float_as_int(c.w); q.omax = m.y; q.code = m.z;
    return q;
}

template <class R, bool MULTI, bool SMEM>
__global__ void __launch_bounds__(RDR_WARPS * 32, 4) rdf_rows_kernel(const RdfGrid* __restrict__ grids, int nsys,
        long long ncells, const int* __restrict__ start, const RdfRec<R>* __restrict__ rec, int S, int nbins,
        const double* __restrict__ e2, double w, float r2pre, float dlt, unsigned long long* __restrict__ hist)
{
    // shared memory: the warps' RdrWarp; dynamic: the FP32 bin edge pairs
    // (e2f[k], e2f[k+1]), k <= nbins (k == nbins: never inside), then, with
    // SMEM, the block's histogram
    __shared__ RdrWarp s_w[RDR_WARPS];
    extern __shared__ float2 s_e2p[];
    unsigned* sh = reinterpret_cast<unsigned*>(s_e2p + nbins + 1);
    const int H = S * S * nbins;
    for (int k = threadIdx.x; k <= nbins; k += blockDim.x)
        s_e2p[k] = k < nbins ? make_float2((float)e2[k], (float)e2[k + 1]) : make_float2(INFINITY, INFINITY);
    if (SMEM)
        for (int k = threadIdx.x; k < H; k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    RdrWarp& W = s_w[wp];
    const double rmax2 = e2[nbins];
    const float inv_wf = (float)(1.0 / w);
    // a candidate at squared FP32 distance >= r2box from the own particles'
    // bounding box passes the FP32 test with none of them (the margin covers
    // the roundings of both distances)
    const float r2box = r2pre * 1.00001f;
    for (long long c = (long long)blockIdx.x * RDR_WARPS + wp; c < ncells; c += (long long)gridDim.x * RDR_WARPS) {
        const int a0 = start[c], a1 = start[c + 1];
        if (a0 == a1) continue;
        int lo = 0, hi = nsys - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (grids[mid].base <= c) lo = mid; else hi = mid - 1;
        }
        const RdfGrid* g = grids + lo;
        const long long lc = c - g->base;
        const int n0 = g->n[0], n1 = g->n[1], n2 = g->n[2];
        const int cx = (int)(lc % n0), cy = (int)((lc / n0) % n1), cz = (int)(lc / ((long long)n0 * n1));
        // the ranges of the 13 rows and the own cell (lane q: slots 2q, 2q+1)
        __syncwarp();
        if (lane < 14) {
            int dy, dz, dxlo, dxhi;
            rdr_row(lane, dy, dz, dxlo, dxhi);
            int yy = cy + dy, zz = cz + dz, code = 0;
            bool skip = false;
            if (yy < 0) { skip |= !g->per[1]; yy += n1; code |= 2 << 2; }
            else if (yy >= n1) { skip |= !g->per[1]; yy -= n1; code |= 1 << 2; }
            if (zz < 0) { skip |= !g->per[2]; zz += n2; code |= 2 << 4; }
            else if (zz >= n2) { skip |= !g->per[2]; zz -= n2; code |= 1 << 4; }
            const int xa = cx + dxlo, xb = cx + dxhi;
            int alo = xa, ahi = xb, acode = code, blo = 0, bhi = -1, bcode = code;
            if (g->per[0]) {
                if (xa < 0) { alo = xa + n0; ahi = n0 - 1; acode = code | 2; blo = 0; bhi = xb; }
                else if (xb >= n0) { ahi = n0 - 1; blo = 0; bhi = xb - n0; bcode = code | 1; }
            } else {
                alo = max(xa, 0);
                ahi = min(xb, n0 - 1);
            }
            const long long row = g->base + ((long long)zz * n1 + yy) * n0;
            int ab = 0, al = 0, bb = 0, bl = 0;
            if (!skip && alo <= ahi) { ab = start[row + alo]; al = start[row + ahi + 1] - ab; }
            if (!skip && blo <= bhi) { bb = start[row + blo]; bl = start[row + bhi + 1] - bb; }
            W.rbase[2 * lane] = ab; W.rlen[2 * lane] = al;
            W.rbase[2 * lane + 1] = bb; W.rlen[2 * lane + 1] = bl;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const int cd = part ? bcode : acode;
                float s[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const int sc = (cd >> (2 * a)) & 3;
                    s[a] = sc == 1 ? (float)g->L[a] : (sc == 2 ? -(float)g->L[a] : 0.f);
                }
                W.rsh[2 * lane + part] = make_float4(s[0], s[1], s[2], __int_as_float(cd));
            }
        }
        __syncwarp();
        {
            const int len = lane < 28 ? W.rlen[lane] : 0;
            int incl = len;
#pragma unroll
            for (int sft = 1; sft < 32; sft <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, sft);
                if (lane >= sft) incl += t;
            }
            W.rpre[lane] = lane < 28 ? incl - len : INT_MAX;
        }
        __syncwarp();
        const int C = W.rpre[27] + W.rlen[27];        // all candidates
        for (int ob = a0; ob < a1; ob += RDR_OWN) {
            const int m = min(RDR_OWN, a1 - ob), np = (m + 1) >> 1;
            // the own particles as packed pairs, and their bounding box
            float p[2][4];
            float bl[3] = {INFINITY, INFINITY, INFINITY}, bh[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = 2 * lane + h;
                if (o < m) {
                    if constexpr (sizeof(R) == 4) {
                        const float4 q = __ldg(&rec[ob + o].p);
                        p[h][0] = q.x; p[h][1] = q.y; p[h][2] = q.z; p[h][3] = q.w;
                    } else {
                        const RdfRec<double> q = rec[ob + o];
                        p[h][0] = (float)q.x; p[h][1] = (float)q.y; p[h][2] = (float)q.z;
                        p[h][3] = __int_as_float(q.t);
                    }
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) { bl[ax] = fminf(bl[ax], p[h][ax]); bh[ax] = fmaxf(bh[ax], p[h][ax]); }
                } else {
                    p[h][0] = p[h][1] = p[h][2] = RDR_FAR_OWN; p[h][3] = 0.f;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    bl[ax] = fminf(bl[ax], __shfl_xor_sync(FULL, bl[ax], o));
                    bh[ax] = fmaxf(bh[ax], __shfl_xor_sync(FULL, bh[ax], o));
                }
            __syncwarp();
            if (lane < 3) {
                W.box[lane] = lane == 0 ? bl[0] : (lane == 1 ? bl[1] : bl[2]);
                W.box[3 + lane] = lane == 0 ? bh[0] : (lane == 1 ? bh[1] : bh[2]);
            }
            if (lane < np) {
                W.oxy[lane] = make_ulonglong2(f2_pack(p[0][0], p[1][0]), f2_pack(p[0][1], p[1][1]));
                W.oz[lane] = f2_pack(p[0][2], p[1][2]);
                W.ot[lane] = make_int2(__float_as_int(p[0][3]), __float_as_int(p[1][3]));
            }
            __syncwarp();
            // The own pairs against the queued candidates qb .. qb + 32 RDR_CPL
            // (those past qn: none).  SELF: some of them are in the own cell and
            // pair with own particles of lower index only.
            auto chunk = [&](int qb, int qn) {
                RdrCand q[RDR_CPL];
                bool any_self = false;
#pragma unroll
                for (int u = 0; u < RDR_CPL; ++u) {
                    const int e = qb + 32 * u + lane;
                    q[u] = e < qn ? rdr_cand(W.cq[e], W.ci[e])
                                  : rdr_cand(make_float4(RDR_FAR_CAND, RDR_FAR_CAND, RDR_FAR_CAND, 0.f),
                                             make_int4(0, RDR_OWN, 0, 0));
                    any_self |= q[u].omax < RDR_OWN;
                }
                auto own_pairs = [&](auto self_tag) {
                    constexpr bool SELF = decltype(self_tag)::value;
                    for (int pp = 0; pp < np; ++pp) {
                        const ulonglong2 a = W.oxy[pp];
                        const f32x2 oz = W.oz[pp];
                        unsigned ex = 0;      // tests (2u + h) left to the exact rule
#pragma unroll
                        for (int u = 0; u < RDR_CPL; ++u) {
                            const f32x2 dX = f2_sub(a.x, q[u].X), dY = f2_sub(a.y, q[u].Y), dZ = f2_sub(oz, q[u].Z);
                            const f32x2 q2 = f2_fma(dZ, dZ, f2_fma(dY, dY, f2_mul(dX, dX)));
                            float r2h[2];
                            f2_unpack(q2, r2h[0], r2h[1]);
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                // the bin of the FP32 distance (rsqrt, then floor by a round-down add of
                                // 2^23), kept when r2 is farther than dlt from both of its edges; computed
                                // for every lane without a branch (a rejected or coincident pair, r2 = 0
                                // or overflowed, gives a NaN distance: bin nbins, whose edges are infinite)
                                const float r2 = r2h[h];
                                const bool acc = (r2 < r2pre) & (!SELF || 2 * pp + h < q[u].omax);
                                const float rr = r2 * rsqrtf(r2);
                                unsigned k = (unsigned)(__float_as_int(__fadd_rd(rr * inv_wf, 8388608.0f)) -
                                                        0x4B000000);
                                k = min(k, (unsigned)nbins);
                                const float2 ed = s_e2p[k];
                                const bool fast = acc & (r2 - dlt >= ed.x) & (r2 + dlt < ed.y);
                                if (fast) {
                                    const int ti = MULTI ? (h ? W.ot[pp].y : W.ot[pp].x) : 0;
                                    rdr_count<MULTI>(ti, q[u].tj, (int)k, S, nbins, SMEM, sh, hist);
                                }
                                ex |= (unsigned)(acc & !fast) << (2 * u + h);
                            }
                        }
                        // the rare pairs near a bin edge (or beyond rmax within the FP32 margin)
                        if (__any_sync(FULL, ex != 0u)) {
#pragma unroll
                            for (int u = 0; u < RDR_CPL; ++u)
#pragma unroll
                                for (int h = 0; h < 2; ++h)
                                    if ((ex >> (2 * u + h)) & 1u) {
                                        const int ti = MULTI ? (h ? W.ot[pp].y : W.ot[pp].x) : 0;
                                        rdr_exact<R, MULTI>(rec, ob + 2 * pp + h, q[u].j, q[u].code, ti, q[u].tj, g,
                                                            S, nbins, rmax2, w, e2, SMEM, sh, hist);
                                    }
                        }
                    }
                };
                if (__any_sync(FULL, any_self)) own_pairs(std::true_type{});
                else own_pairs(std::false_type{});
            };
            // Candidates 32 at a time, one per lane; those whose squared FP32
            // distance to the own particles' bounding box reaches r2box (no
            // own particle can then pass the FP32 test) are dropped, the others
            // queued in order, and the queue is worked off a chunk at a time.
            int qn = 0, slot = 0;
            for (int tb = 0; tb < C; tb += 32) {
                float4 c;
                int4 mi;
                rdr_fetch<R>(W, rec, tb + lane, C, ob, slot, c, mi);
                const float ex = fmaxf(fmaxf(W.box[0] - c.x, c.x - W.box[3]), 0.f);
                const float ey = fmaxf(fmaxf(W.box[1] - c.y, c.y - W.box[4]), 0.f);
                const float ez = fmaxf(fmaxf(W.box[2] - c.z, c.z - W.box[5]), 0.f);
                const bool keep = (tb + lane < C) & (fmaf(ez, ez, fmaf(ey, ey, ex * ex)) < r2box);
                const unsigned mk = __ballot_sync(FULL, keep);
                if (keep) {
                    const int e = qn + __popc(mk & ((1u << lane) - 1u));
                    W.cq[e] = c;
                    W.ci[e] = mi;
                }
                qn += __popc(mk);
                __syncwarp();
                if (qn >= 32 * RDR_CPL) {
                    chunk(0, 32 * RDR_CPL);
                    __syncwarp();
                    qn -= 32 * RDR_CPL;
                    if (lane < qn) {
                        W.cq[lane] = W.cq[32 * RDR_CPL + lane];
                        W.ci[lane] = W.ci[32 * RDR_CPL + lane];
                    }
                    __syncwarp();
                }
            }
            if (qn > 0) chunk(0, qn);
        }
    }
    if (SMEM) {
        __syncthreads();
        for (int k = threadIdx.x; k < H; k += blockDim.x)
            if (sh[k]) atomicAdd(hist + k, (unsigned long long)sh[k]);
    }
}

// ---------------------------------------------------------------------------
// MSD: squared unwrapped displacement per particle (FP64)
// ---------------------------------------------------------------------------
template <class R>
__global__ void msd_kernel(const SysDev* __restrict__ sys, const unsigned short* __restrict__ sys_of, long long ntot,
                           State<R> cur, const double* __restrict__ x0, double* d2, int* types)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = sys[sys_of[i]];
        double u[3];
        int w, id;
        if constexpr (sizeof(R) == 4) {
            const float4 p = cur.pos[i], c = cur.aux[i];
            u[0] = (double)p.x - (double)c.x;
            u[1] = (double)p.y - (double)c.y;
            u[2] = (double)p.z - (double)c.z;
            w = __float_as_int(p.w);
            id = __float_as_int(c.w);
        } else {
            const Rec64 r = cur.rec[i];
            u[0] = r.x; u[1] = r.y; u[2] = r.z;
            w = r.w;
            id = r.id;
        }
        const long long g = s.part_base + id;
        double acc = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int im = (int)(signed char)((w >> (8 + 8 * a)) & 0xff);
            double L;
            if constexpr (sizeof(R) == 4) L = (double)s.Lf[a]; else L = s.L[a];
            const double dd = u[a] + (double)im * L - x0[3 * g + a];
            acc += dd * dd;
        }
        d2[g] = acc;
        types[g] = w & 0xff;
    }
}

// Deterministic per-type sums, in two passes with fixed partitions and fixed
// reduction trees (the result does not depend on scheduling):
// typed_partial_kernel: block (x, y) sums the entries of type y (y == S: all
// entries) in index chunk x; typed_final_kernel: block y sums its partials.
constexpr int TSUM_BLOCK = 256;
__global__ void __launch_bounds__(TSUM_BLOCK) typed_partial_kernel(const double* __restrict__ v,
                                                                   const int* __restrict__ types, long long n, int S,
                                                                   long long chunk, double* __restrict__ part,
                                                                   long long* __restrict__ pcnt)
{
    __shared__ double red[TSUM_BLOCK];
    __shared__ long long cr[TSUM_BLOCK];
    const int want = blockIdx.y;
    const long long a = (long long)blockIdx.x * chunk;
    const long long b = min(n, a + chunk);
    double acc = 0.0;
    long long c = 0;
    for (long long i = a + threadIdx.x; i < b; i += TSUM_BLOCK)
        if (want == S || types[i] == want) { acc += v[i]; ++c; }
    red[threadIdx.x] = acc;
    cr[threadIdx.x] = c;
    __syncthreads();
    for (int o = TSUM_BLOCK / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            red[threadIdx.x] += red[threadIdx.x + o];
            cr[threadIdx.x] += cr[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[(long long)want * gridDim.x + blockIdx.x] = red[0];
        pcnt[(long long)want * gridDim.x + blockIdx.x] = cr[0];
    }
}

__global__ void __launch_bounds__(TSUM_BLOCK) typed_final_kernel(const double* __restrict__ part,
                                                                 const long long* __restrict__ pcnt, int P,
                                                                 double* __restrict__ out, long long* __restrict__ counts)
{
    __shared__ double red[TSUM_BLOCK];
    __shared__ long long cr[TSUM_BLOCK];
    const int want = blockIdx.x;
    double acc = 0.0;
    long long c = 0;
    for (int k = threadIdx.x; k < P; k += TSUM_BLOCK) {
        acc += part[(long long)want * P + k];
        c += pcnt[(long long)want * P + k];
    }
    red[threadIdx.x] = acc;
    cr[threadIdx.x] = c;
    __syncthreads();
    for (int o = TSUM_BLOCK / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            red[threadIdx.x] += red[threadIdx.x + o];
            cr[threadIdx.x] += cr[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[want] = red[0];
        counts[want] = cr[0];
    }
}

// ---------------------------------------------------------------------------
// Pair-list mode.
//
// The cell walk of step_kernel finds the candidates of every particle again in
// every step.  In pair-list mode a list of the pairs closer than
// rl = rc + skin (per type pair) is built from the sorted cell layout, and
// each step evaluates only the listed pairs.  A pair missing from the list
// can come within its cutoff only after its two particles moved by skin
// together, so one of them moved more than about skin/2 (hot): the step
// kernel collects the hot particles, list_check_kernel checks their current
// neighbourhoods against the lists, and a missing pair -- or a particle that
// moved about a full skin, or too many hot particles -- raises a flag; the
// kernels that follow in the same step (gated on the flag, no-ops otherwise)
// re-sort the particles by cell and rebuild the list before the next step.
// Pair displacements are the minimum image with the same IEEE operations as
// the cell walk, so the accepted pairs and the FP32 fixed-point forces are
// identical to the cell walk's.
//
// Between builds a particle keeps its sorted index; each step writes the
// other of two state buffers at the same index, and so does the re-sort.  The
// buffer that holds the input of step t is (t + nreb) & 1, where the parity
// bit nreb flips at every re-sort.
// ---------------------------------------------------------------------------
constexpr int EF_LISTOVF = 16;
constexpr int EF_LISTWIDE = 32;   // a partner's offset needs the 32-bit list entries
constexpr int LIST_CHUNK = 4;     // listed partners whose positions the list step requests together (FP32C)
constexpr int LIST_CHUNK_F64 = 2; // the same for the FP64 step (2 or a multiple of 4)

// List head of particle i (8 bytes): its position at the build on a lattice
// of 2^16 bins per box edge, wrapping (x: bits 0-15 of .x, y: bits 16-31, z:
// bits 0-15 of .y), and its list length (bits 16-31 of .y).  The lattice
// coordinate of any x (also beyond an open axis' bounds) is floor(x 2^16/L)
// mod 2^16; a displacement shorter than L/2 is the wrapped 16-bit difference
// of two lattice coordinates, within 2 bins (the floors and a periodic wrap
// whose L 2^16/L rounds off the integer) of the exact one.
__device__ __forceinline__ unsigned qcoord(float x, float q) { return (unsigned)__float2int_rd(x * q) & 0xffffu; }

template <class R>
__device__ __forceinline__ uint2 make_head(const R x[3], const SysDev& s, int cnt)
{
    const unsigned qx = qcoord((float)x[0], s.qs[0]), qy = qcoord((float)x[1], s.qs[1]);
    const unsigned qz = qcoord((float)x[2], s.qs[2]);
    return make_uint2(qx | (qy << 16), qz | ((unsigned)cnt << 16));
}

__device__ __forceinline__ int head_count(uint2 h) { return (int)(h.y >> 16); }

// squared displacement since the build, lattice estimate
template <class R>
__device__ __forceinline__ float head_disp2(uint2 h, const R x[3], const SysDev& s)
{
    const int dx = (short)(qcoord((float)x[0], s.qs[0]) - (h.x & 0xffffu));
    const int dy = (short)(qcoord((float)x[1], s.qs[1]) - (h.x >> 16));
    const int dz = (short)(qcoord((float)x[2], s.qs[2]) - (h.y & 0xffffu));
    const float ex = (float)dx * s.iqs[0], ey = (float)dy * s.iqs[1], ez = (float)dz * s.iqs[2];
    return ex * ex + ey * ey + ez * ez;
}

// List entries in int4 groups, column-major over i (group g of particle i
// at nbr4[g stride + i]): narrow lists hold 8 signed 16-bit offsets j - i
// per group, wide ones 4 sorted indices j.
__device__ __forceinline__ int group_word(const int4& g, int u)
{
    return u == 0 ? g.x : (u == 1 ? g.y : (u == 2 ? g.z : g.w));
}
__device__ __forceinline__ int list_entry(const int4& g, int u, bool narrow, int i)
{
    if (!narrow) return group_word(g, u);
    const int wd = group_word(g, u >> 1);
    return i + ((u & 1) ? (wd >> 16) : (int)(short)(wd & 0xffff));
}

struct ListCtl {
    int need;        // 1: re-sort and rebuild after this step
    int nreb;        // parity bit, flipped by every re-sort
    int maxcnt;      // longest list met by an overflowing build
    int nbuild;      // builds so far
    int nhot;        // hot particles of the last step (reset by the list check)
    int done;        // blocks of the list check finished (reset by its last block)
};

template <class R> struct ListArgs {
    State<R> b0, b1;     // the two state buffers
    ListCtl* ctl;
    int4* nbr;           // list entries in groups (list_entry); null: sort only
    uint2* head;         // list heads (make_head)
    long long stride;
    int cap;             // list capacity per particle (a multiple of 8)
    int narrow;          // 16-bit offsets, 8 per group (else 32-bit indices, 4 per group)
    const R* rl2t;       // squared list radius (rc + skin) per type pair; 0: no potential, never listed
    R rl2max;            // the largest of them
    float thr2;          // squared displacement since the build above which the list check looks at a particle
    float cap2;          // squared displacement since the build that triggers a rebuild by itself
    int* hot;            // hot particles (moved more than sqrt(thr2)) of the last step, hot_max at most
    int hot_max;         // more hot particles than this: rebuild rather than check them
};

template <class R>
__device__ __forceinline__ int list_sel(const Args<R>& a, const ListArgs<R>& v, long long off)
{
    const long long t = *((volatile const long long*)a.step_ptr) + off;
    return (int)((t + (long long)*((volatile const int*)&v.ctl->nreb)) & 1LL);
}

template <class R>
__device__ __forceinline__ bool list_gate(const Args<R>& a, const ListArgs<R>& v)
{
    return *((volatile const int*)a.err) == 0 && *((volatile const int*)&v.ctl->need) != 0;
}

__device__ __forceinline__ void store_state(const State<float>& st, long long i, const float x[3], int w,
                                            const float c[3], int id)
{
    st.pos[i] = make_float4(x[0], x[1], x[2], __int_as_float(w));
    st.aux[i] = make_float4(c[0], c[1], c[2], __int_as_float(id));
}
__device__ __forceinline__ void store_state(const State<double>& st, long long i, const double x[3], int w,
                                            const double* /*c*/, int id)
{
    Rec64 r;
    r.x = x[0]; r.y = x[1]; r.z = x[2]; r.w = w; r.id = id;
    st.rec[i] = r;
}

// The partners of list entries k0 .. k0 + 3 of sorted particle i (k0 a
// multiple of 4) from the group q that holds them: NARROW, two 32-bit words
// of 16-bit offsets j - i (the low or high half of the group); wide, the 4
// indices of the group.
template <bool NARROW>
__device__ __forceinline__ void quad_entries(const int4& q, int k0, int i, int* jj)
{
    if constexpr (NARROW) {
        const bool hi = (k0 & 4) != 0;
        const int w0 = hi ? q.z : q.x, w1 = hi ? q.w : q.y;
        jj[0] = i + (int)(short)w0;
        jj[1] = i + (w0 >> 16);
        jj[2] = i + (int)(short)w1;
        jj[3] = i + (w1 >> 16);
    } else {
        jj[0] = q.x; jj[1] = q.y; jj[2] = q.z; jj[3] = q.w;
    }
}

// one BD step of every particle over its pair list; ALLPER: every axis of
// every system is periodic (the minimum image needs no per-axis test);
// NARROW: list entries are 16-bit offsets (the handle's list format).  The
// FP32 harmonic-repulsion kernel of all-periodic systems runs 9 blocks of 128
// per SM (56 registers, no spill), measured 4 % faster than 8; 10 spill, and
// so do the other FP32 variants at 9.  Its FP64 twin runs 7 (72 registers,
// 3 % faster than 6 despite a few spilled registers; 8 is slower).
template <class R, bool HREP, bool ALLPER, int BLOCK, bool NARROW>
__global__ void __launch_bounds__(BLOCK, (sizeof(R) == 4 ? (HREP && ALLPER ? 1152 : 1024) : (HREP && ALLPER ? 896 : 768)) /
                                             BLOCK)
    list_step_kernel(Args<R> a, ListArgs<R> v)
{
    __shared__ R s_rc2[MAXT * MAXT];
    __shared__ FastTab<R> s_ft;
    // the error flag, the step counter and the buffer parity, then the
    // particle's inputs, all requested before the pair tables: the block
    // waits on one round of loads, not three
    const int err0 = *((volatile int*)a.err);
    const long long t = *((volatile const long long*)a.step_ptr) + a.step_off;
    const int nreb = *((volatile const int*)&v.ctl->nreb);
    const int sel = (int)((t + (long long)nreb) & 1LL);
    const State<R> cur = sel ? v.b1 : v.b0;
    const State<R> nxt = sel ? v.b0 : v.b1;
    if (err0) return;   // an earlier step failed: keep its input intact
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    const bool live = i < a.ntot;
    int si = 0;
    R xi[3] = {R(0), R(0), R(0)};
    int wi = 0;
    R c[3] = {R(0), R(0), R(0)};
    int id = 0;
    uint2 hd = make_uint2(0, 0);
    int4 q0 = make_int4(0, 0, 0, 0), q1 = q0;
    if (live) {
        si = a.sys_of[i];
        load_pos(cur, i, xi, wi);
        if constexpr (sizeof(R) == 4) {
            const float4 q = __ldg(cur.aux + i);
            c[0] = q.x; c[1] = q.y; c[2] = q.z;
            id = __float_as_int(q.w);
        } else {
            id = __ldg(&cur.rec[i].id);
        }
        hd = __ldg(v.head + i);
        // the first 8 list entries (one narrow group, two wide ones; capacity
        // >= 8), before the list length is known; entries past it are unused
        q0 = __ldg(v.nbr + i);
        q1 = NARROW ? q0 : __ldg(v.nbr + i + v.stride);
    }
    // rows of the S types in use (entries (ti, tj) with ti >= S are never read)
    for (int k = threadIdx.x; k < MAXT * a.tab->S; k += BLOCK) {
        s_rc2[k] = a.tab->rc2[k];
        if (HREP) {
            s_ft.k[k] = a.tab->nterm[k] ? a.tab->term[k * MAX_TERMS].k : R(0);
            s_ft.r0[k] = a.tab->nterm[k] ? a.tab->term[k * MAX_TERMS].r0 : R(0);
        }
    }
    __syncthreads();
    if (!live) return;
    const SysDev& s = a.sys[si];
    const int ti = wi & 0xff;
    Box<R> bx;
    bx.load(s);
    Acc<R> acc;
    acc.zero();
    const int cnt = head_count(hd);
    const int4* nb4 = v.nbr + i;
    PairFrame pf;
    double il[3] = {0.0, 0.0, 0.0};
    if constexpr (sizeof(R) == 4) pf.load(s, xi);
    else { il[0] = s.il[0]; il[1] = s.il[1]; il[2] = s.il[2]; }
    // the partners in chunks of LCHUNK entries (4 or 8): all their positions
    // are requested before the first pair is evaluated
    constexpr int EPG = NARROW ? 8 : 4;      // entries per group
    constexpr int LCHUNK = sizeof(R) == 4 ? LIST_CHUNK : LIST_CHUNK_F64;
    static_assert(LCHUNK == 2 || LCHUNK % 4 == 0, "pairs or whole quads per chunk");
    // FP32 HREP: every lane runs the warp's longest list (its chunks past its
    // own list hold only itself), so the loop needs no per-lane exit (1 %
    // faster on config 4; the FP64 step measured 2 % slower with it)
    const int kend = (HREP && sizeof(R) == 4) ? __reduce_max_sync(__activemask(), cnt) : cnt;
    for (int k0 = 0; k0 < kend; k0 += LCHUNK) {
        int jj[LCHUNK < 4 ? 4 : LCHUNK];
#pragma unroll
        for (int h = 0; h < (LCHUNK + 3) / 4; ++h) {
            const int kq = (k0 & ~3) + 4 * h;       // the quad's first entry
            const int gi = kq / EPG;                // and its group
            int4 q = make_int4(0, 0, 0, 0);
            if (gi == 0) q = q0;
            else if (gi == 1 && !NARROW) q = q1;
            else if (kq < cnt) q = __ldg(nb4 + (long long)gi * v.stride);
            quad_entries<NARROW>(q, kq, i, jj + 4 * h);
        }
        if (LCHUNK == 2 && (k0 & 2)) { jj[0] = jj[2]; jj[1] = jj[3]; }   // the quad's upper pair
        // entries past the list's end: HREP, the particle itself (r^2 = 0,
        // no force, and its position is in L1), which spares the chunk's
        // per-entry branches; otherwise -1 (skipped).  Narrow lists hold
        // offset 0 (the particle itself) in the rest of their last group, and
        // a group past the list's end is not loaded (zeros, offset 0 again),
        // so HREP needs no test there
        if constexpr (!(HREP && NARROW)) {
#pragma unroll
            for (int u = 0; u < LCHUNK; ++u) jj[u] = (k0 + u < cnt) ? jj[u] : (HREP ? i : -1);
        }
        R xj[LCHUNK][3];
        int wj[LCHUNK];
#pragma unroll
        for (int u = 0; u < LCHUNK; ++u) {
            if (HREP || jj[u] >= 0) load_pos(cur, jj[u], xj[u], wj[u]);
            else { xj[u][0] = xj[u][1] = xj[u][2] = R(0); wj[u] = 0; }
        }
#pragma unroll
        for (int u = 0; u < LCHUNK; ++u) {
            if (!HREP && jj[u] < 0) continue;
            R dx, dy, dz, r2;
            if constexpr (sizeof(R) == 4) {
                pair_disp_x2(pf, xj[u][0], xj[u][1], xj[u][2], dx, dy, dz, r2);
            } else {
                dx = mimg_round(xi[0], xj[u][0], bx.L[0], il[0]);
                dy = mimg_round(xi[1], xj[u][1], bx.L[1], il[1]);
                dz = mimg_round(xi[2], xj[u][2], bx.L[2], il[2]);
                r2 = dist2(dx, dy, dz);
            }
            const int pidx = ti * MAXT + (wj[u] & 0xff);
            if (r2 < s_rc2[pidx]) {
                if (HREP) {
                    // pre = k (r - r0) / r; r == 0 has no direction
                    if (r2 > R(0)) {
                        R pre;
                        if constexpr (sizeof(R) == 4) pre = s_ft.k[pidx] * (1.0f - s_ft.r0[pidx] * rsqrtf(r2));
                        else { const R r = sqrt(r2); pre = s_ft.k[pidx] * (r - s_ft.r0[pidx]) / r; }
                        acc.add(pre, dx, dy, dz);
                    }
                } else {
                    const R r = sqrt(r2);
                    const int nt = a.tab->nterm[pidx];
                    for (int m = 0; m < nt; ++m) {
                        R pre, e;
                        pair_term(a.tab->term[pidx * MAX_TERMS + m], r, pre, e);
                        acc.add(pre, dx, dy, dz);
                    }
                }
            }
        }
    }
    if (a.bstart) bond_forces<R, 0>(a, cur, id, xi, s, acc);
    R F[3];
    acc.force(F);
    if (a.n_ext > 0) {
        const ExtTerm<R>* ep = a.ext + (long long)si * a.n_ext;
        R ee = R(0);
        for (int e = 0; e < a.n_ext; ++e)
            if ((ep[e].tmask >> ti) & 1u) ext_force(ep[e], a.tab->prad[ti], xi, F, ee);
    }
    R xn[3];
    if (a.noise) {
        const double* nz = a.noise + 3 * (s.part_base + id);
        xn[0] = (R)nz[0]; xn[1] = (R)nz[1]; xn[2] = (R)nz[2];
    } else {
        bd_normals(s.seed, t, (long long)id, xn);
    }
    const int ef = em_update<ALLPER>(xi, c, wi, F, xn, a.tab->a[ti], a.tab->b[ti], s);
    // displacement since the build (lattice estimate; the thresholds
    // allow for its error)
    const float dd = head_disp2(hd, xi, s);
    if (dd > v.cap2) *((volatile int*)&v.ctl->need) = 1;
    const bool hot = dd > v.thr2;
    const unsigned act = __activemask();
    const unsigned hm = __ballot_sync(act, hot);
    if (hm) {
        const int lane = threadIdx.x & 31;
        const int lead = __ffs(hm) - 1;
        int base = 0;
        if (lane == lead) base = atomicAdd(&v.ctl->nhot, __popc(hm));
        base = __shfl_sync(act, base, lead) + __popc(hm & ((1u << lane) - 1u));
        if (hot && base < v.hot_max) v.hot[base] = i;
    }
    store_state(nxt, i, xi, wi, c, id);
    if (ef) {
        atomicOr(a.err, ef);
        atomicMin((unsigned long long*)a.err_step, (unsigned long long)t);
    }
}

// re-sort, part 1: cell and slot of every particle of the current state
template <class R>
__global__ void list_count_kernel(Args<R> a, ListArgs<R> v, long long off)
{
    if (!list_gate(a, v)) return;
    const State<R> src = list_sel(a, v, off) ? v.b1 : v.b0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const SysDev& s = a.sys[a.sys_of[i]];
        R x[3];
        int w;
        load_pos(src, i, x, w);
        int c[3];
        cell_coords(s, x, c);
        const long long cell = s.cell_base + ((long long)c[2] * s.n[1] + c[1]) * s.n[0] + c[0];
        a.tslot[i] = atomicAdd(a.counts + cell, 1);
        a.tcell[i] = (int)cell;
    }
}

// re-sort, part 3 (after the scan): scatter into the other buffer
template <class R>
__global__ void list_scatter_kernel(Args<R> a, ListArgs<R> v, long long off)
{
    if (!list_gate(a, v)) return;
    const int sel = list_sel(a, v, off);
    const State<R> src = sel ? v.b1 : v.b0;
    const State<R> dst = sel ? v.b0 : v.b1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.ntot;
         i += (long long)gridDim.x * blockDim.x) {
        const long long d = a.start[a.tcell[i]] + a.tslot[i];
        if constexpr (sizeof(R) == 4) {
            const float4 q = src.aux[i];
            dst.pos[d] = src.pos[i];
            dst.aux[d] = q;
            if (a.inv) a.inv[__float_as_int(q.w)] = (int)d;
        } else {
            const Rec64 r = src.rec[i];
            dst.rec[d] = r;
            if (a.inv) a.inv[r.id] = (int)d;
        }
    }
}

// writes the entries of one particle's list (list_entry's layouts); an
// offset that 16 bits cannot hold marks the build as needing wide entries
struct ListWriter {
    int4* nbr;
    long long stride;
    int i, cap;
    bool narrow, wide_need;
    __device__ __forceinline__ void put(int k, int j)
    {
        if (k >= cap) return;
        if (narrow) {
            const int d = j - i;
            if (d < -32768 || d > 32767) { wide_need = true; return; }
            reinterpret_cast<short*>(nbr + (long long)(k >> 3) * stride + i)[k & 7] = (short)d;
        } else {
            reinterpret_cast<int*>(nbr + (long long)(k >> 2) * stride + i)[k & 3] = j;
        }
    }
};

// appends the pairs of one candidate range closer than their list radius
template <class R>
__device__ __forceinline__ void list_range(const State<R>& st, int j0, int j1, int self, const R xi[3], R sx, R sy,
                                           R sz, const R* __restrict__ rl2, ListWriter& lw, int& cnt)
{
    for (int j = j0; j < j1; ++j) {
        R xj[3];
        int wj;
        load_pos(st, j, xj, wj);
        const R dx = sub_rn(xi[0], add_rn(xj[0], sx));
        const R dy = sub_rn(xi[1], add_rn(xj[1], sy));
        const R dz = sub_rn(xi[2], add_rn(xj[2], sz));
        if (dist2(dx, dy, dz) < rl2[wj & 0xff] && j != self) {
            lw.put(cnt, j);
            ++cnt;
        }
    }
}

// Position x in the list's cell grid (>= 3 cells of edge >= rc_max + skin on
// every periodic axis): its cell and offset within it.
template <class R> struct ListCell {
    int c[3];
    R cw[3], fr[3];
    __device__ __forceinline__ void locate(const SysDev& s, const R x[3])
    {
        cell_coords(s, x, c);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if constexpr (sizeof(R) == 4) cw[q] = R(1) / s.invcf[q]; else cw[q] = R(1) / s.invc[q];
            fr[q] = x[q] - (R)c[q] * cw[q];
        }
    }
};

// The cells of row (dz, dy) around x that can hold a sorted particle closer
// than sqrt(lim) to x: f(j0, j1, sx, sy, sz) for every range [j0, j1) of
// sorted particles (two where the row wraps), with the periodic shift of its
// cells.
template <class R, class F>
__device__ __forceinline__ void list_row_ranges(const Args<R>& a, const SysDev& s, const ListCell<R>& g, R lim,
                                                int dz, int dy, F&& f)
{
    const R gz = gap2(dz, g.fr[2], g.cw[2]);
    if (gz >= lim) return;
    Box<R> bx;
    bx.load(s);
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    int z = g.c[2] + dz;
    R sz = R(0);
    if (z < 0 || z >= n2) {
        if (!s.per[2]) return;
        sz = z < 0 ? -bx.L[2] : bx.L[2];
        z = z < 0 ? z + n2 : z - n2;
    }
    const R gyz = gz + gap2(dy, g.fr[1], g.cw[1]);
    if (gyz >= lim) return;
    int y = g.c[1] + dy;
    R sy = R(0);
    if (y < 0 || y >= n1) {
        if (!s.per[1]) return;
        sy = y < 0 ? -bx.L[1] : bx.L[1];
        y = y < 0 ? y + n1 : y - n1;
    }
    const int row = (int)s.cell_base + (z * n1 + y) * n0;
    const R f0 = g.fr[0], w0 = g.cw[0];
    int xa = (gyz + f0 * f0 < lim) ? g.c[0] - 1 : g.c[0];
    int xb = (gyz + (w0 - f0) * (w0 - f0) < lim) ? g.c[0] + 1 : g.c[0];
    const R L0 = bx.L[0];
    if (!s.per[0]) {
        xa = max(xa, 0);
        xb = min(xb, n0 - 1);
    } else {
        if (xa < 0) {
            f(a.start[row + n0 - 1], a.start[row + n0], -L0, sy, sz);
            xa = 0;
        }
        if (xb >= n0) {
            f(a.start[row], a.start[row + 1], L0, sy, sz);
            xb = n0 - 1;
        }
    }
    f(a.start[row + xa], a.start[row + xb + 1], R(0), sy, sz);
}

// the pair list of sorted particle i from its 27-cell neighbourhood
template <class R>
__device__ __forceinline__ void list_build_one(const Args<R>& a, const ListArgs<R>& v, const State<R>& st, int i,
                                               const R* __restrict__ s_rl2, long long off)
{
    const SysDev& s = a.sys[a.sys_of[i]];
    R xi[3];
    int wi;
    load_pos(st, i, xi, wi);
    const R* rl2 = s_rl2 + (wi & 0xff) * MAXT;
    ListWriter lw;
    lw.nbr = v.nbr;
    lw.stride = v.stride;
    lw.i = i;
    lw.cap = v.cap;
    lw.narrow = v.narrow != 0;
    lw.wide_need = false;
    int cnt = 0;
    ListCell<R> g;
    g.locate(s, xi);
    const R lim = v.rl2max * R(1.0001);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            list_row_ranges<R>(a, s, g, lim, dz, dy, [&](int j0, int j1, R sx, R sy, R sz) {
                list_range<R>(st, j0, j1, i, xi, sx, sy, sz, rl2, lw, cnt);
            });
    // narrow lists: the rest of the last group (all of group 0 for an empty
    // list: the list step always loads it) holds offset 0, the particle
    // itself, which the list step reads past the list's end (zero force)
    if (lw.narrow && cnt <= v.cap) {
        const int kfill = cnt == 0 ? 8 : (cnt + 7) & ~7;     // capacity >= 8, a multiple of 8
        for (int k = cnt; k < kfill; ++k) lw.put(k, i);
    }
    v.head[i] = make_head(xi, s, min(cnt, v.cap));
    if (cnt > v.cap || lw.wide_need) {
        if (cnt > v.cap) atomicMax(&v.ctl->maxcnt, cnt);
        atomicOr(a.err, (cnt > v.cap ? EF_LISTOVF : 0) | (lw.wide_need ? EF_LISTWIDE : 0));
        atomicMin((unsigned long long*)a.err_step, (unsigned long long)(*a.step_ptr + off));
    }
}

// re-sort, part 4: the pair list of every particle of the re-sorted state.
// A flattened walk (one candidate sequence per thread, as neighbourhood_flat)
// measured slower here than the per-row loops: the candidate test is short.
// Ranking each tile of particles by list length, so that the step kernel's
// warps walk lists of about the same length, cut the step's instructions by
// a fifth but not its time (it waits on loads, and the ranking adds one).
template <class R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) list_build_kernel(Args<R> a, ListArgs<R> v, long long off)
{
    __shared__ R s_rl2[MAXT * MAXT];
    if (!list_gate(a, v)) return;
    for (int k = threadIdx.x; k < MAXT * MAXT; k += BLOCK) s_rl2[k] = v.rl2t[k];
    __syncthreads();
    const int sel = list_sel(a, v, off);
    const State<R> st = sel ? v.b0 : v.b1;     // the scatter's destination
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    if (i < a.ntot) list_build_one<R>(a, v, st, i, s_rl2, off);
}

// j is in the pair list of i
template <class R>
__device__ __forceinline__ bool listed(const ListArgs<R>& v, int i, int j)
{
    const int cnt = head_count(__ldg(v.head + i));
    const int4* nb4 = v.nbr + i;
    const int epg = v.narrow ? 8 : 4;
    for (int k0 = 0; k0 < cnt; k0 += epg) {
        const int4 q = __ldg(nb4 + (long long)(k0 / epg) * v.stride);
        for (int u = 0; u < epg && k0 + u < cnt; ++u)
            if (list_entry(q, u, v.narrow != 0, i) == j) return true;
    }
    return false;
}

// every particle now closer to hot particle h than their cutoff is in h's
// list, and h in its; one warp per hot particle, lane r < 9 walks cell row r
// of the 27-cell neighbourhood
template <class R>
__device__ __forceinline__ bool hot_pairs_listed(const Args<R>& a, const ListArgs<R>& v, const State<R>& st, int h,
                                                 int lane)
{
    const SysDev& s = a.sys[a.sys_of[h]];
    R xh[3];
    int wh;
    load_pos(st, h, xh, wh);
    bool ok = true;
    if (lane < 9) {
        const R* rc2 = a.tab->rc2 + (wh & 0xff) * MAXT;
        Box<R> bx;
        bx.load(s);
        ListCell<R> g;
        g.locate(s, xh);
        // candidates 4 at a time: their positions are requested together
        // (past the range's end, its last candidate again, not tested)
        list_row_ranges<R>(a, s, g, v.rl2max * R(1.0001), lane / 3 - 1, lane % 3 - 1, [&](int j0, int j1, R, R, R) {
            for (int j = j0; j < j1 && ok; j += 4) {
                R xj[4][3];
                int wj[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) load_pos(st, min(j + u, j1 - 1), xj[u], wj[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = j + u;
                    if (jj >= j1 || jj == h) continue;
                    const R dx = mimg_sel(xh[0], xj[u][0], bx.L[0], bx.half[0], s.per[0]);
                    const R dy = mimg_sel(xh[1], xj[u][1], bx.L[1], bx.half[1], s.per[1]);
                    const R dz = mimg_sel(xh[2], xj[u][2], bx.L[2], bx.half[2], s.per[2]);
                    if (dist2(dx, dy, dz) < rc2[wj[u] & 0xff] * R(1.0001) && !(listed(v, h, jj) && listed(v, jj, h)))
                        ok = false;
                }
            }
        });
    }
    return __all_sync(FULL, ok);
}

// After every step, before the next one's forces: is the pair list still
// complete?  A pair missing from it was farther apart than its cutoff + skin
// at the build, so it can be closer than its cutoff now only if the two
// particles moved by skin together since: one of them moved more than
// sqrt(thr2) ~ skin/2 (a hot particle; the step kernel collects them).  For
// every hot particle h, each particle now within its cutoff of h must be in
// h's list and h in its.  The cell rows around h's current position reach
// every such particle while no particle has moved more than sqrt(cap2) ~
// skin since the build (the step kernel raises the rebuild flag itself
// beyond that).  A missing pair, or more than hot_max hot particles, raise
// the flag.  One warp per hot particle at a time.  The grid is sized for
// hot_max; only the first nb blocks, as many as the step's hot particles
// fill (one when there are none or too many), take part, and the others
// exit at once, so that a step with few hot particles costs a few blocks.
// The last of the nb blocks to finish clears the counts and sets the
// condition of the graph node that holds the re-sort (set_cond).  Every
// block that takes part reads nhot before the last one clears it (the
// clearing waits for the nb blocks' counts); a later block that reads 0
// computes nb = 1 and exits.
template <class R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) list_check_kernel(Args<R> a, ListArgs<R> v, long long off,
                                                           cudaGraphConditionalHandle hc, int set_cond)
{
    constexpr int WPB = BLOCK / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = *((volatile const int*)&v.ctl->nhot);
    const int nb = (n <= 0 || n > v.hot_max) ? 1 : min((int)gridDim.x, (n + WPB - 1) / WPB);
    if ((int)blockIdx.x >= nb) return;
    if (*((volatile const int*)a.err) == 0 && *((volatile const int*)&v.ctl->need) == 0) {
        if (n > v.hot_max) {
            if (threadIdx.x == 0) *((volatile int*)&v.ctl->need) = 1;
        } else if (n > 0) {
            const State<R> st = list_sel(a, v, off) ? v.b1 : v.b0;
            for (int k = blockIdx.x * WPB + warp; k < n; k += nb * WPB) {
                if (!hot_pairs_listed<R>(a, v, st, __ldg(v.hot + k), lane)) {
                    if (lane == 0) *((volatile int*)&v.ctl->need) = 1;
                    break;
                }
            }
        }
    }
    // the last block to finish clears the counts and sets the condition
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&v.ctl->done, 1) == nb - 1) {
            __threadfence();
            v.ctl->done = 0;
            v.ctl->nhot = 0;
            if (set_cond)
                cudaGraphSetConditional(
                    hc, (*((volatile const int*)a.err) == 0 && *((volatile const int*)&v.ctl->need)) ? 1u : 0u);
        }
    }
}

// re-sort, part 5: flip the buffer parity, clear the flag
__global__ void list_finish_kernel(ListCtl* ctl, const int* err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (*((volatile const int*)err) || !*((volatile const int*)&ctl->need)) return;
    ctl->nreb ^= 1;
    ctl->nbuild += 1;
    ctl->need = 0;
}

}  // namespace rdgpu
