// engine_kernels.cuh -- __global__ kernels of the Brownian-dynamics engine.
#pragma once
#include "engine_device.cuh"

namespace rdgpu {

constexpr int CPL_MAX = 8;      // max cells per lane in a work item
constexpr int LIST_CAP = 256;   // per-warp particle list window

// ---------------------------------------------------------------------------
// state access
// ---------------------------------------------------------------------------
template <class R> struct StateBuf;

// FP32C slot record: rec[2s] = (x, y, z, bits(type|images)),
// rec[2s+1] = (cx, cy, cz, bits(id)) -- one 32-byte sector per particle
template <> struct StateBuf<float> {
    float4* rec;
    __device__ __forceinline__ void load_xyzw(long long s, float x[3], int& w) const
    {
        float4 p = __ldg(rec + 2 * s);
        x[0] = p.x; x[1] = p.y; x[2] = p.z;
        w = __float_as_int(p.w);
    }
    __device__ __forceinline__ int load_id(long long s) const { return __float_as_int(__ldg(&rec[2 * s + 1].w)); }
};

template <> struct StateBuf<double> {
    Rec64* st;
    __device__ __forceinline__ void load_xyzw(long long s, double x[3], int& w) const
    {
        const double2* p = reinterpret_cast<const double2*>(st + s);
        double2 a = __ldg(p), b = __ldg(p + 1);
        x[0] = a.x; x[1] = a.y; x[2] = b.x;
        w = __double2loint(b.y);
    }
    __device__ __forceinline__ int load_id(long long s) const { return st[s].id; }
};

template <class R> struct StepArgs {
    const SysDev* sys;
    const WorkItem* items;
    int nitems;
    int n_ext;
    const TypeTab<R>* tab;
    const ExtTerm<R>* ext;        // [sys * n_ext + e]
    StateBuf<R> buf[2];
    int* cnt[3];
    int* work_ctr;                // [3]
    int* err;
    long long* err_step;
    const long long* step_ptr;
    int step_off;
    const double* noise;          // injected noise (3 per global index) or null
};

// force accumulators: FP32 sums pair forces in 2^-32 fixed point (exact,
// order independent); FP64 sums in double.
template <class R> struct Acc;
template <> struct Acc<float> {
    long long fx, fy, fz;
    float e;
    __device__ __forceinline__ void zero() { fx = fy = fz = 0; e = 0.f; }
    __device__ __forceinline__ void add(float pre, float dx, float dy, float dz)
    {
        fx += __float2ll_rn(-pre * dx * FX_SCALE);
        fy += __float2ll_rn(-pre * dy * FX_SCALE);
        fz += __float2ll_rn(-pre * dz * FX_SCALE);
    }
    __device__ __forceinline__ void reduce_xor(int L)
    {
        for (int o = 1; o < L; o <<= 1) {
            fx += __shfl_xor_sync(FULL, fx, o);
            fy += __shfl_xor_sync(FULL, fy, o);
            fz += __shfl_xor_sync(FULL, fz, o);
            e += __shfl_xor_sync(FULL, e, o);
        }
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
    __device__ __forceinline__ void reduce_xor(int L)
    {
        for (int o = 1; o < L; o <<= 1) {
            fx += __shfl_xor_sync(FULL, fx, o);
            fy += __shfl_xor_sync(FULL, fy, o);
            fz += __shfl_xor_sync(FULL, fz, o);
            e += __shfl_xor_sync(FULL, e, o);
        }
    }
    __device__ __forceinline__ void force(double F[3]) const { F[0] = fx; F[1] = fy; F[2] = fz; }
};

// One candidate pair (i, j): minimum image, the bit-exact neighbour predicate
// r^2 < rc(ti,tj)^2, then the pair potentials of (ti, tj).
// MODE 0: forces; 1: forces + energy; 2: neighbour digest (count, hash of id)
template <class R, int MODE>
__device__ __forceinline__ void pair_accum(const R xi[3], int ti, const R xj[3], int wj, const Box<R>& bx,
                                           const int per[3], const TypeTab<R>* __restrict__ tab, Acc<R>& acc,
                                           int& ncount, unsigned long long& hash, int idj)
{
    R dx = mimg(xi[0], xj[0], bx.L[0], bx.half[0], per[0]);
    R dy = mimg(xi[1], xj[1], bx.L[1], bx.half[1], per[1]);
    R dz = mimg(xi[2], xj[2], bx.L[2], bx.half[2], per[2]);
    R r2 = dist2(dx, dy, dz);
    const int pidx = ti * MAXT + (wj & 0xff);
    if (r2 < tab->rc2[pidx]) {
        if (MODE == 2) {
            ncount++;
            hash += splitmix64((unsigned long long)idj);
            return;
        }
        R r = sqrt(r2);
        const int nt = tab->nterm[pidx];
        for (int m = 0; m < nt; ++m) {
            R pre, e;
            pair_term(tab->term[pidx * MAX_TERMS + m], r, pre, e);
            acc.add(pre, dx, dy, dz);
            if (MODE == 1) acc.e += R(0.5) * e;
        }
    }
}

template <class R, int MODE>
__device__ __forceinline__ void cell_pairs(const StateBuf<R>& b, long long sbase, int cnt,
                                           long long self, const R xi[3], int ti, const Box<R>& bx,
                                           const int per[3], const TypeTab<R>* __restrict__ tab,
                                           Acc<R>& acc, int& ncount, unsigned long long& hash)
{
    for (int j = 0; j < cnt; ++j) {
        const long long s = sbase + j;
        if (s == self) continue;
        R xj[3];
        int wj;
        b.load_xyzw(s, xj, wj);
        pair_accum<R, MODE>(xi, ti, xj, wj, bx, per, tab, acc, ncount, hash, MODE == 2 ? b.load_id(s) : 0);
    }
}

// Pair sum over the neighbour cells k = sub, sub+L, ... of the 27-cell stencil
template <class R, int MODE>
__device__ __forceinline__ void neighbourhood(const StateBuf<R>& b, const int* __restrict__ cnt,
                                              const SysDev& s, int cx, int cy, int cz, long long self,
                                              const R xi[3], int ti, const TypeTab<R>* __restrict__ tab,
                                              int sub, int L, Acc<R>& acc, int& ncount,
                                              unsigned long long& hash)
{
    Box<R> bx;
    bx.load(s);
    const int per[3] = {s.per[0], s.per[1], s.per[2]};
    for (int k = sub; k < 27; k += L) {
        const int dz = k / 9 - 1, dy = (k / 3) % 3 - 1, dx = k % 3 - 1;
        int nx, ny, nz;
        if (!axis_cell(cx, dx, s.n[0], per[0], nx)) continue;
        if (!axis_cell(cy, dy, s.n[1], per[1], ny)) continue;
        if (!axis_cell(cz, dz, s.n[2], per[2], nz)) continue;
        const int nc = (nz * s.n[1] + ny) * s.n[0] + nx;
        const int c = min(__ldg(cnt + s.cell_base + nc), 1 << s.cap_log2);
        if (c == 0) continue;
        cell_pairs<R, MODE>(b, s.slot_base + ((long long)nc << s.cap_log2), c, self, xi, ti, bx, per,
                            tab, acc, ncount, hash);
    }
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

// FP32 with Kahan compensation: true position = x - c
__device__ __forceinline__ int em_update(float x[3], float c[3], int& w, const float F[3],
                                         const float xi[3], float A, float B, const SysDev& s)
{
    int ef = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float inc = A * F[a] + B * xi[a];
        float y = inc - c[a];
        float t = x[a] + y;
        c[a] = (t - x[a]) - y;
        x[a] = t;
        if (s.per[a]) {
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

__device__ __forceinline__ int em_update(double x[3], double* /*c*/, int& w, const double F[3],
                                         const double xi[3], double A, double B, const SysDev& s)
{
    int ef = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = x[a] + (A * F[a] + B * xi[a]);
        if (s.per[a]) {
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

template <class R>
__device__ __forceinline__ int cell_index(const SysDev& s, const R x[3])
{
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        R inv;
        if constexpr (sizeof(R) == 4) inv = s.invcf[a]; else inv = s.invc[a];
        int k = (int)(x[a] * inv);
        k = k < 0 ? 0 : (k >= s.n[a] ? s.n[a] - 1 : k);
        c[a] = k;
    }
    return (c[2] * s.n[1] + c[1]) * s.n[0] + c[0];
}

// ---------------------------------------------------------------------------
// The fused step kernel: persistent warps pull work items (runs of cells of
// one system), compact the particles of the run into a shared-memory list,
// then groups of L lanes evaluate one particle each.
// ---------------------------------------------------------------------------
// external forces, Euler-Maruyama update, wrap, claim a slot of the new cell
// in the next layout and write the particle there
template <class R>
__device__ __forceinline__ void finish_particle(const StepArgs<R>& a, const SysDev& s, int si, long long self,
                                                R xi[3], int wi, R F[3], long long t, const StateBuf<R>& cur,
                                                const StateBuf<R>& nxt, int* cnt_nxt)
{
    const int ti = wi & 0xff;
    if (a.n_ext > 0) {
        const ExtTerm<R>* ep = a.ext + (long long)si * a.n_ext;
        R ee = R(0);
        for (int e = 0; e < a.n_ext; ++e) {
            if ((ep[e].tmask >> ti) & 1u) ext_force(ep[e], a.tab->prad[ti], xi, F, ee);
        }
    }
    int id;
    R c[3] = {R(0), R(0), R(0)};
    if constexpr (sizeof(R) == 4) {
        float4 q = __ldg(cur.rec + 2 * self + 1);
        c[0] = q.x; c[1] = q.y; c[2] = q.z;
        id = __float_as_int(q.w);
    } else {
        id = cur.st[self].id;
    }
    R xn[3];
    if (a.noise) {
        const double* nz = a.noise + 3 * (s.part_base + id);
        xn[0] = (R)nz[0]; xn[1] = (R)nz[1]; xn[2] = (R)nz[2];
    } else {
        bd_normals(s.seed, t, (long long)id, xn);
    }
    int ef = em_update(xi, c, wi, F, xn, a.tab->a[ti], a.tab->b[ti], s);
    const int ncell = cell_index(s, xi);
    const int slot = atomicAdd(cnt_nxt + s.cell_base + ncell, 1);
    if (slot >= (1 << s.cap_log2)) {
        ef |= EF_OVERFLOW;
    } else {
        const long long dst = s.slot_base + ((long long)ncell << s.cap_log2) + slot;
        if constexpr (sizeof(R) == 4) {
            nxt.rec[2 * dst] = make_float4(xi[0], xi[1], xi[2], __int_as_float(wi));
            nxt.rec[2 * dst + 1] = make_float4(c[0], c[1], c[2], __int_as_float(id));
        } else {
            Rec64 r;
            r.x = xi[0]; r.y = xi[1]; r.z = xi[2]; r.w = wi; r.id = id;
            nxt.st[dst] = r;
        }
    }
    if (ef) {
        atomicOr(a.err, ef);
        atomicMin((unsigned long long*)a.err_step, (unsigned long long)t);
    }
}

// finish_particle with the compensation (FP32C) or id (FP64) already loaded
template <class R>
__device__ __forceinline__ void finish_particle_pre(const StepArgs<R>& a, const SysDev& s, int si, R xi[3], int wi,
                                                    R F[3], long long t, float4 crec, int idpre,
                                                    const StateBuf<R>& nxt, int* cnt_nxt)
{
    const int ti = wi & 0xff;
    if (a.n_ext > 0) {
        const ExtTerm<R>* ep = a.ext + (long long)si * a.n_ext;
        R ee = R(0);
        for (int e = 0; e < a.n_ext; ++e) {
            if ((ep[e].tmask >> ti) & 1u) ext_force(ep[e], a.tab->prad[ti], xi, F, ee);
        }
    }
    int id;
    R c[3] = {R(0), R(0), R(0)};
    if constexpr (sizeof(R) == 4) {
        c[0] = crec.x; c[1] = crec.y; c[2] = crec.z;
        id = __float_as_int(crec.w);
    } else {
        id = idpre;
    }
    R xn[3];
    if (a.noise) {
        const double* nz = a.noise + 3 * (s.part_base + id);
        xn[0] = (R)nz[0]; xn[1] = (R)nz[1]; xn[2] = (R)nz[2];
    } else {
        bd_normals(s.seed, t, (long long)id, xn);
    }
    int ef = em_update(xi, c, wi, F, xn, a.tab->a[ti], a.tab->b[ti], s);
    const int ncell = cell_index(s, xi);
    const int slot = atomicAdd(cnt_nxt + s.cell_base + ncell, 1);
    if (slot >= (1 << s.cap_log2)) {
        ef |= EF_OVERFLOW;
    } else {
        const long long dst = s.slot_base + ((long long)ncell << s.cap_log2) + slot;
        if constexpr (sizeof(R) == 4) {
            nxt.rec[2 * dst] = make_float4(xi[0], xi[1], xi[2], __int_as_float(wi));
            nxt.rec[2 * dst + 1] = make_float4(c[0], c[1], c[2], __int_as_float(id));
        } else {
            Rec64 r;
            r.x = xi[0]; r.y = xi[1]; r.z = xi[2]; r.w = wi; r.id = id;
            nxt.st[dst] = r;
        }
    }
    if (ef) {
        atomicOr(a.err, ef);
        atomicMin((unsigned long long*)a.err_step, (unsigned long long)t);
    }
}

template <class R>
__device__ __forceinline__ void step_particle(const StepArgs<R>& a, const SysDev& s, int si, int lslot,
                                              bool active, int sub, int L, long long t,
                                              const StateBuf<R>& cur, const StateBuf<R>& nxt,
                                              const int* __restrict__ cnt_cur, int* cnt_nxt)
{
    const long long self = s.slot_base + lslot;
    const int lcell = lslot >> s.cap_log2;
    const int nxy = s.n[0] * s.n[1];
    const int cz = lcell / nxy;
    const int rem = lcell - cz * nxy;
    const int cy = rem / s.n[0];
    const int cx = rem - cy * s.n[0];
    R xi[3] = {R(0), R(0), R(0)};
    int wi = 0;
    if (active) cur.load_xyzw(self, xi, wi);
    const int ti = wi & 0xff;
    Acc<R> acc;
    acc.zero();
    int nc = 0;
    unsigned long long hh = 0;
    if (active)
        neighbourhood<R, 0>(cur, cnt_cur, s, cx, cy, cz, self, xi, ti, a.tab, sub, L, acc, nc, hh);
    acc.reduce_xor(L);
    if (!active || sub != 0) return;
    R F[3];
    acc.force(F);
    finish_particle<R>(a, s, si, self, xi, wi, F, t, cur, nxt, cnt_nxt);
}

template <class R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) step_kernel(StepArgs<R> a)
{
    __shared__ int s_list[BLOCK / 32][LIST_CAP];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (*((volatile int*)a.err)) return;   // an earlier step failed: keep its input intact
    const long long t = (a.step_ptr ? *a.step_ptr : 0LL) + a.step_off;
    const int b3 = (int)(t % 3);
    const int* __restrict__ cnt_cur = a.cnt[b3];
    int* cnt_nxt = a.cnt[(b3 + 1) % 3];
    int* cnt_free = a.cnt[(b3 + 2) % 3];
    int* ctr = a.work_ctr + b3;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.work_ctr[(b3 + 1) % 3] = 0;
    const StateBuf<R> cur = a.buf[t & 1], nxt = a.buf[(t + 1) & 1];

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(ctr, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nitems) break;
        const WorkItem it = a.items[item];
        const SysDev& s = a.sys[it.sys];
        const int cpl = it.cpl;
        const int lg = s.lanes_log2;
        const int L = 1 << lg;
        const int cbeg = it.c0 + lane * cpl;
        int myc[CPL_MAX];
        int tot = 0;
#pragma unroll
        for (int k = 0; k < CPL_MAX; ++k) {
            myc[k] = 0;
            if (k < cpl) {
                const int c = cbeg + k;
                if (c < it.c1) {
                    myc[k] = min(cnt_cur[s.cell_base + c], 1 << s.cap_log2);
                    cnt_free[s.cell_base + c] = 0;
                }
                tot += myc[k];
            }
        }
        const int incl = warp_incl_scan(tot, lane);
        const int excl = incl - tot;
        const int total = __shfl_sync(FULL, incl, 31);
        for (int w0 = 0; w0 < total; w0 += LIST_CAP) {
            int p = excl;
#pragma unroll
            for (int k = 0; k < CPL_MAX; ++k) {
                if (k < cpl) {
                    const int c = cbeg + k;
                    for (int q = 0; q < myc[k]; ++q, ++p) {
                        const int li = p - w0;
                        if (li >= 0 && li < LIST_CAP) s_list[wib][li] = (c << s.cap_log2) + q;
                    }
                }
            }
            __syncwarp();
            const int wn = min(LIST_CAP, total - w0);
            const int G = 32 >> lg;
            for (int r0 = 0; r0 < wn; r0 += G) {
                const int e = r0 + (lane >> lg);
                const bool active = e < wn;
                const int lslot = active ? s_list[wib][e] : 0;
                step_particle<R>(a, s, it.sys, lslot, active, lane & (L - 1), L, t, cur, nxt, cnt_cur, cnt_nxt);
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// Brick-staged step kernel: a block takes a brick of ex*ey*ez cells of one
// system, stages the positions of the brick and its one-cell halo into shared
// memory (coalesced loads, all in flight together), then groups of L lanes
// evaluate one particle each from shared memory and reduce with shuffles.
// Bricks are strided statically over a persistent grid.
// ---------------------------------------------------------------------------
constexpr int MAXH = 512;     // halo cells per brick
constexpr int MAXP = 1024;    // staged particles per brick (FP32)
constexpr int MAXP64 = 896;   // staged particles per brick (FP64, 48 KB static smem)
template <class R> struct StageCap { static constexpr int value = sizeof(R) == 4 ? MAXP : MAXP64; };

struct BrickItem {
    int sys;
    int xy;       // x0 | y0 << 16
    int z;        // z0
    int ext;      // ex | ey << 8 | ez << 16 | lanes_log2 << 24
};

template <class R> struct SPos;
template <> struct alignas(16) SPos<float> { float x, y, z; int w; };
template <> struct alignas(16) SPos<double> { double x, y, z; int w, pad; };

template <int BLOCK>
__device__ __forceinline__ int block_excl_scan(const int* in, int* out, int n, int* s_warp)
{
    // out[0..n]: exclusive prefix of in[0..n), out[n] = total
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = (n + BLOCK - 1) / BLOCK;
    const int b0 = tid * per;
    int sum = 0;
    for (int k = 0; k < per; ++k)
        if (b0 + k < n) sum += in[b0 + k];
    int incl = warp_incl_scan(sum, lane);
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int v = lane < BLOCK / 32 ? s_warp[lane] : 0;
        int vi = warp_incl_scan(v, lane);
        if (lane < BLOCK / 32) s_warp[lane] = vi - v;
    }
    __syncthreads();
    int run = s_warp[wid] + incl - sum;
    for (int k = 0; k < per; ++k) {
        if (b0 + k < n) {
            out[b0 + k] = run;
            run += in[b0 + k];
        }
    }
    __syncthreads();
    if (tid == BLOCK - 1) out[n] = run;
    __syncthreads();
    return out[n];
}

__device__ __forceinline__ bool halo_axis(int v, int n, int per, int& out)
{
    if (v >= 0 && v < n) { out = v; return true; }
    if (!per) return false;
    v %= n;
    if (v < 0) v += n;
    out = v;
    return true;
}

// offsets valid on a periodic axis with fewer than 3 cells (each neighbour
// cell once)
__device__ __forceinline__ bool small_axis_ok(int d, int n, int per)
{
    if (!per || n >= 3) return true;
    if (n == 2) return d != -1;
    return d == 0;
}

// Pair term accumulation for a staged neighbour (image already applied)
template <class R>
__device__ __forceinline__ void staged_pair(R xi0, R xi1, R xi2, int ti, const SPos<R>& pj, bool notself,
                                            const R* __restrict__ s_rc2, const TypeTab<R>* __restrict__ tab,
                                            Acc<R>& acc)
{
    const R dx = sub_rn(xi0, pj.x), dy = sub_rn(xi1, pj.y), dz = sub_rn(xi2, pj.z);
    const R r2 = dist2(dx, dy, dz);
    const int pidx = ti * MAXT + (pj.w & 0xff);
    if (r2 < s_rc2[pidx] && notself) {
        const R r = sqrt(r2);
        const int nt = tab->nterm[pidx];
        for (int m = 0; m < nt; ++m) {
            R pre, e;
            pair_term(tab->term[pidx * MAX_TERMS + m], r, pre, e);
            acc.add(pre, dx, dy, dz);
        }
    }
}

template <class R>
__device__ __noinline__ void brick_fallback(const StateBuf<R> cur, const int* __restrict__ cnt_cur, const SysDev& s,
                                            int gc, long long self, const TypeTab<R>* __restrict__ tab, int sub,
                                            int L, Acc<R>& acc, R& xi0, R& xi1, R& xi2, int& wi)
{
    R xi[3];
    cur.load_xyzw(self, xi, wi);
    xi0 = xi[0]; xi1 = xi[1]; xi2 = xi[2];
    const int cx = gc % s.n[0], cy = (gc / s.n[0]) % s.n[1], cz = gc / (s.n[0] * s.n[1]);
    int nc = 0;
    unsigned long long hh = 0;
    neighbourhood<R, 0>(cur, cnt_cur, s, cx, cy, cz, self, xi, wi & 0xff, tab, sub, L, acc, nc, hh);
}

// asynchronous 16-byte global -> shared copy (no register round trip)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <class R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) brick_step_kernel(StepArgs<R> a, const BrickItem* __restrict__ bricks,
                                                           int nbricks)
{
    constexpr int SCAP = StageCap<R>::value;
    constexpr int HPT = MAXH / BLOCK;   // halo cells per thread
    __shared__ int s_cnt[MAXH];
    __shared__ int s_off[MAXH + 1];
    __shared__ int s_gc[MAXH];          // global cell | image code << 26 (2 bits per axis)
    __shared__ int s_icnt[MAXH];
    __shared__ int s_ioff[MAXH + 1];
    __shared__ int s_warp[BLOCK / 32];
    __shared__ int s_ilist[SCAP];       // inner particle -> staged index | halo cell << 12
    __shared__ SPos<R> s_p[SCAP];
    __shared__ R s_rc2[MAXT * MAXT];

    if (*((volatile int*)a.err)) return;   // an earlier step failed: keep its input intact
    const int tid = threadIdx.x;
    const long long t = (a.step_ptr ? *a.step_ptr : 0LL) + a.step_off;
    const int b3 = (int)(t % 3);
    const int* __restrict__ cnt_cur = a.cnt[b3];
    int* __restrict__ cnt_nxt = a.cnt[(b3 + 1) % 3];
    int* __restrict__ cnt_free = a.cnt[(b3 + 2) % 3];
    const StateBuf<R> cur = a.buf[t & 1], nxt = a.buf[(t + 1) & 1];
    for (int i = tid; i < MAXT * MAXT; i += BLOCK) s_rc2[i] = a.tab->rc2[i];

    for (int bi = blockIdx.x; bi < nbricks; bi += gridDim.x) {
        const BrickItem it = bricks[bi];
        const SysDev& s = a.sys[it.sys];
        const int x0 = it.xy & 0xffff, y0 = it.xy >> 16, z0 = it.z;
        const int ex = it.ext & 0xff, ey = (it.ext >> 8) & 0xff, ez = (it.ext >> 16) & 0xff;
        const int lg = (it.ext >> 24) & 0x7;
        const int hx = ex + 2, hy = ey + 2, hz = ez + 2;
        const int H = hx * hy * hz, NI = ex * ey * ez;
        const int cap_log2 = s.cap_log2, cap = 1 << cap_log2;
        const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
        const int per0 = s.per[0], per1 = s.per[1], per2 = s.per[2];

        // 1. halo cells: global cell, image shift, count -- all count loads in
        //    flight together, then the shared-memory stores
        int gcode[HPT], cval[HPT];
#pragma unroll
        for (int k = 0; k < HPT; ++k) {
            const int h = tid + k * BLOCK;
            gcode[k] = -1;
            cval[k] = 0;
            if (h < H) {
                const int r = h / hx, ix = h - r * hx;
                const int iz = r / hy, iy = r - iz * hy;
                int gx = x0 - 1 + ix, gy = y0 - 1 + iy, gz = z0 - 1 + iz, kx = 0, ky = 0, kz = 0;
                bool v = true;
                if (gx < 0) { if (per0) { gx += n0; kx = -1; } else v = false; }
                else if (gx >= n0) { if (per0) { gx -= n0; kx = 1; } else v = false; }
                if (gy < 0) { if (per1) { gy += n1; ky = -1; } else v = false; }
                else if (gy >= n1) { if (per1) { gy -= n1; ky = 1; } else v = false; }
                if (gz < 0) { if (per2) { gz += n2; kz = -1; } else v = false; }
                else if (gz >= n2) { if (per2) { gz -= n2; kz = 1; } else v = false; }
                if (v) {
                    const int gc = (gz * n1 + gy) * n0 + gx;
                    gcode[k] = gc | (((kx + 1) | ((ky + 1) << 2) | ((kz + 1) << 4)) << 26);
                    cval[k] = __ldg(cnt_cur + s.cell_base + gc);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < HPT; ++k) {
            const int h = tid + k * BLOCK;
            if (h < H) {
                const int c = min(cval[k], cap);
                s_gc[h] = gcode[k];
                s_cnt[h] = c;
                const int r = h / hx, ix = h - r * hx;
                const int iz = r / hy, iy = r - iz * hy;
                if (ix >= 1 && ix <= ex && iy >= 1 && iy <= ey && iz >= 1 && iz <= ez) {
                    s_icnt[((iz - 1) * ey + (iy - 1)) * ex + (ix - 1)] = c;
                    cnt_free[s.cell_base + (gcode[k] & ((1 << 26) - 1))] = 0;
                }
            }
        }
        __syncthreads();
        const int T = block_excl_scan<BLOCK>(s_cnt, s_off, H, s_warp);
        const int TI = block_excl_scan<BLOCK>(s_icnt, s_ioff, NI, s_warp);
        // systems with fewer than 3 cells on a periodic axis take the global path
        const bool small = (per0 && n0 < 3) || (per1 && n1 < 3) || (per2 && n2 < 3);
        const bool staged = T <= SCAP && !small;

        // 2. stage brick + halo with asynchronous copies; list the inner particles
        if (staged) {
            for (int h = tid; h < H; h += BLOCK) {
                const int c = s_cnt[h];
                if (c == 0) continue;
                const long long g = s.slot_base + ((long long)(s_gc[h] & ((1 << 26) - 1)) << cap_log2);
                const int o = s_off[h];
                for (int q = 0; q < c; ++q) {
                    if constexpr (sizeof(R) == 4) {
                        cp_async16(&s_p[o + q], cur.rec + 2 * (g + q));
                    } else {
                        cp_async16(&s_p[o + q], cur.st + g + q);
                        cp_async16(reinterpret_cast<char*>(&s_p[o + q]) + 16,
                                   reinterpret_cast<const char*>(cur.st + g + q) + 16);
                    }
                }
            }
        }
        for (int kin = tid; kin < NI; kin += BLOCK) {
            const int c = s_icnt[kin];
            if (c == 0) continue;
            const int ix = kin % ex, rest = kin / ex, iy = rest % ey, iz = rest / ey;
            const int h = ((iz + 1) * hy + (iy + 1)) * hx + (ix + 1);
            const int o = s_off[h], io = s_ioff[kin];
            for (int q = 0; q < c; ++q) s_ilist[io + q] = (o + q) | (h << 12);
        }
        if (staged) {
            cp_async_wait_all();
            // apply the periodic image shift of wrapped halo cells to the copies
            // this thread issued (the FP64 record's w/id word comes along as is)
            R Lx, Ly, Lz;
            if constexpr (sizeof(R) == 4) { Lx = s.Lf[0]; Ly = s.Lf[1]; Lz = s.Lf[2]; }
            else { Lx = s.L[0]; Ly = s.L[1]; Lz = s.L[2]; }
            for (int h = tid; h < H; h += BLOCK) {
                const int code = s_gc[h];
                const int c = s_cnt[h];
                if (c == 0 || (((unsigned)code >> 26) == 0x15u)) continue;   // 0x15: no shift on any axis
                const int kx = ((code >> 26) & 3) - 1, ky = ((code >> 28) & 3) - 1, kz = ((code >> 30) & 3) - 1;
                const int o = s_off[h];
                for (int q = 0; q < c; ++q) {
                    SPos<R>& sp = s_p[o + q];
                    if (kx) sp.x = add_rn(sp.x, kx > 0 ? Lx : -Lx);
                    if (ky) sp.y = add_rn(sp.y, ky > 0 ? Ly : -Ly);
                    if (kz) sp.z = add_rn(sp.z, kz > 0 ? Lz : -Lz);
                }
            }
        }
        __syncthreads();

        // 3. groups of L lanes, one particle each: 9 contiguous row ranges
        const int L = 1 << lg, G = BLOCK >> lg, g = tid >> lg, sub = tid & (L - 1);
        for (int base = 0; base < TI; base += G) {
            const int p = base + g;
            const bool active = p < TI;
            Acc<R> acc;
            acc.zero();
            int si = 0, h = 0;
            R xi0 = R(0), xi1 = R(0), xi2 = R(0);
            int wi = 0;
            if (active) {
                const int e = s_ilist[p];
                si = e & 0xfff;
                h = e >> 12;
            }
            const int q = si - s_off[h];
            const long long self = s.slot_base + ((long long)(s_gc[h] & ((1 << 26) - 1)) << cap_log2) + q;
            // the particle's compensation/id record, fetched before the pair loop
            float4 crec = make_float4(0.f, 0.f, 0.f, 0.f);
            int idpre = 0;
            if (active && sub == 0) {
                if constexpr (sizeof(R) == 4) crec = __ldg(cur.rec + 2 * self + 1);
                else idpre = __ldg(&cur.st[self].id);
            }
            if (active && staged) {
                const SPos<R> sp = s_p[si];
                xi0 = sp.x; xi1 = sp.y; xi2 = sp.z;
                wi = sp.w;
                const int ti = wi & 0xff;
                for (int rr = sub; rr < 9; rr += L) {
                    const int dz = rr / 3 - 1, dy = rr - (rr / 3) * 3 - 1;
                    const int hrow = h + (dz * hy + dy) * hx;
                    const int t0 = s_off[hrow - 1], t1 = s_off[hrow + 2];
                    for (int tj = t0; tj < t1; ++tj)
                        staged_pair<R>(xi0, xi1, xi2, ti, s_p[tj], tj != si, s_rc2, a.tab, acc);
                }
            } else if (active) {
                // brick too dense for the stage, or a tiny periodic box: global loads
                brick_fallback<R>(cur, cnt_cur, s, s_gc[h] & ((1 << 26) - 1), self, a.tab, sub, L, acc,
                                  xi0, xi1, xi2, wi);
            }
            acc.reduce_xor(L);
            if (active && sub == 0) {
                R F[3];
                acc.force(F);
                R xi[3] = {xi0, xi1, xi2};
                finish_particle_pre<R>(a, s, it.sys, xi, wi, F, t, crec, idpre, nxt, cnt_nxt);
            }
        }
        __syncthreads();
    }
}

// advances the device step counter after a captured run of n steps, unless a
// step failed (the host then resumes from the failing step)
__global__ void advance_kernel(long long* step, const int* err, int n)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && *err == 0) *step += n;
}

// ---------------------------------------------------------------------------
// binning of dense per-particle arrays into the cell layout of a buffer
// ---------------------------------------------------------------------------
__device__ __forceinline__ int find_sys_by_part(const SysDev* sys, int nsys, long long g)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sys[mid].part_base <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int find_sys_by_cell(const SysDev* sys, int nsys, long long c)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sys[mid].cell_base <= c) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <class R> struct Dense;
template <> struct Dense<float> { float4* pos; float4* cmp; };
template <> struct Dense<double> { Rec64* st; };

template <class R>
__global__ void bin_kernel(const SysDev* sys, int nsys, long long ntot, Dense<R> d, StateBuf<R> b,
                           int* cnt, int* err)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const int si = find_sys_by_part(sys, nsys, g);
        const SysDev& s = sys[si];
        R x[3];
        if constexpr (sizeof(R) == 4) {
            float4 p = d.pos[g];
            x[0] = p.x; x[1] = p.y; x[2] = p.z;
        } else {
            x[0] = d.st[g].x; x[1] = d.st[g].y; x[2] = d.st[g].z;
        }
        const int c = cell_index(s, x);
        const int slot = atomicAdd(cnt + s.cell_base + c, 1);
        if (slot >= (1 << s.cap_log2)) { atomicOr(err, EF_OVERFLOW); continue; }
        const long long dst = s.slot_base + ((long long)c << s.cap_log2) + slot;
        if constexpr (sizeof(R) == 4) { b.rec[2 * dst] = d.pos[g]; b.rec[2 * dst + 1] = d.cmp[g]; }
        else { b.st[dst] = d.st[g]; }
    }
}

constexpr int EF_BADINPUT = 8;

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

template <class R>
__global__ void ingest_kernel(const SysDev* sys, int nsys, long long ntot, const double* __restrict__ xyz,
                              const int* __restrict__ types, int ntypes, Dense<R> d, double* x0, int* err)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const int si = find_sys_by_part(sys, nsys, g);
        const SysDev& s = sys[si];
        const int t = types[g];
        bool ok = t >= 0 && t < ntypes;
        const int id = (int)(g - s.part_base);
        if constexpr (sizeof(R) == 4) {
            float h[3], c[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float Lf = s.Lf[a];
                double xr = __dsub_rn(xyz[3 * g + a], s.lo[a]);
                ok = ok && isfinite(xr) && wrap_rel_dev(xr, (double)Lf, s.per[a]);
                float hh = __double2float_rn(xr);
                if (s.per[a] && hh >= Lf) { hh = 0.0f; xr = __dsub_rn(xr, (double)Lf); }
                h[a] = hh;
                c[a] = __double2float_rn(__dsub_rn((double)hh, xr));
                x0[3 * g + a] = xr;
            }
            d.pos[g] = make_float4(h[0], h[1], h[2], __int_as_float(t));
            d.cmp[g] = make_float4(c[0], c[1], c[2], __int_as_float(id));
        } else {
            double x[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                double xr = __dsub_rn(xyz[3 * g + a], s.lo[a]);
                ok = ok && isfinite(xr) && wrap_rel_dev(xr, s.L[a], s.per[a]);
                x[a] = xr;
                x0[3 * g + a] = xr;
            }
            Rec64 r;
            r.x = x[0]; r.y = x[1]; r.z = x[2]; r.w = t; r.id = id;
            d.st[g] = r;
        }
        if (!ok) atomicOr(err, EF_BADINPUT);
    }
}

// dense arrays -> absolute coordinates and types (by global index)
template <class R>
__global__ void emit_kernel(const SysDev* sys, int nsys, long long ntot, Dense<R> d, double* xyz, int* types)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const int si = find_sys_by_part(sys, nsys, g);
        const SysDev& s = sys[si];
        if constexpr (sizeof(R) == 4) {
            const float4 p = d.pos[g], c = d.cmp[g];
            xyz[3 * g + 0] = __dadd_rn(__dsub_rn((double)p.x, (double)c.x), s.lo[0]);
            xyz[3 * g + 1] = __dadd_rn(__dsub_rn((double)p.y, (double)c.y), s.lo[1]);
            xyz[3 * g + 2] = __dadd_rn(__dsub_rn((double)p.z, (double)c.z), s.lo[2]);
            types[g] = __float_as_int(p.w) & 0xff;
        } else {
            const Rec64 r = d.st[g];
            xyz[3 * g + 0] = __dadd_rn(r.x, s.lo[0]);
            xyz[3 * g + 1] = __dadd_rn(r.y, s.lo[1]);
            xyz[3 * g + 2] = __dadd_rn(r.z, s.lo[2]);
            types[g] = r.w & 0xff;
        }
    }
}

// cell layout -> dense arrays (by global particle index)
template <class R>
__global__ void gather_kernel(const SysDev* sys, int nsys, long long ncells_tot, StateBuf<R> b,
                              const int* cnt, Dense<R> d)
{
    for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncells_tot;
         gc += (long long)gridDim.x * blockDim.x) {
        const int n = cnt[gc];
        if (n == 0) continue;
        const int si = find_sys_by_cell(sys, nsys, gc);
        const SysDev& s = sys[si];
        const int cap = 1 << s.cap_log2;
        const long long base = s.slot_base + ((gc - s.cell_base) << s.cap_log2);
        for (int q = 0; q < n && q < cap; ++q) {
            if constexpr (sizeof(R) == 4) {
                float4 c = b.rec[2 * (base + q) + 1];
                long long g = s.part_base + __float_as_int(c.w);
                d.pos[g] = b.rec[2 * (base + q)];
                d.cmp[g] = c;
            } else {
                Rec64 r = b.st[base + q];
                d.st[s.part_base + r.id] = r;
            }
        }
    }
}

// per-cell counts -> max occupancy
__global__ void max_count_kernel(const int* cnt, long long n, int* out)
{
    int m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = max(m, cnt[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ---------------------------------------------------------------------------
// diagnostics: forces + energy, neighbour digest (same pair code as the step)
// ---------------------------------------------------------------------------
template <class R, int MODE>
__global__ void diag_kernel(StepArgs<R> a, int nsys, long long ncells_tot, int buf, int cntbuf,
                            double* forces, double* energy, int* ncount, unsigned long long* hashes)
{
    const StateBuf<R> cur = a.buf[buf];
    const int* cnt = a.cnt[cntbuf];
    for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncells_tot;
         gc += (long long)gridDim.x * blockDim.x) {
        int n = cnt[gc];
        if (n == 0) continue;
        const int si = find_sys_by_cell(a.sys, nsys, gc);
        const SysDev& s = a.sys[si];
        n = min(n, 1 << s.cap_log2);
        const int lcell = (int)(gc - s.cell_base);
        const int nxy = s.n[0] * s.n[1];
        const int cz = lcell / nxy, rem = lcell - cz * nxy, cy = rem / s.n[0], cx = rem - cy * s.n[0];
        for (int q = 0; q < n; ++q) {
            const long long self = s.slot_base + ((long long)lcell << s.cap_log2) + q;
            R xi[3];
            int wi;
            cur.load_xyzw(self, xi, wi);
            const int ti = wi & 0xff;
            const long long g = s.part_base + cur.load_id(self);
            Acc<R> acc;
            acc.zero();
            int nc = 0;
            unsigned long long hh = 0;
            neighbourhood<R, MODE>(cur, cnt, s, cx, cy, cz, self, xi, ti, a.tab, 0, 1, acc, nc, hh);
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
}

// Gaussian draws of step `t` by global particle index
template <class R>
__global__ void noise_kernel(const SysDev* sys, int nsys, long long ntot, long long t, double* out)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
         g += (long long)gridDim.x * blockDim.x) {
        const int si = find_sys_by_part(sys, nsys, g);
        R xn[3];
        bd_normals(sys[si].seed, t, g - sys[si].part_base, xn);
        out[3 * g] = xn[0];
        out[3 * g + 1] = xn[1];
        out[3 * g + 2] = xn[2];
    }
}

// ---------------------------------------------------------------------------
// RDF: counts of ordered pairs by (ti, tj, bin), FP64 predicate on the stored
// positions, stencil of +-R cells (CudaSimulation.cu:1784-1827 semantics).
// ---------------------------------------------------------------------------
template <class R>
__global__ void rdf_kernel(const SysDev* sys, int nsys, long long ncells_tot, StateBuf<R> b,
                           const int* cnt, int S, int nbins, const double* __restrict__ e2,
                           double w, int use_smem, unsigned long long* hist)
{
    extern __shared__ unsigned int sh[];
    const int H = S * S * nbins;
    if (use_smem) {
        for (int i = threadIdx.x; i < H; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    const double rmax2 = e2[nbins];
    const double rmax = w * nbins;
    for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncells_tot;
         gc += (long long)gridDim.x * blockDim.x) {
        int n = cnt[gc];
        if (n == 0) continue;
        const int si = find_sys_by_cell(sys, nsys, gc);
        const SysDev& s = sys[si];
        n = min(n, 1 << s.cap_log2);
        double L[3], half[3];
        int rng[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if constexpr (sizeof(R) == 4) L[a] = (double)s.Lf[a]; else L[a] = s.L[a];
            half[a] = 0.5 * L[a];
            // cells to search each way; the whole axis once if the stencil wraps onto itself
            int r = (int)ceil(rmax * s.invc[a]) ;
            if (r < 1) r = 1;
            rng[a] = r;
        }
        const int lcell = (int)(gc - s.cell_base);
        const int nxy = s.n[0] * s.n[1];
        const int cc[3] = {lcell % s.n[0], (lcell / s.n[0]) % s.n[1], lcell / nxy};
        int lo3[3], cntax[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (s.per[a]) {
                if (2 * rng[a] + 1 >= s.n[a]) { lo3[a] = 0; cntax[a] = s.n[a]; rng[a] = -1; }
                else { lo3[a] = cc[a] - rng[a]; cntax[a] = 2 * rng[a] + 1; }
            } else {
                int l = max(0, cc[a] - rng[a]), h = min(s.n[a] - 1, cc[a] + rng[a]);
                lo3[a] = l; cntax[a] = h - l + 1;
            }
        }
        for (int q = 0; q < n; ++q) {
            const long long self = s.slot_base + ((long long)lcell << s.cap_log2) + q;
            R xr[3];
            int wi;
            b.load_xyzw(self, xr, wi);
            const double xi0 = (double)xr[0], xi1 = (double)xr[1], xi2 = (double)xr[2];
            const int ti = wi & 0xff;
            for (int iz = 0; iz < cntax[2]; ++iz) {
                int z = lo3[2] + iz;
                if (s.per[2]) z = (z % s.n[2] + s.n[2]) % s.n[2];
                for (int iy = 0; iy < cntax[1]; ++iy) {
                    int y = lo3[1] + iy;
                    if (s.per[1]) y = (y % s.n[1] + s.n[1]) % s.n[1];
                    for (int ix = 0; ix < cntax[0]; ++ix) {
                        int x = lo3[0] + ix;
                        if (s.per[0]) x = (x % s.n[0] + s.n[0]) % s.n[0];
                        const int nc = (z * s.n[1] + y) * s.n[0] + x;
                        const int m = min(__ldg(cnt + s.cell_base + nc), 1 << s.cap_log2);
                        const long long sb = s.slot_base + ((long long)nc << s.cap_log2);
                        for (int j = 0; j < m; ++j) {
                            if (sb + j == self) continue;
                            R xq[3];
                            int wj;
                            b.load_xyzw(sb + j, xq, wj);
                            double dx = mimg(xi0, (double)xq[0], L[0], half[0], s.per[0]);
                            double dy = mimg(xi1, (double)xq[1], L[1], half[1], s.per[1]);
                            double dz = mimg(xi2, (double)xq[2], L[2], half[2], s.per[2]);
                            double r2 = dist2(dx, dy, dz);
                            if (!(r2 < rmax2)) continue;
                            int k = (int)(sqrt(r2) / w);
                            k = min(max(k, 0), nbins - 1);
                            while (k > 0 && e2[k] > r2) --k;
                            while (k < nbins - 1 && e2[k + 1] <= r2) ++k;
                            const int hidx = (ti * S + (wj & 0xff)) * nbins + k;
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

// ---------------------------------------------------------------------------
// MSD: squared unwrapped displacement per particle (FP64)
// ---------------------------------------------------------------------------
template <class R>
__global__ void msd_kernel(const SysDev* sys, int nsys, long long ncells_tot, StateBuf<R> b,
                           const int* cnt, const double* x0, double* d2, int* types)
{
    for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncells_tot;
         gc += (long long)gridDim.x * blockDim.x) {
        int n = cnt[gc];
        if (n == 0) continue;
        const int si = find_sys_by_cell(sys, nsys, gc);
        const SysDev& s = sys[si];
        n = min(n, 1 << s.cap_log2);
        const long long base = s.slot_base + ((gc - s.cell_base) << s.cap_log2);
        for (int q = 0; q < n; ++q) {
            double u[3];
            int w, id;
            if constexpr (sizeof(R) == 4) {
                float4 p = b.rec[2 * (base + q)], c = b.rec[2 * (base + q) + 1];
                u[0] = (double)p.x - (double)c.x;
                u[1] = (double)p.y - (double)c.y;
                u[2] = (double)p.z - (double)c.z;
                w = __float_as_int(p.w);
                id = __float_as_int(c.w);
            } else {
                Rec64 r = b.st[base + q];
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
}

// deterministic per-type sums in index order: block b sums the entries of
// type b (b == S: all entries)
__global__ void typed_sum_kernel(const double* v, const int* types, long long n, int S, double* out,
                                 long long* counts)
{
    extern __shared__ double red[];
    const int want = blockIdx.x;
    double acc = 0.0;
    long long c = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        if (want == S || types[i] == want) { acc += v[i]; ++c; }
    }
    red[threadIdx.x] = acc;
    long long* cr = reinterpret_cast<long long*>(red + blockDim.x);
    cr[threadIdx.x] = c;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
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

}  // namespace rdgpu
