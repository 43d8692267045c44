// engine_device.cuh -- device-side types and helpers of the B200
// Brownian-dynamics engine: per-system constants (SysDev), per-type tables,
// pair and external potentials with the Java semantics, Philox-4x32-10 noise
// and Box-Muller, IEEE-exact minimum image and distance, error flags.
//
// Data layout in HBM (per handle; all systems of a batch share the arrays):
//   cells:  every system owns n0*n1*n2 cells of edge L/n (>= the cutoff, or
//           the cutoff + skin with the pair list), cell id (z*n1 + y)*n0 + x
//           placed at cell_base in the global cell arrays.
//   state:  sorted by cell (CSR: particles of cell c are start[c] ..
//           start[c+1]); FP32C pos[i] = float4(x, y, z, bits(type | images)),
//           aux[i] = float4(cx, cy, cz, bits(id)), true position x - cx;
//           FP64 Rec64{double x, y, z; int w (type | images); int id}.
//           Coordinates are box-relative, in [0, L) on periodic axes.
//   Two state buffers: a step reads one and writes the other.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rdgpu {

constexpr int MAXT = 16;
constexpr int MAX_TERMS = 4;
constexpr unsigned FULL = 0xffffffffu;

// error flags
constexpr int EF_NONFINITE = 2;
constexpr int EF_JUMP = 4;

// fixed-point scale of the FP32 force accumulator (2^32): order-independent,
// hence deterministic, sums of FP32 pair forces.
constexpr float FX_SCALE = 4294967296.0f;
constexpr float FX_INV = 2.3283064365386963e-10f;

struct SysDev {
    int n[3];
    int per[3];
    int ncells;
    long long cell_base;
    long long part_base;
    int npart;
    float Lf[3], halff[3], invcf[3];
    float ilf[3];     // 1/Lf on periodic axes, 0 on open ones (image by rounding)
    double L[3], half[3], invc[3];
    double il[3];     // 1/L on periodic axes, 0 on open ones (image by rounding)
    double lo[3];
    unsigned long long seed;
    float qs[3];      // 2^16 / L: bins of the 16-bit build-position lattice per unit length
    float iqs[3];     // L / 2^16
};

template <class R> struct PairTerm {
    int kind, sub;
    R k, r0, l, d, q;
};

template <class R> struct ExtTerm {
    int kind, sub;
    R k;
    R c[3], nrm[3];
    R rad, h;
    R blo[3], bhi[3];
    int consider;
    unsigned tmask;
    R rad2h, rad2l;   // rad^2 as an unevaluated sum hi + lo (FP32 sphere distance)
};

template <class R> struct TypeTab {
    int S;
    int n_ext;
    R a[MAXT];        // D dt / (kB T)
    R b[MAXT];        // sqrt(2 D dt)
    R prad[MAXT];     // default collision radius (external potentials)
    R rc2[MAXT * MAXT];
    int nterm[MAXT * MAXT];
    PairTerm<R> term[MAXT * MAXT * MAX_TERMS];
};

struct alignas(32) Rec64 {
    double x, y, z;
    int w;
    int id;
};

struct WorkItem {
    int sys;
    int c0, c1;
    int cpl;          // cells per lane
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Counter (index lo, index hi, step lo, step hi),
// key = the system seed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

__device__ __forceinline__ uint4 bd_words(unsigned long long seed, long long step, long long index)
{
    uint4 c = make_uint4((unsigned)index, (unsigned)((unsigned long long)index >> 32),
                         (unsigned)step, (unsigned)((unsigned long long)step >> 32));
    return philox4x32_10(c, make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
}

// -2 ln u of the uniform u = (w + 1/2) 2^-32 of Philox word w, in FP32.
// Near u = 1 the logarithm is small and an absolute error in it becomes a
// large relative error in sqrt(-2 ln u), so for v = 1 - u < 1/16 it is the
// Taylor series -ln(1 - v) = v + v^2/2 + ... + v^6/6 (truncation below
// v^6/7 relative, 9e-9), with v = (~w + 1/2) 2^-32 taken from the
// complement of the word (exact where it matters; u itself, rounded to 24
// bits, would be off by up to 2^-25).  Elsewhere, |ln u| >= ln(16/15), the
// hardware log2 (__log2f) times ln 2.  Both values are computed and one is
// selected, so the warp does not diverge.
__device__ __forceinline__ float bm_minus2ln(unsigned w)
{
    const float s = 2.3283064365386963e-10f;    // 2^-32
    const float u = ((float)w + 0.5f) * s;
    const float v = ((float)(~w) + 0.5f) * s;
    float p = 1.0f / 6.0f;
    p = fmaf(p, v, 0.2f);
    p = fmaf(p, v, 0.25f);
    p = fmaf(p, v, 1.0f / 3.0f);
    p = fmaf(p, v, 0.5f);
    p = fmaf(p, v, 1.0f);
    const float series = 2.0f * v * p;
    const float hw = -1.3862943611198906f * __log2f(u);    // -2 ln 2 log2(u)
    return v < 0.0625f ? series : hw;
}

// Box-Muller on the uniforms (w + 1/2) 2^-32 of the four Philox words.  The
// FP32 transform takes the angle from the hardware sin/cos approximation on
// the argument 2 pi u - pi in [-pi, pi], where its absolute error is about
// 4e-7, and flips the sign back; the radius is sqrt(bm_minus2ln(w)).
__device__ __forceinline__ void bd_normals(unsigned long long seed, long long step, long long index,
                                           float out[3])
{
    uint4 w = bd_words(seed, step, index);
    const float s = 2.3283064365386963e-10f;
    const float two_pi = 6.283185307179586f, pi = 3.141592653589793f;
    const float u1 = ((float)w.y + 0.5f) * s, u3 = ((float)w.w + 0.5f) * s;
    const float ra = sqrtf(bm_minus2ln(w.x)), rb = sqrtf(bm_minus2ln(w.z));
    float sa, ca, sb, cb;
    __sincosf(fmaf(u1, two_pi, -pi), &sa, &ca);
    __sincosf(fmaf(u3, two_pi, -pi), &sb, &cb);
    out[0] = -ra * ca;
    out[1] = -ra * sa;
    out[2] = -rb * cb;
}

__device__ __forceinline__ void bd_normals(unsigned long long seed, long long step, long long index,
                                           double out[3])
{
    uint4 w = bd_words(seed, step, index);
    const double s = 2.3283064365386963e-10;
    double u0 = ((double)w.x + 0.5) * s, u1 = ((double)w.y + 0.5) * s;
    double u2 = ((double)w.z + 0.5) * s, u3 = ((double)w.w + 0.5) * s;
    double ra = sqrt(-2.0 * log(u0)), rb = sqrt(-2.0 * log(u2));
    double sa, ca, sb, cb;
    sincospi(2.0 * u1, &sa, &ca);
    sincospi(2.0 * u3, &sb, &cb);
    out[0] = ra * ca;
    out[1] = ra * sa;
    out[2] = rb * cb;
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// ---------------------------------------------------------------------------
// Non-contracted arithmetic: the neighbour predicate must round exactly like
// the CPU oracle (no FMA), so dx, r^2 use explicit _rn intrinsics.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// ---------------------------------------------------------------------------
// Packed FP32 pairs: add/sub/mul/fma.rn.f32x2 of sm_100 work on two floats
// held in one 64-bit register pair, each lane rounded as the scalar op (an
// instruction with an explicit rounding mode is never contracted).
// ---------------------------------------------------------------------------
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Operands of pair_disp_x2 for one particle i of system s.
struct PairFrame {
    f32x2 xy, il_xy, l_xy;   // (x, y) of i, 1/L or 0, L
    float z, il_z, l_z;
    __device__ __forceinline__ void load(const SysDev& s, const float xi[3])
    {
        xy = f2_pack(xi[0], xi[1]);
        il_xy = f2_pack(s.ilf[0], s.ilf[1]);
        l_xy = f2_pack(s.Lf[0], s.Lf[1]);
        z = xi[2];
        il_z = s.ilf[2];
        l_z = s.Lf[2];
    }
};

// FP64 minimum-image displacement of a listed pair along one axis: the image
// k in {-1, 0, 1} is rint((xi - xj)/L), rounded by adding and subtracting
// 1.5 2^52 to the exact product with il = 1/L (0 on an open axis), then
// xi - (xj + k L), one rounding per operation as in mimg.  As for the FP32
// pair_disp_x2 below, k differs from mimg's comparison with L/2 only for
// pairs about L/2 apart on that axis, which no cutoff reaches.
__device__ __forceinline__ double mimg_round(double xi, double xj, double L, double il)
{
    const double M = 6755399441055744.0;   // 1.5 2^52
    const double k = __dadd_rn(__fma_rn(__dsub_rn(xi, xj), il, M), -M);
    return __dsub_rn(xi, __fma_rn(k, L, xj));
}

// FP32 minimum-image displacement and squared distance of a listed pair, x
// and y as one packed pair.  The image k in {-1, 0, 1} is rint((xi - xj)/L),
// rounded by adding and subtracting 1.5 2^23 to the exact product with 1/L
// (0 on open axes, so k = 0); then dx = xi - (xj + k L) and r^2 = (dx^2 +
// dy^2) + dz^2, one rounding per operation as in mimg and dist2.  k differs
// from the comparison with L/2 of mimg only when |xi - xj| is within a few
// ulp of L/2, and then both images are at least L/2 >= 1.5 (rc + skin) apart
// on that axis (the pair list needs >= 3 cells of edge rc + skin on every
// periodic axis): the pair is rejected either way, the forces are unchanged.
__device__ __forceinline__ void pair_disp_x2(const PairFrame& f, float xj, float yj, float zj, float& dx, float& dy,
                                             float& dz, float& r2)
{
    const float M = 12582912.0f;     // 1.5 2^23
    const f32x2 M2 = f2_pack(M, M), NM2 = f2_pack(-M, -M);
    const f32x2 xyj = f2_pack(xj, yj);
    const f32x2 k = f2_add(f2_fma(f2_sub(f.xy, xyj), f.il_xy, M2), NM2);
    const f32x2 d = f2_sub(f.xy, f2_fma(k, f.l_xy, xyj));
    float px, py;
    f2_unpack(f2_mul(d, d), px, py);
    f2_unpack(d, dx, dy);
    const float kz = __fadd_rn(__fmaf_rn(__fsub_rn(f.z, zj), f.il_z, M), -M);
    dz = __fsub_rn(f.z, __fmaf_rn(kz, f.l_z, zj));
    r2 = __fadd_rn(__fadd_rn(px, py), __fmul_rn(dz, dz));
}

template <class R> struct Box;
template <> struct Box<float> {
    float L[3], half[3];
    __device__ __forceinline__ void load(const SysDev& s)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) { L[a] = s.Lf[a]; half[a] = s.halff[a]; }
    }
};
template <> struct Box<double> {
    double L[3], half[3];
    __device__ __forceinline__ void load(const SysDev& s)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) { L[a] = s.L[a]; half[a] = s.half[a]; }
    }
};

// Minimum-image displacement of one component (CudaSimulation.cu:996-1002):
// the image k in {-1, 0, +1} is chosen by comparing xi - xj with half a box,
// the displacement is then formed as xi - (xj + k L).  The CPU oracle rounds
// the same sequence, which keeps the neighbour predicate bit-exact.
template <class R>
__device__ __forceinline__ R mimg(R xi, R xj, R L, R half, int per)
{
    R d = sub_rn(xi, xj);
    if (per) {
        if (d > half) d = sub_rn(xi, add_rn(xj, L));
        else if (d < -half) d = sub_rn(xi, sub_rn(xj, L));
    }
    return d;
}

// Minimum-image displacement for the RDF, symmetric in i and j: d = xi - xj,
// then d -/+ L when |d| > L/2, each step rounded once.  Swapping i and j
// negates every intermediate exactly, so both orientations of a pair get the
// same r^2 and the same bin, and a pair can be evaluated once for both.
template <class R>
__device__ __forceinline__ R mimg_sym(R xi, R xj, R L, R half, int per)
{
    const R d = sub_rn(xi, xj);
    if (per) {
        if (d > half) return sub_rn(d, L);
        if (d < -half) return add_rn(d, L);
    }
    return d;
}

// The same displacement as mimg, with the image chosen first and one
// subtraction path: xj + (-L) == xj - L exactly, and xj + 0 == xj up to the
// sign of a zero (which no force or distance sees).
template <class R>
__device__ __forceinline__ R mimg_sel(R xi, R xj, R L, R half, int per)
{
    const R d0 = sub_rn(xi, xj);
    const R s = (per && d0 > half) ? L : ((per && d0 < -half) ? -L : R(0));
    return sub_rn(xi, add_rn(xj, s));
}

// r^2 = (dx*dx + dy*dy) + dz*dz, rounded after every operation
template <class R>
__device__ __forceinline__ R dist2(R dx, R dy, R dz)
{
    return add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
}

// pair term: the force on particle i is pre * (x_j - x_i); energy e.
// P2_Harmonic.java:144-234, P2_WeakInteractionPiecewiseHarmonic.java:114-206.
template <class R>
__device__ __forceinline__ void pair_term(const PairTerm<R>& t, R r, R& pre, R& e)
{
    pre = R(0);
    e = R(0);
    if (t.kind == 1) {
        R rr = (r == R(0)) ? R(1e-6) : r;
        bool act = (t.sub == 3) || (t.sub == 2 && rr < t.r0) || (t.sub == 1 && rr > t.r0);
        if (act) {
            R dr = rr - t.r0;
            pre = t.k * dr / rr;
            e = R(0.5) * t.k * dr * dr;
        }
    } else {
        const R r0 = t.r0, l = t.l, d = t.d, q = t.q;
        if (r < r0) {
            pre = (r > R(0)) ? t.k * (r - r0) / r : R(0);
            e = t.k / R(2) * (r - r0) * (r - r0) - d;
        } else if (r < r0 + R(0.5) * l) {
            pre = d * q * (r - r0) / r;
            e = R(0.5) * d * q * (r - r0) * (r - r0) - d;
        } else if (r < r0 + l) {
            pre = -d * q * (r - r0 - l) / r;
            e = -R(0.5) * d * q * (r - r0 - l) * (r - r0 - l);
        }
    }
}

// external potential force (-grad V) and energy at box-relative x.
// P1_Disk.java:112-320, P1_Cylinder.java:109-340, P1_Sphere.java:202-340,
// P1_Cube.java:187-273.
template <class R>
__device__ __forceinline__ void ext_force(const ExtTerm<R>& p, R prad, const R x[3], R g[3], R& e)
{
    const R k = p.k;
    if (p.kind == 1 || p.kind == 2) {
        R s = (x[0] - p.c[0]) * p.nrm[0] + (x[1] - p.c[1]) * p.nrm[1] + (x[2] - p.c[2]) * p.nrm[2];
        R pp[3] = {x[0] - p.nrm[0] * s, x[1] - p.nrm[1] * s, x[2] - p.nrm[2] * s};
        R dpl = fabs(s);
        R cp0 = pp[0] - p.c[0], cp1 = pp[1] - p.c[1], cp2 = pp[2] - p.c[2];
        R din = sqrt(cp0 * cp0 + cp1 * cp1 + cp2 * cp2);
        if (p.kind == 1) {
            if (p.sub == 1) {
                if (dpl > R(0)) {
                    R pre = k;   // k (r - 0) / r
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                    e += R(0.5) * k * dpl * dpl;
                }
                R r = din + prad;
                if (r > p.rad) {
                    R pre = k * (r - p.rad) / r;
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p.c[a] - pp[a]);
                    e += R(0.5) * k * (r - p.rad) * (r - p.rad);
                }
            } else {
                R r1 = din - prad;
                if (dpl < prad && r1 < p.rad) {
                    R pre = (dpl > R(0)) ? k * (dpl - prad) / dpl : R(0);
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                    e += R(0.5) * k * (dpl - prad) * (dpl - prad);
                }
            }
        } else {
            if (p.sub == 1) {
                R r = dpl + prad, r0 = R(0.5) * p.h;
                if (r > r0) {
                    R pre = k * (r - r0) / r;
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                }
                r = din + prad;
                if (r > p.rad) {
                    R pre = k * (r - p.rad) / r;
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p.c[a] - pp[a]);
                }
                if (dpl > p.h) e += R(0.5) * k * (dpl - p.h) * (dpl - p.h);
                if (r > p.rad) e += R(0.5) * k * (r - p.rad) * (r - p.rad);
            } else {
                R r0 = prad + R(0.5) * p.h;
                R r1 = din - prad;
                if (r1 < p.rad) {
                    R pre = (r1 != R(0)) ? k * (r1 - p.rad) / r1 : R(0);
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p.c[a] - pp[a]);
                }
                if (dpl < r0) {
                    R pre = (dpl > R(0)) ? k * (dpl - r0) / dpl : R(0);
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                }
                R r0e = prad + p.h;
                if (dpl < r0e) e += R(0.5) * k * (dpl - r0e) * (dpl - r0e);
                if (r1 < p.rad) e += R(0.5) * k * (r1 - p.rad) * (r1 - p.rad);
            }
        }
    } else if (p.kind == 3) {
        R pr = p.consider ? prad : R(0);
        R d0 = x[0] - p.c[0], d1 = x[1] - p.c[1], d2 = x[2] - p.c[2];
        R d, dr;   // distance to the centre, and d - rad
        if constexpr (sizeof(R) == 4) {
            // d - rad without the cancellation of FP32 d near the shell:
            // d^2 - rad^2 from the exact products (fma residues) and the
            // two-part rad^2, divided by d + rad
            // (the _rn intrinsics keep the compiler from fusing the
            // products into the sums, which the two-sums rely on)
            const float h0 = __fmul_rn(d0, d0), h1 = __fmul_rn(d1, d1), h2 = __fmul_rn(d2, d2);
            const float l = fmaf(d0, d0, -h0) + fmaf(d1, d1, -h1) + fmaf(d2, d2, -h2);
            const float s01 = __fadd_rn(h0, h1);
            const float b01 = __fsub_rn(s01, h0);
            const float e01 = __fadd_rn(__fsub_rn(h0, __fsub_rn(s01, b01)), __fsub_rn(h1, b01));   // two-sum residue
            const float s = __fadd_rn(s01, h2);
            const float bs = __fsub_rn(s, s01);
            const float es = __fadd_rn(__fsub_rn(s01, __fsub_rn(s, bs)), __fsub_rn(h2, bs));
            d = sqrtf(s);
            const float num = __fsub_rn(s, p.rad2h) + ((e01 + es + l) - p.rad2l);
            dr = num / (d + p.rad);
        } else {
            d = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            dr = d - p.rad;
        }
        R r, rr;   // r and r - r0 of the Java potential
        bool act;
        if (p.sub == 1) { r = d + pr; rr = dr + pr; act = rr > R(0); }
        else if (p.sub == 2) { r = d; rr = dr - pr; act = rr < R(0); }
        else { r = d; rr = dr; act = rr != R(0); }
        if (act) {
            R pre = (r != R(0)) ? k * rr / r : R(0);
            g[0] += pre * (p.c[0] - x[0]);
            g[1] += pre * (p.c[1] - x[1]);
            g[2] += pre * (p.c[2] - x[2]);
            e += R(0.5) * k * rr * rr;
        }
    } else {
        R pr = p.consider ? prad : R(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            R gi = R(0);
            if (x[a] - pr >= p.blo[a] && x[a] + pr <= p.bhi[a]) {
                gi = R(0);
            } else if (x[a] - pr < p.blo[a]) {
                R r = x[a] - pr;
                gi = k * (r - p.blo[a]);
                e += R(0.5) * k * (r - p.blo[a]) * (r - p.blo[a]);
            } else {
                R r = x[a] + pr;
                gi = k * (r - p.bhi[a]);
                e += R(0.5) * k * (r - p.bhi[a]) * (r - p.bhi[a]);
            }
            g[a] += (p.sub == 1) ? -gi : gi;
        }
    }
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

}  // namespace rdgpu
