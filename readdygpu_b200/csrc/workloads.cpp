// workloads.cpp -- seeded synthetic inputs for the benchmark workloads.
#include <cmath>
#include <cstdint>
#include <vector>

#include "readdy_b200_workloads.h"

namespace {
struct SplitMix {
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
}  // namespace

extern "C" int64_t rdgpu_rsa_spheres(int64_t n, double L, double diam, uint64_t seed,
                                     int64_t max_attempts, double* xyz)
{
    int nc = (int)std::floor(L / diam);
    if (nc < 3) nc = 3 > (int)(L / diam) ? (int)(L / diam) : 3;
    if (nc < 1) nc = 1;
    const double c = L / nc;
    const int cap = 16;
    std::vector<int32_t> cnt((size_t)nc * nc * nc, 0);
    std::vector<int64_t> slot((size_t)nc * nc * nc * cap, -1);
    SplitMix rng{seed};
    const double d2 = diam * diam;
    int64_t placed = 0;
    for (int64_t att = 0; att < max_attempts && placed < n; ++att) {
        double p[3] = {rng.uniform() * L, rng.uniform() * L, rng.uniform() * L};
        int ci[3];
        for (int a = 0; a < 3; ++a) {
            int k = (int)(p[a] / c);
            ci[a] = k >= nc ? nc - 1 : k;
        }
        bool ok = true;
        for (int dz = -1; dz <= 1 && ok; ++dz)
            for (int dy = -1; dy <= 1 && ok; ++dy)
                for (int dx = -1; dx <= 1 && ok; ++dx) {
                    int x = (ci[0] + dx + nc) % nc, y = (ci[1] + dy + nc) % nc, z = (ci[2] + dz + nc) % nc;
                    size_t cell = ((size_t)z * nc + y) * nc + x;
                    for (int q = 0; q < cnt[cell]; ++q) {
                        const double* o = xyz + 3 * slot[cell * cap + q];
                        double r2 = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            double d = p[a] - o[a];
                            if (d > 0.5 * L) d -= L;
                            else if (d < -0.5 * L) d += L;
                            r2 += d * d;
                        }
                        if (r2 < d2) { ok = false; break; }
                    }
                }
        if (!ok) continue;
        size_t cell = ((size_t)ci[2] * nc + ci[1]) * nc + ci[0];
        if (cnt[cell] >= cap) continue;
        slot[cell * cap + cnt[cell]++] = placed;
        for (int a = 0; a < 3; ++a) xyz[3 * placed + a] = p[a];
        ++placed;
    }
    return placed;
}
