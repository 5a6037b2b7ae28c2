// Force-form Langevin thermostat of langevin_debug_intel (Source/mod_langevin.f90:15-43):
// f += -gamma m v / kcal2amu + sqrt(12 * 2 m gamma kT kcal2amu / dt) U / kcal2amu with U
// uniform in [-1/2, 1/2).  The uniforms come from Philox4x32-10 keyed by (seed, atom,
// step), so the noise is reproducible; the reference draws clock-seeded MKL uniforms.
// Shared by the MD step (md.cu) and the pair path's force unpack (mixed.cu), which
// applies it while it writes each atom's forces.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace sofia {

constexpr double KCAL2AMU = (double)0.0004184f;      // real*4 literal (get_started.f90:32)
constexpr double KBOLTZ = (double)0.001987204181f;   // real*4 variable (global.f90:133)

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter-based RNG.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
__device__ __forceinline__ double u01m(unsigned b) {  // uniform in [-1/2, 1/2)
    return (double)(b >> 8) * (1.0 / 16777216.0) - 0.5;
}

// Thermostat parameters of one step; on == 0 switches the term off.
struct LangevinArgs {
    int on;
    double gamma, gsig;  // friction (1/fs), noise amplitude
    unsigned long long seed;
    const long long *step;  // device step counter
    const double *mass, *vx, *vy, *vz;
};

// Langevin force on atom i in 64-bit fixed point (scale 2^32).
__device__ __forceinline__ void langevin_force(const LangevinArgs &a, int i, long long &fx,
                                               long long &fy, long long &fz) {
    const long long step = a.step[0];
    const uint4 r = philox(make_uint4((unsigned)i, (unsigned)step, (unsigned)(step >> 32), 0x5EED5EEDu),
                           make_uint2((unsigned)a.seed, (unsigned)(a.seed >> 32)));
    const double m = a.mass[i];
    const double g1 = -a.gamma * m / KCAL2AMU;
    const double g2 = a.gsig * sqrt(m);
    fx = __double2ll_rn((g1 * a.vx[i] + g2 * u01m(r.x)) * 4294967296.0);
    fy = __double2ll_rn((g1 * a.vy[i] + g2 * u01m(r.y)) * 4294967296.0);
    fz = __double2ll_rn((g1 * a.vz[i] + g2 * u01m(r.z)) * 4294967296.0);
}

}  // namespace sofia
