// md.cu -- device-resident MD step: velocity Verlet, force-form Langevin,
// SHAKE and bonded terms around the nonbonded path, so a trajectory segment
// runs without host round trips (and is captured once into a CUDA graph).
//
// Step order follows the reference's NVE loop (Source/mod_integrate.f90:270-298):
// nve_v(dt/2), nve_x, [list maintenance], forces, shake(1), nve_v(dt/2).
//   nve_v / nve_x          Source/mod_ensemble.f90:11-87
//   Langevin force          Source/mod_langevin.f90:15-43 (force form, gconst of
//                           Source/get_started.f90:81-84); the reference draws
//                           clock-seeded MT19937 uniforms, here a counter-based
//                           Philox4x32-10 keyed by (seed, atom, step)
//   SHAKE                   Source/mod_shake.f90:8-913 (shake2/3/4/3angle)
//   bond / angle            Source/mod_force_bond.f90:6-75, mod_force_angle.f90:10-122
//   torsion + 1-4 pair      Source/mod_force_dihed.f90:816-1092
// The reference's DSF driver drops the bond, angle and improper forces
// (Source/mod_force.f90:549-553); here every enabled term acts on the atoms.
// State is FP64 (positions, velocities) with 64-bit fixed-point forces; all
// force contributions are added in integers, so a step is bit-reproducible.
#include <algorithm>
#include <cmath>
#include <vector>

#include "improper.cuh"
#include "langevin.cuh"
#include "system.cuh"

namespace sofia {
namespace {


__device__ __forceinline__ long long fixd(double v) { return __double2ll_rn(v * FIX_SCALE); }
__device__ __forceinline__ double unfix(long long v) { return (double)v * FIX_INV; }

__device__ __forceinline__ void fadd(long long *f, double v) {
    atomicAdd(reinterpret_cast<unsigned long long *>(f), (unsigned long long)fixd(v));
}

// Minimum image.  d * (1/L) instead of d / L: the compiler hoists 1/L, so a
// bonded term or SHAKE group takes one FP64 division instead of one per
// component.  The two quotients differ by an ulp at most, which can change
// rint only where d is within rounding of half a box, far beyond any bonded
// distance.
__device__ __forceinline__ double mimg(double d, double L) { return d - L * rint(d * (1.0 / L)); }


// nve_v: v += (dt/2) * kcal2amu * f / m
__device__ __forceinline__ void kick_body(int bx, int n, double h, const double *__restrict__ invm,
                       const long long *__restrict__ fx, const long long *__restrict__ fy,
                       const long long *__restrict__ fz, double *__restrict__ vx,
                       double *__restrict__ vy, double *__restrict__ vz) {
    const int i = bx * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double c = h * invm[i];
    vx[i] += c * unfix(fx[i]);
    vy[i] += c * unfix(fy[i]);
    vz[i] += c * unfix(fz[i]);
}
__global__ void k_kick(int n, double h, const double *__restrict__ invm,
                       const long long *__restrict__ fx, const long long *__restrict__ fy,
                       const long long *__restrict__ fz, double *__restrict__ vx,
                       double *__restrict__ vy, double *__restrict__ vz) {
    SOFIA_PDL_ENTRY();
    kick_body(blockIdx.x, n, h, invm, fx, fy, fz, vx, vy, vz);
}

// First half-kick and drift of a step fused with the step counter and the
// list triggers: v += h f / m (nve_v), x += dt v (nve_x), then bit 0 of the
// trigger word if an atom moved more than skin/2 since the list build, bit 1
// if more than margin/2 since the last prune (the word was cleared after the
// previous step's list decisions).  TWICE: the previous step's closing
// half-kick first, as its own rounded addition (v += h f / m twice with the same
// forces), so a segment that skips the separate closing kick gives the same bits.
template <bool TWICE = false>
__device__ __forceinline__ void kick_drift_body(int bx, int n, double h, const double *__restrict__ invm,
                             const long long *__restrict__ fx, const long long *__restrict__ fy,
                             const long long *__restrict__ fz, double *__restrict__ vx,
                             double *__restrict__ vy, double *__restrict__ vz, double dt,
                             double *__restrict__ x, double *__restrict__ y,
                             double *__restrict__ z, const double *__restrict__ rx,
                             const double *__restrict__ ry, const double *__restrict__ rz,
                             const double *__restrict__ px, const double *__restrict__ py,
                             const double *__restrict__ pz, double L, double lim2, double plim2,
                             int *__restrict__ flag, long long *__restrict__ step) {
    const int i = bx * blockDim.x + threadIdx.x;
    if (i == 0) step[0] += 1;
    bool far = false, pfar = false;
    if (i < n) {
        const double c = h * invm[i];
        double ux = vx[i], uy = vy[i], uz = vz[i];
        const double gx = c * unfix(fx[i]), gy = c * unfix(fy[i]), gz = c * unfix(fz[i]);
        if (TWICE) {
            ux = ux + gx;
            uy = uy + gy;
            uz = uz + gz;
        }
        ux = ux + gx;
        uy = uy + gy;
        uz = uz + gz;
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        const double xn = x[i] + dt * ux, yn = y[i] + dt * uy, zn = z[i] + dt * uz;
        x[i] = xn;
        y[i] = yn;
        z[i] = zn;
        far = disp2(xn, yn, zn, rx[i], ry[i], rz[i], L) > lim2;
        pfar = disp2(xn, yn, zn, px[i], py[i], pz[i], L) > plim2;
    }
    const bool a = __any_sync(0xffffffffu, far), b = __any_sync(0xffffffffu, pfar);
    if ((threadIdx.x & 31) == 0 && (a || b)) atomicOr(flag, (a ? 1 : 0) | (b ? 2 : 0));
}
template <bool TWICE>
__global__ void k_kick_drift(int n, double h, const double *__restrict__ invm,
                             const long long *__restrict__ fx, const long long *__restrict__ fy,
                             const long long *__restrict__ fz, double *__restrict__ vx,
                             double *__restrict__ vy, double *__restrict__ vz, double dt,
                             double *__restrict__ x, double *__restrict__ y,
                             double *__restrict__ z, const double *__restrict__ rx,
                             const double *__restrict__ ry, const double *__restrict__ rz,
                             const double *__restrict__ px, const double *__restrict__ py,
                             const double *__restrict__ pz, double L, double lim2, double plim2,
                             int *__restrict__ flag, long long *__restrict__ step) {
    SOFIA_PDL_ENTRY();
    kick_drift_body<TWICE>(blockIdx.x, n, h, invm, fx, fy, fz, vx, vy, vz, dt, x, y, z, rx, ry, rz, px, py, pz, L, lim2, plim2, flag, step);
}



template <bool EN>
__device__ __forceinline__ void bond_term(int m, int nb, const int *__restrict__ bl, const double *__restrict__ bc,
                       const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, double L, long long *__restrict__ fx,
                       long long *__restrict__ fy, long long *__restrict__ fz,
                       double *__restrict__ e) {
    if (m >= nb) return;
    const int i1 = bl[3 * m] - 1, i2 = bl[3 * m + 1] - 1, t = bl[3 * m + 2] - 1;
    const double dx = mimg(x[i1] - x[i2], L), dy = mimg(y[i1] - y[i2], L), dz = mimg(z[i1] - z[i2], L);
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double dr = r - bc[2 * t + 1];
    const double rk = bc[2 * t] * dr;
    const double force = (r > 0.0) ? -2.0 * rk / r : 0.0;
    fadd(&fx[i1], dx * force);
    fadd(&fy[i1], dy * force);
    fadd(&fz[i1], dz * force);
    fadd(&fx[i2], -dx * force);
    fadd(&fy[i2], -dy * force);
    fadd(&fz[i2], -dz * force);
    if (EN) e[m] = rk * dr;
}

template <bool EN>
__device__ __forceinline__ void angle_term(int m, int na, const int *__restrict__ al, const double *__restrict__ ac,
                        const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, double L, long long *__restrict__ fx,
                        long long *__restrict__ fy, long long *__restrict__ fz,
                        double *__restrict__ e) {
    if (m >= na) return;
    const int i1 = al[4 * m] - 1, i2 = al[4 * m + 1] - 1, i3 = al[4 * m + 2] - 1,
              t = al[4 * m + 3] - 1;
    const double dx1 = mimg(x[i1] - x[i2], L), dy1 = mimg(y[i1] - y[i2], L),
                 dz1 = mimg(z[i1] - z[i2], L);
    const double dx2 = mimg(x[i3] - x[i2], L), dy2 = mimg(y[i3] - y[i2], L),
                 dz2 = mimg(z[i3] - z[i2], L);
    const double rsq1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1, r1 = sqrt(rsq1);
    const double rsq2 = dx2 * dx2 + dy2 * dy2 + dz2 * dz2, r2 = sqrt(rsq2);
    double c = (dx1 * dx2 + dy1 * dy2 + dz1 * dz2) / (r1 * r2);
    c = fmin(1.0, fmax(-1.0, c));
    double s = sqrt(1.0 - c * c);
    if (s < 0.001) s = 0.001;
    s = 1.0 / s;
    const double dtheta = acos(c) - ac[2 * t + 1];
    const double tk = ac[2 * t] * dtheta;
    const double a = 2.0 * tk * s;
    const double a11 = a * c / rsq1, a12 = -a / (r1 * r2), a22 = a * c / rsq2;
    const double vx1 = a11 * dx1 + a12 * dx2, vx2 = a22 * dx2 + a12 * dx1;
    const double vy1 = a11 * dy1 + a12 * dy2, vy2 = a22 * dy2 + a12 * dy1;
    const double vz1 = a11 * dz1 + a12 * dz2, vz2 = a22 * dz2 + a12 * dz1;
    fadd(&fx[i1], -vx1);
    fadd(&fy[i1], -vy1);
    fadd(&fz[i1], -vz1);
    fadd(&fx[i2], vx2 + vx1);
    fadd(&fy[i2], vy2 + vy1);
    fadd(&fz[i2], vz2 + vz1);
    fadd(&fx[i3], -vx2);
    fadd(&fy[i3], -vy2);
    fadd(&fz[i3], -vz2);
    if (EN) e[m] = tk * dtheta;
}

// improper_harmonic_lammps14 (mod_force_dihed.f90:1546-1724) on the FP64 state.
template <bool EN>
__device__ __forceinline__ void improper_term(int m, int ni, const int *__restrict__ il, const double *__restrict__ ic,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, double L, long long *__restrict__ fx,
                           long long *__restrict__ fy, long long *__restrict__ fz,
                           double *__restrict__ e) {
    if (m >= ni) return;
    const int i1 = il[5 * m] - 1, i2 = il[5 * m + 1] - 1, i3 = il[5 * m + 2] - 1,
              i4 = il[5 * m + 3] - 1, t = il[5 * m + 4] - 1;
    const double v1[3] = {mimg(x[i1] - x[i2], L), mimg(y[i1] - y[i2], L), mimg(z[i1] - z[i2], L)};
    const double v2[3] = {mimg(x[i3] - x[i2], L), mimg(y[i3] - y[i2], L), mimg(z[i3] - z[i2], L)};
    const double v3[3] = {mimg(x[i4] - x[i3], L), mimg(y[i4] - y[i3], L), mimg(z[i4] - z[i3], L)};
    const ImproperOut r = improper_harmonic(v1, v2, v3, ic[2 * t], ic[2 * t + 1]);
    long long *f[3] = {fx, fy, fz};
    for (int d = 0; d < 3; ++d) {
        fadd(&f[d][i1], r.f1[d]);
        fadd(&f[d][i2], r.f2[d]);
        fadd(&f[d][i3], r.f3[d]);
        fadd(&f[d][i4], r.f4[d]);
    }
    if (EN) e[m] = r.e;
}


// dihedral_opls_DSF (mod_force_dihed.f90:849-1068) on the FP64 state.
template <bool EN>
__device__ __forceinline__ void dihedral_term(int n, const DihArgs &a) {
    if (n >= a.nd) return;
    const int i1 = a.dl[5 * n] - 1, i2 = a.dl[5 * n + 1] - 1, i3 = a.dl[5 * n + 2] - 1,
              i4 = a.dl[5 * n + 3] - 1, type = a.dl[5 * n + 4] - 1;
    const double *x = a.x, *y = a.y, *z = a.z;
    const double L = a.L;
    const double vb1x = mimg(x[i1] - x[i2], L), vb1y = mimg(y[i1] - y[i2], L), vb1z = mimg(z[i1] - z[i2], L);
    const double vb2x = mimg(x[i3] - x[i2], L), vb2y = mimg(y[i3] - y[i2], L), vb2z = mimg(z[i3] - z[i2], L);
    const double vb2xm = -vb2x, vb2ym = -vb2y, vb2zm = -vb2z;
    const double vb3x = mimg(x[i4] - x[i3], L), vb3y = mimg(y[i4] - y[i3], L), vb3z = mimg(z[i4] - z[i3], L);
    double f1[3] = {0, 0, 0}, f2[3] = {0, 0, 0}, f3[3] = {0, 0, 0}, f4[3] = {0, 0, 0};
    double pp = 0.0;
    if (a.terms & 4) {
        const double sb1 = 1.0 / (vb1x * vb1x + vb1y * vb1y + vb1z * vb1z);
        const double sb2 = 1.0 / (vb2x * vb2x + vb2y * vb2y + vb2z * vb2z);
        const double sb3 = 1.0 / (vb3x * vb3x + vb3y * vb3y + vb3z * vb3z);
        const double rb1 = sqrt(sb1), rb3 = sqrt(sb3);
        const double c0 = (vb1x * vb3x + vb1y * vb3y + vb1z * vb3z) * rb1 * rb3;
        const double b1mag = sqrt(vb1x * vb1x + vb1y * vb1y + vb1z * vb1z);
        const double b2mag = sqrt(vb2x * vb2x + vb2y * vb2y + vb2z * vb2z);
        const double b3mag = sqrt(vb3x * vb3x + vb3y * vb3y + vb3z * vb3z);
        const double r12c1 = 1.0 / (b1mag * b2mag);
        const double c1mag = (vb1x * vb2x + vb1y * vb2y + vb1z * vb2z) * r12c1;
        const double r12c2 = 1.0 / (b2mag * b3mag);
        const double c2mag = (vb2xm * vb3x + vb2ym * vb3y + vb2zm * vb3z) * r12c2;
        double sc1 = sqrt(fmax(1.0 - c1mag * c1mag, 0.0));
        if (sc1 < 0.001) sc1 = 0.001;
        sc1 = 1.0 / sc1;
        double sc2 = sqrt(fmax(1.0 - c2mag * c2mag, 0.0));
        if (sc2 < 0.001) sc2 = 0.001;
        sc2 = 1.0 / sc2;
        const double s1 = sc1 * sc1, s2 = sc2 * sc2;
        double s12 = sc1 * sc2;
        double c = (c0 + c1mag * c2mag) * s12;
        c = fmin(1.0, fmax(-1.0, c));
        const double phi = acos(c);
        double si = sin(phi);
        if (fabs(si) < 0.0001) si = 0.0001;
        const double siinv = 1.0 / si;
        const double *kc = a.dc + 4 * type;
        pp = kc[0] * (1.0 + c) + kc[1] * (1.0 - cos(2.0 * phi)) + kc[2] * (1.0 + cos(3.0 * phi)) +
             kc[3] * (1.0 - cos(4.0 * phi));
        const double pd = kc[0] - 2.0 * kc[1] * sin(2.0 * phi) * siinv +
                          3.0 * kc[2] * sin(3.0 * phi) * siinv - 4.0 * kc[3] * sin(4.0 * phi) * siinv;
        c *= pd;
        s12 *= pd;
        const double a11 = c * sb1 * s1, a22 = -sb2 * (2.0 * c0 * s12 - c * (s1 + s2)),
                     a33 = c * sb3 * s2;
        const double a12 = -r12c1 * (c1mag * c * s1 + c2mag * s12), a13 = -rb1 * rb3 * s12,
                     a23 = r12c2 * (c2mag * c * s2 + c1mag * s12);
        const double sx2 = a12 * vb1x + a22 * vb2x + a23 * vb3x;
        const double sy2 = a12 * vb1y + a22 * vb2y + a23 * vb3y;
        const double sz2 = a12 * vb1z + a22 * vb2z + a23 * vb3z;
        f1[0] = a11 * vb1x + a12 * vb2x + a13 * vb3x;
        f1[1] = a11 * vb1y + a12 * vb2y + a13 * vb3y;
        f1[2] = a11 * vb1z + a12 * vb2z + a13 * vb3z;
        f2[0] = -sx2 - f1[0];
        f2[1] = -sy2 - f1[1];
        f2[2] = -sz2 - f1[2];
        f4[0] = a13 * vb1x + a23 * vb2x + a33 * vb3x;
        f4[1] = a13 * vb1y + a23 * vb2y + a33 * vb3y;
        f4[2] = a13 * vb1z + a23 * vb2z + a33 * vb3z;
        f3[0] = sx2 - f4[0];
        f3[1] = sy2 - f4[1];
        f3[2] = sz2 - f4[2];
    }
    double ec14 = 0.0, p14 = 0.0;
    if (a.terms & 8) {
        const double ddx = mimg(x[i1] - x[i4], L), ddy = mimg(y[i1] - y[i4], L),
                     ddz = mimg(z[i1] - z[i4], L);
        const double dr2 = ddx * ddx + ddy * ddy + ddz * ddz;
        double force = 0.0;
        if (dr2 < a.cut_coulsq) {
            const double r = sqrt(dr2), dr2i = 1.0 / dr2;
            // coulpre*q(i1)*q(i4) is a real*4 product in the reference
            // (mod_force_dihed.f90:1010), promoted by the division by r
            const double pref = (double)__fmul_rn(__fmul_rn(a.coulpre, a.q[i1]), a.q[i4]) / r;
            const double erfcd = exp(-a.alpha * a.alpha * dr2);
            const double t = 1.0 / (1.0 + a.EWALD_P * a.alpha * r);
            const double erfcc = t * (a.A1 + t * (a.A2 + t * (a.A3 + t * (a.A4 + t * a.A5)))) * erfcd;
            const double fc = 0.5 * pref * (erfcc / r + 2.0 * a.alpha / a.MY_PIS * erfcd + r * a.f_shift) * r;
            ec14 = 0.5 * pref * (erfcc - r * a.e_shift - dr2 * a.f_shift);
            double flj = 0.0;
            if (dr2 < a.rcut2) {
                const double dr6i = dr2i * dr2i * dr2i;
                const size_t o = (size_t)(a.type[i1] - 1) * a.ntypes + (size_t)(a.type[i4] - 1);
                const size_t tn = (size_t)a.ntypes * a.ntypes;
                flj = dr6i * (a.lj14[o] * dr6i - a.lj14[tn + o]);
                p14 = dr6i * (dr6i * a.lj14[2 * tn + o] - a.lj14[3 * tn + o]);
            }
            force = (fc + flj) * dr2i;
        }
        f1[0] += ddx * force;
        f1[1] += ddy * force;
        f1[2] += ddz * force;
        f4[0] -= ddx * force;
        f4[1] -= ddy * force;
        f4[2] -= ddz * force;
    }
    long long *F[3] = {a.fx, a.fy, a.fz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fadd(&F[d][i1], f1[d]);
        fadd(&F[d][i2], f2[d]);
        fadd(&F[d][i3], f3[d]);
        fadd(&F[d][i4], f4[d]);
    }
    if (EN) {
        a.e[3 * n] = pp;
        a.e[3 * n + 1] = ec14;
        a.e[3 * n + 2] = p14;
    }
}

// SHAKE (force form) per group; each atom belongs to at most one group, so the
// owning thread adds its constraint forces without atomics.
// Constraint c of a SHAKE group of type NUM joins group atoms shake_cp and
// shake_cq: NUM 1 = one bond (atoms 0-1), 3 = two bonds from atom 0, 4 = three
// bonds from atom 0, -3 = a rigid triangle (0-1, 0-2, 1-2; mod_shake.f90).
__host__ __device__ constexpr int shake_nc(int num) { return num == 1 ? 1 : (num == 3 ? 2 : 3); }
__host__ __device__ constexpr int shake_na(int num) { return num == 1 ? 2 : (num == 4 ? 4 : 3); }
__host__ __device__ constexpr int shake_cp(int num, int c) { return (num == -3 && c == 2) ? 1 : 0; }
__host__ __device__ constexpr int shake_cq(int num, int c) { return (num == -3 && c == 2) ? 2 : c + 1; }

// One SHAKE group of type NUM: the group's size and constraint pairs are
// compile-time constants, so every loop unrolls and the small matrices live in
// registers.  The operations and their order are those of the general solver.
template <int NUM>
__device__ __forceinline__ void shake_group(int g, const int (&at)[4], const double *__restrict__ sb,
                        const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const double *__restrict__ vx,
                        const double *__restrict__ vy, const double *__restrict__ vz,
                        const double *__restrict__ invm, double L, double dt, double dtsq,
                        int maxiter, double tol, long long *__restrict__ fx,
                        long long *__restrict__ fy, long long *__restrict__ fz,
                        int *__restrict__ status) {
    constexpr int nc = shake_nc(NUM), na = shake_na(NUM);
    constexpr int cp[3] = {shake_cp(NUM, 0), shake_cp(NUM, 1), shake_cp(NUM, 2)};
    constexpr int cq[3] = {shake_cq(NUM, 0), shake_cq(NUM, 1), shake_cq(NUM, 2)};
    double bl[3];
#pragma unroll
    for (int k = 0; k < nc; ++k) bl[k] = sb[3 * g + k];
    double im[4], xs[4][3], xc[4][3];
#pragma unroll
    for (int a = 0; a < na; ++a) {
        const int i = at[a];
        im[a] = invm[i];
        const double c = dtsq * im[a];
        xc[a][0] = x[i];
        xc[a][1] = y[i];
        xc[a][2] = z[i];
        xs[a][0] = x[i] + dt * vx[i] + c * unfix(fx[i]);
        xs[a][1] = y[i] + dt * vy[i] + c * unfix(fy[i]);
        xs[a][2] = z[i] + dt * vz[i] + c * unfix(fz[i]);
    }
    double r[3][3], s[3][3], C[3][3];
#pragma unroll
    for (int c = 0; c < nc; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            r[c][d] = mimg(xc[cp[c]][d] - xc[cq[c]][d], L);
            s[c][d] = mimg(xs[cp[c]][d] - xs[cq[c]][d], L);
        }
#pragma unroll
    for (int c = 0; c < nc; ++c)
#pragma unroll
        for (int d = 0; d < nc; ++d) {
            double e = 0.0;
            if (cp[c] == cp[d]) e += im[cp[c]];
            if (cp[c] == cq[d]) e -= im[cp[c]];
            if (cq[c] == cp[d]) e -= im[cq[c]];
            if (cq[c] == cq[d]) e += im[cq[c]];
            C[c][d] = e;
        }
    double lam[3] = {0.0, 0.0, 0.0};
    if constexpr (nc == 1) {
        const double rr = r[0][0] * r[0][0] + r[0][1] * r[0][1] + r[0][2] * r[0][2];
        const double ss = s[0][0] * s[0][0] + s[0][1] * s[0][1] + s[0][2] * s[0][2];
        const double sr = s[0][0] * r[0][0] + s[0][1] * r[0][1] + s[0][2] * r[0][2];
        const double aa = C[0][0] * C[0][0] * rr, bb = 2.0 * C[0][0] * sr, cc = ss - bl[0] * bl[0];
        double det = bb * bb - 4.0 * aa * cc;
        if (det < 0.0) {
            atomicAdd(&status[ST_SHAKE], 1);
            det = 0.0;
        }
        const double l1 = (-bb + sqrt(det)) / (2.0 * aa), l2 = (-bb - sqrt(det)) / (2.0 * aa);
        lam[0] = (fabs(l1) <= fabs(l2)) ? l1 : l2;
    } else {
        double A[3][3], Ai[3][3], ss[3], rd[3][3];
#pragma unroll
        for (int c = 0; c < nc; ++c) {
            ss[c] = s[c][0] * s[c][0] + s[c][1] * s[c][1] + s[c][2] * s[c][2];
#pragma unroll
            for (int d = 0; d < nc; ++d) {
                A[c][d] = 2.0 * C[c][d] * (s[c][0] * r[d][0] + s[c][1] * r[d][1] + s[c][2] * r[d][2]);
                rd[c][d] = r[c][0] * r[d][0] + r[c][1] * r[d][1] + r[c][2] * r[d][2];
            }
        }
        if constexpr (nc == 2) {
            const double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
            if (det == 0.0) {
                atomicAdd(&status[ST_SHAKE], 1);
                return;
            }
            const double di = 1.0 / det;
            Ai[0][0] = A[1][1] * di; Ai[0][1] = -A[0][1] * di;
            Ai[1][0] = -A[1][0] * di; Ai[1][1] = A[0][0] * di;
        } else {
            const double det = A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
                               A[0][2] * A[1][0] * A[2][1] - A[0][0] * A[1][2] * A[2][1] -
                               A[0][1] * A[1][0] * A[2][2] - A[0][2] * A[1][1] * A[2][0];
            if (det == 0.0) {
                atomicAdd(&status[ST_SHAKE], 1);
                return;
            }
            const double di = 1.0 / det;
            Ai[0][0] = di * (A[1][1] * A[2][2] - A[1][2] * A[2][1]);
            Ai[0][1] = -di * (A[0][1] * A[2][2] - A[0][2] * A[2][1]);
            Ai[0][2] = di * (A[0][1] * A[1][2] - A[0][2] * A[1][1]);
            Ai[1][0] = -di * (A[1][0] * A[2][2] - A[1][2] * A[2][0]);
            Ai[1][1] = di * (A[0][0] * A[2][2] - A[0][2] * A[2][0]);
            Ai[1][2] = -di * (A[0][0] * A[1][2] - A[0][2] * A[1][0]);
            Ai[2][0] = di * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
            Ai[2][1] = -di * (A[0][0] * A[2][1] - A[0][1] * A[2][0]);
            Ai[2][2] = di * (A[0][0] * A[1][1] - A[0][1] * A[1][0]);
        }
        bool done = false;
        for (int it = 0; it < maxiter && !done; ++it) {
            double bvec[3], ln[3];
#pragma unroll
            for (int c = 0; c < nc; ++c) {
                double qd = 0.0;
#pragma unroll
                for (int d = 0; d < nc; ++d)
#pragma unroll
                    for (int e = 0; e < nc; ++e) qd += C[c][d] * C[c][e] * rd[d][e] * lam[d] * lam[e];
                bvec[c] = bl[c] * bl[c] - ss[c] - qd;
            }
            done = true;
#pragma unroll
            for (int c = 0; c < nc; ++c) {
                ln[c] = 0.0;
#pragma unroll
                for (int d = 0; d < nc; ++d) ln[c] += Ai[c][d] * bvec[d];
                if (fabs(ln[c] - lam[c]) > tol) done = false;
            }
#pragma unroll
            for (int c = 0; c < nc; ++c) lam[c] = ln[c];
        }
        if (!done) atomicAdd(&status[ST_SHAKE_NC], 1);  // warning only (mod_shake.f90:322-324)
    }
    long long *F[3] = {fx, fy, fz};
#pragma unroll
    for (int c = 0; c < nc; ++c) {
        const double l = lam[c] / dtsq;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            F[d][at[cp[c]]] += fixd(l * r[c][d]);
            F[d][at[cq[c]]] -= fixd(l * r[c][d]);
        }
    }
}

__device__ __forceinline__ void shake_body(int bx, int ns, const int *__restrict__ sa, const double *__restrict__ sb,
                        const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const double *__restrict__ vx,
                        const double *__restrict__ vy, const double *__restrict__ vz,
                        const double *__restrict__ invm, double L, double dt, double dtsq,
                        int maxiter, double tol, long long *__restrict__ fx,
                        long long *__restrict__ fy, long long *__restrict__ fz,
                        int *__restrict__ status) {
    const int g = bx * blockDim.x + threadIdx.x;
    if (g >= ns) return;
    const int num = sa[5 * g];
    const int at[4] = {sa[5 * g + 1] - 1, sa[5 * g + 2] - 1, sa[5 * g + 3] - 1, sa[5 * g + 4] - 1};
#define SOFIA_SHAKE_ARGS g, at, sb, x, y, z, vx, vy, vz, invm, L, dt, dtsq, maxiter, tol, fx, fy, fz, status
    switch (num) {
    case 1: shake_group<1>(SOFIA_SHAKE_ARGS); break;
    case 3: shake_group<3>(SOFIA_SHAKE_ARGS); break;
    case 4: shake_group<4>(SOFIA_SHAKE_ARGS); break;
    case -3: shake_group<-3>(SOFIA_SHAKE_ARGS); break;
    default: break;
    }
#undef SOFIA_SHAKE_ARGS
}
__global__ void k_shake(int ns, const int *__restrict__ sa, const double *__restrict__ sb,
                        const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const double *__restrict__ vx,
                        const double *__restrict__ vy, const double *__restrict__ vz,
                        const double *__restrict__ invm, double L, double dt, double dtsq,
                        int maxiter, double tol, long long *__restrict__ fx,
                        long long *__restrict__ fy, long long *__restrict__ fz,
                        int *__restrict__ status) {
    SOFIA_PDL_ENTRY();
    shake_body(blockIdx.x, ns, sa, sb, x, y, z, vx, vy, vz, invm, L, dt, dtsq, maxiter, tol, fx, fy, fz, status);
}

// RATTLE velocity stage (Andersen, J. Comput. Phys. 52 (1983) 24; the scheme of
// LAMMPS fix rattle) after the second half-kick: the full-step velocities of
// each constraint group are projected so that every constrained distance has
// zero time derivative, (v_p - v_q) . r_pq = 0, solving C_cd (r_c . r_d) mu_d =
// -(v_p - v_q) . r_c for the impulses mu (C as in k_shake, nc <= 3, Cramer's
// rule).  The positions of SHAKE and RATTLE are the same sequence, so the
// impulse m dv is taken back out of the force the next step's first half-kick
// applies (f -= m dv / h): the next half-step velocity, and with it every later
// position, is what the plain SHAKE step gives; only the full-step velocities
// (and the kinetic energy measured from them) change.
__device__ __forceinline__ void rattle_body(int bx, int ns, const int *__restrict__ sa, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ z,
                         double *__restrict__ vx, double *__restrict__ vy,
                         double *__restrict__ vz, const double *__restrict__ invm, double L,
                         double h, long long *__restrict__ fx, long long *__restrict__ fy,
                         long long *__restrict__ fz) {
    const int g = bx * blockDim.x + threadIdx.x;
    if (g >= ns) return;
    const int num = sa[5 * g];
    const int at[4] = {sa[5 * g + 1] - 1, sa[5 * g + 2] - 1, sa[5 * g + 3] - 1,
                       sa[5 * g + 4] - 1};
    int nc, na, cp[3], cq[3];
    if (num == 1) {
        nc = 1; na = 2; cp[0] = 0; cq[0] = 1;
    } else if (num == 3) {
        nc = 2; na = 3; cp[0] = 0; cq[0] = 1; cp[1] = 0; cq[1] = 2;
    } else if (num == 4) {
        nc = 3; na = 4;
        for (int k = 0; k < 3; ++k) { cp[k] = 0; cq[k] = k + 1; }
    } else if (num == -3) {
        nc = 3; na = 3; cp[0] = 0; cq[0] = 1; cp[1] = 0; cq[1] = 2; cp[2] = 1; cq[2] = 2;
    } else {
        return;
    }
    double im[4], xv[4][3], vv[4][3];
    for (int a = 0; a < na; ++a) {
        const int i = at[a];
        im[a] = invm[i];
        xv[a][0] = x[i]; xv[a][1] = y[i]; xv[a][2] = z[i];
        vv[a][0] = vx[i]; vv[a][1] = vy[i]; vv[a][2] = vz[i];
    }
    double r[3][3], M[3][3], rhs[3];
    for (int c = 0; c < nc; ++c) {
        double gdot = 0.0;
        for (int d = 0; d < 3; ++d) {
            r[c][d] = mimg(xv[cp[c]][d] - xv[cq[c]][d], L);
            gdot += (vv[cp[c]][d] - vv[cq[c]][d]) * r[c][d];
        }
        rhs[c] = -gdot;
    }
    for (int c = 0; c < nc; ++c)
        for (int d = 0; d < nc; ++d) {
            double e = 0.0;
            if (cp[c] == cp[d]) e += im[cp[c]];
            if (cp[c] == cq[d]) e -= im[cp[c]];
            if (cq[c] == cp[d]) e -= im[cq[c]];
            if (cq[c] == cq[d]) e += im[cq[c]];
            M[c][d] = e * (r[c][0] * r[d][0] + r[c][1] * r[d][1] + r[c][2] * r[d][2]);
        }
    double mu[3] = {0.0, 0.0, 0.0};
    if (nc == 1) {
        if (M[0][0] == 0.0) return;
        mu[0] = rhs[0] / M[0][0];
    } else if (nc == 2) {
        const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        if (det == 0.0) return;
        mu[0] = (rhs[0] * M[1][1] - M[0][1] * rhs[1]) / det;
        mu[1] = (M[0][0] * rhs[1] - rhs[0] * M[1][0]) / det;
    } else {
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        if (det == 0.0) return;
        for (int c = 0; c < 3; ++c) {
            double A[3][3];
            for (int u = 0; u < 3; ++u)
                for (int w = 0; w < 3; ++w) A[u][w] = (w == c) ? rhs[u] : M[u][w];
            mu[c] = (A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0])) / det;
        }
    }
    double dv[4][3] = {};
    for (int c = 0; c < nc; ++c)
        for (int d = 0; d < 3; ++d) {
            dv[cp[c]][d] += mu[c] * im[cp[c]] * r[c][d];
            dv[cq[c]][d] -= mu[c] * im[cq[c]] * r[c][d];
        }
    double *V[3] = {vx, vy, vz};
    long long *F[3] = {fx, fy, fz};
    for (int a = 0; a < na; ++a) {
        const double mh = 1.0 / (im[a] * h);
        for (int d = 0; d < 3; ++d) {
            V[d][at[a]] = vv[a][d] + dv[a][d];
            F[d][at[a]] -= fixd(dv[a][d] * mh);
        }
    }
}
__global__ void k_rattle(int ns, const int *__restrict__ sa, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ z,
                         double *__restrict__ vx, double *__restrict__ vy,
                         double *__restrict__ vz, const double *__restrict__ invm, double L,
                         double h, long long *__restrict__ fx, long long *__restrict__ fy,
                         long long *__restrict__ fz) {
    SOFIA_PDL_ENTRY();
    rattle_body(blockIdx.x, ns, sa, x, y, z, vx, vy, vz, invm, L, h, fx, fy, fz);
}

// Langevin force alone (friction + noise of the current step counter) as the
// whole force: the forces-only query's way to the thermostat term.
__global__ void k_langevin_only(int n, LangevinArgs lg, long long *__restrict__ fx,
                                long long *__restrict__ fy, long long *__restrict__ fz) {
    SOFIA_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long a, b, c;
    langevin_force(lg, i, a, b, c);
    fx[i] = a;
    fy[i] = b;
    fz[i] = c;
}

__device__ __forceinline__ void ke_body(int bx, int n, const double *__restrict__ mass, const double *__restrict__ vx,
                     const double *__restrict__ vy, const double *__restrict__ vz,
                     double *__restrict__ ke) {
    const int i = bx * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ke[i] = 0.5 * mass[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]) / KCAL2AMU;
}
__global__ void k_ke(int n, const double *__restrict__ mass, const double *__restrict__ vx,
                     const double *__restrict__ vy, const double *__restrict__ vz,
                     double *__restrict__ ke) {
    SOFIA_PDL_ENTRY();
    ke_body(blockIdx.x, n, mass, vx, vy, vz, ke);
}


// Two-stage deterministic sum of column c of in[n][w] into out[slot].
constexpr int MRED = 64;
__device__ __forceinline__ void mred1_body(int bx, int n, int w, int c, const double *__restrict__ in,
                        double *__restrict__ part, int nblk) {
    __shared__ double s[256];
    const int chunk = (n + nblk - 1) / nblk;
    const int b0 = bx * chunk, b1 = min(n, b0 + chunk);
    double acc = 0.0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += in[(size_t)i * w + c];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[bx] = s[0];
}
__global__ void k_mred1(int n, int w, int c, const double *__restrict__ in,
                        double *__restrict__ part) {
    SOFIA_PDL_ENTRY();
    mred1_body(blockIdx.x, n, w, c, in, part, (int)gridDim.x);
}
__device__ __forceinline__ void mred2_body(int bx, const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double s[MRED];
    s[threadIdx.x] = part[threadIdx.x];
    __syncthreads();
    for (int off = MRED / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0];
}
__global__ void k_mred2(const double *__restrict__ part, double *__restrict__ out) {
    SOFIA_PDL_ENTRY();
    mred2_body(blockIdx.x, part, out);
}

}  // namespace

static void md_reduce(cudaStream_t st, int n, int w, int c, const double *in, double *part,
                      double *out) {
    if (n <= 0) return;
    sofia::launch_pdl(k_mred1, MRED, 256, 0, st, n, w, c, in, part);
    sofia::launch_pdl(k_mred2, 1, MRED, 0, st, part, out);
}

// energies slots in md.ered: 0 lj, 1 coul, (2..4 pair virial), 5 bond, 6 angle,
// 7 torsion, 8 coul14, 9 lj14, 10 kinetic; partials after slot 16.
// All bonded terms of a step in one launch: threads [0, nb) take bonds, the
// next na angles, then nd dihedrals (torsion and 1-4 pair), then ni impropers.
// A count of 0 switches a term off.
template <bool EN>
// Threads take the torsions (the longest terms) first, then impropers, angles
// and bonds, so the last wave of blocks holds the short terms.  Every term
// adds fixed-point forces and writes its energy to its own slot, so the order
// does not change any result.
__device__ __forceinline__ void bonded_body(int bx, const BondedArgs &b) {
    int t = bx * blockDim.x + threadIdx.x;
    const DihArgs &d = b.dih;
    if (t < b.nd) {
        dihedral_term<EN>(t, d);
        return;
    }
    t -= b.nd;
    if (t < b.ni) {
        improper_term<EN>(t, b.ni, b.il, b.ic, d.x, d.y, d.z, d.L, d.fx, d.fy, d.fz, b.ei);
        return;
    }
    t -= b.ni;
    if (t < b.na) {
        angle_term<EN>(t, b.na, b.al, b.ac, d.x, d.y, d.z, d.L, d.fx, d.fy, d.fz, b.ea);
        return;
    }
    t -= b.na;
    if (t < b.nb) bond_term<EN>(t, b.nb, b.bl, b.bc, d.x, d.y, d.z, d.L, d.fx, d.fy, d.fz, b.eb);
}
// 6 resident blocks of 128 per SM (at most 85 registers): the kernel's time is
// a few waves of latency-bound torsion threads, and more resident blocks per SM
// shorten it more than the few spills cost (MD 433 -> 436.5 M atom-steps/s at
// 275k atoms; 8 blocks measured the same)
#ifndef SOFIA_BONDED_MINB
#define SOFIA_BONDED_MINB 6
#endif
template <bool EN>
__global__ void __launch_bounds__(128, SOFIA_BONDED_MINB) k_bonded(BondedArgs b) {
    SOFIA_PDL_ENTRY();
    bonded_body<EN>(blockIdx.x, b);
}

// Arguments of the torsion / 1-4 term (everything but the dihedral count).
static void md_dih_args(Sys *s, double *et, DihArgs *ap) {
    Md &md = s->md;
    DihArgs &a = *ap;
    a.ntypes = s->ntypes;
    a.terms = md.terms;
    a.dl = md.diheds.as<int>();
    a.dc = md.dcoef.as<double>();
    a.lj14 = md.lj14.as<double>();
    a.x = s->x[0].as<double>();
    a.y = s->x[1].as<double>();
    a.z = s->x[2].as<double>();
    a.type = s->type.as<int>();
    a.q = s->q.as<float>();
    a.L = s->L;
    a.alpha = s->alpha;
    a.EWALD_P = (double)0.3275911f;
    a.A1 = (double)0.254829592f;
    a.A2 = (double)-0.284496736f;
    a.A3 = (double)1.421413741f;
    a.A4 = (double)-1.453152027f;
    a.A5 = (double)1.061405429f;
    a.MY_PIS = (double)1.77245385090551602729f;
    a.e_shift = s->e_shift;
    a.f_shift = s->f_shift;
    a.cut_coulsq = (double)(float)(s->rc * s->rc);
    a.rcut2 = a.cut_coulsq;
    a.coulpre = s->coulpre;
    a.fx = s->f[0].as<long long>();
    a.fy = s->f[1].as<long long>();
    a.fz = s->f[2].as<long long>();
    a.e = et + md.nbond + md.nangle;
}

// Parts of a step's force evaluation (all of them in an MD step; the
// forces-only query selects).
constexpr int MDF_PAIR = 1, MDF_LANGEVIN = 2, MDF_SHAKE = 4, MDF_ALL = 7;

static int md_forces(Sys *s, bool energy, bool force_build, bool disp_done = false,
                     int sel = MDF_ALL) {
    Md &md = s->md;
    cudaStream_t st = s->ctx->stream;
    // the Langevin force is added by the pair path's force unpack
    LangevinArgs lg{};
    if (md.gamma > 0.0 && (sel & MDF_LANGEVIN)) {
        const double kT = KBOLTZ * md.temperature;
        lg.on = 1;
        lg.gamma = md.gamma;
        lg.gsig = sqrt(12.0 * 2.0 * md.gamma * kT * KCAL2AMU / md.dt) / KCAL2AMU;
        lg.seed = md.seed;
        lg.step = md.step_dev.as<long long>();
        lg.mass = s->mass.as<double>();
        lg.vx = s->v[0].as<double>();
        lg.vy = s->v[1].as<double>();
        lg.vz = s->v[2].as<double>();
    }
    long long *fx = s->f[0].as<long long>(), *fy = s->f[1].as<long long>(),
              *fz = s->f[2].as<long long>();
    if (sel & MDF_PAIR) {
        int rc = sys_step_forces(s, s->precision, energy, false, force_build, disp_done, &lg);
        if (rc) return rc;
    } else {
        const size_t nb = sizeof(long long) * (size_t)s->n;
        SOFIA_CUDA(s->ctx, cudaMemsetAsync(fx, 0, nb, st));
        SOFIA_CUDA(s->ctx, cudaMemsetAsync(fy, 0, nb, st));
        SOFIA_CUDA(s->ctx, cudaMemsetAsync(fz, 0, nb, st));
        SOFIA_CUDA(s->ctx, cudaMemsetAsync(s->red.p, 0, sizeof(double) * 5, st));
        if (lg.on) {
            sofia::launch_pdl(k_langevin_only, grid_for(s->n, 256), 256, 0, st, s->n, lg, fx, fy,
                              fz);
            s->launches += 1;
        }
    }
    const double *x = s->x[0].as<double>(), *y = s->x[1].as<double>(), *z = s->x[2].as<double>();
    double *et = md.eterm.as<double>();
    const int nb = md.nbond, na = md.nangle, nd = md.ndihed;
    BondedArgs b;
    b.nb = (md.terms & 1) ? nb : 0;
    b.na = (md.terms & 2) ? na : 0;
    b.nd = (md.terms & 12) ? nd : 0;
    b.ni = (md.terms & 16) ? md.nimpro : 0;
    b.bl = md.bonds.as<int>();
    b.bc = md.bcoef.as<double>();
    b.al = md.angles.as<int>();
    b.ac = md.acoef.as<double>();
    b.il = md.impros.as<int>();
    b.ic = md.icoef.as<double>();
    b.eb = et;
    b.ea = et + nb;
    b.ei = et + nb + na + 3 * (size_t)nd;
    DihArgs &a = b.dih;
    md_dih_args(s, et, &a);
    a.nd = b.nd;
    const long nterm = (long)b.nb + b.na + b.nd + b.ni;
    if (nterm > 0) {
        if (energy)
            sofia::launch_pdl(k_bonded<true>, grid_for(nterm, 128), 128, 0, st, b);
        else
            sofia::launch_pdl(k_bonded<false>, grid_for(nterm, 128), 128, 0, st, b);
    }
    if (md.nshake && (sel & MDF_SHAKE)) {
        sofia::launch_pdl(k_shake, grid_for(md.nshake, 128), 128, 0, st,
            md.nshake, md.shake.as<int>(), md.sbond.as<double>(), x, y, z, s->v[0].as<double>(),
            s->v[1].as<double>(), s->v[2].as<double>(), s->invm.as<double>(), s->L, md.dt,
            md.dt * md.dt * KCAL2AMU, md.shake_maxiter, md.shake_tol, fx, fy, fz,
            s->status_local.as<int>());
    }
    SOFIA_CUDA(s->ctx, cudaGetLastError());
    return SOFIA_OK;
}

static void md_energy_reduce(Sys *s) {
    Md &md = s->md;
    cudaStream_t st = s->ctx->stream;
    double *red = md.ered.as<double>();
    double *part = red + 16;
    double *et = md.eterm.as<double>();
    // nonbonded pair energies were reduced into s->red by the pair path
    cudaMemcpyAsync(red, s->red.p, sizeof(double) * 5, cudaMemcpyDeviceToDevice, st);  // checked with the step's launches
    if (md.nbond && (md.terms & 1)) md_reduce(st, md.nbond, 1, 0, et, part, red + 5);
    if (md.nangle && (md.terms & 2)) md_reduce(st, md.nangle, 1, 0, et + md.nbond, part, red + 6);
    if (md.ndihed && (md.terms & 12)) {
        const double *ed = et + md.nbond + md.nangle;
        md_reduce(st, md.ndihed, 3, 0, ed, part, red + 7);
        md_reduce(st, md.ndihed, 3, 1, ed, part, red + 8);
        md_reduce(st, md.ndihed, 3, 2, ed, part, red + 9);
    }
    if (md.nimpro && (md.terms & 16))
        md_reduce(st, md.nimpro, 1, 0, et + md.nbond + md.nangle + 3 * (size_t)md.ndihed, part,
                  red + 11);
    double *ke = md.eterm.as<double>() + (md.nbond + md.nangle + 3 * (size_t)md.ndihed +
                                          (size_t)md.nimpro);
    sofia::launch_pdl(k_ke, grid_for(s->n, 256), 256, 0, st, s->n, s->mass.as<double>(), s->v[0].as<double>(),
                                              s->v[1].as<double>(), s->v[2].as<double>(), ke);
    md_reduce(st, s->n, 1, 0, ke, part, red + 10);
}

// Reduced device energies (red slots: 0-1 pair, 5 bond, 6 angle, 7-9 torsion,
// coul14, lj14, 10 kinetic, 11 improper) -> the SOFIA_MD_NE output layout.
static void md_fill_energies(const Md &md, const double *e, double *o) {
    const double pot = e[0] + e[1] + md.e_self + e[5] + e[6] + e[7] + e[8] + e[9] + e[11];
    o[0] = e[0];
    o[1] = e[1];
    o[2] = md.e_self;
    o[3] = e[5];
    o[4] = e[6];
    o[5] = e[7];
    o[6] = e[8];
    o[7] = e[9];
    o[8] = e[10];
    o[9] = pot + e[10];
    o[10] = 2.0 * e[10] / ((double)md.ndof * KBOLTZ);
    o[11] = (double)md.step;
    o[12] = e[11];
}

// One MD step (all device work; capturable).
// One step.  twice: this step opens with the previous step's closing half-kick
// (that step ran with close = false); close: launch this step's closing
// half-kick (and RATTLE).  A segment of steps chains (close = false, twice =
// true) pairs and gives the same bits as separate steps.
static int md_step(Sys *s, bool energy, bool twice = false, bool close = true) {
    Md &md = s->md;
    cudaStream_t st = s->ctx->stream;
    const int n = s->n;
    const double h = 0.5 * md.dt * KCAL2AMU;
    double *vx = s->v[0].as<double>(), *vy = s->v[1].as<double>(), *vz = s->v[2].as<double>();
    const long long *fx = s->f[0].as<long long>(), *fy = s->f[1].as<long long>(),
                    *fz = s->f[2].as<long long>();
    const double half = 0.5 * s->skin, phalf = 0.5 * s->margin;
    sofia::launch_pdl(twice ? k_kick_drift<true> : k_kick_drift<false>, grid_for(n, 256), 256, 0, st,
        n, h, s->invm.as<double>(), fx, fy, fz, vx, vy, vz, md.dt, s->x[0].as<double>(),
        s->x[1].as<double>(), s->x[2].as<double>(), s->xref[0].as<double>(),
        s->xref[1].as<double>(), s->xref[2].as<double>(), s->xprn[0].as<double>(),
        s->xprn[1].as<double>(), s->xprn[2].as<double>(), s->L, half * half, phalf * phalf,
        s->flag.as<int>(), md.step_dev.as<long long>());
    int rc = md_forces(s, energy, false, true);
    if (rc) return rc;
    if (!close) {
        s->launches += 1;
        SOFIA_CUDA(s->ctx, cudaGetLastError());
        return SOFIA_OK;
    }
    sofia::launch_pdl(k_kick, grid_for(n, 256), 256, 0, st, n, h, s->invm.as<double>(), fx, fy, fz, vx, vy, vz);
    if (md.rattle && md.nshake) {
        sofia::launch_pdl(k_rattle, grid_for(md.nshake, 128), 128, 0, st, md.nshake,
                          md.shake.as<int>(), s->x[0].as<double>(), s->x[1].as<double>(),
                          s->x[2].as<double>(), vx, vy, vz, s->invm.as<double>(), s->L, h,
                          s->f[0].as<long long>(), s->f[1].as<long long>(),
                          s->f[2].as<long long>());
        s->launches += 1;
    }
    if (energy) md_energy_reduce(s);
    s->launches += 2;
    SOFIA_CUDA(s->ctx, cudaGetLastError());
    return SOFIA_OK;
}

static void md_drop_graphs(Sys *s) {
    for (auto &g : s->md.graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    s->md.graph_ok = 0;
}

static int md_capture(Sys *s) {
    md_drop_graphs(s);
    cudaStream_t st = s->ctx->stream;
    const int timing = s->timing;
    s->timing = 0;  // no event records inside the graph
    // RATTLE rewrites the full-step velocities after the closing kick, so its
    // steps keep separate kicks
    const bool fuse = !(s->md.rattle && s->md.nshake);
    const int nsteps_g[4] = {1, 1, s->md.seg, s->md.seg};
    for (int e = 0; e < 4; ++e) {
        cudaGraph_t g = nullptr;
        const long long l0 = s->launches;
        SOFIA_CUDA(s->ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = SOFIA_OK;
        for (int k = 0; k < nsteps_g[e] && !rc; ++k) {
            const bool last = k == nsteps_g[e] - 1;
            rc = md_step(s, (e & 1) && last, fuse && k > 0, !fuse || last);
        }
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        s->md.graph_launches[e] = s->launches - l0;
        s->launches = l0;
        s->timing = timing;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(s->ctx, ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&s->md.graph[e], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(s->ctx, ce, "cudaGraphInstantiate");
    }
    s->md.graph_ok = 1;
    return SOFIA_OK;
}

}  // namespace sofia

using sofia::Md;
using sofia::Sys;

template <class T>
static int up(sofia_nb_ctx *ctx, sofia::DevBuf &b, const T *src, size_t count) {
    SOFIA_CUDA(ctx, b.ensure(sizeof(T) * (count ? count : 1)));
    if (count && src)
        SOFIA_CUDA(ctx, cudaMemcpy(b.p, src, sizeof(T) * count, cudaMemcpyDefault));
    return SOFIA_OK;
}

extern "C" int sofia_system_md_setup(sofia_system *ss, const sofia_md_desc *d) {
    if (!ss || !d || !(d->dt > 0.0) || d->temperature < 0.0 || d->gamma < 0.0) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    Md &md = s->md;
    sofia::md_drop_graphs(s);
    md.dt = d->dt;
    md.temperature = d->temperature;
    md.gamma = d->gamma;
    md.seed = d->seed;
    md.nbond = d->bonds ? d->nbond : 0;
    md.nangle = d->angles ? d->nangle : 0;
    md.ndihed = d->dihedrals ? d->ndihed : 0;
    md.nshake = d->shake ? d->nshake : 0;
    md.nimpro = d->impropers ? d->nimpro : 0;
    md.terms = d->terms;
    if (d->flags & ~(SOFIA_MD_RATTLE | SOFIA_MD_LJ_SHIFT))
        return sofia::fail(ctx, SOFIA_EINVAL, "unknown sofia_md_desc flags%s");
    md.rattle = (d->flags & SOFIA_MD_RATTLE) ? 1 : 0;
    s->lj_shift = (d->flags & SOFIA_MD_LJ_SHIFT) ? 1 : 0;
    sofia::dropin_drop(s);  // the captured drop-in graphs hold the pair constants
    md.shake_maxiter = d->shake_maxiter > 0 ? d->shake_maxiter : 25;
    md.shake_tol = d->shake_tol > 0.0 ? d->shake_tol : (double)0.0001f;
    int rc;
    if ((rc = up(ctx, md.bonds, d->bonds, (size_t)md.nbond * 3))) return rc;
    if ((rc = up(ctx, md.bcoef, d->bond_coeff, (size_t)(d->nbondtypes > 0 ? d->nbondtypes : 0) * 2))) return rc;
    if ((rc = up(ctx, md.angles, d->angles, (size_t)md.nangle * 4))) return rc;
    if ((rc = up(ctx, md.acoef, d->angle_coeff, (size_t)(d->nangletypes > 0 ? d->nangletypes : 0) * 2))) return rc;
    if ((rc = up(ctx, md.diheds, d->dihedrals, (size_t)md.ndihed * 5))) return rc;
    if ((rc = up(ctx, md.dcoef, d->dihed_coeff, (size_t)(d->ndihedtypes > 0 ? d->ndihedtypes : 0) * 4))) return rc;
    if ((rc = up(ctx, md.lj14, d->lj14, d->lj14 ? (size_t)4 * s->ntypes * s->ntypes : 0))) return rc;
    if ((rc = up(ctx, md.shake, d->shake, (size_t)md.nshake * 5))) return rc;
    if ((rc = up(ctx, md.sbond, d->shake_bond, (size_t)md.nshake * 3))) return rc;
    if ((rc = up(ctx, md.impros, d->impropers, (size_t)md.nimpro * 5))) return rc;
    if ((rc = up(ctx, md.icoef, d->impro_coeff, (size_t)(d->nimprotypes > 0 ? d->nimprotypes : 0) * 2))) return rc;
    // validate indices on the host (no kernel ever sees an out-of-range id)
    {
        const int n = s->n;
        auto bad = [n](const int32_t *l, int cnt, int stride, int nid, int tcol, int ntyp) {
            for (int m = 0; m < cnt; ++m) {
                for (int k = 0; k < nid; ++k)
                    if (l[m * stride + k] < 1 || l[m * stride + k] > n) return true;
                if (tcol >= 0 && (l[m * stride + tcol] < 1 || l[m * stride + tcol] > ntyp)) return true;
            }
            return false;
        };
        if ((md.nbond && bad(d->bonds, md.nbond, 3, 2, 2, d->nbondtypes)) ||
            (md.nangle && bad(d->angles, md.nangle, 4, 3, 3, d->nangletypes)) ||
            (md.ndihed && bad(d->dihedrals, md.ndihed, 5, 4, 4, d->ndihedtypes)) ||
            (md.nimpro && bad(d->impropers, md.nimpro, 5, 4, 4, d->nimprotypes)))
            return sofia::fail(ctx, SOFIA_EINVAL, "bonded list index or type out of range%s");
        if ((md.terms & 8) && md.ndihed && !d->lj14)
            return sofia::fail(ctx, SOFIA_EINVAL, "1-4 pairs need lj14 tables%s");
        for (int g = 0; g < md.nshake; ++g) {
            const int num = d->shake[5 * g];
            const int na = (num == 1) ? 2 : (num == 4 ? 4 : 3);
            if (num != 1 && num != 3 && num != 4 && num != -3)
                return sofia::fail(ctx, SOFIA_EINVAL, "unknown SHAKE group kind%s");
            for (int k = 0; k < na; ++k)
                if (d->shake[5 * g + 1 + k] < 1 || d->shake[5 * g + 1 + k] > n)
                    return sofia::fail(ctx, SOFIA_EINVAL, "SHAKE atom index out of range%s");
        }
    }
    const size_t nterm = (size_t)md.nbond + md.nangle + 3 * (size_t)md.ndihed +
                         (size_t)md.nimpro + (size_t)s->n;
    SOFIA_CUDA(ctx, md.eterm.ensure(sizeof(double) * nterm));
    SOFIA_CUDA(ctx, md.ered.ensure(sizeof(double) * (16 + sofia::MRED)));
    SOFIA_CUDA(ctx, md.bpart.ensure(sizeof(double) * sofia::MD_NJOB * sofia::MRED));
    SOFIA_CUDA(ctx, cudaMemset(md.ered.p, 0, sizeof(double) * 16));
    SOFIA_CUDA(ctx, md.step_dev.ensure(sizeof(long long)));
    SOFIA_CUDA(ctx, cudaMemset(md.step_dev.p, 0, sizeof(long long)));
    for (int k = 0; k < 6; ++k) SOFIA_CUDA(ctx, md.snap[k].ensure(sizeof(double) * s->n));
    SOFIA_CUDA(ctx, md.snap[6].ensure(sizeof(long long)));
    // DSF self energy (Source/mod_assign_types.f90:59-62) and degrees of freedom
    {
        std::vector<float> hq(s->n);
        SOFIA_CUDA(ctx, cudaMemcpy(hq.data(), s->q.p, sizeof(float) * s->n, cudaMemcpyDeviceToHost));
        const double my_pis = (double)1.77245385090551602729f;
        double es = 0.0;
        for (int i = 0; i < s->n; ++i)
            es -= (0.5 * s->e_shift + s->alpha / my_pis) * (double)hq[i] * (double)hq[i] *
                  (double)s->coulpre;
        md.e_self = es;
        int ncons = 0;
        for (int g = 0; g < md.nshake; ++g) {
            const int num = d->shake[5 * g];
            ncons += (num == 1) ? 1 : (num == 3 ? 2 : 3);
        }
        md.ndof = 3 * s->n - ncons - 3;
    }
    md.step = 0;
    md.forces_valid = 0;
    md.ready = 1;
    return SOFIA_OK;
}

// Runs nsteps MD steps on the device.  energies[SOFIA_MD_NE] receives the
// energies of the last step (if energy_every > 0 and it divides the step).
extern "C" int sofia_system_md_run(sofia_system *ss, int nsteps, int energy_every, int use_graph,
                                   double *energies) {
    if (!ss || nsteps < 0) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    Md &md = s->md;
    if (!md.ready) return sofia::fail(ctx, SOFIA_EINVAL, "sofia_system_md_setup first%s");
    if (!s->mass.p) return sofia::fail(ctx, SOFIA_EINVAL, "system created without masses%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t nb = sizeof(double) * (size_t)s->n;
    for (int attempt = 0; attempt < 4; ++attempt) {
        // snapshot for a redo after a list-capacity overflow
        for (int d = 0; d < 3; ++d) {
            SOFIA_CUDA(ctx, cudaMemcpyAsync(md.snap[d].p, s->x[d].p, nb, cudaMemcpyDeviceToDevice, st));
            SOFIA_CUDA(ctx, cudaMemcpyAsync(md.snap[3 + d].p, s->v[d].p, nb, cudaMemcpyDeviceToDevice, st));
        }
        SOFIA_CUDA(ctx, cudaMemcpyAsync(md.snap[6].p, md.step_dev.p, sizeof(long long), cudaMemcpyDeviceToDevice, st));
        SOFIA_CUDA(ctx, cudaMemsetAsync(s->status_local.p, 0, sizeof(int) * sofia::ST_NSLOTS, st));
        int rc = SOFIA_OK;
        if (!md.forces_valid) {
            // initial forces (force_driver(0) + shake(1) before the loop, mod_integrate.f90:237-240)
            rc = sofia::md_forces(s, false, true);
            if (rc) return rc;
            md.forces_valid = 1;
        }
        if (use_graph && !md.graph_ok) {
            rc = sofia::md_capture(s);
            if (rc) return rc;
        }
        for (int k = 0; k < nsteps;) {
            const bool en = energy_every > 0 && ((k + 1) % energy_every == 0 || k + 1 == nsteps);
            if (use_graph) {
                // a whole segment when steps k .. k + seg - 1 hold no energy step but
                // possibly the last one
                const int sg = md.seg;
                int first_e = nsteps;  // first energy step at or after k
                if (energy_every > 0)
                    first_e = std::min(((k + energy_every) / energy_every) * energy_every - 1,
                                       nsteps - 1);
                if (sg > 1 && k + sg <= nsteps && first_e >= k + sg - 1) {
                    const int g = (first_e == k + sg - 1) ? 3 : 2;
                    SOFIA_CUDA(ctx, cudaGraphLaunch(md.graph[g], st));
                    s->launches += md.graph_launches[g];
                    k += sg;
                    continue;
                }
                SOFIA_CUDA(ctx, cudaGraphLaunch(md.graph[en ? 1 : 0], st));
                s->launches += md.graph_launches[en ? 1 : 0];
            } else {
                rc = sofia::md_step(s, en);
                if (rc) return rc;
            }
            ++k;
        }
        rc = sofia::sys_list_overflow(s);
        if (rc == SOFIA_ENEEDGROW) {
            // list row capacity grew: restore the segment start and run it again
            sofia::md_drop_graphs(s);
            for (int d = 0; d < 3; ++d) {
                SOFIA_CUDA(ctx, cudaMemcpyAsync(s->x[d].p, md.snap[d].p, nb, cudaMemcpyDeviceToDevice, st));
                SOFIA_CUDA(ctx, cudaMemcpyAsync(s->v[d].p, md.snap[3 + d].p, nb, cudaMemcpyDeviceToDevice, st));
            }
            SOFIA_CUDA(ctx, cudaMemcpyAsync(md.step_dev.p, md.snap[6].p, sizeof(long long), cudaMemcpyDeviceToDevice, st));
            md.forces_valid = 0;
            continue;
        }
        if (rc) return rc;
        int hs[sofia::ST_NSLOTS];
        SOFIA_CUDA(ctx, cudaMemcpyAsync(hs, s->status_local.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
        SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
        if (hs[sofia::ST_SHAKE])
            return sofia::fail(ctx, SOFIA_ESTATE, "SHAKE determinant <= 0 (mod_shake.f90:146-153, :267)%s");
        s->shake_nc += hs[sofia::ST_SHAKE_NC];
        md.step += nsteps;
        if (energies && energy_every > 0) {
            double e[16];
            SOFIA_CUDA(ctx, cudaMemcpy(e, md.ered.p, sizeof(double) * 16, cudaMemcpyDeviceToHost));
            sofia::md_fill_energies(md, e, energies);
        }
        return SOFIA_OK;
    }
    return sofia::fail(ctx, SOFIA_ENEEDGROW, "list capacity kept overflowing%s");
}

// Forces of one MD step at the resident positions and velocities, without
// stepping: the step's force evaluation (force_wrapper_DSF's zero / nonbond /
// bonded / 1-4 merge, Source/mod_force.f90:510-554, plus the Langevin force
// and SHAKE's constraint forces for the next step) restricted to the selected
// terms, all summed in 64-bit fixed point as in the step.
extern "C" int sofia_system_md_forces(sofia_system *ss, int terms, double *f, double *energies) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    Md &md = s->md;
    if (!md.ready) return sofia::fail(ctx, SOFIA_EINVAL, "sofia_system_md_setup first%s");
    if (!s->mass.p) return sofia::fail(ctx, SOFIA_EINVAL, "system created without masses%s");
    if (terms & ~(SOFIA_TERM_BOND | SOFIA_TERM_ANGLE | SOFIA_TERM_TORSION | SOFIA_TERM_PAIR14 |
                  SOFIA_TERM_IMPROPER | SOFIA_TERM_NONBOND | SOFIA_TERM_LANGEVIN |
                  SOFIA_TERM_SHAKE))
        return sofia::fail(ctx, SOFIA_EINVAL, "unknown force term bits%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int sel = 0;
    if (terms & SOFIA_TERM_NONBOND) sel |= sofia::MDF_PAIR;
    if (terms & SOFIA_TERM_LANGEVIN) sel |= sofia::MDF_LANGEVIN;
    if (terms & SOFIA_TERM_SHAKE) sel |= sofia::MDF_SHAKE;
    const int saved = md.terms;
    md.terms = saved & terms & 31;
    SOFIA_CUDA(ctx, cudaMemsetAsync(s->status_local.p, 0, sizeof(int) * sofia::ST_NSLOTS, st));
    // terms left out keep no energy from an earlier step
    SOFIA_CUDA(ctx, cudaMemsetAsync(md.ered.p, 0, sizeof(double) * 16, st));
    int rc = sofia::md_forces(s, energies != nullptr, false, false, sel);
    if (!rc && energies) sofia::md_energy_reduce(s);
    md.terms = saved;
    if (rc) return rc;
    // the step's forces are replaced: the next MD run recomputes its own
    md.forces_valid = 0;
    rc = sofia::sys_list_overflow(s);
    if (rc == SOFIA_ENEEDGROW) {
        // the row capacity grew: evaluate again on the rebuilt list
        md.terms = saved & terms & 31;
        rc = sofia::md_forces(s, energies != nullptr, true, false, sel);
        if (!rc && energies) sofia::md_energy_reduce(s);
        md.terms = saved;
        if (!rc) rc = sofia::sys_list_overflow(s);
    }
    if (rc) return rc;
    int hs[sofia::ST_NSLOTS];
    SOFIA_CUDA(ctx, cudaMemcpyAsync(hs, s->status_local.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    if (hs[sofia::ST_SHAKE])
        return sofia::fail(ctx, SOFIA_ESTATE, "SHAKE determinant <= 0 (mod_shake.f90:146-153, :267)%s");
    if (f) {
        const size_t n = (size_t)s->n;
        std::vector<long long> h(3 * n);
        for (int d = 0; d < 3; ++d)
            SOFIA_CUDA(ctx, cudaMemcpy(h.data() + d * n, s->f[d].p, sizeof(long long) * n,
                                       cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) f[3 * i + d] = (double)h[d * n + i] * sofia::FIX_INV;
    }
    if (energies) {
        double e[16];
        SOFIA_CUDA(ctx, cudaMemcpy(e, md.ered.p, sizeof(double) * 16, cudaMemcpyDeviceToHost));
        sofia::md_fill_energies(md, e, energies);
    }
    return SOFIA_OK;
}

// ---------------------------------------------------------------------------
// Batches of independent replicas.  Every kernel of an MD step runs once for all
// replicas of the batch (BatchDev in system.cuh): a launch walks its virtual
// blocks in a grid-stride loop over the replicas' own buffers, with the block
// size and body of the single-system kernel, so a replica's trajectory is
// bit-identical to the same replica run alone.  Steps are captured as CUDA
// graphs of `seg` steps (100 by default); the graphs hold only the address of
// the device table, which the host rewrites when membership changes or a list
// grows, so neither needs a recapture.  Replicas never exchange data (the
// reference runs one replica per MPI rank, Source/MD.f90:26-44).
namespace sofia {
namespace {

#define SOFIA_BATCH_LOOP(KIND)                                                   \
    const int nrep_ = tab->nrep;                                                 \
    const int *pre_ = tab->pre[KIND];                                            \
    const int tot_ = pre_[nrep_];                                                \
    for (int vb = blockIdx.x; vb < tot_; vb += gridDim.x) {                      \
        const int r_ = batch_rep(pre_, nrep_, vb);                               \
        const RepDev &d = tab->rep[r_];                                          \
        const int lb = vb - pre_[r_];
#define SOFIA_BATCH_END }

// Segment start for every replica in one launch: the snapshot a list regrow
// restarts from (positions, velocities, step counter) and cleared status words.
__global__ void k_snapshot_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_A256)
    const int i = lb * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.snap[0][i] = d.x[i];
        d.snap[1][i] = d.y[i];
        d.snap[2][i] = d.z[i];
        d.snap[3][i] = d.vx[i];
        d.snap[4][i] = d.vy[i];
        d.snap[5][i] = d.vz[i];
    }
    if (lb == 0 && threadIdx.x == 0) d.snap_step[0] = d.step[0];
    if (lb == 0 && threadIdx.x < ST_NSLOTS) d.status[threadIdx.x] = 0;
    SOFIA_BATCH_END
}

// The status words and the 16 energy sums of every replica into two arrays
// (replica r at r * ST_NSLOTS and r * 16), each read back with one copy.
__global__ void k_status_b(const BatchDev *__restrict__ tab, int *__restrict__ out,
                           double *__restrict__ eout) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_REP)
    const int r = (int)(&d - tab->rep);
    if (threadIdx.x < ST_NSLOTS) out[r * ST_NSLOTS + threadIdx.x] = d.status[threadIdx.x];
    if (threadIdx.x < 16) eout[r * 16 + threadIdx.x] = d.ered[threadIdx.x];
    SOFIA_BATCH_END
}

template <bool TWICE>
__global__ void __launch_bounds__(256, SOFIA_BATCH_STREAM_MINB) k_kick_drift_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_A256)
    kick_drift_body<TWICE>(lb, d.n, d.h, d.invm, d.fx, d.fy, d.fz, d.vx, d.vy, d.vz, d.dt, d.x, d.y,
                    d.z, d.rx, d.ry, d.rz, d.px, d.py, d.pz, d.L, d.lim2, d.plim2, d.flag,
                    d.step);
    SOFIA_BATCH_END
}

template <bool EN>
// The batched bonded and SHAKE kernels walk their virtual blocks in a static
// grid-stride order: one thread per term or group is short, uniform work, and
// popping a work queue per block cost more than it balanced (64 replicas:
// 363 -> 365 M atom-steps/s with the static order).
__global__ void __launch_bounds__(128, SOFIA_BONDED_MINB) k_bonded_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_B128)
    bonded_body<EN>(lb, d.b);
    SOFIA_BATCH_END
}

__global__ void k_shake_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_G128)
    shake_body(lb, d.nshake, d.shake, d.sbond, d.x, d.y, d.z, d.vx, d.vy, d.vz, d.invm, d.L,
               d.dt, d.dtsq, d.shake_maxiter, d.shake_tol, d.fx, d.fy, d.fz, d.status);
    SOFIA_BATCH_END
}

__global__ void k_kick_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_A256)
    kick_body(lb, d.n, d.h, d.invm, d.fx, d.fy, d.fz, d.vx, d.vy, d.vz);
    SOFIA_BATCH_END
}

__global__ void k_rattle_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_G128)
    if (d.rattle)
        rattle_body(lb, d.nshake, d.shake, d.x, d.y, d.z, d.vx, d.vy, d.vz, d.invm, d.L, d.h,
                    d.fx, d.fy, d.fz);
    SOFIA_BATCH_END
}

// Energy steps: pair sums to their slots, kinetic energy, then the per-term sums
// with the same two-stage trees (MRED blocks, then one block) as md_reduce.
__global__ void k_copyred_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_REP)
    if (threadIdx.x < 5) d.ered[threadIdx.x] = d.red[threadIdx.x];
    SOFIA_BATCH_END
}

__global__ void k_ke_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_A256)
    ke_body(lb, d.n, d.mass, d.vx, d.vy, d.vz, d.ke);
    SOFIA_BATCH_END
}

__global__ void k_mred1_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_MRED)
    const int job = lb / MRED, blk = lb - job * MRED;
    if (d.job_n[job] > 0)
        mred1_body(blk, d.job_n[job], d.job_w[job], d.job_c[job], d.job_in[job],
                   d.ebpart + job * MRED, MRED);
    __syncthreads();
    SOFIA_BATCH_END
}

__global__ void k_mred2_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_MJOB)
    if (d.job_n[lb] > 0) mred2_body(0, d.ebpart + lb * MRED, d.ered + d.job_slot[lb]);
    __syncthreads();
    SOFIA_BATCH_END
}

#undef SOFIA_BATCH_LOOP
#undef SOFIA_BATCH_END

}  // namespace

// The MD part of a replica's table entry (step constants, thermostat, bonded
// terms, SHAKE, energy-sum jobs); the argument values of md_forces / md_step.
static void repdev_fill_md(Sys *s, RepDev *d) {
    Md &md = s->md;
    d->h = 0.5 * md.dt * KCAL2AMU;
    d->dt = md.dt;
    d->dtsq = md.dt * md.dt * KCAL2AMU;
    d->shake_maxiter = md.shake_maxiter;
    d->shake_tol = md.shake_tol;
    d->nshake = md.nshake;
    d->rattle = md.rattle;
    d->shake = md.shake.as<int>();
    d->sbond = md.sbond.as<double>();
    d->step = md.step_dev.as<long long>();
    for (int c = 0; c < 6; ++c) d->snap[c] = md.snap[c].as<double>();
    d->snap_step = md.snap[6].as<long long>();
    LangevinArgs lg{};
    if (md.gamma > 0.0) {
        const double kT = KBOLTZ * md.temperature;
        lg.on = 1;
        lg.gamma = md.gamma;
        lg.gsig = sqrt(12.0 * 2.0 * md.gamma * kT * KCAL2AMU / md.dt) / KCAL2AMU;
        lg.seed = md.seed;
        lg.step = md.step_dev.as<long long>();
        lg.mass = s->mass.as<double>();
        lg.vx = s->v[0].as<double>();
        lg.vy = s->v[1].as<double>();
        lg.vz = s->v[2].as<double>();
    }
    d->lg = lg;
    double *et = md.eterm.as<double>();
    const int nb = md.nbond, na = md.nangle, nd = md.ndihed;
    BondedArgs &b = d->b;
    b.nb = (md.terms & 1) ? nb : 0;
    b.na = (md.terms & 2) ? na : 0;
    b.nd = (md.terms & 12) ? nd : 0;
    b.ni = (md.terms & 16) ? md.nimpro : 0;
    b.bl = md.bonds.as<int>();
    b.bc = md.bcoef.as<double>();
    b.al = md.angles.as<int>();
    b.ac = md.acoef.as<double>();
    b.il = md.impros.as<int>();
    b.ic = md.icoef.as<double>();
    b.eb = et;
    b.ea = et + nb;
    b.ei = et + nb + na + 3 * (size_t)nd;
    DihArgs &a = b.dih;
    md_dih_args(s, et, &a);
    a.nd = b.nd;
    d->ered = md.ered.as<double>();
    d->ebpart = md.bpart.as<double>();
    d->ke = et + (nb + na + 3 * (size_t)nd + (size_t)md.nimpro);
    const int jn[MD_NJOB] = {(nb && (md.terms & 1)) ? nb : 0, (na && (md.terms & 2)) ? na : 0,
                             (nd && (md.terms & 12)) ? nd : 0, (nd && (md.terms & 12)) ? nd : 0,
                             (nd && (md.terms & 12)) ? nd : 0,
                             (md.nimpro && (md.terms & 16)) ? md.nimpro : 0, s->n};
    const int jw[MD_NJOB] = {1, 1, 3, 3, 3, 1, 1}, jc[MD_NJOB] = {0, 0, 0, 1, 2, 0, 0};
    const int js[MD_NJOB] = {5, 6, 7, 8, 9, 11, 10};
    const double *jin[MD_NJOB] = {et, et + nb, et + nb + na, et + nb + na, et + nb + na,
                                  et + nb + na + 3 * (size_t)nd, d->ke};
    for (int k = 0; k < MD_NJOB; ++k) {
        d->job_n[k] = jn[k];
        d->job_w[k] = jw[k];
        d->job_c[k] = jc[k];
        d->job_slot[k] = js[k];
        d->job_in[k] = jin[k];
    }
}

// One batched MD step: the same kernels, in the same order, as md_step.
// One batch step; twice and close as for md_step (a segment chains its steps'
// closing half-kicks into the next steps' kick and drift).
static void batch_step(BatchDev *tab, Sys *s0, bool energy, bool rattle, cudaStream_t st,
                       int nsm, int pair_blocks, bool twice = false, bool close = true) {
    const int g256 = nsm * 8, g128 = nsm * 16;
    if (twice)
        launch_pdl(k_kick_drift_b<true>, g256, 256, 0, st, tab);
    else
        launch_pdl(k_kick_drift_b<false>, g256, 256, 0, st, tab);
    batch_pair_path(tab, s0, s0->precision, energy, st, nsm, pair_blocks);
    if (energy)
        launch_pdl(k_bonded_b<true>, g128, 128, 0, st, tab);
    else
        launch_pdl(k_bonded_b<false>, g128, 128, 0, st, tab);
    launch_pdl(k_shake_b, g128, 128, 0, st, tab);
    if (!close) return;
    launch_pdl(k_kick_b, g256, 256, 0, st, tab);
    if (rattle) launch_pdl(k_rattle_b, g128, 128, 0, st, tab);
    if (energy) {
        launch_pdl(k_copyred_b, nsm, 32, 0, st, tab);
        launch_pdl(k_ke_b, g256, 256, 0, st, tab);
        launch_pdl(k_mred1_b, g256, 256, 0, st, tab);
        launch_pdl(k_mred2_b, nsm * 8, MRED, 0, st, tab);
    }
}

}  // namespace sofia

struct sofia_batch {
    sofia_nb_ctx *ctx = nullptr;
    std::vector<sofia_system *> sys;
    sofia::DevBuf tab;                  // BatchDev on the device
    std::vector<unsigned char> htab;    // its host image
    sofia::DevBuf stat, estat;          // every replica's status words and energy sums
    std::vector<int> hstat;             // their host copies
    std::vector<double> hestat;
    int seg = 100;                      // steps per captured segment graph
    int nsm = 148;
    // captured graphs: [0] one step, [1] one step with energies, [2] seg steps,
    // [3] seg steps with energies on the last
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    int graph_ok = 0;
    int graph_rattle = 0;               // the graphs hold the RATTLE launch
    sofia::PairKey graph_key{};         // the pair constants the graphs hold
    long long graph_launches[4] = {0, 0, 0, 0};  // kernel launches each graph holds
};

static void batch_drop_graphs(sofia_batch *b) {
    for (auto &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    b->graph_ok = 0;
}

static int batch_check_members(sofia_nb_ctx *ctx, sofia_system *const *systems, int n) {
    if (n <= 0 || n > sofia::MAXREP)
        return sofia::fail(ctx, SOFIA_EINVAL, "a batch holds 1 to 256 replicas%s");
    for (int i = 0; i < n; ++i) {
        if (!systems[i]) return sofia::fail(ctx, SOFIA_EINVAL, "null system in batch%s");
        if (systems[i]->s.ctx->device != ctx->device)
            return sofia::fail(ctx, SOFIA_EINVAL, "batch systems must share the device%s");
        if (!systems[i]->s.md.ready)
            return sofia::fail(ctx, SOFIA_EINVAL, "sofia_system_md_setup every system first%s");
        if (!systems[i]->s.mass.p)
            return sofia::fail(ctx, SOFIA_EINVAL, "system created without masses%s");
        if (!sofia::pair_const_compatible(&systems[0]->s, &systems[i]->s))
            return sofia::fail(ctx, SOFIA_EINVAL,
                               "batch systems must share precision, types, cut-off and DSF "
                               "constants%s");
        for (int j = 0; j < i; ++j)
            if (systems[j] == systems[i]) return sofia::fail(ctx, SOFIA_EINVAL, "system listed twice%s");
    }
    return SOFIA_OK;
}

// Rewrites the device table from the members' current buffers and sizes.
static int batch_upload(sofia_batch *b) {
    sofia_nb_ctx *ctx = b->ctx;
    const int n = (int)b->sys.size();
    if (b->htab.size() != sizeof(sofia::BatchDev)) b->htab.assign(sizeof(sofia::BatchDev), 0);
    auto *h = reinterpret_cast<sofia::BatchDev *>(b->htab.data());
    h->nrep = n;
    for (int k = 0; k < sofia::BK_N; ++k) h->pre[k][0] = 0;
    for (int r = 0; r < n; ++r) {
        Sys *s = &b->sys[r]->s;
        sofia::RepDev &d = h->rep[r];
        sofia::repdev_fill_pair(s, &d);
        sofia::repdev_fill_md(s, &d);
        const long nterm = (long)d.b.nb + d.b.na + d.b.nd + d.b.ni;
        const int cnt[sofia::BK_N] = {
            sofia::grid_for(s->n, 256), 1, s->ncols, sofia::grid_for((long)s->max_clusters * 8, 256),
            sofia::grid_for((long)s->max_clusters * 32, 256),
            sofia::grid_for(nterm, 128), sofia::grid_for(s->md.nshake, 128), sofia::RED_BLOCKS,
            1, sofia::MD_NJOB * sofia::MRED, sofia::MD_NJOB};
        for (int k = 0; k < sofia::BK_N; ++k) h->pre[k][r + 1] = h->pre[k][r] + cnt[k];
    }
    SOFIA_CUDA(ctx, b->tab.ensure(sizeof(sofia::BatchDev)));
    const size_t used = offsetof(sofia::BatchDev, rep) + sizeof(sofia::RepDev) * (size_t)n;
    SOFIA_CUDA(ctx, cudaMemcpyAsync(b->tab.p, h, used, cudaMemcpyHostToDevice, ctx->stream));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SOFIA_OK;
}

extern "C" int sofia_batch_create(sofia_nb_ctx *ctx, sofia_system *const *systems, int n,
                                  sofia_batch **out) {
    if (!ctx || !systems || !out) return SOFIA_EINVAL;
    *out = nullptr;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    int rc = batch_check_members(ctx, systems, n);
    if (rc) return rc;
    SOFIA_CUDA(ctx, sofia::batch_pair_smem_optin(systems[0]->s.ntypes));
    sofia_batch *b = new sofia_batch();
    b->ctx = ctx;
    b->sys.assign(systems, systems + n);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    *out = b;
    return SOFIA_OK;
}

extern "C" int sofia_batch_destroy(sofia_batch *b) {
    if (!b) return SOFIA_OK;
    if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
    batch_drop_graphs(b);
    b->tab.release();
    b->stat.release();
    b->estat.release();
    delete b;
    return SOFIA_OK;
}

// Replaces the batch's members (continuous batching).  The captured graphs stay
// valid when the new members share the first member's pair constants and need
// no RATTLE launch the graphs lack.
extern "C" int sofia_batch_set_systems(sofia_batch *b, sofia_system *const *systems, int n) {
    if (!b || !systems) return SOFIA_EINVAL;
    sofia_nb_ctx *ctx = b->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    int rc = batch_check_members(ctx, systems, n);
    if (rc) return rc;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    b->sys.assign(systems, systems + n);
    if (b->graph_ok) {
        bool rat = false;
        for (auto *s : b->sys) rat = rat || (s->s.md.rattle && s->s.md.nshake);
        const bool keep = (!rat || b->graph_rattle) && b->graph_key == sofia::pair_key(&b->sys[0]->s);
        if (!keep) batch_drop_graphs(b);
    }
    return SOFIA_OK;
}

extern "C" int sofia_batch_set_segment(sofia_batch *b, int steps) {
    if (!b || steps < 1 || steps > 1000) return SOFIA_EINVAL;
    if (steps != b->seg) {
        sofia_nb_ctx *ctx = b->ctx;
        SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        batch_drop_graphs(b);
        b->seg = steps;
    }
    return SOFIA_OK;
}

static int batch_capture(sofia_batch *b) {
    batch_drop_graphs(b);
    sofia_nb_ctx *ctx = b->ctx;
    cudaStream_t ms = ctx->stream;
    auto *tab = b->tab.as<sofia::BatchDev>();
    Sys *s0 = &b->sys[0]->s;
    bool rat = false;
    for (auto *s : b->sys) rat = rat || (s->s.md.rattle && s->s.md.nshake);
    const int nsteps[4] = {1, 1, b->seg, b->seg};
    const auto *h = reinterpret_cast<const sofia::BatchDev *>(b->htab.data());
    const int pair_blocks = h->pre[sofia::BK_W256][h->nrep];
    for (int g = 0; g < 4; ++g) {
        cudaGraph_t graph = nullptr;
        SOFIA_CUDA(ctx, cudaStreamBeginCapture(ms, cudaStreamCaptureModeThreadLocal));
        // without RATTLE the steps of a segment chain their closing half-kicks
        const bool fuse = !rat;
        for (int k = 0; k < nsteps[g]; ++k) {
            const bool last = k == nsteps[g] - 1;
            sofia::batch_step(tab, s0, (g & 1) && last, rat, ms, b->nsm, pair_blocks,
                              fuse && k > 0, !fuse || last);
        }
        cudaError_t ce = cudaStreamEndCapture(ms, &graph);
        if (ce != cudaSuccess) return sofia::cuda_fail(ctx, ce, "cudaStreamEndCapture (batch)");
        ce = cudaGraphInstantiate(&b->graph[g], graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return sofia::cuda_fail(ctx, ce, "cudaGraphInstantiate (batch)");
    }
    // a step: kick+drift, the pair path (active-replica compaction, bin, scan,
    // scatter, sort, pack with the cluster boxes, search, prune, pair, unpack),
    // bonded, SHAKE; then the closing kick (+ RATTLE), once per segment when the
    // kicks are chained; energies add the two pair-energy and four MD-energy
    // reductions
    const long long body = 1 + 10 + 2, closing = 1 + (rat ? 1 : 0);
    b->graph_launches[0] = body + closing;
    b->graph_launches[1] = body + closing + 6;
    b->graph_launches[2] = rat ? b->seg * (body + closing) : b->seg * body + closing;
    b->graph_launches[3] = b->graph_launches[2] + 6;
    b->graph_rattle = rat;
    b->graph_key = sofia::pair_key(s0);
    b->graph_ok = 1;
    return SOFIA_OK;
}

// Runs nsteps steps of every replica: segments of `seg` steps as one graph
// launch each, the rest one step per launch.  energies[n*SOFIA_MD_NE] (may be
// NULL) receive each replica's energies of the last step when energy_every > 0
// (only that step computes them).
extern "C" int sofia_batch_md_run(sofia_batch *b, int nsteps, int energy_every,
                                  double *energies) {
    if (!b || nsteps < 0) return SOFIA_EINVAL;
    sofia_nb_ctx *ctx = b->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t ms = ctx->stream;
    const int n = (int)b->sys.size();
    const bool want_e = energy_every > 0 && nsteps > 0;
    SOFIA_CUDA(ctx, b->stat.ensure(sizeof(int) * sofia::ST_NSLOTS * sofia::MAXREP));
    SOFIA_CUDA(ctx, b->estat.ensure(sizeof(double) * 16 * sofia::MAXREP));
    b->hstat.resize((size_t)sofia::ST_NSLOTS * n);
    b->hestat.resize((size_t)16 * n);
    for (int attempt = 0; attempt < 4; ++attempt) {
        // work the caller queued on the members' own streams comes first
        for (int i = 0; i < n; ++i) SOFIA_CUDA(ctx, cudaStreamSynchronize(b->sys[i]->s.ctx->stream));
        int rc = batch_upload(b);
        if (rc) return rc;
        auto *tab = b->tab.as<sofia::BatchDev>();
        // snapshots and cleared status words for all members in one launch, before
        // any initial force evaluation (whose list build reports into the status)
        SOFIA_CUDA(ctx, sofia::launch_pdl(sofia::k_snapshot_b, b->nsm * 8, 256, 0, ms, tab));
        bool stale = false;
        for (int i = 0; i < n; ++i) stale = stale || !b->sys[i]->s.md.forces_valid;
        if (stale) {
            SOFIA_CUDA(ctx, cudaStreamSynchronize(ms));
            for (int i = 0; i < n; ++i) {
                Sys *s = &b->sys[i]->s;
                if (s->md.forces_valid) continue;
                rc = sofia::md_forces(s, false, true);
                if (rc) return rc;
                s->md.forces_valid = 1;
                SOFIA_CUDA(ctx, cudaStreamSynchronize(s->ctx->stream));
            }
        }
        if (!b->graph_ok) {
            rc = batch_capture(b);
            if (rc) return rc;
        }
        int left = nsteps;
        long long launched = 0;
        while (left > 0) {
            const bool full = left >= b->seg;
            const int k = full ? b->seg : 1;
            const bool en = want_e && left == k;
            SOFIA_CUDA(ctx, cudaGraphLaunch(b->graph[(full ? 2 : 0) + (en ? 1 : 0)], ms));
            launched += b->graph_launches[(full ? 2 : 0) + (en ? 1 : 0)];
            left -= k;
        }
        SOFIA_CUDA(ctx, sofia::launch_pdl(sofia::k_status_b, b->nsm, 32, 0, ms, tab,
                                          b->stat.as<int>(), b->estat.as<double>()));
        launched += 2;  // the snapshot and status kernels
        SOFIA_CUDA(ctx, cudaMemcpyAsync(b->hstat.data(), b->stat.p,
                                        sizeof(int) * sofia::ST_NSLOTS * (size_t)n,
                                        cudaMemcpyDeviceToHost, ms));
        if (energies && want_e)
            SOFIA_CUDA(ctx, cudaMemcpyAsync(b->hestat.data(), b->estat.p,
                                            sizeof(double) * 16 * (size_t)n,
                                            cudaMemcpyDeviceToHost, ms));
        SOFIA_CUDA(ctx, cudaStreamSynchronize(ms));
        bool regrow = false;
        for (int i = 0; i < n; ++i) {
            Sys *s = &b->sys[i]->s;
            s->launches += launched / (n > 0 ? n : 1);
            const int r2 = sofia::sys_list_overflow(s, &b->hstat[(size_t)sofia::ST_NSLOTS * i]);
            if (r2 == SOFIA_ENEEDGROW) {
                regrow = true;
                continue;
            }
            if (r2) return r2;
        }
        if (regrow) {
            // a list row overflowed: every replica restarts the segment from its
            // snapshot (the table is rewritten with the grown lists)
            for (int i = 0; i < n; ++i) {
                Sys *s = &b->sys[i]->s;
                Md &md = s->md;
                cudaStream_t st = s->ctx->stream;
                const size_t nb = sizeof(double) * (size_t)s->n;
                sofia::md_drop_graphs(s);
                for (int d = 0; d < 3; ++d) {
                    SOFIA_CUDA(ctx, cudaMemcpyAsync(s->x[d].p, md.snap[d].p, nb, cudaMemcpyDeviceToDevice, st));
                    SOFIA_CUDA(ctx, cudaMemcpyAsync(s->v[d].p, md.snap[3 + d].p, nb, cudaMemcpyDeviceToDevice, st));
                }
                SOFIA_CUDA(ctx, cudaMemcpyAsync(md.step_dev.p, md.snap[6].p, sizeof(long long), cudaMemcpyDeviceToDevice, st));
                md.forces_valid = 0;
                s->built = 0;
                SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
            }
            continue;
        }
        for (int i = 0; i < n; ++i) {
            Sys *s = &b->sys[i]->s;
            Md &md = s->md;
            const int *hs = &b->hstat[(size_t)sofia::ST_NSLOTS * i];
            if (hs[sofia::ST_SHAKE])
                return sofia::fail(ctx, SOFIA_ESTATE, "SHAKE determinant <= 0 in a batch replica%s");
            s->shake_nc += hs[sofia::ST_SHAKE_NC];
            md.step += nsteps;
            if (energies && want_e) {
                double *o = energies + (size_t)i * SOFIA_MD_NE;
                sofia::md_fill_energies(md, &b->hestat[(size_t)16 * i], o);
            }
        }
        return SOFIA_OK;
    }
    return sofia::fail(ctx, SOFIA_ENEEDGROW, "list capacity kept overflowing (batch)%s");
}

// Prune margin (A) of the pruned inner list: the per-size-class tuning knob.
namespace sofia {
void md_invalidate(Sys *s) {
    s->built = 0;
    s->md.forces_valid = 0;  // the next run rebuilds and recomputes before any capture
    md_drop_graphs(s);
    dropin_drop(s);
}
}  // namespace sofia

extern "C" int sofia_system_set_margin(sofia_system *ss, double margin) {
    if (!ss || !(margin >= 0.05) || !(margin <= ss->s.skin)) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    SOFIA_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    s->margin = margin;
    sofia::md_invalidate(s);
    return SOFIA_OK;
}

// In-memory snapshot / rollback of one replica, the accept/reject pattern of
// nuc_move (mod_nucleation.f90:318-389 saves position, v and the lists;
// :453-531 restores them on reject).  The snapshot holds positions, velocities
// and the thermostat step counter on the device; the lists are rebuilt from
// the saved positions after the snapshot and after a rollback alike, so
// nothing else needs saving.
extern "C" int sofia_system_snapshot(sofia_system *ss) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia::Md &md = s->md;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t nb = sizeof(double) * (size_t)s->n;
    cudaStream_t st = ctx->stream;
    for (int d = 0; d < 3; ++d) {
        SOFIA_CUDA(ctx, md.keep[d].ensure(nb));
        SOFIA_CUDA(ctx, md.keep[3 + d].ensure(nb));
        SOFIA_CUDA(ctx, cudaMemcpyAsync(md.keep[d].p, s->x[d].p, nb, cudaMemcpyDeviceToDevice, st));
        SOFIA_CUDA(ctx, cudaMemcpyAsync(md.keep[3 + d].p, s->v[d].p, nb, cudaMemcpyDeviceToDevice, st));
    }
    SOFIA_CUDA(ctx, md.keep[6].ensure(sizeof(long long)));
    if (md.ready) {
        SOFIA_CUDA(ctx, cudaMemcpyAsync(md.keep[6].p, md.step_dev.p, sizeof(long long),
                                        cudaMemcpyDeviceToDevice, st));
    }
    md.keep_step = md.step;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    md.has_keep = 1;
    // The snapshot is a restart point: the next evaluation rebuilds the lists
    // and recomputes the forces from these positions, exactly as it will after
    // a rollback, so both continuations take identical steps.
    s->built = 0;
    md.forces_valid = 0;
    return SOFIA_OK;
}

extern "C" int sofia_system_rollback(sofia_system *ss) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia::Md &md = s->md;
    sofia_nb_ctx *ctx = s->ctx;
    if (!md.has_keep) return sofia::fail(ctx, SOFIA_ESTATE, "rollback: no snapshot was taken");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t nb = sizeof(double) * (size_t)s->n;
    cudaStream_t st = ctx->stream;
    for (int d = 0; d < 3; ++d) {
        SOFIA_CUDA(ctx, cudaMemcpyAsync(s->x[d].p, md.keep[d].p, nb, cudaMemcpyDeviceToDevice, st));
        SOFIA_CUDA(ctx, cudaMemcpyAsync(s->v[d].p, md.keep[3 + d].p, nb, cudaMemcpyDeviceToDevice, st));
    }
    if (md.ready) {
        SOFIA_CUDA(ctx, cudaMemcpyAsync(md.step_dev.p, md.keep[6].p, sizeof(long long),
                                        cudaMemcpyDeviceToDevice, st));
    }
    md.step = md.keep_step;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    s->built = 0;
    md.forces_valid = 0;
    return SOFIA_OK;
}

namespace sofia {
namespace {
// Resident FP64 positions -> real*4 ainfo records wrapped into (0, box] (the
// state the reference's pbc leaves, Source/mod_pbc.f90:6-39, from the
// double-precision wrap x - L floor(x / L)), and global ids 1..n.
__global__ void k_resident_ainfo(int n, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const int *__restrict__ type, double L, float box,
                                 float4 *__restrict__ out, int *__restrict__ gid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float w[3];
    const double p[3] = {x[i], y[i], z[i]};
    for (int d = 0; d < 3; ++d) {
        float f = (float)(p[d] - L * floor(p[d] / L));
        if (f <= 0.0f) f += box;
        w[d] = f;
    }
    out[i] = make_float4(w[0], w[1], w[2], __int_as_float(type[i]));
    gid[i] = i + 1;
}

// ptta_full[i*3 + d] = the current FP64 position of glycine atom i (first call).
__global__ void k_ptta_init(int na, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, double *__restrict__ ptta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= na) return;
    ptta[3 * i + 0] = x[i];
    ptta[3 * i + 1] = y[i];
    ptta[3 * i + 2] = z[i];
}
}  // namespace
}  // namespace sofia

// Largest-cluster analysis (get_greatestCluster, Source/mod_cluster.f90:15-83)
// on a resident system's current positions: the positions never leave the
// device, as nuc_move keeps them between segments
// (Source/mod_nucleation.f90:396-449).  Glycine molecules are the first
// n_gly * atoms_per_gly atoms; ptta_full (host or device) and
// *greatest_belongsto are in/out as in sofia_greatest_cluster.
extern "C" int sofia_system_greatest_cluster(sofia_system *ss, int n_gly, int atoms_per_gly,
                                             double mrcut, double denscut, int densmin,
                                             double *ptta_full, int32_t *greatest_belongsto,
                                             int32_t *size_out) {
    if (!ss || !size_out) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    if (n_gly < 0 || atoms_per_gly <= 0 || (size_t)n_gly * atoms_per_gly > (size_t)s->n)
        return sofia::fail(ctx, SOFIA_EINVAL, "glycine atoms beyond the system%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, s->cl_pos.ensure(sizeof(float4) * (size_t)s->n));
    SOFIA_CUDA(ctx, s->cl_gid.ensure(sizeof(int) * (size_t)s->n));
    sofia::k_resident_ainfo<<<sofia::grid_for(s->n, 256), 256, 0, ctx->stream>>>(
        s->n, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(),
        s->type.as<int>(), s->L, s->box, s->cl_pos.as<float4>(), s->cl_gid.as<int>());
    SOFIA_CUDA(ctx, cudaGetLastError());
    if (!ptta_full) {
        // the system keeps its own ptta_full on the device, set from the current
        // positions by the first call
        const int na = n_gly * atoms_per_gly;
        if (s->ptta_atoms != na) {
            SOFIA_CUDA(ctx, s->ptta.ensure(sizeof(double) * 3 * (size_t)(na > 0 ? na : 1)));
            if (na > 0)
                sofia::k_ptta_init<<<sofia::grid_for(na, 256), 256, 0, ctx->stream>>>(
                    na, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(),
                    s->ptta.as<double>());
            SOFIA_CUDA(ctx, cudaGetLastError());
            s->ptta_atoms = na;
        }
        ptta_full = s->ptta.as<double>();
    }
    return sofia_greatest_cluster(ctx, s->n, s->cl_pos.as<sofia_ainfo>(), s->cl_gid.as<int32_t>(),
                                  n_gly, atoms_per_gly, s->box, mrcut, denscut, densmin,
                                  ptta_full, greatest_belongsto, size_out, nullptr, nullptr);
}

// Device memory a system holds (all its buffers, lists and MD state).
extern "C" int sofia_system_device_bytes(sofia_system *ss, int64_t *bytes) {
    if (!ss || !bytes) return SOFIA_EINVAL;
    const Sys *s = &ss->s;
    const Md &md = s->md;
    const sofia::DevBuf *bufs[] = {
        &s->x[0], &s->x[1], &s->x[2], &s->v[0], &s->v[1], &s->v[2], &s->f[0], &s->f[1], &s->f[2],
        &s->xref[0], &s->xref[1], &s->xref[2], &s->img[0], &s->img[1], &s->img[2], &s->type,
        &s->q, &s->invm, &s->mass, &s->specbond, &s->num3bond, &s->ljtab, &s->col_count,
        &s->col_start, &s->col_fill, &s->col_atoms, &s->col_key, &s->cl_start, &s->slot_orig,
        &s->rec, &s->bb, &s->jlist, &s->jmask, &s->jcount, &s->nclusters, &s->recf, &s->fslot,
        &s->atom_slot, &s->status_local, &s->energy, &s->red, &s->flag, &s->stage_pos,
        &s->stage_ff, &s->cl_pos, &s->cl_gid, &s->ptta, &s->ilist, &s->imask, &s->icount,
        &s->xprn[0], &s->xprn[1], &s->xprn[2], &s->part, &s->dcount, &md.bonds, &md.bcoef,
        &md.angles, &md.acoef, &md.diheds, &md.dcoef, &md.lj14, &md.shake, &md.sbond, &md.impros,
        &md.icoef, &md.eterm, &md.ered, &md.bpart, &md.step_dev, &md.snap[0], &md.snap[1],
        &md.snap[2], &md.snap[3], &md.snap[4], &md.snap[5], &md.snap[6], &md.keep[0], &md.keep[1],
        &md.keep[2], &md.keep[3], &md.keep[4], &md.keep[5], &md.keep[6]};
    int64_t total = 0;
    for (const sofia::DevBuf *b : bufs) total += (int64_t)b->bytes;
    *bytes = total;
    return SOFIA_OK;
}

// Thermostat step counter (the Philox counter of the Langevin noise): read it
// for a checkpoint, set it when resuming one so the noise sequence continues.
extern "C" int sofia_system_md_get_step(sofia_system *ss, long long *step) {
    if (!ss || !step) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    if (!s->md.ready) return sofia::fail(s->ctx, SOFIA_ESTATE, "md_get_step: MD is not set up");
    SOFIA_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
    SOFIA_CUDA(s->ctx, cudaMemcpyAsync(step, s->md.step_dev.p, sizeof(long long),
                                       cudaMemcpyDeviceToHost, s->ctx->stream));
    SOFIA_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return SOFIA_OK;
}

extern "C" int sofia_system_md_set_step(sofia_system *ss, long long step) {
    if (!ss || step < 0) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    if (!s->md.ready) return sofia::fail(s->ctx, SOFIA_ESTATE, "md_set_step: MD is not set up");
    SOFIA_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
    SOFIA_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    SOFIA_CUDA(s->ctx, cudaMemcpy(s->md.step_dev.p, &step, sizeof(long long),
                                  cudaMemcpyHostToDevice));
    s->md.step = step;
    return SOFIA_OK;
}
