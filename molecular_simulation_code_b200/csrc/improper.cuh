// Harmonic improper torsion of improper_harmonic_lammps14
// (Source/mod_force_dihed.f90:1546-1724), FP64, shared by the reference-semantics
// entry point (ref_kernels.cu) and the device MD term (md.cu).
//
// Atoms 1..4 with bond vectors v1 = x1 - x2, v2 = x3 - x2, v3 = x4 - x3 (minimum
// image taken by the caller).  The angle omega between the planes (1,2,3) and
// (2,3,4) gives E = k (omega - omega0)^2; f1..f4 receive the forces and vir the
// diagonal virial v1*f1 + v2*f3 + (v3 + v2)*f4.  Degenerate geometries are
// floored at 0.001 like the reference (its SMALL); cos(omega) is clamped to
// [-1, 1] (the reference only prints when it is out of range).
#pragma once

namespace sofia {

struct ImproperOut {
    double e;
    double f1[3], f2[3], f3[3], f4[3];
    double vir[3];
};

__host__ __device__ inline ImproperOut improper_harmonic(const double v1[3], const double v2[3],
                                                         const double v3[3], double k,
                                                         double omega0) {
    const double SMALL = (double)0.001f;  // real*4 literal in the reference
    const double ss1 = 1.0 / (v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
    const double ss2 = 1.0 / (v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
    const double ss3 = 1.0 / (v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
    const double r1 = sqrt(ss1), r2 = sqrt(ss2), r3 = sqrt(ss3);
    const double c0 = (v1[0] * v3[0] + v1[1] * v3[1] + v1[2] * v3[2]) * r1 * r3;
    const double c1 = (v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2]) * r1 * r2;
    const double c2 = -(v3[0] * v2[0] + v3[1] * v2[1] + v3[2] * v2[2]) * r3 * r2;
    double s1 = 1.0 - c1 * c1;
    if (s1 < SMALL) s1 = SMALL;
    s1 = 1.0 / s1;
    double s2 = 1.0 - c2 * c2;
    if (s2 < SMALL) s2 = SMALL;
    s2 = 1.0 / s2;
    double s12 = sqrt(s1 * s2);
    double c = (c1 * c2 + c0) * s12;
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    double s = sqrt(1.0 - c * c);
    if (s < SMALL) s = SMALL;
    const double domega = acos(c) - omega0;
    double a = k * domega;
    ImproperOut o;
    o.e = a * domega;
    a = -a * 2.0 / s;
    c = c * a;
    s12 = s12 * a;
    const double a11 = c * ss1 * s1;
    const double a22 = -ss2 * (2.0 * c0 * s12 - c * (s1 + s2));
    const double a33 = c * ss3 * s2;
    const double a12 = -r1 * r2 * (c1 * c * s1 + c2 * s12);
    const double a13 = -r1 * r3 * s12;
    const double a23 = r2 * r3 * (c2 * c * s2 + c1 * s12);
    for (int d = 0; d < 3; ++d) {
        const double sx2 = a22 * v2[d] + a23 * v3[d] + a12 * v1[d];
        o.f1[d] = a12 * v2[d] + a13 * v3[d] + a11 * v1[d];
        o.f2[d] = -sx2 - o.f1[d];
        o.f4[d] = a23 * v2[d] + a33 * v3[d] + a13 * v1[d];
        o.f3[d] = sx2 - o.f4[d];
        o.vir[d] = v1[d] * o.f1[d] + v2[d] * o.f3[d] + (v3[d] + v2[d]) * o.f4[d];
    }
    return o;
}

}  // namespace sofia
