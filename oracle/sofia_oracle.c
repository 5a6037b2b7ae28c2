/*
 * sofia_oracle.c -- CPU restatement of the Sofia nonbonded hot path.
 *
 * TEST INFRASTRUCTURE ONLY (checker + timed CPU baseline).  PARITY UNPINNED:
 * the Fortran reference cannot be built here and ships no golden outputs.
 *
 * Every routine names the reference file:line it restates.  Arithmetic keeps
 * the Fortran types and evaluation order: real*4 where the reference stores or
 * computes in real*4, real*8 otherwise, single-precision literals rounded to
 * float, no FMA contraction (build with -ffp-contract=off, no fast-math).
 */
#include "sofia_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO23F 8388608.0f            /* 1/epsilon(real*4) */
#define TWO52 4503599627370496.0     /* 1/epsilon(real*8) */

/* get_started.f90:25-117 (init): constants with the reference's literal precision. */
void orc_init_params(orc_params *p, double alpha, float box, float cut_coul, float rcut,
                     float neighbor_pad) {
    memset(p, 0, sizeof(*p));
    p->alpha = alpha;
    p->EWALD_F = (double)1.12837917f;
    p->EWALD_P = (double)0.3275911f;
    p->A1 = (double)0.254829592f;
    p->A2 = (double)-0.284496736f;
    p->A3 = (double)1.421413741f;
    p->A4 = (double)-1.453152027f;
    p->A5 = (double)1.061405429f;
    p->MY_PIS = (double)1.77245385090551602729f; /* single-precision literal (:109) */
    p->MY_PIS_INV = 1.0 / p->MY_PIS;
    p->coulpre = 332.06371f; /* real*4 (global.f90:73) */
    p->box = box;
    p->ibox = (float)(1.0 / (double)box);         /* ibox = 1.0d0/box stored real*4 (:66) */
    p->vol = (box * box) * box;                   /* vol = box**3, real*4 (:64) */
    p->cut_coul = cut_coul;
    p->rcut = rcut;
    p->neighbor_pad = neighbor_pad;
    p->rcut2 = (double)(rcut * rcut);             /* real*4 product (:74) */
    p->cut_coulsq = (double)(cut_coul * cut_coul);
    p->rv = (double)(neighbor_pad + cut_coul);    /* real*4 sum (:45) */
    p->rv2 = p->rv * p->rv;
    p->rvrc2 = (double)neighbor_pad * (double)neighbor_pad;
    {
        double cc = (double)cut_coul;
        double erfcc = erfc(alpha * cc);
        double erfcd = exp(-(((alpha * alpha) * cc) * cc));
        p->f_shift = -(erfcc / p->cut_coulsq + (((2.0 / p->MY_PIS) * alpha) * erfcd) / cc);
        p->e_shift = erfcc / cc - p->f_shift * cc;
    }
}

/* get_started.f90:147-173 (calculate_gewald): bisection for erfc(g rc)/rc = 1e-6 */
double orc_calculate_gewald(float cut_coul) {
    double tol = (double)0.000001f;
    double cc = (double)cut_coul;
    double lo = 0.0, hi = 1.0, g = 1.0;
    for (int i = 0; i < 100; ++i) {
        g = 0.5 * (lo + hi);
        if (erfc(g * cc) / cc > tol) lo = g;
        else hi = g;
    }
    return g;
}

/* mod_neighbor.f90:1434-1452 (check_allocation): cell edge and counts. */
void orc_cell_grid(float box, float vol, float cut_coul, float rcut, float *rn, int *ncellT,
                   int *ncellD) {
    float c = (cut_coul > rcut) ? cut_coul : rcut;
    int nside = (int)(box / c);                 /* int() truncates */
    float r = box / (float)nside;               /* real*4 / integer in real*4 */
    float r3 = (r * r) * r;
    *rn = r;
    *ncellT = (int)lroundf(vol / r3);           /* nint */
    *ncellD = (int)lround(pow((double)(*ncellT), 1.0 / 3.0));
}

/* mod_neighbor.f90:1309-1378 (neighcell_nonewton): self cell, then the 26
 * neighbours in (iz,iy,ix) loop order with periodic wrap. */
void orc_stencil(int ncellT, int ncellD, int32_t *cnum) {
    int count = 0;
    for (int ic = 0; ic < ncellT; ++ic) {
        cnum[count] = ic;
        int icz = ic / (ncellD * ncellD);
        int icy = (ic - icz * ncellD * ncellD) / ncellD;
        int icx = ic - icy * ncellD - icz * ncellD * ncellD;
        for (int iz = -1; iz <= 1; ++iz)
            for (int iy = -1; iy <= 1; ++iy)
                for (int ix = -1; ix <= 1; ++ix) {
                    int zc = icz + iz, yc = icy + iy, xc = icx + ix;
                    zc = zc < 0 ? zc + ncellD : (zc >= ncellD ? zc - ncellD : zc);
                    yc = yc < 0 ? yc + ncellD : (yc >= ncellD ? yc - ncellD : yc);
                    xc = xc < 0 ? xc + ncellD : (xc >= ncellD ? xc - ncellD : xc);
                    if (iz != 0 || iy != 0 || ix != 0) {
                        count++;
                        cnum[count] = xc + yc * ncellD + zc * ncellD * ncellD;
                    }
                }
        count++;
    }
}

/* mod_neighbor.f90:1381-1424 (xyz2bin): binning in double from real*4 coordinates. */
int orc_xyz2bin(float x, float y, float z, float box, float rn, int ncellD) {
    double irn = 1.0 / (double)rn, b = (double)box;
    int ix = ((double)x < b) ? (int)((double)x * irn) : ncellD - 1;
    int iy = ((double)y < b) ? (int)((double)y * irn) : ncellD - 1;
    int iz = ((double)z < b) ? (int)((double)z * irn) : ncellD - 1;
    if (ix == ncellD) ix = ncellD - 1;
    if (iy == ncellD) iy = ncellD - 1;
    if (iz == ncellD) iz = ncellD - 1;
    return ix + iy * ncellD + iz * ncellD * ncellD;
}

/* mod_neighbor.f90:923-942 (new_nlist) + :946-1005 (sort_posit_charge):
 * head-of-chain linked cells (LIFO), then cells in ascending order. */
void orc_bin_sort(int np, const orc_ainfo *pos, float box, float rn, int ncellT, int ncellD,
                  int32_t *tt, int32_t *ttb, int32_t *start, int32_t *endposit,
                  int32_t *atombin) {
    int32_t *hoc = (int32_t *)calloc((size_t)ncellT + 1, sizeof(int32_t));
    int32_t *ll = (int32_t *)malloc(sizeof(int32_t) * (size_t)(np + 1));
    for (int i = 1; i <= np; ++i) {
        int icell = orc_xyz2bin(pos[i - 1].x, pos[i - 1].y, pos[i - 1].z, box, rn, ncellD);
        ll[i] = hoc[icell];
        hoc[icell] = i;
    }
    int count = 1;
    for (int c = 0; c < ncellT; ++c) {
        int j = hoc[c];
        start[c] = count;
        while (j != 0) {
            tt[j - 1] = count;
            ttb[count - 1] = j;
            atombin[count - 1] = c;
            j = ll[j];
            count++;
        }
        endposit[c] = count - 1;
    }
    free(hoc);
    free(ll);
}

/* mod_neighbor.f90:622-809 (build_neighbor_nonewton_nomic): pass 1 fills the
 * float32 dr2 of every 27-cell candidate (magic-number minimum image,
 * :688-705), pass 2 keeps z /= i, dr2 < rv2 (double) and z not in
 * specbond(1:num3bond(i)) (:714-742).  The two passes are fused here; the
 * value tested is the same real*4 dr2. */
int orc_build_neighbor_nonewton(const orc_params *p, int np, const orc_ainfo *pos,
                                const int32_t *atombin, const int32_t *start,
                                const int32_t *endposit, const int32_t *cnum,
                                const int32_t *specbond, const int32_t *num3bond,
                                int32_t *nlist, int32_t *numneigh, int neigh_alloc,
                                int nthreads) {
    const float box = p->box, ibox = p->ibox;
    const double rv2 = p->rv2;
    int maxn = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(max : maxn)
#endif
    for (int i = 1; i <= np; ++i) {
        const float x1 = pos[i - 1].x, y1 = pos[i - 1].y, z1 = pos[i - 1].z;
        const int bin = atombin[i - 1];
        const int n3 = num3bond[i - 1];
        const int32_t *bonds = specbond + (size_t)(i - 1) * 12;
        const size_t n0 = (size_t)(i - 1) * (size_t)neigh_alloc;
        int nnpt = 0;
        for (int k = bin * 27; k <= bin * 27 + 26; ++k) {
            int cell = cnum[k];
            for (int z = start[cell]; z <= endposit[cell]; ++z) {
                float dx = x1 - pos[z - 1].x;
                float dy = y1 - pos[z - 1].y;
                float dz = z1 - pos[z - 1].z;
                float bx = dx * ibox, by = dy * ibox, bz = dz * ibox;
                bx = (bx + copysignf(TWO23F, bx)) - copysignf(TWO23F, dx);
                by = (by + copysignf(TWO23F, by)) - copysignf(TWO23F, dy);
                bz = (bz + copysignf(TWO23F, bz)) - copysignf(TWO23F, dz);
                dx = dx - bx * box;
                dy = dy - by * box;
                dz = dz - bz * box;
                float dr2 = dx * dx + dy * dy + dz * dz;
                if (z != i && (double)dr2 < rv2) {
                    int keep = 1;
                    for (int l = 0; l < n3; ++l)
                        if (bonds[l] == z) keep = 0;
                    if (keep) {
                        nnpt++;
                        if (nnpt <= neigh_alloc) nlist[n0 + (size_t)nnpt - 1] = z;
                    }
                }
            }
        }
        numneigh[i - 1] = nnpt;
        if (nnpt > maxn) maxn = nnpt;
    }
    return maxn;
}

/* neighbor_wrapper (mod_neighbor.f90:8-86) on unsorted input: bin, sort,
 * remap specbond through tt (sort_specbond_numbond :1011-1039), build, then map
 * the list back to the input index space. */
int orc_neighbor_wrapper(const orc_params *p, int np, const orc_ainfo *pos,
                         const int32_t *specbond, const int32_t *num3bond, int32_t *nlist,
                         int32_t *numneigh, int neigh_alloc, int nthreads) {
    float rn;
    int ncellT, ncellD;
    orc_cell_grid(p->box, p->vol, p->cut_coul, p->rcut, &rn, &ncellT, &ncellD);
    int32_t *cnum = (int32_t *)malloc(sizeof(int32_t) * 27 * (size_t)ncellT);
    orc_stencil(ncellT, ncellD, cnum);
    int32_t *tt = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    int32_t *ttb = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    int32_t *st = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncellT);
    int32_t *en = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncellT);
    int32_t *ab = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    orc_bin_sort(np, pos, p->box, rn, ncellT, ncellD, tt, ttb, st, en, ab);
    orc_ainfo *ps = (orc_ainfo *)malloc(sizeof(orc_ainfo) * (size_t)np);
    int32_t *sb = (int32_t *)calloc((size_t)np * 12, sizeof(int32_t));
    int32_t *n3 = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    for (int s = 0; s < np; ++s) {
        int o = ttb[s] - 1;
        ps[s] = pos[o];
        n3[s] = num3bond[o];
        for (int l = 0; l < num3bond[o]; ++l) sb[(size_t)s * 12 + l] = tt[specbond[(size_t)o * 12 + l] - 1];
    }
    int32_t *nl = (int32_t *)malloc(sizeof(int32_t) * (size_t)np * (size_t)neigh_alloc);
    int32_t *nn = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    int maxn = orc_build_neighbor_nonewton(p, np, ps, ab, st, en, cnum, sb, n3, nl, nn,
                                           neigh_alloc, nthreads);
    for (int s = 0; s < np; ++s) {
        int o = ttb[s] - 1;
        numneigh[o] = nn[s];
        int m = nn[s] < neigh_alloc ? nn[s] : neigh_alloc;
        for (int j = 0; j < m; ++j)
            nlist[(size_t)o * neigh_alloc + j] = ttb[nl[(size_t)s * neigh_alloc + j] - 1];
    }
    free(cnum); free(tt); free(ttb); free(st); free(en); free(ab); free(ps); free(sb);
    free(n3); free(nl); free(nn);
    return maxn;
}

/* mod_neighbor.f90:814-861 (build_neighbor_n2_nonewton): all-pairs list. */
int orc_build_neighbor_n2(const orc_params *p, int np, const orc_ainfo *pos,
                          const int32_t *specbond, const int32_t *num3bond, int32_t *nlist,
                          int32_t *numneigh, int neigh_alloc) {
    const float box = p->box, ibox = p->ibox;
    int maxn = 0;
    for (int i = 1; i <= np; ++i) {
        const float x1 = pos[i - 1].x, y1 = pos[i - 1].y, z1 = pos[i - 1].z;
        int nnpt = 0;
        for (int j = 1; j <= np; ++j) {
            if (i == j) continue;
            float dx = x1 - pos[j - 1].x, dy = y1 - pos[j - 1].y, dz = z1 - pos[j - 1].z;
            float bx = dx * ibox, by = dy * ibox, bz = dz * ibox;
            bx = (bx + copysignf(TWO23F, bx)) - copysignf(TWO23F, dx);
            by = (by + copysignf(TWO23F, by)) - copysignf(TWO23F, dy);
            bz = (bz + copysignf(TWO23F, bz)) - copysignf(TWO23F, dz);
            dx = dx - box * bx;
            dy = dy - box * by;
            dz = dz - box * bz;
            float dr2 = dx * dx + dy * dy + dz * dz;
            int excl = 0;
            for (int m = 0; m < num3bond[i - 1]; ++m)
                if (specbond[(size_t)(i - 1) * 12 + m] == j) excl = 1;
            if (!excl && (double)dr2 < p->rv2) {
                nnpt++;
                if (nnpt <= neigh_alloc) nlist[(size_t)(i - 1) * neigh_alloc + nnpt - 1] = j;
            }
        }
        numneigh[i - 1] = nnpt;
        if (nnpt > maxn) maxn = nnpt;
    }
    return maxn;
}

/* mod_neighbor.f90:895-913 (check_neighbor): any atom moved >= the full skin. */
int orc_check_neighbor(int np, const float *drx, const float *dry, const float *drz,
                       double rvrc2) {
    int flag = 0;
    for (int i = 0; i < np; ++i) {
        double dr2 = (double)(drx[i] * drx[i] + dry[i] * dry[i] + drz[i] * drz[i]);
        if (dr2 >= rvrc2) flag = 1;
    }
    return flag;
}

/* mod_force_nonbond.f90:105-196 (lj_cut_coul_dsf_nonewton_NOMIC): FP64 pair
 * arithmetic on the real*4 module arrays over the full list.  The reference
 * accumulates potential/e_coul in an OpenMP reduction of unspecified order;
 * here per-atom partial sums are added in atom order so the result does not
 * depend on the thread count. */
void orc_force_dsf_nonewton(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                            const float *lj1, const float *lj2, const float *lj3,
                            const float *lj4, int ntypes, const int32_t *nlist,
                            const int32_t *numneigh, int neigh_alloc, float *ff,
                            double *potential, double *e_coul, double *virial3,
                            double *ff64, int nthreads) {
    const double box = (double)p->box, ibox = (double)p->ibox;
    const double rcut2 = p->rcut2, cut_coulsq = p->cut_coulsq, alpha = p->alpha;
    const double coulpre = (double)p->coulpre;
    const double EWALD_P = p->EWALD_P, A1 = p->A1, A2 = p->A2, A3 = p->A3, A4 = p->A4,
                 A5 = p->A5, MY_PIS_INV = p->MY_PIS_INV, e_shift = p->e_shift,
                 f_shift = p->f_shift;
    double *pe = (double *)malloc(sizeof(double) * (size_t)np * 5);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 32) num_threads(nthreads)
#endif
    for (int i = 1; i <= np; ++i) {
        const double x1 = pos[i - 1].x, y1 = pos[i - 1].y, z1 = pos[i - 1].z;
        const int itype = pos[i - 1].type;
        const double qtmp = q[i - 1];
        const int ioffset = (itype - 1) * ntypes;
        const size_t neigh_off = (size_t)neigh_alloc * (size_t)(i - 1);
        const int num = numneigh[i - 1];
        double ffx = 0.0, ffy = 0.0, ffz = 0.0, pot = 0.0, ec = 0.0;
        double vx = 0.0, vy = 0.0, vz = 0.0;
        for (int j = 1; j <= num; ++j) {
            const int neigh = nlist[neigh_off + j - 1];
            double dx = x1 - (double)pos[neigh - 1].x;
            double dy = y1 - (double)pos[neigh - 1].y;
            double dz = z1 - (double)pos[neigh - 1].z;
            const int jtype = pos[neigh - 1].type;
            double bx = dx * ibox, by = dy * ibox, bz = dz * ibox;
            bx = (bx + copysign(TWO52, bx)) - copysign(TWO52, dx);
            by = (by + copysign(TWO52, by)) - copysign(TWO52, dy);
            bz = (bz + copysign(TWO52, bz)) - copysign(TWO52, dz);
            dx = dx - box * bx;
            dy = dy - box * by;
            dz = dz - box * bz;
            const double dr2 = dx * dx + dy * dy + dz * dz;
            const double dr2i = 1.0 / dr2;
            double dr6i = dr2i * dr2i * dr2i;
            if (dr2 > rcut2) dr6i = 0.0;
            const int offset = ioffset + jtype - 1;
            const double forcelj = dr6i * ((double)lj1[offset] * dr6i - (double)lj2[offset]);
            pot = pot + dr6i * (dr6i * (double)lj3[offset] - (double)lj4[offset]);
            const double r = sqrt(dr2);
            const double dri = 1.0 / r;
            double prefactor = coulpre * qtmp * (double)q[neigh - 1] * dri;
            if (dr2 > cut_coulsq) prefactor = 0.0;
            const double erfcd = exp(-(((alpha * alpha) * r) * r));
            const double t = 1.0 / (1.0 + (EWALD_P * alpha) * r);
            const double erfcc = t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * erfcd;
            const double forcecoul =
                prefactor * (erfcc * dri + ((2.0 * alpha) * MY_PIS_INV) * erfcd + r * f_shift) * r;
            ec = ec + prefactor * ((erfcc - r * e_shift) - dr2 * f_shift);
            const double force = (forcecoul + forcelj) * dr2i;
            ffx = ffx + dx * force;
            ffy = ffy + dy * force;
            ffz = ffz + dz * force;
            vx += dx * dx * force;
            vy += dy * dy * force;
            vz += dz * dz * force;
        }
        ff[(size_t)(i - 1) * 3 + 0] = (float)ffx;
        ff[(size_t)(i - 1) * 3 + 1] = (float)ffy;
        ff[(size_t)(i - 1) * 3 + 2] = (float)ffz;
        if (ff64) {
            ff64[(size_t)(i - 1) * 3 + 0] = ffx;
            ff64[(size_t)(i - 1) * 3 + 1] = ffy;
            ff64[(size_t)(i - 1) * 3 + 2] = ffz;
        }
        pe[(size_t)(i - 1) * 5 + 0] = pot;
        pe[(size_t)(i - 1) * 5 + 1] = ec;
        pe[(size_t)(i - 1) * 5 + 2] = vx;
        pe[(size_t)(i - 1) * 5 + 3] = vy;
        pe[(size_t)(i - 1) * 5 + 4] = vz;
    }
    double sp = 0.0, se = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 0; i < np; ++i) {
        sp += pe[(size_t)i * 5 + 0];
        se += pe[(size_t)i * 5 + 1];
        sx += pe[(size_t)i * 5 + 2];
        sy += pe[(size_t)i * 5 + 3];
        sz += pe[(size_t)i * 5 + 4];
    }
    free(pe);
    *potential = 0.50 * sp; /* :193-194 */
    *e_coul = 0.50 * se;
    if (virial3) {
        virial3[0] = 0.5 * sx;
        virial3[1] = 0.5 * sy;
        virial3[2] = 0.5 * sz;
    }
}

/* mod_force_nonbond.f90:300-400 (lj_cut_coul_long_nonewton_NOMIC; the _MIC
 * variant at :201-298 has the same arithmetic): real-space Ewald/PME pair term
 * with LJ over the full list, all pair arithmetic in real*4.  Mixed-mode
 * statements follow Fortran promotion: dr2i = 1.0d0/dr2, grij = gewald*r,
 * t = 1.0/(1.0+EWALD_P*grij), the erfc polynomial and forcecoul are computed
 * in double and stored to real*4; the real*4 exp(-grij*grij) is taken as the
 * correctly rounded single-precision exponential, (float)exp((double)x).
 * Force and virial terms are real*4 products added into double sums. */
void orc_force_long_nonewton(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                             const float *lj1, const float *lj2, const float *lj3,
                             const float *lj4, int ntypes, const int32_t *nlist,
                             const int32_t *numneigh, int neigh_alloc, double gewald, float *ff,
                             double *potential, double *e_coul, double *virial3,
                             double *ff64, int nthreads) {
    const float box = p->box, ibox = p->ibox, coulpre = p->coulpre;
    const double rcut2 = p->rcut2, cut_coulsq = p->cut_coulsq;
    const double EWALD_F = p->EWALD_F, EWALD_P = p->EWALD_P, A1 = p->A1, A2 = p->A2,
                 A3 = p->A3, A4 = p->A4, A5 = p->A5;
    const float TWO23 = 8388608.0f; /* 1/epsilon(real*4) */
    double *pe = (double *)malloc(sizeof(double) * (size_t)np * 5);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 32) num_threads(nthreads)
#endif
    for (int i = 1; i <= np; ++i) {
        const float x1 = pos[i - 1].x, y1 = pos[i - 1].y, z1 = pos[i - 1].z;
        const int itype = pos[i - 1].type;
        const float qtmp = q[i - 1];
        const int ioffset = (itype - 1) * ntypes;
        const size_t neigh_off = (size_t)neigh_alloc * (size_t)(i - 1);
        const int num = numneigh[i - 1];
        double ffx = 0.0, ffy = 0.0, ffz = 0.0, pot = 0.0, ec = 0.0;
        double vx = 0.0, vy = 0.0, vz = 0.0;
        for (int j = 1; j <= num; ++j) {
            const int neigh = nlist[neigh_off + j - 1];
            float dx = x1 - pos[neigh - 1].x;
            float dy = y1 - pos[neigh - 1].y;
            float dz = z1 - pos[neigh - 1].z;
            const int jtype = pos[neigh - 1].type;
            float bx = dx * ibox, by = dy * ibox, bz = dz * ibox;
            bx = (bx + copysignf(TWO23, bx)) - copysignf(TWO23, dx);
            by = (by + copysignf(TWO23, by)) - copysignf(TWO23, dy);
            bz = (bz + copysignf(TWO23, bz)) - copysignf(TWO23, dz);
            dx = dx - box * bx;
            dy = dy - box * by;
            dz = dz - box * bz;
            const float dr2 = dx * dx + dy * dy + dz * dz;
            const float dr2i = (float)(1.0 / (double)dr2);
            float dr6i = dr2i * dr2i * dr2i;
            if ((double)dr2 > rcut2) dr6i = 0.0f;
            const int offset = ioffset + jtype - 1;
            const float forcelj = dr6i * (lj1[offset] * dr6i - lj2[offset]);
            pot = pot + (double)(dr6i * (dr6i * lj3[offset] - lj4[offset]));
            const float r = sqrtf(dr2);
            float prefactor = coulpre * qtmp * q[neigh - 1] / r;
            const float grij = (float)(gewald * (double)r);
            const float expm2 = (float)exp((double)(-(grij * grij)));
            const float t = (float)(1.0 / (1.0 + EWALD_P * (double)grij));
            const double td = (double)t;
            const float erfc_ = (float)(td * (A1 + td * (A2 + td * (A3 + td * (A4 + td * A5)))) *
                                        (double)expm2);
            if ((double)dr2 > cut_coulsq) prefactor = 0.0f;
            const float forcecoul = (float)((double)prefactor *
                                            ((double)erfc_ + EWALD_F * (double)grij * (double)expm2));
            ec = ec + (double)(prefactor * erfc_);
            const float force = (forcecoul + forcelj) * dr2i;
            ffx = ffx + (double)(dx * force);
            ffy = ffy + (double)(dy * force);
            ffz = ffz + (double)(dz * force);
            vx += (double)(dx * dx * force);
            vy += (double)(dy * dy * force);
            vz += (double)(dz * dz * force);
        }
        ff[(size_t)(i - 1) * 3 + 0] = (float)ffx;
        ff[(size_t)(i - 1) * 3 + 1] = (float)ffy;
        ff[(size_t)(i - 1) * 3 + 2] = (float)ffz;
        if (ff64) {
            ff64[(size_t)(i - 1) * 3 + 0] = ffx;
            ff64[(size_t)(i - 1) * 3 + 1] = ffy;
            ff64[(size_t)(i - 1) * 3 + 2] = ffz;
        }
        pe[(size_t)(i - 1) * 5 + 0] = pot;
        pe[(size_t)(i - 1) * 5 + 1] = ec;
        pe[(size_t)(i - 1) * 5 + 2] = vx;
        pe[(size_t)(i - 1) * 5 + 3] = vy;
        pe[(size_t)(i - 1) * 5 + 4] = vz;
    }
    double sp = 0.0, se = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 0; i < np; ++i) {
        sp += pe[(size_t)i * 5 + 0];
        se += pe[(size_t)i * 5 + 1];
        sx += pe[(size_t)i * 5 + 2];
        sy += pe[(size_t)i * 5 + 3];
        sz += pe[(size_t)i * 5 + 4];
    }
    free(pe);
    *potential = 0.50 * sp; /* :395-397 */
    *e_coul = 0.50 * se;
    if (virial3) {
        virial3[0] = 0.5 * sx; /* virialx = 0.50*vvx, :387-389 */
        virial3[1] = 0.5 * sy;
        virial3[2] = 0.5 * sz;
    }
}

/* mod_force_nonbond.f90:409-502 (lj_cut_coul_dsf_N2): O(N^2) pairs i<j with
 * NINT minimum image, a single dr2 < rcut2 gate, 1-2/1-3 weight 0 and 1-4
 * weight 0.5 from specbond.  Accumulates in double (the reference rounds ff to
 * real*4 at every pair). */
void orc_force_dsf_n2(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                      const float *lj1, const float *lj2, const float *lj3, const float *lj4,
                      int ntypes, const int32_t *specbond, const int32_t *num1bond,
                      const int32_t *num2bond, const int32_t *num3bond, double *ff64,
                      double *potential, double *e_coul) {
    (void)num1bond;
    const double box = (double)p->box, ibox = (double)p->ibox;
    const double alpha = p->alpha, coulpre = (double)p->coulpre;
    double pot = 0.0, ec = 0.0;
    memset(ff64, 0, sizeof(double) * 3 * (size_t)np);
    for (int i = 1; i < np; ++i) {
        const double x1 = pos[i - 1].x, y1 = pos[i - 1].y, z1 = pos[i - 1].z;
        const int itype = pos[i - 1].type;
        const double qtmp = q[i - 1];
        const int n2 = num2bond[i - 1], n3 = num3bond[i - 1];
        for (int j = i + 1; j <= np; ++j) {
            double dx = x1 - (double)pos[j - 1].x;
            double dy = y1 - (double)pos[j - 1].y;
            double dz = z1 - (double)pos[j - 1].z;
            dx = dx - box * (double)lround(dx * ibox);
            dy = dy - box * (double)lround(dy * ibox);
            dz = dz - box * (double)lround(dz * ibox);
            const double dr2 = dx * dx + dy * dy + dz * dz;
            if (!(dr2 < p->rcut2)) continue;
            double fudge = 1.0;
            for (int l = 1; l <= n3; ++l) {
                if (specbond[(size_t)(i - 1) * 12 + l - 1] == j) fudge = (l <= n2) ? 0.0 : 0.5;
            }
            const int jtype = pos[j - 1].type;
            const double dr2i = 1.0 / dr2;
            const double dr6i = dr2i * dr2i * dr2i;
            const int offset = ntypes * (itype - 1) + jtype - 1;
            const double forcelj = dr6i * ((double)lj1[offset] * dr6i - (double)lj2[offset]);
            pot = pot + fudge * dr6i * ((double)lj3[offset] * dr6i - (double)lj4[offset]);
            const double r = sqrt(dr2);
            const double dri = 1.0 / r;
            double prefactor = coulpre * qtmp * (double)q[j - 1] * dri;
            if (dr2 > p->cut_coulsq) prefactor = 0.0;
            const double erfcd = exp(-(((alpha * alpha) * r) * r));
            const double t = 1.0 / (1.0 + (p->EWALD_P * alpha) * r);
            const double erfcc =
                t * (p->A1 + t * (p->A2 + t * (p->A3 + t * (p->A4 + t * p->A5)))) * erfcd;
            const double forcecoul =
                prefactor * (erfcc * dri + ((2.0 * alpha) * p->MY_PIS_INV) * erfcd + r * p->f_shift) * r;
            ec = ec + fudge * prefactor * ((erfcc - r * p->e_shift) - dr2 * p->f_shift);
            const double force = fudge * (forcecoul + forcelj) * dr2i;
            ff64[(size_t)(i - 1) * 3 + 0] += dx * force;
            ff64[(size_t)(i - 1) * 3 + 1] += dy * force;
            ff64[(size_t)(i - 1) * 3 + 2] += dz * force;
            ff64[(size_t)(j - 1) * 3 + 0] -= dx * force;
            ff64[(size_t)(j - 1) * 3 + 1] -= dy * force;
            ff64[(size_t)(j - 1) * 3 + 2] -= dz * force;
        }
    }
    *potential = pot;
    *e_coul = ec;
}

/* mod_minimg.f90:5-15: d -= box*nint(ibox*d); box*nint() is a real*4 product. */
static inline double minimg1(double d, float box, float ibox) {
    long k = lround((double)ibox * d);
    float s = box * (float)k;
    return d - (double)s;
}

/* mod_force_dihed.f90:1546-1724 (improper_harmonic_lammps14): bond vectors from
 * real*4 coordinate differences with the NINT minimum image, FP64 angle math,
 * forces added to the real*4 ff_impro after every improper, energy and the
 * diagonal virial into double accumulators.  omega0 = improcoeff(2,type). */
void orc_improper_harmonic(const orc_params *p, int np, const orc_ainfo *pos, int nimpro,
                           const int32_t *improlist, const double *improcoeff, float *ff_impro,
                           double *e_improper, double *v_impro3) {
    (void)np;
    const float box = p->box, ibox = p->ibox;
    const double SMALL = (double)0.001f;
    for (int m = 0; m < nimpro; ++m) {
        const int i1 = improlist[5 * m] - 1, i2 = improlist[5 * m + 1] - 1,
                  i3 = improlist[5 * m + 2] - 1, i4 = improlist[5 * m + 3] - 1,
                  t = improlist[5 * m + 4] - 1;
        const double v1x = minimg1((double)(pos[i1].x - pos[i2].x), box, ibox);
        const double v1y = minimg1((double)(pos[i1].y - pos[i2].y), box, ibox);
        const double v1z = minimg1((double)(pos[i1].z - pos[i2].z), box, ibox);
        const double v2x = minimg1((double)(pos[i3].x - pos[i2].x), box, ibox);
        const double v2y = minimg1((double)(pos[i3].y - pos[i2].y), box, ibox);
        const double v2z = minimg1((double)(pos[i3].z - pos[i2].z), box, ibox);
        const double v3x = minimg1((double)(pos[i4].x - pos[i3].x), box, ibox);
        const double v3y = minimg1((double)(pos[i4].y - pos[i3].y), box, ibox);
        const double v3z = minimg1((double)(pos[i4].z - pos[i3].z), box, ibox);
        const double ss1 = 1.0 / (v1x * v1x + v1y * v1y + v1z * v1z);
        const double ss2 = 1.0 / (v2x * v2x + v2y * v2y + v2z * v2z);
        const double ss3 = 1.0 / (v3x * v3x + v3y * v3y + v3z * v3z);
        const double r1 = sqrt(ss1), r2 = sqrt(ss2), r3 = sqrt(ss3);
        const double c0 = (v1x * v3x + v1y * v3y + v1z * v3z) * r1 * r3;
        const double c1 = (v1x * v2x + v1y * v2y + v1z * v2z) * r1 * r2;
        const double c2 = -(v3x * v2x + v3y * v2y + v3z * v2z) * r3 * r2;
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
        const double domega = acos(c) - improcoeff[2 * t + 1];
        double a = improcoeff[2 * t] * domega;
        *e_improper += a * domega;
        a = -a * 2.0 / s;
        c = c * a;
        s12 = s12 * a;
        const double a11 = c * ss1 * s1;
        const double a22 = -ss2 * (2.0 * c0 * s12 - c * (s1 + s2));
        const double a33 = c * ss3 * s2;
        const double a12 = -r1 * r2 * (c1 * c * s1 + c2 * s12);
        const double a13 = -r1 * r3 * s12;
        const double a23 = r2 * r3 * (c2 * c * s2 + c1 * s12);
        const double v1[3] = {v1x, v1y, v1z}, v2[3] = {v2x, v2y, v2z}, v3[3] = {v3x, v3y, v3z};
        float *f = ff_impro;
        for (int d = 0; d < 3; ++d) {
            const double sx2 = a22 * v2[d] + a23 * v3[d] + a12 * v1[d];
            const double f1 = a12 * v2[d] + a13 * v3[d] + a11 * v1[d];
            const double f2 = -sx2 - f1;
            const double f4 = a23 * v2[d] + a33 * v3[d] + a13 * v1[d];
            const double f3 = sx2 - f4;
            /* ff_impro(i)%x = f + ff_impro(i)%x : real*4 store after a double add */
            f[3 * i1 + d] = (float)(f1 + (double)f[3 * i1 + d]);
            f[3 * i2 + d] = (float)(f2 + (double)f[3 * i2 + d]);
            f[3 * i3 + d] = (float)(f3 + (double)f[3 * i3 + d]);
            f[3 * i4 + d] = (float)(f4 + (double)f[3 * i4 + d]);
            /* v_improx = v_improx + v1x*f1 + v2x*f3 + (v3x+v2x)*f4, left to right */
            if (v_impro3) v_impro3[d] = v_impro3[d] + v1[d] * f1 + v2[d] * f3 + (v3[d] + v2[d]) * f4;
        }
    }
}

/* mod_force_dihed.f90:816-1092 (dihedral_opls_DSF): OPLS torsion plus the
 * 0.5-scaled DSF Coulomb and lj14 LJ of the dihedral's 1-4 pair, into ffh. */
void orc_dihedral_opls_dsf(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                           int ntypes, const double *lj14, int ndihed,
                           const int32_t *dihedlist, const double *dihedcoeff, float *ffh,
                           double *e_dihedral, double *e_coul_14, double *pot_14,
                           double *ffh64) {
    (void)np;
    const float box = p->box, ibox = p->ibox;
    const double alpha = p->alpha;
    const double TOLERANCE = (double)0.001f, SMALL = (double)0.001f, SMALLER = (double)0.0001f;
    double edih = 0.0, ec14 = 0.0, p14 = 0.0;
    for (int n = 0; n < ndihed; ++n) {
        const int i1 = dihedlist[n * 5 + 0] - 1, i2 = dihedlist[n * 5 + 1] - 1,
                  i3 = dihedlist[n * 5 + 2] - 1, i4 = dihedlist[n * 5 + 3] - 1,
                  type = dihedlist[n * 5 + 4];
        double vb1x = minimg1((double)(pos[i1].x - pos[i2].x), box, ibox);
        double vb1y = minimg1((double)(pos[i1].y - pos[i2].y), box, ibox);
        double vb1z = minimg1((double)(pos[i1].z - pos[i2].z), box, ibox);
        double vb2x = minimg1((double)(pos[i3].x - pos[i2].x), box, ibox);
        double vb2y = minimg1((double)(pos[i3].y - pos[i2].y), box, ibox);
        double vb2z = minimg1((double)(pos[i3].z - pos[i2].z), box, ibox);
        double vb2xm = minimg1(-vb2x, box, ibox);
        double vb2ym = minimg1(-vb2y, box, ibox);
        double vb2zm = minimg1(-vb2z, box, ibox);
        double vb3x = minimg1((double)(pos[i4].x - pos[i3].x), box, ibox);
        double vb3y = minimg1((double)(pos[i4].y - pos[i3].y), box, ibox);
        double vb3z = minimg1((double)(pos[i4].z - pos[i3].z), box, ibox);
        /* 1-4 pair (:887-895): real*4 difference, then minimum image in double */
        double ddx = minimg1((double)(pos[i1].x - pos[i4].x), box, ibox);
        double ddy = minimg1((double)(pos[i1].y - pos[i4].y), box, ibox);
        double ddz = minimg1((double)(pos[i1].z - pos[i4].z), box, ibox);
        double dr2 = ddx * ddx + ddy * ddy + ddz * ddz;
        int itype = pos[i1].type, jtype = pos[i4].type;

        double sb1 = 1.0 / (vb1x * vb1x + vb1y * vb1y + vb1z * vb1z);
        double sb2 = 1.0 / (vb2x * vb2x + vb2y * vb2y + vb2z * vb2z);
        double sb3 = 1.0 / (vb3x * vb3x + vb3y * vb3y + vb3z * vb3z);
        double rb1 = sqrt(sb1), rb3 = sqrt(sb3);
        double c0 = (vb1x * vb3x + vb1y * vb3y + vb1z * vb3z) * rb1 * rb3;
        double b1mag2 = vb1x * vb1x + vb1y * vb1y + vb1z * vb1z;
        double b1mag = sqrt(b1mag2);
        double b2mag2 = vb2x * vb2x + vb2y * vb2y + vb2z * vb2z;
        double b2mag = sqrt(b2mag2);
        double b3mag2 = vb3x * vb3x + vb3y * vb3y + vb3z * vb3z;
        double b3mag = sqrt(b3mag2);
        double ctmp = vb1x * vb2x + vb1y * vb2y + vb1z * vb2z;
        double r12c1 = 1.0 / (b1mag * b2mag);
        double c1mag = ctmp * r12c1;
        ctmp = vb2xm * vb3x + vb2ym * vb3y + vb2zm * vb3z;
        double r12c2 = 1.0 / (b2mag * b3mag);
        double c2mag = ctmp * r12c2;
        double sin2 = fmax(1.0 - c1mag * c1mag, 0.0);
        double sc1 = sqrt(sin2);
        if (sc1 < SMALL) sc1 = SMALL;
        sc1 = 1.0 / sc1;
        sin2 = fmax(1.0 - c2mag * c2mag, 0.0);
        double sc2 = sqrt(sin2);
        if (sc2 < SMALL) sc2 = SMALL;
        sc2 = 1.0 / sc2;
        double s1 = sc1 * sc1, s2 = sc2 * sc2, s12 = sc1 * sc2;
        double c = (c0 + c1mag * c2mag) * s12;
        (void)TOLERANCE;
        if (c > 1.0) c = 1.0;
        if (c < -1.0) c = -1.0;
        double phi = acos(c);
        double si = sin(phi);
        if (fabs(si) < SMALLER) si = SMALLER;
        double siinv = 1.0 / si;
        const double *kc = dihedcoeff + (size_t)(type - 1) * 4;
        double k1 = kc[0], k2 = kc[1], k3 = kc[2], k4 = kc[3];
        double pp = k1 * (1.0 + c) + k2 * (1.0 - cos(2.0 * phi)) + k3 * (1.0 + cos(3.0 * phi)) +
                    k4 * (1.0 - cos(4.0 * phi));
        double pd = k1 - 2.0 * k2 * sin(2.0 * phi) * siinv + 3.0 * k3 * sin(3.0 * phi) * siinv -
                    4.0 * k4 * sin(4.0 * phi) * siinv;
        edih += pp;
        double a = pd;
        c = c * a;
        s12 = s12 * a;
        double a11 = c * sb1 * s1;
        double a22 = -sb2 * (2.0 * c0 * s12 - c * (s1 + s2));
        double a33 = c * sb3 * s2;
        double a12 = -r12c1 * (c1mag * c * s1 + c2mag * s12);
        double a13 = -rb1 * rb3 * s12;
        double a23 = r12c2 * (c2mag * c * s2 + c1mag * s12);
        double sx2 = a12 * vb1x + a22 * vb2x + a23 * vb3x;
        double sy2 = a12 * vb1y + a22 * vb2y + a23 * vb3y;
        double sz2 = a12 * vb1z + a22 * vb2z + a23 * vb3z;
        double f1[3], f2[3], f3[3], f4[3];
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
        /* :1003-1048 */
        double force = 0.0;
        if (dr2 < p->cut_coulsq) {
            double r = sqrt(dr2);
            double dr2i = 1.0 / dr2;
            double prefactor = (double)((p->coulpre * q[i1]) * q[i4]) / r;
            double erfcd = exp(-(((alpha * alpha) * r) * r));
            double t = 1.0 / (1.0 + (p->EWALD_P * alpha) * r);
            double erfcc = t * (p->A1 + t * (p->A2 + t * (p->A3 + t * (p->A4 + t * p->A5)))) * erfcd;
            double forcecoul = (0.50 * prefactor) *
                               ((erfcc / r + ((2.0 * alpha) / p->MY_PIS) * erfcd) + r * p->f_shift) * r;
            ec14 = ec14 + (0.50 * prefactor) * ((erfcc - r * p->e_shift) - dr2 * p->f_shift);
            double forcelj = 0.0;
            if (dr2 < p->rcut2) {
                double dr6i = dr2i * dr2i * dr2i;
                size_t o = (size_t)(itype - 1) * ntypes + (size_t)(jtype - 1);
                size_t tn = (size_t)ntypes * ntypes;
                forcelj = dr6i * (lj14[0 * tn + o] * dr6i - lj14[1 * tn + o]);
                p14 = p14 + dr6i * (dr6i * lj14[2 * tn + o] - lj14[3 * tn + o]);
            }
            force = (forcecoul + forcelj) * dr2i;
        }
        f1[0] += ddx * force;
        f1[1] += ddy * force;
        f1[2] += ddz * force;
        f4[0] -= ddx * force;
        f4[1] -= ddy * force;
        f4[2] -= ddz * force;
        for (int c3 = 0; c3 < 3; ++c3) {
            ffh[(size_t)i1 * 3 + c3] = (float)((double)ffh[(size_t)i1 * 3 + c3] + f1[c3]);
            ffh[(size_t)i2 * 3 + c3] = (float)((double)ffh[(size_t)i2 * 3 + c3] + f2[c3]);
            ffh[(size_t)i3 * 3 + c3] = (float)((double)ffh[(size_t)i3 * 3 + c3] + f3[c3]);
            ffh[(size_t)i4 * 3 + c3] = (float)((double)ffh[(size_t)i4 * 3 + c3] + f4[c3]);
            if (ffh64) {
                /* the same per-dihedral terms summed in double (for FP64 comparisons) */
                ffh64[(size_t)i1 * 3 + c3] += f1[c3];
                ffh64[(size_t)i2 * 3 + c3] += f2[c3];
                ffh64[(size_t)i3 * 3 + c3] += f3[c3];
                ffh64[(size_t)i4 * 3 + c3] += f4[c3];
            }
        }
    }
    *e_dihedral += edih;
    *e_coul_14 += ec14;
    *pot_14 += p14;
}

/* mod_force_correction.f90:6-93 / 95-184 / 187-278 (correct_12/13/14_bonds):
 * Ewald real-space erfc part minus (1-fudge) of the bare Coulomb, per bonded
 * pair (i1[m*stride], i2[m*stride]). */
void orc_correct_pairs(const orc_params *p, const orc_ainfo *pos, const float *q, int npairs,
                       const int32_t *i1v, const int32_t *i2v, int stride, double gewald,
                       double fudge, float *ffc, double *e_corr, double *virial3) {
    const double box = (double)p->box, ibox = (double)p->ibox;
    double e = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
    for (int m = 0; m < npairs; ++m) {
        int i1 = i1v[(size_t)m * stride] - 1, i2 = i2v[(size_t)m * stride] - 1;
        double dx = (double)(pos[i1].x - pos[i2].x);
        double dy = (double)(pos[i1].y - pos[i2].y);
        double dz = (double)(pos[i1].z - pos[i2].z);
        double bx = dx * ibox, by = dy * ibox, bz = dz * ibox;
        bx = (bx + copysign(TWO52, bx)) - copysign(TWO52, dx);
        by = (by + copysign(TWO52, by)) - copysign(TWO52, dy);
        bz = (bz + copysign(TWO52, bz)) - copysign(TWO52, dz);
        dx = dx - box * bx;
        dy = dy - box * by;
        dz = dz - box * bz;
        double dr2 = dx * dx + dy * dy + dz * dz;
        double dr2i = 1.0 / dr2;
        double r = sqrt(dr2);
        double prefactor = (double)((p->coulpre * q[i1]) * q[i2]) / r;
        double grij = gewald * r;
        double expm2 = exp(-(grij * grij));
        double t = 1.0 / (1.0 + p->EWALD_P * grij);
        double erfcv = t * (p->A1 + t * (p->A2 + t * (p->A3 + t * (p->A4 + t * p->A5)))) * expm2;
        if (dr2 > p->cut_coulsq) prefactor = 0.0;
        double forcecoul = prefactor * (erfcv + (p->EWALD_F * grij) * expm2);
        forcecoul = forcecoul - (1.0 - fudge) * prefactor;
        e = e + prefactor * erfcv;
        e = e - (1.0 - fudge) * prefactor;
        double force = forcecoul * dr2i;
        ffc[(size_t)i1 * 3 + 0] = (float)((double)ffc[(size_t)i1 * 3 + 0] + dx * force);
        ffc[(size_t)i1 * 3 + 1] = (float)((double)ffc[(size_t)i1 * 3 + 1] + dy * force);
        ffc[(size_t)i1 * 3 + 2] = (float)((double)ffc[(size_t)i1 * 3 + 2] + dz * force);
        ffc[(size_t)i2 * 3 + 0] = (float)((double)ffc[(size_t)i2 * 3 + 0] - dx * force);
        ffc[(size_t)i2 * 3 + 1] = (float)((double)ffc[(size_t)i2 * 3 + 1] - dy * force);
        ffc[(size_t)i2 * 3 + 2] = (float)((double)ffc[(size_t)i2 * 3 + 2] - dz * force);
        vx = vx + dx * dx * force;
        vy = vy + dy * dy * force;
        vz = vz + dz * dz * force;
    }
    *e_corr += e;
    if (virial3) {
        virial3[0] += vx;
        virial3[1] += vy;
        virial3[2] += vz;
    }
}

/* mod_assign_types.f90:50-62 (assign_charge_types, coul_flag = 1) */
double orc_e_self_dsf(const orc_params *p, int np, const float *q) {
    double e = 0.0;
    for (int i = 0; i < np; ++i)
        e = e - (((0.5 * p->e_shift + p->alpha / p->MY_PIS) * (double)q[i]) * (double)q[i]) *
                    (double)p->coulpre;
    return e;
}

/* ------------------------------------------------------------------------ */
/* Largest cluster: mod_cluster.f90:15-83 with build_ptta_wrap_cluster2
 * (mod_build_ptta.f90:116-164), xyzcenter_molecule (mod_cluster.f90:803-836),
 * pbc_molcom (:841-884), cluster_neighbor_wrapper and callees
 * (mod_neighbor_cluster.f90:15-37,57-199,538-709), buildClusters/harvestCluster
 * (mod_cluster.f90:200-247) and append_surface_molecules (:163-194). */
typedef struct {
    int n, *stack;
} orc_stack;

int orc_greatest_cluster(int np, const orc_ainfo *pos, const int32_t *global_id, int n_gly,
                         int apg, float box, float ibox, float vol, double mrcut,
                         double denscut, int densmin, double *ptta, int32_t *greatest_belongsto,
                         int32_t *denstrack_out, int32_t *belongsto_out) {
    const int flag = n_gly * apg;
    /* build_ptta_wrap_cluster2: the atom with global id == flag is never refreshed (:127) */
    for (int i = 0; i < np; ++i) {
        int id = global_id[i];
        if (id < flag) {
            ptta[(size_t)(id - 1) * 3 + 0] = (double)pos[i].x;
            ptta[(size_t)(id - 1) * 3 + 1] = (double)pos[i].y;
            ptta[(size_t)(id - 1) * 3 + 2] = (double)pos[i].z;
        }
    }
    for (int m = 0; m < n_gly; ++m) {
        double x1 = ptta[(size_t)(m * apg) * 3 + 0], y1 = ptta[(size_t)(m * apg) * 3 + 1],
               z1 = ptta[(size_t)(m * apg) * 3 + 2];
        for (int j = 1; j < apg; ++j) {
            double *pj = ptta + (size_t)(m * apg + j) * 3;
            double x2 = pj[0], y2 = pj[1], z2 = pj[2];
            double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
            pj[0] = x2 - (double)(box * (float)lround(dx * (double)ibox));
            pj[1] = y2 - (double)(box * (float)lround(dy * (double)ibox));
            pj[2] = z2 - (double)(box * (float)lround(dz * (double)ibox));
        }
    }
    /* xyzcenter_molecule + pbc_molcom */
    double *com = (double *)malloc(sizeof(double) * 3 * (size_t)(n_gly > 0 ? n_gly : 1));
    const double b = (double)box;
    for (int m = 0; m < n_gly; ++m) {
        double xc = 0.0, yc = 0.0, zc = 0.0;
        for (int j = 0; j < apg; ++j) {
            xc += ptta[(size_t)(m * apg + j) * 3 + 0];
            yc += ptta[(size_t)(m * apg + j) * 3 + 1];
            zc += ptta[(size_t)(m * apg + j) * 3 + 2];
        }
        double c[3] = {xc / (double)(float)apg, yc / (double)(float)apg, zc / (double)(float)apg};
        for (int d = 0; d < 3; ++d) {
            while (c[d] > b) c[d] = c[d] - b;
            while (c[d] < 0.0) c[d] = c[d] + b;
            com[(size_t)m * 3 + d] = c[d];
        }
    }
    /* check_allocation_cluster: mrn = box/int(box/mrcut) in real*4 */
    int nside = (int)((double)box / mrcut);
    double mrn = (double)(box / (float)nside);
    int mncellT = (int)lround((double)vol / ((mrn * mrn) * mrn));
    int mncellD = (int)lround(pow((double)mncellT, 1.0 / 3.0));
    int32_t *mcnum = (int32_t *)malloc(sizeof(int32_t) * 26 * (size_t)mncellT);
    {
        int itel = 0;
        for (int cell = 0; cell < mncellT; ++cell) {
            int icz = cell / (mncellD * mncellD);
            int icy = (cell - icz * mncellD * mncellD) / mncellD;
            int icx = cell - icy * mncellD - icz * mncellD * mncellD;
            for (int iz = -1; iz <= 1; ++iz)
                for (int iy = -1; iy <= 1; ++iy)
                    for (int ix = -1; ix <= 1; ++ix) {
                        int zc = icz + iz, yc = icy + iy, xc = icx + ix;
                        zc = zc < 0 ? zc + mncellD : (zc >= mncellD ? zc - mncellD : zc);
                        yc = yc < 0 ? yc + mncellD : (yc >= mncellD ? yc - mncellD : yc);
                        xc = xc < 0 ? xc + mncellD : (xc >= mncellD ? xc - mncellD : xc);
                        if (iz != 0 || iy != 0 || ix != 0)
                            mcnum[itel++] = xc + yc * mncellD + zc * mncellD * mncellD;
                    }
        }
    }
    /* mol_new_nlist (LIFO chains) with mol_xyz2bin */
    int32_t *mhoc = (int32_t *)calloc((size_t)mncellT + 1, sizeof(int32_t));
    int32_t *mll = (int32_t *)calloc((size_t)n_gly + 1, sizeof(int32_t));
    double imrn = 1.0 / mrn;
    for (int i = 1; i <= n_gly; ++i) {
        const double *c = com + (size_t)(i - 1) * 3;
        int ix = (c[0] < b) ? (int)(c[0] * imrn) : mncellD - 1;
        int iy = (c[1] < b) ? (int)(c[1] * imrn) : mncellD - 1;
        int iz = (c[2] < b) ? (int)(c[2] * imrn) : mncellD - 1;
        if (ix == mncellD) ix = mncellD - 1;
        if (iy == mncellD) iy = mncellD - 1;
        if (iz == mncellD) iz = mncellD - 1;
        int icell = ix + iy * mncellD + iz * mncellD * mncellD;
        mll[i] = mhoc[icell];
        mhoc[icell] = i;
    }
    /* mol_build_neighbor_nosort: denstrack and densvl (dens list in discovery order) */
    const double mrcut2 = mrcut * mrcut, denscut2 = denscut * denscut;
    int32_t *denstrack = (int32_t *)calloc((size_t)n_gly + 1, sizeof(int32_t));
    size_t dcap = 64;
    int32_t **densvl = (int32_t **)calloc((size_t)n_gly + 1, sizeof(int32_t *));
    size_t *dlen_cap = (size_t *)calloc((size_t)n_gly + 1, sizeof(size_t));
    for (int cell = 0; cell < mncellT; ++cell) {
        for (int p1 = mhoc[cell]; p1 != 0; p1 = mll[p1]) {
            const double *c1 = com + (size_t)(p1 - 1) * 3;
            for (int k = cell * 26; k <= cell * 26 + 25; ++k) {
                for (int p2 = mhoc[mcnum[k]]; p2 != 0; p2 = mll[p2]) {
                    const double *c2 = com + (size_t)(p2 - 1) * 3;
                    double dx = c1[0] - c2[0], dy = c1[1] - c2[1], dz = c1[2] - c2[2];
                    double sx = -(double)(box * (float)lround(dx * (double)ibox));
                    double sy = -(double)(box * (float)lround(dy * (double)ibox));
                    double sz = -(double)(box * (float)lround(dz * (double)ibox));
                    dx = dx + sx;
                    dy = dy + sy;
                    dz = dz + sz;
                    double dr2 = dx * dx + dy * dy + dz * dz;
                    if (dr2 < mrcut2 && dr2 < denscut2) {
                        int d = denstrack[p1]++;
                        if ((size_t)d >= dlen_cap[p1]) {
                            dlen_cap[p1] = dlen_cap[p1] ? 2 * dlen_cap[p1] : dcap;
                            densvl[p1] = (int32_t *)realloc(densvl[p1], sizeof(int32_t) * dlen_cap[p1]);
                        }
                        densvl[p1][d] = p2;
                    }
                }
            }
            for (int p2 = mhoc[cell]; p2 != 0; p2 = mll[p2]) {
                if (p2 == p1) continue;
                const double *c2 = com + (size_t)(p2 - 1) * 3;
                double dx = c1[0] - c2[0], dy = c1[1] - c2[1], dz = c1[2] - c2[2];
                double dr2 = dx * dx + dy * dy + dz * dz;
                if (dr2 < mrcut2 && dr2 < denscut2) {
                    int d = denstrack[p1]++;
                    if ((size_t)d >= dlen_cap[p1]) {
                        dlen_cap[p1] = dlen_cap[p1] ? 2 * dlen_cap[p1] : dcap;
                        densvl[p1] = (int32_t *)realloc(densvl[p1], sizeof(int32_t) * dlen_cap[p1]);
                    }
                    densvl[p1][d] = p2;
                }
            }
        }
    }
    /* buildClusters: seeds in ascending index, depth-first harvest (explicit stack
     * in place of the recursion; the visited set is the same). */
    int32_t *belongsto = (int32_t *)calloc((size_t)n_gly + 1, sizeof(int32_t));
    int32_t *stk = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n_gly + 1));
    int nclus = 0;
    for (int ti = 1; ti <= n_gly; ++ti) {
        if (belongsto[ti] == 0 && denstrack[ti] >= densmin) {
            nclus++;
            belongsto[ti] = nclus;
            int sp = 0;
            stk[sp++] = ti;
            while (sp > 0) {
                int u = stk[--sp];
                for (int l = 0; l < denstrack[u]; ++l) {
                    int nb = densvl[u][l];
                    if (belongsto[nb] == 0 && denstrack[nb] >= densmin) {
                        belongsto[nb] = nclus;
                        stk[sp++] = nb;
                    }
                }
            }
        }
    }
    /* histogram and largest (strict >, first in label order) */
    int32_t *histo = (int32_t *)calloc((size_t)nclus + 2, sizeof(int32_t));
    for (int ti = 1; ti <= n_gly; ++ti)
        if (belongsto[ti] != 0) histo[belongsto[ti]]++;
    int greatest = 0;
    for (int c = 1; c <= nclus; ++c)
        if (histo[c] > greatest) {
            greatest = histo[c];
            *greatest_belongsto = c;
        }
    /* append_surface_molecules */
    int cluster = *greatest_belongsto;
    int32_t *surf = (int32_t *)calloc((size_t)n_gly + 1, sizeof(int32_t));
    for (int ti = 1; ti <= n_gly; ++ti)
        if (belongsto[ti] == cluster)
            for (int l = 0; l < denstrack[ti]; ++l) {
                int nb = densvl[ti][l];
                if (denstrack[nb] < densmin) surf[nb]++;
            }
    int surface = 0;
    for (int i = 1; i <= n_gly; ++i)
        if (surf[i] >= 1) {
            surface++;
            belongsto[i] = cluster;
        }
    if (denstrack_out)
        for (int i = 0; i < n_gly; ++i) denstrack_out[i] = denstrack[i + 1];
    if (belongsto_out)
        for (int i = 0; i < n_gly; ++i) belongsto_out[i] = belongsto[i + 1];
    for (int i = 0; i <= n_gly; ++i) free(densvl[i]);
    free(densvl); free(dlen_cap); free(denstrack); free(belongsto); free(stk); free(histo);
    free(surf); free(mhoc); free(mll); free(mcnum); free(com);
    return greatest + surface;
}

/* ------------------------------------------------------------------------ */
/* mod_force_bond.f90:6-75 (bond_harmonic) into a double force array. */
void orc_bond_harmonic(const orc_params *p, const orc_ainfo *pos, int nbond,
                       const int32_t *bl, const double *bc, double *f, double *e_bond) {
    double e = 0.0;
    for (int m = 0; m < nbond; ++m) {
        int i1 = bl[m * 3] - 1, i2 = bl[m * 3 + 1] - 1, t = bl[m * 3 + 2] - 1;
        double dx = minimg1((double)(pos[i1].x - pos[i2].x), p->box, p->ibox);
        double dy = minimg1((double)(pos[i1].y - pos[i2].y), p->box, p->ibox);
        double dz = minimg1((double)(pos[i1].z - pos[i2].z), p->box, p->ibox);
        double rsq = dx * dx + dy * dy + dz * dz;
        double r = sqrt(rsq);
        double dr = r - bc[t * 2 + 1];
        double rk = bc[t * 2 + 0] * dr;
        e = e + rk * dr;
        double force = (r > 0.0) ? -2.0 * rk / r : 0.0;
        f[i1 * 3 + 0] += dx * force; f[i1 * 3 + 1] += dy * force; f[i1 * 3 + 2] += dz * force;
        f[i2 * 3 + 0] -= dx * force; f[i2 * 3 + 1] -= dy * force; f[i2 * 3 + 2] -= dz * force;
    }
    *e_bond += e;
}

/* mod_force_angle.f90:10-122 (angle_harmonic) into a double force array. */
void orc_angle_harmonic(const orc_params *p, const orc_ainfo *pos, int nangle,
                        const int32_t *al, const double *ac, double *f, double *e_angle) {
    const double small = (double)0.001f;
    double e = 0.0;
    for (int m = 0; m < nangle; ++m) {
        int i1 = al[m * 4] - 1, i2 = al[m * 4 + 1] - 1, i3 = al[m * 4 + 2] - 1, t = al[m * 4 + 3] - 1;
        double dx1 = minimg1((double)(pos[i1].x - pos[i2].x), p->box, p->ibox);
        double dy1 = minimg1((double)(pos[i1].y - pos[i2].y), p->box, p->ibox);
        double dz1 = minimg1((double)(pos[i1].z - pos[i2].z), p->box, p->ibox);
        double rsq1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1, r1 = sqrt(rsq1);
        double dx2 = minimg1((double)(pos[i3].x - pos[i2].x), p->box, p->ibox);
        double dy2 = minimg1((double)(pos[i3].y - pos[i2].y), p->box, p->ibox);
        double dz2 = minimg1((double)(pos[i3].z - pos[i2].z), p->box, p->ibox);
        double rsq2 = dx2 * dx2 + dy2 * dy2 + dz2 * dz2, r2 = sqrt(rsq2);
        double c = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
        c = c / (r1 * r2);
        if (c > 1.0) c = 1.0;
        if (c < -1.0) c = -1.0;
        double s = sqrt(1.0 - c * c);
        if (s < small) s = small;
        s = 1.0 / s;
        double dtheta = acos(c) - ac[t * 2 + 1];
        double tk = ac[t * 2 + 0] * dtheta;
        e = e + tk * dtheta;
        double a = 2.0 * tk * s;
        double a11 = a * c / rsq1, a12 = -a / (r1 * r2), a22 = a * c / rsq2;
        double vx1 = a11 * dx1 + a12 * dx2, vx2 = a22 * dx2 + a12 * dx1;
        double vy1 = a11 * dy1 + a12 * dy2, vy2 = a22 * dy2 + a12 * dy1;
        double vz1 = a11 * dz1 + a12 * dz2, vz2 = a22 * dz2 + a12 * dz1;
        f[i1 * 3 + 0] -= vx1; f[i1 * 3 + 1] -= vy1; f[i1 * 3 + 2] -= vz1;
        f[i2 * 3 + 0] += vx2 + vx1; f[i2 * 3 + 1] += vy2 + vy1; f[i2 * 3 + 2] += vz2 + vz1;
        f[i3 * 3 + 0] -= vx2; f[i3 * 3 + 1] -= vy2; f[i3 * 3 + 2] -= vz2;
    }
    *e_angle += e;
}

/* ------------------------------------------------------------------------ */
/* SHAKE (mod_shake.f90:8-85 driver, shake2 :89-187, shake3 :194-355, shake4
 * :361-628, shake3angle :637-880, shake_update :888-913) on FP64 state.
 * Each group is written as a list of constraints (p,q) with reference vectors
 * r_pq = x_p - x_q (minimum image) and predicted s_pq; the linearised matrix
 * A_cd = 2 C_cd (s_c . r_d), C_cd = e(p_c,d)/m_p - e(q_c,d)/m_q, and the
 * quadratic correction |sum_d lambda_d C_cd r_d|^2 are those of the reference
 * routines; one-constraint groups use the exact quadratic root of shake2. */
static inline double mi_d(double d, double box) { return d - box * (double)lround(d / box); }

int orc_shake(int np, const double *x, const double *v, double *f, const double *mass,
              double box, int nshake, const int32_t *sa, const double *sbond, double dt,
              double kcal2amu, int iflag, int maxiter, double tolerance) {
    (void)np;
    int status = 0;
    double dtsq = (iflag == 0) ? 0.5 * dt * dt * kcal2amu : dt * dt * kcal2amu;
    for (int g = 0; g < nshake; ++g) {
        int num = sa[g * 5];
        int at[4] = {sa[g * 5 + 1] - 1, sa[g * 5 + 2] - 1, sa[g * 5 + 3] - 1, sa[g * 5 + 4] - 1};
        int nc, cp[3], cq[3];
        double bl[3];
        if (num == 1) { nc = 1; cp[0] = 0; cq[0] = 1; bl[0] = sbond[g * 3]; }
        else if (num == 3) { nc = 2; cp[0] = 0; cq[0] = 1; cp[1] = 0; cq[1] = 2; bl[0] = sbond[g * 3]; bl[1] = sbond[g * 3 + 1]; }
        else if (num == 4) { nc = 3; for (int k = 0; k < 3; ++k) { cp[k] = 0; cq[k] = k + 1; bl[k] = sbond[g * 3 + k]; } }
        else if (num == -3) { nc = 3; cp[0] = 0; cq[0] = 1; cp[1] = 0; cq[1] = 2; cp[2] = 1; cq[2] = 2; for (int k = 0; k < 3; ++k) bl[k] = sbond[g * 3 + k]; }
        else continue;
        int na = (num == 1) ? 2 : (num == 4 ? 4 : 3);
        double im[4], xs[4][3];
        for (int a = 0; a < na; ++a) {
            im[a] = 1.0 / mass[at[a]];
            for (int d = 0; d < 3; ++d)
                xs[a][d] = x[at[a] * 3 + d] + dt * v[at[a] * 3 + d] + dtsq * im[a] * f[at[a] * 3 + d];
        }
        double r[3][3], s[3][3];
        for (int c = 0; c < nc; ++c)
            for (int d = 0; d < 3; ++d) {
                r[c][d] = mi_d(x[at[cp[c]] * 3 + d] - x[at[cq[c]] * 3 + d], box);
                s[c][d] = mi_d(xs[cp[c]][d] - xs[cq[c]][d], box);
            }
        double C[3][3];
        for (int c = 0; c < nc; ++c)
            for (int d = 0; d < nc; ++d) {
                double e = 0.0;
                if (cp[c] == cp[d]) e += im[cp[c]];
                if (cp[c] == cq[d]) e -= im[cp[c]];
                if (cq[c] == cp[d]) e -= im[cq[c]];
                if (cq[c] == cq[d]) e += im[cq[c]];
                C[c][d] = e;
            }
        double lam[3] = {0, 0, 0};
        if (nc == 1) {
            double rr = r[0][0] * r[0][0] + r[0][1] * r[0][1] + r[0][2] * r[0][2];
            double ss = s[0][0] * s[0][0] + s[0][1] * s[0][1] + s[0][2] * s[0][2];
            double sr = s[0][0] * r[0][0] + s[0][1] * r[0][1] + s[0][2] * r[0][2];
            double a = C[0][0] * C[0][0] * rr, b = 2.0 * C[0][0] * sr, cc = ss - bl[0] * bl[0];
            double det = b * b - 4.0 * a * cc;
            if (det < 0.0) { status = 1; det = 0.0; }
            double l1 = (-b + sqrt(det)) / (2.0 * a), l2 = (-b - sqrt(det)) / (2.0 * a);
            lam[0] = (fabs(l1) <= fabs(l2)) ? l1 : l2;
        } else {
            double A[3][3], Ai[3][3], ss[3], rd[3][3];
            for (int c = 0; c < nc; ++c) {
                ss[c] = s[c][0] * s[c][0] + s[c][1] * s[c][1] + s[c][2] * s[c][2];
                for (int d = 0; d < nc; ++d) {
                    A[c][d] = 2.0 * C[c][d] * (s[c][0] * r[d][0] + s[c][1] * r[d][1] + s[c][2] * r[d][2]);
                    rd[c][d] = r[c][0] * r[d][0] + r[c][1] * r[d][1] + r[c][2] * r[d][2];
                }
            }
            if (nc == 2) {
                double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
                if (det == 0.0) { status = 2; continue; }
                double di = 1.0 / det;
                Ai[0][0] = A[1][1] * di; Ai[0][1] = -A[0][1] * di;
                Ai[1][0] = -A[1][0] * di; Ai[1][1] = A[0][0] * di;
            } else {
                double det = A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
                             A[0][2] * A[1][0] * A[2][1] - A[0][0] * A[1][2] * A[2][1] -
                             A[0][1] * A[1][0] * A[2][2] - A[0][2] * A[1][1] * A[2][0];
                if (det == 0.0) { status = 2; continue; }
                double di = 1.0 / det;
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
            int niter = 0, done = 0;
            while (!done && niter < maxiter) {
                double bvec[3], ln[3];
                for (int c = 0; c < nc; ++c) {
                    double qd = 0.0;
                    for (int d = 0; d < nc; ++d)
                        for (int e = 0; e < nc; ++e) qd += C[c][d] * C[c][e] * rd[d][e] * lam[d] * lam[e];
                    bvec[c] = bl[c] * bl[c] - ss[c] - qd;
                }
                done = 1;
                for (int c = 0; c < nc; ++c) {
                    ln[c] = 0.0;
                    for (int d = 0; d < nc; ++d) ln[c] += Ai[c][d] * bvec[d];
                    if (fabs(ln[c] - lam[c]) > tolerance) done = 0;
                }
                for (int c = 0; c < nc; ++c) lam[c] = ln[c];
                niter++;
            }
            if (!done) status = 3;
        }
        for (int c = 0; c < nc; ++c) {
            double l = lam[c] / dtsq;
            for (int d = 0; d < 3; ++d) {
                f[at[cp[c]] * 3 + d] += l * r[c][d];
                f[at[cq[c]] * 3 + d] -= l * r[c][d];
            }
        }
    }
    return status;
}
