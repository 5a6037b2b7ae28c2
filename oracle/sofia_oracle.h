/*
 * sofia_oracle.h -- CPU restatement of the Sofia nonbonded hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * and the timed CPU baseline; nothing in the product library links it.
 *
 * PARITY UNPINNED: the reference is Fortran 90 (Intel ifport/MKL/MPI/LEO) and
 * cannot be compiled in this environment, and the reference ships no tests,
 * golden vectors or logged outputs.  The restatement is therefore pinned only
 * by its own cross-checks (list-based vs O(N^2) forces, Newton's third law,
 * finite differences) and by matching the reference source line by line.
 *
 * Conventions mirror the reference module state:
 *   - ainfo records {float x,y,z; int32 type}       Source/global.f90:82-85
 *   - specbond[i*12 + l] holds 1-based partner ids   Source/global.f90:446
 *   - nlist[i*neigh_alloc + j] holds 1-based ids     Source/mod_neighbor.f90:669,736
 *   - ff[i*3 + c] float                              Source/global.f90:87-89,102
 * All arithmetic follows the Fortran evaluation order with strict IEEE
 * semantics (compiled with -ffp-contract=off, no fast-math).
 */
#ifndef SOFIA_ORACLE_H
#define SOFIA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float x, y, z;
    int32_t type;
} orc_ainfo;

typedef struct {
    /* DSF constants (Source/get_started.f90:101-117) */
    double alpha, EWALD_F, EWALD_P, A1, A2, A3, A4, A5, MY_PIS, MY_PIS_INV;
    double e_shift, f_shift;
    float coulpre;
    /* geometry (Source/global.f90:128-135, get_started.f90:45-75) */
    float box, ibox, vol, cut_coul, rcut, neighbor_pad;
    double rcut2, cut_coulsq, rv, rv2, rvrc2;
} orc_params;

void orc_init_params(orc_params *p, double alpha, float box, float cut_coul, float rcut,
                     float neighbor_pad);

/* ---- neighbor list (Source/mod_neighbor.f90) ---- */
void orc_cell_grid(float box, float vol, float cut_coul, float rcut, float *rn, int *ncellT,
                   int *ncellD);
void orc_stencil(int ncellT, int ncellD, int32_t *cnum /* 27*ncellT */);
int orc_xyz2bin(float x, float y, float z, float box, float rn, int ncellD);
/* new_nlist + sort_posit_charge: tt[orig] = sorted (1-based), ttb[sorted-1] = orig (1-based),
 * start/endposit per cell (1-based sorted ids), atombin per sorted atom. */
void orc_bin_sort(int np, const orc_ainfo *pos, float box, float rn, int ncellT, int ncellD,
                  int32_t *tt, int32_t *ttb, int32_t *start, int32_t *endposit, int32_t *atombin);
/* full neighbour build of build_neighbor_nonewton_nomic on already cell-sorted arrays.
 * Returns max row length; rows longer than neigh_alloc are truncated. */
int orc_build_neighbor_nonewton(const orc_params *p, int np, const orc_ainfo *pos,
                                const int32_t *atombin, const int32_t *start,
                                const int32_t *endposit, const int32_t *cnum,
                                const int32_t *specbond, const int32_t *num3bond,
                                int32_t *nlist, int32_t *numneigh, int neigh_alloc, int nthreads);
/* whole neighbor_wrapper on unsorted input: returns the list in INPUT index space */
int orc_neighbor_wrapper(const orc_params *p, int np, const orc_ainfo *pos,
                         const int32_t *specbond, const int32_t *num3bond, int32_t *nlist,
                         int32_t *numneigh, int neigh_alloc, int nthreads);
int orc_build_neighbor_n2(const orc_params *p, int np, const orc_ainfo *pos,
                          const int32_t *specbond, const int32_t *num3bond, int32_t *nlist,
                          int32_t *numneigh, int neigh_alloc);
int orc_check_neighbor(int np, const float *drx, const float *dry, const float *drz,
                       double rvrc2);

/* ---- nonbonded forces (Source/mod_force_nonbond.f90) ---- */
void orc_force_dsf_nonewton(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                            const float *lj1, const float *lj2, const float *lj3,
                            const float *lj4, int ntypes, const int32_t *nlist,
                            const int32_t *numneigh, int neigh_alloc, float *ff,
                            double *potential, double *e_coul, double *virial3,
                            double *ff64 /* optional (np,3) double accumulators */,
                            int nthreads);
/* lj_cut_coul_long_nonewton_NOMIC (mod_force_nonbond.f90:300-400): real*4 real-space Ewald */
void orc_force_long_nonewton(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                             const float *lj1, const float *lj2, const float *lj3,
                             const float *lj4, int ntypes, const int32_t *nlist,
                             const int32_t *numneigh, int neigh_alloc, double gewald, float *ff,
                             double *potential, double *e_coul, double *virial3,
                             double *ff64, int nthreads);
/* improper_harmonic_lammps14 (mod_force_dihed.f90:1546-1724) */
void orc_improper_harmonic(const orc_params *p, int np, const orc_ainfo *pos, int nimpro,
                           const int32_t *improlist, const double *improcoeff, float *ff_impro,
                           double *e_improper, double *v_impro3);
void orc_force_dsf_n2(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                      const float *lj1, const float *lj2, const float *lj3, const float *lj4,
                      int ntypes, const int32_t *specbond, const int32_t *num1bond,
                      const int32_t *num2bond, const int32_t *num3bond, double *ff64,
                      double *potential, double *e_coul);

/* ---- 1-4 pairs of dihedral_opls_DSF (Source/mod_force_dihed.f90:816-1092) ---- */
void orc_dihedral_opls_dsf(const orc_params *p, int np, const orc_ainfo *pos, const float *q,
                           int ntypes, const double *lj14 /* [4][ntypes][ntypes] */,
                           int ndihed, const int32_t *dihedlist /* [n][5] */,
                           const double *dihedcoeff /* [ntype][4] */, float *ffh,
                           double *e_dihedral, double *e_coul_14, double *pot_14,
                           double *ffh64 /* optional (np,3) double sums, may be NULL */);

/* ---- PME exclusion corrections (Source/mod_force_correction.f90) ---- */
void orc_correct_pairs(const orc_params *p, const orc_ainfo *pos, const float *q, int npairs,
                       const int32_t *i1, const int32_t *i2, int stride, double gewald,
                       double fudge, float *ffc, double *e_coul_corr, double *virial3);
double orc_calculate_gewald(float cut_coul);

/* ---- self energy (Source/mod_assign_types.f90:50-62) ---- */
double orc_e_self_dsf(const orc_params *p, int np, const float *q);

/* ---- largest cluster (Source/mod_cluster.f90:15-83 and callees) ---- */
int orc_greatest_cluster(int np, const orc_ainfo *pos, const int32_t *global_id, int n_gly,
                         int atoms_per_gly, float box, float ibox, float vol, double mrcut,
                         double denscut, int densmin, double *ptta_full /* [n_gly*apg*3] in/out */,
                         int32_t *greatest_belongsto /* in/out */, int32_t *denstrack_out,
                         int32_t *belongsto_out);

/* ---- residency kernels (Source/mod_ensemble.f90, mod_pbc.f90, mod_shake.f90, ...) ---- */
void orc_bond_harmonic(const orc_params *p, const orc_ainfo *pos, int nbond,
                       const int32_t *bondlist /* [n][3] */, const double *bondcoeff /* [t][2] */,
                       double *f64, double *e_bond);
void orc_angle_harmonic(const orc_params *p, const orc_ainfo *pos, int nangle,
                        const int32_t *anglelist /* [n][4] */, const double *anglecoeff,
                        double *f64, double *e_angle);
/* SHAKE on FP64 state: x (np,3), v (np,3), f (np,3) in/out; masses per atom */
int orc_shake(int np, const double *x, const double *v, double *f, const double *mass_atom,
              double box, int nshake, const int32_t *shakeatom /* [n][5] */,
              const double *shake_bond /* [n][3] */, double dt, double kcal2amu, int iflag,
              int maxiter, double tolerance);

#ifdef __cplusplus
}
#endif
#endif
