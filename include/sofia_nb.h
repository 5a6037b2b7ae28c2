/*
 * sofia_nb.h -- C ABI of the B200 (sm_100a) nonbonded hot path of Sofia.
 *
 * The reference exposes this path as argument-less Fortran subroutines over
 * module state (Source/mod_neighbor.f90:8 neighbor_wrapper,
 * Source/mod_force_nonbond.f90:105 lj_cut_coul_dsf_nonewton_NOMIC,
 * Source/mod_force_dihed.f90:816 dihedral_opls_DSF,
 * Source/mod_force_correction.f90:6,95,187 correct_12/13/14_bonds,
 * Source/mod_cluster.f90:15 get_greatestCluster).  Each entry point below takes
 * exactly the module arrays those subroutines read and write, with the
 * reference's layout and 1-based indices, so a Fortran shim can pass its
 * module arrays through ISO_C_BINDING unchanged (the precedent is the
 * bind(c) PME interface at Source/mod_force.f90:14-23).
 *
 * Pointers may be host memory (copied to and from the GPU inside the call, like
 * the reference's LEO `in`/`inout` transfers, Source/mod_force.f90:446-462) or
 * device memory (used in place).  Calls are ordered on the context's CUDA
 * stream and return after their results are visible to the caller.
 *
 * Return codes: SOFIA_OK, or an error with a message in sofia_last_error().
 * No call aborts or traps.
 */
#ifndef SOFIA_NB_H
#define SOFIA_NB_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOFIA_OK 0
#define SOFIA_ENEEDGROW 1 /* output capacity too small; *needed_* holds the size to grow to */
#define SOFIA_EINVAL 2    /* invalid argument */
#define SOFIA_ECUDA 3     /* CUDA runtime error */
#define SOFIA_ETIMEOUT 4  /* a bounded device wait gave up */
#define SOFIA_ESTATE 5    /* device state check failed (non-finite values, SHAKE failure, ...) */
#define SOFIA_ETOOBIG 6   /* size beyond the fixed capacity of an allocation-free call */

/* type(ainfo) of Source/global.f90:82-85: {real*4 x,y,z; integer type}, 16 bytes. */
typedef struct {
    float x, y, z;
    int32_t type;
} sofia_ainfo;

typedef struct {
    int device; /* CUDA device ordinal */
    int flags;  /* reserved, 0 */
} sofia_nb_params;

typedef struct sofia_nb_ctx sofia_nb_ctx;

/* Context: one per host thread / replica (Source/mod_memory.f90:236-286 device setup). */
int sofia_nb_create(const sofia_nb_params *params, sofia_nb_ctx **out);
int sofia_nb_destroy(sofia_nb_ctx *ctx);
const char *sofia_last_error(const sofia_nb_ctx *ctx);
/* Blocks until all work of the context is done (offload_wait, Source/mod_force.f90:496). */
int sofia_wait(sofia_nb_ctx *ctx);
/* The context's cudaStream_t, for callers that order their own work with it. */
void *sofia_stream(sofia_nb_ctx *ctx);

/* DSF shift constants of init (Source/get_started.f90:112-116). */
int sofia_dsf_constants(double alpha, float cut_coul, double *e_shift, double *f_shift);

/* Cell grid of check_allocation (Source/mod_neighbor.f90:1446-1452). */
int sofia_cell_grid(float box, float cut_coul, float rcut, float *rn, int32_t *ncellT,
                    int32_t *ncellD);

/*
 * new_nlist + sort_posit_charge (Source/mod_neighbor.f90:923-1005): bins atoms
 * (xyz2bin, :1381-1424) and returns the cell-sorted order.  Outputs (any may be
 * NULL): tt[np] old->new 1-based, ttb[np] new->old 1-based, start/endposit[ncellT]
 * 1-based per cell, atombin[np] cell of each sorted atom, position_sorted[np].
 * Within a cell atoms follow the reference's linked-list order (descending
 * input index).
 */
int sofia_cell_sort(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position, float box,
                    float cut_coul, float rcut, int32_t *tt, int32_t *ttb, int32_t *start,
                    int32_t *endposit, int32_t *atombin, sofia_ainfo *position_sorted);

/*
 * build_neighbor_nonewton_nomic (Source/mod_neighbor.f90:622-809), with the
 * cell grid, stencil and binning of :1309-1526: full (non-Newton) list of every
 * z /= i in the 27 cells around atom i with real*4 minimum-image dr2 < rv2 and
 * z not in specbond(1:num3bond(i), i).
 *   specbond[i*12 + l] : 1-based partners (Fortran specbond(12,np) column-major)
 *   nlist[i*neigh_alloc + j] : 1-based neighbours in INPUT index order; may be
 *       NULL, in which case the list stays resident in the context for
 *       sofia_force_nonbond_dsf (the reference's `nocopy(nlist)`).
 * Rows are ordered by stencil cell, then by ascending input index inside a cell;
 * for input that is already cell sorted (sofia_cell_sort) this is exactly the
 * reference's row order.  If a row exceeds neigh_alloc the call returns
 * SOFIA_ENEEDGROW with *needed_alloc = roundup16(1.2*max) like the redo loop
 * (:767-802); the caller grows and calls again.
 */
int sofia_neighbor_build(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                         const int32_t *specbond, const int32_t *num3bond, float box, double rv2,
                         float cut_coul, float rcut, int32_t *nlist, int32_t *numneigh,
                         int32_t neigh_alloc, int32_t *needed_alloc);

/*
 * check_neighbor (Source/mod_neighbor.f90:895-913): *nflag = 1 if any atom's
 * accumulated displacement (real*4 drx, dry, drz) has drx^2+dry^2+drz^2 >= rvrc2
 * (rvrc2 = neighbor_pad^2, the full skin, Source/get_started.f90:47-48).
 */
int sofia_check_neighbor(sofia_nb_ctx *ctx, int np, const float *drx, const float *dry,
                         const float *drz, double rvrc2, int32_t *nflag);

/*
 * The permutations that follow the cell sort (sofia_cell_sort returns tt and ttb):
 *   sofia_sort_gather   -- sort_posit_charge (Source/mod_neighbor.f90:946-1005):
 *       out[new] = in[ttb[new]-1] for rows of elem_bytes (a multiple of 4, at most
 *       256); use it for position (16 B), v (12 B), q, mol, global_id, ...;
 *   sofia_sort_specbond -- sort_specbond_numbond (:1011-1039), in place: row i
 *       moves to tt[i] and its first num3bond entries are mapped through tt
 *       (entries past num3bond come back 0; the reference leaves stale values);
 *   sofia_remap_ids     -- sort_bondlist / anglelist / dihedlist / improlist
 *       (:1043-1168), in place: the first ncols of each row's stride entries are
 *       mapped through tt (0 stays 0).
 * tt and ttb are 1-based like the reference; ids outside 1..np give SOFIA_EINVAL.
 */
int sofia_sort_gather(sofia_nb_ctx *ctx, int np, int elem_bytes, const int32_t *ttb,
                      const void *in, void *out);
int sofia_sort_specbond(sofia_nb_ctx *ctx, int np, const int32_t *tt, int32_t *specbond,
                        int32_t *num1bond, int32_t *num2bond, int32_t *num3bond);
int sofia_remap_ids(sofia_nb_ctx *ctx, int np, const int32_t *tt, int nrows, int stride,
                    int ncols, int32_t *list);

/*
 * pbc (Source/mod_pbc.f90:6-39), in place: each real*4 coordinate is wrapped into
 * (0, box] by repeated subtraction / addition of box, as the reference loops do.
 * A coordinate that is non-finite or more than 64 boxes outside gives SOFIA_ESTATE.
 */
int sofia_pbc(sofia_nb_ctx *ctx, int np, sofia_ainfo *position, float box);

/*
 * lj_cut_coul_dsf_nonewton_NOMIC (Source/mod_force_nonbond.f90:105-196): LJ
 * 12-6 + damped-shifted-force Coulomb over the full list, FP64 pair arithmetic
 * on the real*4 arrays.  lj1..lj4 are [ntypes*ntypes] real*4 tables indexed
 * (itype-1)*ntypes + jtype.  ff[i*3+c] receives the per-atom force (real*4),
 * potential/e_coul the halved pair sums (:193-194), virial_diag3 (may be NULL)
 * the halved sum of dx*dx*force per axis.  nlist == NULL uses the list left
 * resident by the last sofia_neighbor_build.
 */
int sofia_force_nonbond_dsf(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                            const float *q, const float *lj1, const float *lj2,
                            const float *lj3, const float *lj4, int ntypes,
                            const int32_t *nlist, const int32_t *numneigh, int32_t neigh_alloc,
                            float box, float ibox, double rcut2, double cut_coulsq, double alpha,
                            double e_shift, double f_shift, float coulpre, float *ff,
                            double *potential, double *e_coul, double *virial_diag3);

/*
 * lj_cut_coul_long_nonewton_NOMIC (Source/mod_force_nonbond.f90:300-400; the
 * _MIC variant at :201-298 computes the same): the real-space Ewald term of
 * the PME path (coul_flag = 2) with LJ, over the same full list.  Pair
 * arithmetic is real*4 as in the reference, promoted to double where the
 * reference's mixed-mode statements promote; the A&S 7.1.26 erfc uses
 * gewald (calculate_gewald, Source/get_started.f90:153-173).  Outputs and list
 * handling as in sofia_force_nonbond_dsf; the reciprocal-space part
 * (cal_e_pme_kspace) and the excluded-pair corrections (sofia_correct_1x)
 * are separate calls.
 */
int sofia_force_nonbond_long(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                             const float *q, const float *lj1, const float *lj2,
                             const float *lj3, const float *lj4, int ntypes,
                             const int32_t *nlist, const int32_t *numneigh, int32_t neigh_alloc,
                             float box, float ibox, double rcut2, double cut_coulsq,
                             double gewald, float coulpre, float *ff, double *potential,
                             double *e_coul, double *virial_diag3);

/*
 * improper_harmonic_lammps14 (Source/mod_force_dihed.f90:1546-1724): harmonic
 * improper torsions E = k (omega - omega0)^2 over improlist[nimpro*5] (i1..i4,
 * type; 1-based), improcoeff[nimprotypes*2] = (k, omega0 in rad).  Forces are
 * ADDED to ff_impro (real*4 [np][3], the reference's ff_impro), the energy to
 * *e_improper and the diagonal virial to virial3 (may be NULL).  The reference
 * reads no omega0 from its topology (read_topol leaves theta0 unset,
 * Source/mod_readfile.f90:433), so the caller supplies it.
 */
int sofia_improper_harmonic(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position, int nimpro,
                            const int32_t *improlist, const double *improcoeff, int nimprotypes,
                            float box, float ibox, float *ff_impro, double *e_improper,
                            double *virial3);

/*
 * Allocation-free form of sofia_force_nonbond_dsf.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot allocate device
 * memory when they need forces: hosts that give the library a fixed device
 * arena or enforce a memory budget from outside (an allocation inside the call
 * would bypass the arena or break the budget), and drivers that keep every
 * device array themselves and must know the library's footprint up front.  It
 * needs no context and allocates nothing: no cudaMalloc, no cudaFree, no
 * allocating library routine.
 *   - stream: the caller's cudaStream_t (NULL = the legacy default stream).
 *   - position, q, lj1..lj4, nlist, numneigh and ff must be device memory of
 *     the current device (or managed memory); host pointers and buffers on
 *     another GPU are rejected with SOFIA_EINVAL, because using them would need
 *     a staging buffer or peer access.  potential, e_coul, virial_diag3 are host
 *     scalars and may be NULL.  Meaning of every argument as in
 *     sofia_force_nonbond_dsf.
 *   - np may be at most SOFIA_NOALLOC_MAX_ATOMS; larger systems get
 *     SOFIA_ETOOBIG.  The per-atom energy partials live in a fixed array of
 *     (5*SOFIA_NOALLOC_MAX_ATOMS + 1040) doubles (about 2.6 MB) compiled into
 *     the library, which every GPU that loads the library holds until exit.
 *   - The first call on a device does a one-time set-up: it looks up that
 *     array's device address (cudaGetSymbolAddress, with that device current)
 *     and caches it for the process.  Make that first call before any stream
 *     capture.  After a cudaDeviceReset of that device the cached address is
 *     stale, so do not call it across a device reset.
 *   - All calls share the one array: calls that overlap on the GPU (on
 *     different streams, threads or processes sharing the context) race and
 *     corrupt each other's energies; order them on one stream or serialise.
 *   - The call copies the energies to host memory and synchronises the stream
 *     before it returns.
 */
#define SOFIA_NOALLOC_MAX_ATOMS 65536
int sofia_force_nonbond_dsf_noalloc(void *stream, int np, const sofia_ainfo *position,
                                    const float *q, const float *lj1, const float *lj2,
                                    const float *lj3, const float *lj4, int ntypes,
                                    const int32_t *nlist, const int32_t *numneigh,
                                    int32_t neigh_alloc, float box, float ibox, double rcut2,
                                    double cut_coulsq, double alpha, double e_shift,
                                    double f_shift, float coulpre, float *ff, double *potential,
                                    double *e_coul, double *virial_diag3);

/*
 * dihedral_opls_DSF (Source/mod_force_dihed.f90:816-1092): OPLS torsion with
 * dihedcoeff[type][4] plus the 0.5-scaled DSF Coulomb and lj14 LJ of each
 * dihedral's 1-4 pair (:1003-1048).  dihedlist[n*5 + k] = i1,i2,i3,i4,type
 * (1-based, type <= ndihedtypes); dihedcoeff = [ndihedtypes][4] real*8;
 * lj14 = [4][ntypes][ntypes] real*8.  Forces are ADDED to ffh; energies are
 * ADDED to *e_dihedral, *e_coul_14, *pot_14.
 */
int sofia_pair14_dsf(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position, const float *q,
                     int ntypes, const double *lj14, int ndihed, const int32_t *dihedlist,
                     const double *dihedcoeff, int ndihedtypes, float box, float ibox, double rcut2,
                     double cut_coulsq, double alpha, double e_shift, double f_shift,
                     float coulpre, float *ffh, double *e_dihedral, double *e_coul_14,
                     double *pot_14);

/*
 * correct_12_bonds / correct_13_bonds / correct_14_bonds
 * (Source/mod_force_correction.f90:6-93, 95-184, 187-278): for each row m of
 * `list` (row stride `stride` ints, 1-based atom ids in columns col_a, col_b)
 * add the Ewald real-space erfc term minus (1-fudge) of the bare Coulomb to ffc
 * and the energy to *e_corr, the diagonal virial to virial3 (may be NULL).
 */
int sofia_correct_1x(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position, const float *q,
                     int npairs, const int32_t *list, int stride, int col_a, int col_b,
                     float box, float ibox, double cut_coulsq, double gewald, double fudge,
                     float coulpre, float *ffc, double *e_corr, double *virial3);

/*
 * get_greatestCluster (Source/mod_cluster.f90:15-83) with
 * build_ptta_wrap_cluster2 (Source/mod_build_ptta.f90:116-164), the molecule
 * centre/cell list (Source/mod_neighbor_cluster.f90:15-709) and the flood fill
 * and surface append (Source/mod_cluster.f90:163-247).  Returns the integer
 * size in *size_out.  ptta_full[n_gly*atoms_per_gly*3] (real*8) and
 * *greatest_belongsto are in/out exactly like the module variable and the
 * caller's `greatest` argument.  mrcut/denscut in Angstrom, densmin integer.
 * denstrack/belongsto (may be NULL) receive the per-molecule arrays.
 */
int sofia_greatest_cluster(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                           const int32_t *global_id, int n_gly, int atoms_per_gly, float box,
                           double mrcut, double denscut, int densmin, double *ptta_full,
                           int32_t *greatest_belongsto, int32_t *size_out, int32_t *denstrack,
                           int32_t *belongsto);

/* ------------------------------------------------------------------------ */
/*
 * Production path (device-resident system).  Replaces the same call,
 * lj_cut_coul_dsf_nonewton (Source/mod_force_nonbond.f90:105-196) with the list
 * kept by neighbor_wrapper (Source/mod_neighbor.f90:8-86), but keeps the list,
 * the static per-atom data and the positions resident on the GPU, the way the
 * reference's MIC path keeps `nlist` resident (`nocopy`, Source/mod_force.f90:446-461).
 * The list is a cluster-pair list over rlist = cut_coul + neighbor_pad and is
 * rebuilt on the device whenever an atom has moved more than neighbor_pad/2.
 *   precision SOFIA_PREC_MIXED: FP64 positions, FP64 displacement rounded to
 *       FP32, FP32 pair arithmetic, 64-bit fixed-point force sums (2^-32 units).
 *   precision SOFIA_PREC_FP64: the same kernel with FP64 pair arithmetic.
 * Pair terms, cutoffs and energies are those of lj_cut_coul_dsf_nonewton
 * (potential and e_coul are halved sums over the full list).
 */
#define SOFIA_PREC_MIXED 0
#define SOFIA_PREC_FP64 1

typedef struct {
    int np;              /* atoms */
    int ntypes;          /* atom types (<= 48) */
    float box;           /* cubic box edge, Angstrom (real*4 box) */
    double alpha;        /* DSF damping, 1/Angstrom */
    float cut_coul;      /* Coulomb cutoff (== rcut) */
    float rcut;          /* LJ cutoff */
    float neighbor_pad;  /* list skin */
    int precision;       /* SOFIA_PREC_MIXED or SOFIA_PREC_FP64 */
    const int32_t *type; /* [np] 1-based */
    const float *q;      /* [np] */
    const float *lj1, *lj2, *lj3, *lj4; /* [ntypes*ntypes] real*4 */
    const int32_t *specbond; /* [np*12] 1-based 1-2/1-3/1-4 partners */
    const int32_t *num3bond; /* [np] */
    const double *mass;      /* [ntypes] amu; may be NULL for force-only use */
} sofia_system_desc;

typedef struct sofia_system sofia_system;

int sofia_system_create(sofia_nb_ctx *ctx, const sofia_system_desc *desc, sofia_system **out);
int sofia_system_destroy(sofia_system *sys);
/* Drop-in for lj_cut_coul_dsf_nonewton (Source/mod_force_nonbond.f90:105-196):
 * reference AoS positions in (host or device), real*4 forces ff[np*3] out,
 * energies (each may be NULL).  Like the reference routine, pass
 * virial_diag3 = NULL unless the virial is wanted: a non-NULL pointer selects
 * the kernel that also accumulates it.  Returns after one stream
 * synchronization, with ff and the energies written. */
int sofia_force_nonbond_mixed(sofia_system *sys, const sofia_ainfo *position, float *ff,
                              double *potential, double *e_coul, double *virial_diag3);
/* Resident state: x, v as [np*3] doubles (host or device). */
int sofia_system_set_state(sofia_system *sys, const double *x, const double *v);
int sofia_system_get_state(sofia_system *sys, double *x, double *v, double *f);
/* Forces on the resident positions with the given precision.  flags:
 * SOFIA_EVAL_REBUILD forces a list rebuild, SOFIA_EVAL_VIRIAL adds the
 * diagonal virial.  energies[5] (may be NULL; energies are computed only when
 * given) = potential, e_coul, virial x, y, z. */
#define SOFIA_EVAL_REBUILD 1
#define SOFIA_EVAL_VIRIAL 2
int sofia_system_compute_forces(sofia_system *sys, int precision, int flags, double *energies);
/* stats[0..10]: list builds, clusters, list entries, row capacity, columns per
 * side, cluster capacity, column reach, kernels launched so far, prunes,
 * entries of the pruned (rc + margin) list, SHAKE groups that reached maxiter
 * (a warning, as the reference prints, Source/mod_shake.f90:322-324). */
int sofia_system_stats(sofia_system *sys, int64_t *stats, int nstats);
/* The resident cluster-pair list as atom pairs (a diagnostic query; copies the
 * list to the host).  which = 0: the outer list over rc + neighbor_pad made at
 * the last build; 1: the pruned list over rc + margin made at the last prune.
 * Each listed unordered pair appears once (half list): pairs[2k], pairs[2k+1]
 * are its 0-based atom ids, *npairs the number of pairs; SOFIA_ENEEDGROW when
 * capacity is smaller (only the first `capacity` are written).  xlist[np*3]
 * (may be NULL) receives the positions that list was made at.  The reference's
 * counterpart is the full list nlist/numneigh of build_neighbor_nonewton_nomic
 * (Source/mod_neighbor.f90:622-809), which holds every pair twice. */
int sofia_system_list_pairs(sofia_system *sys, int which, int64_t capacity, int32_t *pairs,
                            int64_t *npairs, double *xlist);
/* Ballistic drift x += dt*v of the resident positions, nsteps times (no forces). */
int sofia_system_drift(sofia_system *sys, double dt, int nsteps);
/* CUDA-event timers of the list build and the pair kernel on the system's
 * stream: returns and resets timers[4] = {build ms, builds, pair ms, pair
 * launches}; enable != 0 keeps timing on. */
int sofia_system_timers(sofia_system *sys, int enable, double *timers);

/* ------------------------------------------------------------------------ */
/*
 * Device-resident MD around the production path (residency kernels): velocity
 * Verlet (Source/mod_ensemble.f90:11-87), force-form Langevin
 * (Source/mod_langevin.f90:15-43; counter-based Philox4x32-10 noise keyed by
 * seed, atom and step instead of the reference's clock-seeded MT19937),
 * SHAKE (Source/mod_shake.f90:8-913), harmonic bonds and angles
 * (Source/mod_force_bond.f90:6-75, Source/mod_force_angle.f90:10-122), OPLS
 * torsions with their 0.5-scaled DSF/LJ 1-4 pairs
 * (Source/mod_force_dihed.f90:816-1092).  Step order of the reference loop
 * (Source/mod_integrate.f90:270-298).  Lists are 1-based like the reference's
 * bondlist(3,:), anglelist(4,:), dihedlist(5,:), shakeatom.
 */
#define SOFIA_TERM_BOND 1
#define SOFIA_TERM_ANGLE 2
#define SOFIA_TERM_TORSION 4
#define SOFIA_TERM_PAIR14 8
#define SOFIA_TERM_IMPROPER 16
/* Terms only sofia_system_md_forces selects (an MD step always has them). */
#define SOFIA_TERM_NONBOND 32  /* LJ + DSF pair forces of the production path */
#define SOFIA_TERM_LANGEVIN 128 /* Langevin friction + noise at the current step counter */
#define SOFIA_TERM_SHAKE 64    /* SHAKE constraint forces for the next step, on the sum of the others */
/* sofia_md_desc.flags */
#define SOFIA_MD_RATTLE 1   /* RATTLE velocity stage after the second half-kick */
#define SOFIA_MD_LJ_SHIFT 2 /* LJ pair energies shifted to zero at the cut-off (energy only) */
#define SOFIA_MD_NE 13 /* lj, coul, self, bond, angle, torsion, coul14, lj14, kinetic, total, T(K), step, improper */

typedef struct {
    double dt;          /* fs */
    double temperature; /* K (Langevin bath) */
    double gamma;       /* Langevin friction, 1/fs (0 = NVE) */
    uint64_t seed;      /* Langevin noise stream */
    int terms;          /* SOFIA_TERM_* bitmask */
    int nbond;
    const int32_t *bonds;      /* [nbond*3] i1, i2, type */
    int nbondtypes;
    const double *bond_coeff;  /* [nbondtypes*2] k (kcal/mol/A^2), r0 (A) */
    int nangle;
    const int32_t *angles;     /* [nangle*4] i1, i2 (middle), i3, type */
    int nangletypes;
    const double *angle_coeff; /* [nangletypes*2] k (kcal/mol/rad^2), theta0 (rad) */
    int ndihed;
    const int32_t *dihedrals;  /* [ndihed*5] i1..i4, type */
    int ndihedtypes;
    const double *dihed_coeff; /* [ndihedtypes*4] OPLS k1..k4 */
    const double *lj14;        /* [4*ntypes*ntypes] lj14_1..4 (needed for SOFIA_TERM_PAIR14) */
    int nshake;
    const int32_t *shake;      /* [nshake*5] num (1, 3, 4, -3), atoms */
    const double *shake_bond;  /* [nshake*3] bond lengths */
    int shake_maxiter;         /* 0 = 25 like the reference */
    double shake_tol;          /* 0 = 1e-4 like the reference */
    int nimpro;                /* harmonic impropers (SOFIA_TERM_IMPROPER) */
    const int32_t *impropers;  /* [nimpro*5] i1..i4, type */
    int nimprotypes;
    const double *impro_coeff; /* [nimprotypes*2] k (kcal/mol/rad^2), omega0 (rad) */
    /* SOFIA_MD_* options, 0 = the reference's scheme.  Neither changes positions:
     * SOFIA_MD_RATTLE projects the full-step velocities onto the constraints
     * (Andersen's RATTLE; the positions of SHAKE and RATTLE are the same
     * sequence, the reference has SHAKE alone, Source/mod_shake.f90:888-913),
     * SOFIA_MD_LJ_SHIFT subtracts E_LJ(rc) from every pair inside the cut-off
     * (the reference truncates, Source/mod_force_nonbond.f90:155). */
    int flags;
} sofia_md_desc;

int sofia_system_md_setup(sofia_system *sys, const sofia_md_desc *md);
/* Runs nsteps steps on the device (use_graph != 0: one CUDA graph per step kind);
 * energies (may be NULL) receive the last step's SOFIA_MD_NE values when
 * energy_every > 0.  Positions and velocities stay resident
 * (sofia_system_get_state / set_state move them). */
int sofia_system_md_run(sofia_system *sys, int nsteps, int energy_every, int use_graph,
                        double *energies);
/* Forces of one MD step at the resident positions and velocities, without
 * stepping: zero, nonbonded pairs, bonded terms and 1-4 pairs, merged like
 * force_wrapper_DSF (Source/mod_force.f90:510-554), plus the Langevin force
 * (Source/mod_langevin.f90:15-43) and SHAKE's constraint forces for the next
 * step (Source/mod_shake.f90:8-85, 888-913), restricted to the SOFIA_TERM_*
 * bits in `terms` (bonded bits only act where md_setup enabled them; SHAKE acts
 * on the sum of the other selected terms).  f[np*3] (may be NULL) receives the
 * fixed-point sum as doubles in atom order; energies[SOFIA_MD_NE] (may be
 * NULL; computed only when given) the selected terms' energies and the
 * kinetic energy.  The next sofia_system_md_run recomputes its own forces. */
int sofia_system_md_forces(sofia_system *sys, int terms, double *f, double *energies);

/*
 * Batches of independent replicas (no reference counterpart: the reference
 * runs one replica per MPI rank, Source/MD.f90:26-44, with no exchange).
 * Each kernel of an MD step runs once for all replicas (up to 256, of any
 * sizes and boxes) over a device table of the replicas' buffers, so a batch
 * step is one launch per kernel; steps run as captured CUDA graphs of `seg`
 * steps (default 100).  A replica's trajectory is bit-identical to the same
 * replica run alone.  All replicas must share precision, atom types, cut-off
 * and DSF constants (the box may differ) and be set up for MD.
 *   sofia_batch_md_run: nsteps steps of every replica; energies = [n][SOFIA_MD_NE]
 *       (may be NULL) receive each replica's energies of the last step when
 *       energy_every > 0 (only that step computes them).
 *   sofia_batch_set_systems: new members for the next run (continuous
 *       batching); the captured graphs are kept when the new members share the
 *       pair constants, so membership changes need no recapture.
 *   sofia_batch_set_segment: steps per captured graph (1..1000).
 */
typedef struct sofia_batch sofia_batch;
int sofia_batch_create(sofia_nb_ctx *ctx, sofia_system *const *systems, int n, sofia_batch **out);
int sofia_batch_destroy(sofia_batch *batch);
int sofia_batch_md_run(sofia_batch *batch, int nsteps, int energy_every, double *energies);
int sofia_batch_set_systems(sofia_batch *batch, sofia_system *const *systems, int n);
int sofia_batch_set_segment(sofia_batch *batch, int steps);
/* Prune margin (A) of the pruned inner list (default 0.4): the tuning knob
 * the autotuner picks per size class.  Any margin > 0 gives the same forces:
 * the list is re-pruned as soon as an atom has moved more than margin/2. */
int sofia_system_set_margin(sofia_system *sys, double margin);
/* Cluster shape: the xy column width as a multiple (0.5..2) of the cube side of
 * 8 atoms (1 = default; < 1 taller, > 1 flatter clusters).  Reallocates the
 * column and list buffers; the next evaluation rebuilds the lists.  The
 * autotuner's geometry knob, chosen per size class with the prune margin. */
int sofia_system_set_cluster_shape(sofia_system *sys, double aspect);

/*
 * Snapshot / rollback of the resident replica state, replacing the in-memory
 * copies nuc_move makes before a trial segment and restores on rejection
 * (Source/mod_nucleation.f90:318-389 and :453-531).  The snapshot holds
 * positions, velocities and the thermostat step counter.  Both calls make the
 * next evaluation rebuild the neighbor structures and recompute the forces
 * from the (saved) positions, so the run continued after a snapshot and the
 * run repeated after a rollback take bit-identical steps.
 * sofia_system_rollback returns SOFIA_ESTATE when no snapshot was taken.
 */
int sofia_system_snapshot(sofia_system *sys);
int sofia_system_rollback(sofia_system *sys);
/* get_greatestCluster (Source/mod_cluster.f90:15-83) on the resident positions
 * of a system, which never leave the device (nuc_move keeps the replica state
 * between segments, Source/mod_nucleation.f90:396-449): the FP64 positions are
 * wrapped into (0, box] as real*4 (x - L floor(x/L), then +box if <= 0) and
 * analysed like sofia_greatest_cluster with global ids 1..np.  The glycine
 * molecules are the first n_gly * atoms_per_gly atoms.  ptta_full (host or
 * device) and *greatest_belongsto are in/out as in sofia_greatest_cluster;
 * ptta_full == NULL uses the system's own device copy, set from its current
 * positions by the first such call. */
int sofia_system_greatest_cluster(sofia_system *sys, int n_gly, int atoms_per_gly, double mrcut,
                                  double denscut, int densmin, double *ptta_full,
                                  int32_t *greatest_belongsto, int32_t *size_out);
/* Device memory the system holds now (buffers grow with the list capacity). */
int sofia_system_device_bytes(sofia_system *sys, int64_t *bytes);
/* Thermostat step counter (counter of the Langevin noise).  Reading it with
 * the state and setting it on resume continues the same noise sequence; the
 * reference restart (read_dump_global_id_v, Source/mod_datadump.f90:216-252)
 * holds no such counter.  SOFIA_ESTATE before sofia_system_md_setup. */
int sofia_system_md_get_step(sofia_system *sys, long long *step);
int sofia_system_md_set_step(sofia_system *sys, long long step);

#ifdef __cplusplus
}
#endif
#endif
