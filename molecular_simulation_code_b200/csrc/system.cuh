// system.cuh -- device-resident system (one replica) of the production path.
//
// HBM layout (per system):
//   global-order atom state   x/v (double SoA), f (int64 fixed point SoA),
//                             type (int32), q (float), inverse mass (double),
//                             positions at the last list build (double SoA)
//   cluster order             AtomRec[slot] = {double x,y,z; float q; int type}
//                             (32 B, two 16 B loads), slot -> global index,
//                             8 slots per cluster, clusters grouped by xy column
//                             and sorted by z inside a column; an FP32 copy for
//                             the prune as float x[8], y[8], z[8] per cluster
//                             (96 B, six 16 B loads)
//   cluster-pair list         per i-cluster a row of jcap entries:
//                             int32 {j cluster | image << 26} + uint64 pair mask
#pragma once
#include <stdint.h>

#include "common.cuh"
#include "langevin.cuh"

namespace sofia {

constexpr int CL = 8;                  // atoms per cluster
constexpr double FIX_SCALE = 4294967296.0;  // 2^32 fixed-point units per kcal/mol/A
constexpr double FIX_INV = 1.0 / 4294967296.0;
constexpr int IMG_SHIFT = 26;

struct __align__(16) AtomRec {
    double x, y, z;
    float q;
    int type;
};

// Device-resident MD state (velocity Verlet + force-form Langevin + SHAKE +
// bonded terms) of one system.
struct Md {
    int ready = 0;
    double dt = 2.0, temperature = 300.0, gamma = 0.0;  // fs, K, 1/fs
    unsigned long long seed = 0;
    int nbond = 0, nangle = 0, ndihed = 0, nshake = 0, nimpro = 0;
    int nbt = 0, nat = 0, ndt = 0;
    DevBuf bonds, bcoef, angles, acoef, diheds, dcoef, lj14, shake, sbond, impros, icoef;
    int shake_maxiter = 25;
    double shake_tol = 1e-4;
    int terms = 15;
    int rattle = 0;        // RATTLE velocity stage after the second half-kick (SOFIA_MD_RATTLE)
    DevBuf eterm;          // per-term energy partials
    DevBuf ered;           // reduced energies
    DevBuf bpart;          // stage-1 partials of the batched energy sums
    DevBuf step_dev;       // device step counter (RNG counter inside graphs)
    DevBuf snap[7];        // x, v (3 each) and the step counter at segment start
    DevBuf keep[7];        // caller-requested snapshot (same layout), for rollback
    long long keep_step = 0;
    int has_keep = 0;
    double e_self = 0.0;
    int ndof = 0;
    long long step = 0;
    int forces_valid = 0;
    // captured graphs: [0] one step, [1] one step with energies, [2] seg steps,
    // [3] seg steps with energies on the last; inside a segment each step's
    // closing half-kick is fused into the next step's kick and drift
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    long long graph_launches[4] = {0, 0, 0, 0};
    int seg = 10;
    int graph_ok = 0;
};

struct Sys {
    sofia_nb_ctx *ctx = nullptr;
    int n = 0, ntypes = 0, precision = 0;
    double L = 0.0;
    float box = 0.0f;
    double alpha = 0.0, rc = 0.0, rlist = 0.0, skin = 0.0, e_shift = 0.0, f_shift = 0.0;
    float coulpre = 0.0f;
    double r_excl = 6.0;
    // column grid
    int ncx = 0, ncols = 0, max_clusters = 0, jcap = 0, ncol_reach = 0;
    double s_col = 0.0;
    double aspect = 1.0;              // column width / cube side of 8 atoms (cluster shape)
    // global-order state
    DevBuf x[3], v[3], f[3], xref[3], img[3];
    DevBuf type, q, invm, mass, specbond, num3bond;
    DevBuf ljtab;                      // float4 {lj1,lj2,lj3,lj4} per type pair
    // cluster structures
    DevBuf col_count, col_start, col_fill, col_atoms, col_key, cl_start;
    DevBuf slot_orig, rec, bb, jlist, jmask, jcount, nclusters;
    DevBuf recf;                        // FP32 positions per cluster: x[8], y[8], z[8]
    DevBuf fslot;                       // pair forces in cluster-slot order, 64-bit fixed point [3][slots]
    DevBuf sref;                        // build-time data in slot order (see pack_body)
    DevBuf atom_slot;                   // cluster slot of every atom (inverse of slot_orig)
    DevBuf status_local;
    DevBuf energy;                      // per-i-cluster energy partials (pot, ecoul, vir x,y,z)
    DevBuf red;                         // reduced energies
    DevBuf flag;                        // rebuild flag (int)
    DevBuf stage_pos, stage_ff;
    DevBuf cl_pos, cl_gid;              // resident positions as real*4 ainfo records, ids 1..n (cluster analysis)
    DevBuf ptta;                        // resident ptta_full of the cluster analysis
    int ptta_atoms = 0;                 // glycine atoms ptta holds (0 = not yet set)
    // pruned inner list (rc + margin) and the positions it was pruned at
    DevBuf ilist, imask, icount, xprn[3], part, dcount;
    double margin = 0.4;
    // LJ energy of every pair inside the cut-off shifted by -E_LJ(rc) (SOFIA_MD_LJ_SHIFT);
    // forces are unchanged, so only the energy bookkeeping differs
    int lj_shift = 0;
    long long n_prunes = 0;
    int built = 0;
    long long n_builds = 0;
    long long launches = 0;             // kernels launched by this system (all paths)
    long long shake_nc = 0;             // SHAKE groups that reached maxiter (warnings)
    // optional CUDA-event timing of the list build and the pair kernel
    int timing = 0;
    cudaGraphExec_t dropin[3] = {nullptr, nullptr, nullptr};  // drop-in force call: forces / +energy / +virial
    long long dropin_launches[3] = {0, 0, 0};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double t_build_ms = 0.0, t_pair_ms = 0.0;
    long long n_pair = 0, n_build_timed = 0;
    int pending_build = 0, pending_pair = 0;
    Md md;
};


// Arguments of the bonded-term kernel (md.cu): torsions with their 1-4 pairs.
struct DihArgs {
    int nd, ntypes, terms;
    const int *dl;
    const double *dc, *lj14;
    const double *x, *y, *z;
    const int *type;
    const float *q;
    double L, alpha, EWALD_P, A1, A2, A3, A4, A5, MY_PIS, e_shift, f_shift, cut_coulsq, rcut2;
    float coulpre;
    long long *fx, *fy, *fz;
    double *e;  // [nd][3] torsion, coul14, lj14
};

// All bonded terms of a step in one launch: threads [0, nb) take bonds, the
// next na angles, then nd dihedrals (torsion and 1-4 pair), then ni impropers.
// A count of 0 switches a term off.
struct BondedArgs {
    int nb, na, nd, ni;
    const int *bl, *al, *il;
    const double *bc, *ac, *ic;
    double *eb, *ea, *ei;
    DihArgs dih;
};

// ---------------------------------------------------------------------------
// Batched replicas: every kernel of an MD step runs once for all replicas of a
// batch.  The launch walks "virtual blocks" in a grid-stride loop; the blocks of
// kernel kind K for replica r are [pre[K][r], pre[K][r+1]), each with the block
// size of the single-system kernel, so a block never spans two replicas and the
// single-system kernel bodies run unchanged on replica r's buffers.  Replica
// data live in a device table that the host rewrites when membership or a
// buffer changes; the captured graphs only hold the table's address.
enum BatchKind {
    BK_A256 = 0,  // ceil(n / 256): per-atom kernels
    BK_SCAN,      // 1: the column scans (1024 threads)
    BK_COLS,      // ncols: the column sort
    BK_S256,      // ceil(max_clusters * 8 / 256): per-slot kernels
    BK_W256,      // ceil(max_clusters * 32 / 256): warp-per-cluster kernels
    BK_B128,      // ceil(bonded terms / 128)
    BK_G128,      // ceil(SHAKE groups / 128)
    BK_RED,       // RED_BLOCKS: stage 1 of the pair-energy sums
    BK_REP,       // 1 per replica
    BK_MRED,      // MD_NJOB * MRED: stage 1 of the MD energy sums
    BK_MJOB,      // MD_NJOB: stage 2 of the MD energy sums
    BK_N
};
constexpr int MAXREP = 256;
// resident 256-thread blocks per SM of the batched per-atom streaming kernels
// (kick and drift, pack, unpack): their replica arguments come from the device
// table, and without a bound the compiler keeps them all in registers (70-87),
// which halves the warps that hide memory latency (64 replicas: 380.5 -> 386.7 M
// atom-steps/s with the bound)
#ifndef SOFIA_BATCH_STREAM_MINB
#define SOFIA_BATCH_STREAM_MINB 4
#endif
constexpr int RED_BLOCKS = 128;  // blocks of stage 1 of the pair-energy sums
constexpr int MD_NJOB = 7;  // bonds, angles, torsion, coul14, lj14, impropers, kinetic

struct RepDev {
    int n, ncols, ncx, maxcl, jcap, reach, nslots, nshake, rattle, shake_maxiter;
    double L, s_col, lim2, plim2, h, dt, dtsq, shake_tol;
    float rl, rl2, rexcl2, rin2, rfar2;
    // global-order atom state
    double *x, *y, *z, *vx, *vy, *vz;
    long long *fx, *fy, *fz;
    double *rx, *ry, *rz, *ix, *iy, *iz, *px, *py, *pz;
    const double *invm, *mass;
    const float *q;
    const int *type, *specbond, *num3bond;
    // list build and cluster order
    int *col_count, *col_start, *col_fill, *col_atoms, *col_of, *cl_start, *slot_orig, *cl_col,
        *atom_slot;
    float *col_key;
    AtomRec *rec;
    double *sref;
    float *recf;
    float4 *bb;
    int *jlist, *jcount, *ilist, *icount;
    unsigned long long *jmask, *imask, *fslot;
    int *ncl, *flag, *status, *ctx_status;
    long long *dcount;
    const float4 *ljtab;
    double *energy, *part, *red;
    // MD
    long long *step;
    LangevinArgs lg;
    BondedArgs b;
    const int *shake;
    const double *sbond;
    double *ered, *ebpart, *ke;
    // segment-start snapshot (x, y, z, vx, vy, vz; the step counter)
    double *snap[6];
    long long *snap_step;
    // energy-sum jobs: column count n (0 = off), width, column, input, output slot of ered
    int job_n[MD_NJOB], job_w[MD_NJOB], job_c[MD_NJOB], job_slot[MD_NJOB];
    const double *job_in[MD_NJOB];
};

// Replicas whose list trigger fired this step, per trigger mask: BA_BUILD
// (bit 0: rebuild) and BA_PRUNE (bits 0-1: rebuild or prune).  The conditional
// kernels walk only the virtual blocks of these replicas: apre[m][K] is the
// prefix of kind-K blocks over the active replicas act[m][0 .. nact[m]).
enum BatchActive { BA_BUILD = 0, BA_PRUNE = 1, BA_N = 2 };

struct BatchDev {
    int nrep;
    int nact[BA_N];
    int act[BA_N][MAXREP];
    int apre[BA_N][BK_N][MAXREP + 1];
    int pre[BK_N][MAXREP + 1];
    RepDev rep[MAXREP];
};

// Batched kernels walk virtual blocks in grid-stride order: block b takes
// virtual blocks b, b + gridDim.x, ...  The pair, search and prune kernels are
// launched with one block per virtual block of all members at capture time, so
// each block takes at most one and the hardware block scheduler balances the
// uneven rows; members added later without a recapture are covered by the
// stride.  ACTIVE_LOOP walks the kind-KIND blocks of the replicas active for
// trigger mask M (BatchActive).  Inside, d is the replica's entry and lb the
// block index within that replica.
#define SOFIA_BATCH_ACTIVE_LOOP(KIND, M)                                         \
    for (int vb = blockIdx.x;; vb += gridDim.x) {                                \
        const int na_ = *reinterpret_cast<const volatile int *>(&tab->nact[M]);  \
        const int *ap_ = tab->apre[M][KIND];                                     \
        if (vb >= ap_[na_]) break;                                               \
        const int a_ = batch_rep(ap_, na_, vb);                                  \
        const RepDev &d = tab->rep[tab->act[M][a_]];                             \
        const int lb = vb - ap_[a_];
// Replica of virtual block vb: the last r with pre[r] <= vb.
__device__ __forceinline__ int batch_rep(const int *__restrict__ pre, int nrep, int vb) {
    int lo = 0, hi = nrep - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= vb)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Fills the nonbonded-path part of a replica's table entry (mixed.cu).
void repdev_fill_pair(const Sys *s, RepDev *d);
// The nonbonded part of one batched MD step (mixed.cu): list build and prune on
// each replica's trigger, record pack, pair kernel, force unpack with the
// Langevin force, and (energy) the pair-energy sums.  All replicas share the
// pair constants k (all but the box) and the precision.
// nsm: multiprocessors of the device (the grid-stride launches are sized from it).
// pair_blocks: the warp-per-cluster virtual blocks over all members when the graph
// is captured, the grid of the pair, search and prune kernels (later members that
// need more are covered by the kernels' grid-stride loops).
void batch_pair_path(BatchDev *tab, const Sys *s0, int precision, bool energy,
                     cudaStream_t st, int nsm, int pair_blocks);
// raises the batched pair kernels' dynamic shared-memory limit for nt atom types
cudaError_t batch_pair_smem_optin(int nt);
// The pair constants a captured batch graph holds (everything but the box).
struct PairKey {
    int precision, ntypes, lj_shift;
    double rc, alpha, e_shift, f_shift;
    float coulpre;
};
inline PairKey pair_key(const Sys *s) {
    return PairKey{s->precision, s->ntypes, s->lj_shift, s->rc, s->alpha, s->e_shift,
                   s->f_shift, s->coulpre};
}
inline bool operator==(const PairKey &a, const PairKey &b) {
    return a.precision == b.precision && a.ntypes == b.ntypes && a.lj_shift == b.lj_shift &&
           a.rc == b.rc && a.alpha == b.alpha && a.e_shift == b.e_shift &&
           a.f_shift == b.f_shift && a.coulpre == b.coulpre;
}
// True when two systems' pair constants agree in everything but the box.
inline bool pair_const_compatible(const Sys *a, const Sys *b) { return pair_key(a) == pair_key(b); }

// evaluation entry points (mixed.cu)
int sys_eval(Sys *s, int precision, bool energy, bool virial, bool force_build);
// count_flag (may be NULL): the trigger word whose build/prune bits are counted
// and then cleared; lg (may be NULL): Langevin force added to the pair forces;
// ff_out (may be NULL): the forces also written as real*4 [n][3] in atom order.
int sys_pair(Sys *s, int precision, bool energy, bool virial, int *count_flag = nullptr,
             const LangevinArgs *lg = nullptr, float *ff_out = nullptr);
// disp_done: the caller already ORed the displacement-trigger bits into a
// cleared trigger word (the MD step's fused kick/drift kernel does).
// lg (may be NULL): Langevin force added while the pair forces are written.
// ff_out (may be NULL): as for sys_pair.
int sys_step_forces(Sys *s, int precision, bool energy, bool virial, bool force_build,
                    bool disp_done = false, const LangevinArgs *lg = nullptr,
                    float *ff_out = nullptr);
// After a device segment: SOFIA_ENEEDGROW (and a larger row capacity) if a list
// row overflowed.  status: the segment's status words already on the host, or
// nullptr to copy them (one stream synchronization).
int sys_list_overflow(Sys *s, const int32_t *status = nullptr);
// Frees the captured drop-in force graphs (they bake in list pointers and the margin).
void dropin_drop(Sys *s);
// Column grid and list capacities for a cluster shape (mixed.cu).
bool sys_geometry(Sys *s, double aspect);
// After a change of list geometry or margin (md.cu): drops the system's captured
// graphs and makes the next MD run start with a fresh build and force evaluation.
void md_invalidate(Sys *s);

}  // namespace sofia

namespace sofia {
// Squared minimum-image displacement since a reference position; non-finite
// positions give a huge value so that they trigger a rebuild.
__device__ __forceinline__ double disp2(double x, double y, double z, double rx, double ry,
                                        double rz, double L) {
    double dx = x - rx, dy = y - ry, dz = z - rz;
    dx -= L * rint(dx / L);
    dy -= L * rint(dy / L);
    dz -= L * rint(dz / L);
    const double d2 = dx * dx + dy * dy + dz * dz;
    return (d2 == d2) ? d2 : 1e300;
}
}  // namespace sofia

struct sofia_system {
    sofia::Sys s;
};
