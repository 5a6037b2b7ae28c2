// system.cuh -- device-resident system (one replica) of the production path.
//
// HBM layout (per system):
//   global-order atom state   x/v (double SoA), f (int64 fixed point SoA),
//                             type (int32), q (float), inverse mass (double),
//                             positions at the last list build (double SoA)
//   cluster order             AtomRec[slot] = {double x,y,z; float q; int type}
//                             (32 B, two 16 B loads), slot -> global index,
//                             8 slots per cluster, clusters grouped by xy column
//                             and sorted by z inside a column
//   cluster-pair list         per i-cluster a row of jcap entries:
//                             int32 {j cluster | image << 26} + uint64 pair mask
#pragma once
#include <stdint.h>

#include "common.cuh"

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
    // global-order state
    DevBuf x[3], v[3], f[3], xref[3], img[3];
    DevBuf type, q, invm, mass, specbond, num3bond;
    DevBuf ljtab;                      // float4 {lj1,lj2,lj3,lj4} per type pair
    // cluster structures
    DevBuf col_count, col_start, col_fill, col_atoms, col_key, cl_start;
    DevBuf slot_orig, rec, recf, bb, jlist, jmask, jcount, nclusters;
    DevBuf status_local;
    DevBuf energy;                      // per-i-cluster energy partials (pot, ecoul, vir x,y,z)
    DevBuf red;                         // reduced energies
    DevBuf flag;                        // rebuild flag (int)
    DevBuf stage_pos, stage_ff;
    // pruned inner list (rc + margin) and the positions it was pruned at
    DevBuf ilist, imask, icount, xprn[3], part;
    double margin = 0.6;
    long long n_prunes = 0;
    int built = 0;
    long long n_builds = 0;
    long long launches = 0;             // kernels launched by this system (all paths)
    // optional CUDA-event timing of the list build and the pair kernel
    int timing = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double t_build_ms = 0.0, t_pair_ms = 0.0;
    long long n_pair = 0, n_build_timed = 0;
    int pending_build = 0, pending_pair = 0;
};

}  // namespace sofia
