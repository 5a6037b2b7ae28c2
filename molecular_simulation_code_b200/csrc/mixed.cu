// mixed.cu -- production nonbonded path: cluster-pair list + LJ/DSF kernel.
//
// The reference evaluates LJ + damped-shifted-force Coulomb over a full
// per-atom Verlet list in FP64 (Source/mod_force_nonbond.f90:105-196).  Here
// atoms are grouped into clusters of 8 (xy columns, sorted by z) and the half
// list holds each cluster pair whose bounding boxes come within
// rlist = rc + skin once, with a 64-bit mask of the interacting atom pairs
// (padding, self pairs and 1-2/1-3/1-4 exclusions removed).  A prune keeps the
// entries with pairs inside rc + margin and their in-range bits.  One warp
// works on one i-cluster: lane = (i atom, j atom pair) covers the 8x8 pair
// tile, the i force stays in registers and each entry's j forces are reduced
// over lanes and added with 64-bit fixed-point atomics.  Positions are FP64 in
// HBM; each pair displacement is formed in FP64 and rounded to FP32 (mixed) or
// kept in FP64 (plain FP64 twin); FP32 partial sums are flushed to 64-bit fixed
// point (2^-32 kcal/mol/A), so forces are bit-reproducible and independent of
// the order of the atomics.
//
// The list stays valid while no atom has moved more than skin/2 since the
// build (checked every step on the device; the reference triggers at the full
// skin, Source/mod_neighbor.f90:895-913).
#include <cmath>
#include <algorithm>
#include <vector>

#include "system.cuh"

namespace sofia {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAX_COL = 2048;  // atoms per xy column handled by the in-column sort

// Build and prune kernels take an optional device flag: when `cond` is given
// they return at once unless (cond[0] & cmask) != 0, so a whole step can be
// launched (or captured into a CUDA graph) without a host round trip.
#define SOFIA_COND_RETURN \
    if (cond && !(cond[0] & cmask)) return
// List entries between the pair kernel's FP32 -> fixed-point flushes of the i
// forces: one flush per 32-entry batch of a list row (at 275k atoms, 16 ->
// 32: force-only MD +0.9 %, the energy kernel 0.531 -> 0.517 ms).
#ifndef SOFIA_PAIR_FLUSH
#define SOFIA_PAIR_FLUSH 32
#endif
#ifndef SOFIA_PAIR_MINB
#define SOFIA_PAIR_MINB 4
#endif
#ifndef SOFIA_PAIR_MINB_EN
#define SOFIA_PAIR_MINB_EN 4
#endif
// Threads per block of the single-system pair kernels (one warp per i-cluster):
// the force-only kernel runs 8 blocks of 128 per SM (0.449 -> 0.447 ms at 275k,
// MD +0.4 %); the energy kernels keep 4 blocks of 256, because every block
// refills the 16 KB three-index LJ table (with 128 threads: 0.526 -> 0.556 ms).
#ifndef SOFIA_PAIR_BLOCK
#define SOFIA_PAIR_BLOCK 128
#endif
#ifndef SOFIA_PAIR_BLOCK_EN
#define SOFIA_PAIR_BLOCK_EN 256
#endif
template <typename T, bool EN>
constexpr int pair_block() { return (sizeof(T) == 4 && !EN) ? SOFIA_PAIR_BLOCK : SOFIA_PAIR_BLOCK_EN; }
template <typename T, bool EN>
constexpr int pair_minb() {
    return sizeof(T) == 4 ? (EN ? SOFIA_PAIR_MINB_EN : SOFIA_PAIR_MINB * 256 / SOFIA_PAIR_BLOCK)
                          : 2 * 256 / SOFIA_PAIR_BLOCK_EN;
}
#ifndef SOFIA_PAIR_HYBRID
#define SOFIA_PAIR_HYBRID 1
#endif
#ifndef SOFIA_PRUNE_MINB
#define SOFIA_PRUNE_MINB 4
#endif
// FP32 energy kernels of systems with at most this many atom types read their
// LJ parameters from a three-index table (i type pair, j type): one 16-byte
// load gives both packed operands of a lane's two pairs, where the two-index
// tables take two 8-byte loads for the force and two for the energy (0 = never).
// The force-only kernel keeps the two-index tables: there the 16-byte loads
// from many distinct addresses cost more shared-memory wavefronts than they
// save instructions (0.468 -> 0.478 ms per launch at 275k atoms; the energy
// kernel 0.556 -> 0.549 ms).
#ifndef SOFIA_PAIR_TRI_MAX
#define SOFIA_PAIR_TRI_MAX 10
#endif
#ifndef SOFIA_SEARCH_ZWIN
#define SOFIA_SEARCH_ZWIN 1
#endif
constexpr int FLUSH = SOFIA_PAIR_FLUSH;  // list entries between FP32 -> fixed-point flushes of the i forces
static_assert(FLUSH >= 1 && FLUSH <= 32 && (32 % FLUSH) == 0, "FLUSH must divide 32");

__device__ __forceinline__ double wrap_shift(double x, double L) {
    // shift s with x + s in [0, L)
    return -L * floor(x / L);
}

__device__ __forceinline__ void wrap_bin_body(int bx, const int *__restrict__ cond, int cmask, int n,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, double L, double s_col, int ncx,
                           double *__restrict__ ix, double *__restrict__ iy,
                           double *__restrict__ iz, double *__restrict__ rx,
                           double *__restrict__ ry, double *__restrict__ rz,
                           int *__restrict__ col_of, int *__restrict__ col_count,
                           float *__restrict__ zkey) {
    SOFIA_COND_RETURN;
    int i = bx * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = x[i], py = y[i], pz = z[i];
    double sx = wrap_shift(px, L), sy = wrap_shift(py, L), sz = wrap_shift(pz, L);
    double wx = px + sx, wy = py + sy, wz = pz + sz;
    // guard the upper edge after rounding
    if (wx >= L) { wx -= L; sx -= L; }
    if (wy >= L) { wy -= L; sy -= L; }
    if (wz >= L) { wz -= L; sz -= L; }
    ix[i] = sx;
    iy[i] = sy;
    iz[i] = sz;
    rx[i] = px;
    ry[i] = py;
    rz[i] = pz;
    int cx = min((int)(wx / s_col), ncx - 1);
    int cy = min((int)(wy / s_col), ncx - 1);
    cx = max(cx, 0);
    cy = max(cy, 0);
    const int c = cx + cy * ncx;
    col_of[i] = c;
    zkey[i] = (float)wz;
    atomicAdd(&col_count[c], 1);
}
__global__ void k_wrap_bin(const int *__restrict__ cond, int cmask, int n,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, double L, double s_col, int ncx,
                           double *__restrict__ ix, double *__restrict__ iy,
                           double *__restrict__ iz, double *__restrict__ rx,
                           double *__restrict__ ry, double *__restrict__ rz,
                           int *__restrict__ col_of, int *__restrict__ col_count,
                           float *__restrict__ zkey) {
    SOFIA_PDL_ENTRY();
    wrap_bin_body(blockIdx.x, cond, cmask, n, x, y, z, L, s_col, ncx, ix, iy, iz, rx, ry, rz, col_of, col_count, zkey);
}

// Column scans of a build, one block: col_start = exclusive scan of the atom
// counts, cl_start = exclusive scan of the cluster counts (ceil(count/8)), the
// total cluster count into ncl.  The counts are cleared for the next build.
__device__ __forceinline__ void scan_cols_body(int bx, const int *__restrict__ cond, int cmask, int n,
                            int *__restrict__ col_count, int *__restrict__ col_start,
                            int *__restrict__ cl_start, int *__restrict__ ncl) {
    SOFIA_COND_RETURN;
    __shared__ int s1[1024], s2[1024];
    __shared__ int carry1, carry2;
    const int t = threadIdx.x;
    if (t == 0) carry1 = carry2 = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        const int v = (base + t < n) ? col_count[base + t] : 0;
        const int w = (v + CL - 1) / CL;
        s1[t] = v;
        s2[t] = w;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const int a1 = (t >= off) ? s1[t - off] : 0;
            const int a2 = (t >= off) ? s2[t - off] : 0;
            __syncthreads();
            s1[t] += a1;
            s2[t] += a2;
            __syncthreads();
        }
        if (base + t < n) {
            col_start[base + t] = carry1 + s1[t] - v;
            cl_start[base + t] = carry2 + s2[t] - w;
            col_count[base + t] = 0;
        }
        __syncthreads();
        if (t == 1023) {
            carry1 += s1[1023];
            carry2 += s2[1023];
        }
        __syncthreads();
    }
    if (t == 0) {
        col_start[n] = carry1;
        cl_start[n] = carry2;
        ncl[0] = carry2;
    }
}
__global__ void k_scan_cols(const int *__restrict__ cond, int cmask, int n,
                            int *__restrict__ col_count, int *__restrict__ col_start,
                            int *__restrict__ cl_start, int *__restrict__ ncl) {
    SOFIA_PDL_ENTRY();
    scan_cols_body(blockIdx.x, cond, cmask, n, col_count, col_start, cl_start, ncl);
}

__device__ __forceinline__ void col_scatter_body(int bx, const int *__restrict__ cond, int cmask, int n,
                              const int *__restrict__ col_of,
                              const int *__restrict__ col_start, int *__restrict__ col_fill,
                              int *__restrict__ col_atoms) {
    SOFIA_COND_RETURN;
    int i = bx * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = col_of[i];
    const int s = atomicAdd(&col_fill[c], 1);
    col_atoms[col_start[c] + s] = i;
}
__global__ void k_col_scatter(const int *__restrict__ cond, int cmask, int n,
                              const int *__restrict__ col_of,
                              const int *__restrict__ col_start, int *__restrict__ col_fill,
                              int *__restrict__ col_atoms) {
    SOFIA_PDL_ENTRY();
    col_scatter_body(blockIdx.x, cond, cmask, n, col_of, col_start, col_fill, col_atoms);
}

// Sort each column by (z, index); then lay the column out as clusters of 8.
__device__ __forceinline__ void col_sort_assign_body(int bx, const int *__restrict__ cond, int cmask, int ncols,
                                  const int *__restrict__ col_start,
                                  int *__restrict__ col_atoms, const float *__restrict__ zkey,
                                  const int *__restrict__ cl_start, int *__restrict__ slot_orig,
                                  int *__restrict__ cl_col, int *__restrict__ atom_slot,
                                  int *__restrict__ col_fill, int *__restrict__ status) {
    SOFIA_COND_RETURN;
    __shared__ unsigned long long s[MAX_COL];
    const int c = bx;
    if (c >= ncols) return;
    // the scatter is done with this column's fill counter: clear it for the next build
    if (threadIdx.x == 0) col_fill[c] = 0;
    const int b = col_start[c], nc = col_start[c + 1] - b;
    if (nc > MAX_COL) {
        if (threadIdx.x == 0) atomicAdd(&status[ST_CELLOVER], 1);
        return;
    }
    int m = 1;
    while (m < nc) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        if (t < nc) {
            const int i = col_atoms[b + t];
            const unsigned zb = __float_as_uint(fmaxf(zkey[i], 0.0f));
            s[t] = ((unsigned long long)zb << 32) | (unsigned)i;
        } else {
            s[t] = ~0ull;
        }
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < m; t += blockDim.x) {
                const int ix = t ^ j;
                if (ix > t) {
                    const bool up = ((t & k) == 0);
                    const unsigned long long a = s[t], bb = s[ix];
                    if ((a > bb) == up) {
                        s[t] = bb;
                        s[ix] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    const int c0 = cl_start[c], ncl = cl_start[c + 1] - c0;
    for (int t = threadIdx.x; t < ncl * CL; t += blockDim.x) {
        const int o = (t < nc) ? (int)(s[t] & 0xffffffffu) : -1;
        slot_orig[c0 * CL + t] = o;
        if (o >= 0) atom_slot[o] = c0 * CL + t;
        if ((t & (CL - 1)) == 0) cl_col[c0 + t / CL] = c;
    }
}
__global__ void k_col_sort_assign(const int *__restrict__ cond, int cmask, int ncols,
                                  const int *__restrict__ col_start,
                                  int *__restrict__ col_atoms, const float *__restrict__ zkey,
                                  const int *__restrict__ cl_start, int *__restrict__ slot_orig,
                                  int *__restrict__ cl_col, int *__restrict__ atom_slot,
                                  int *__restrict__ col_fill, int *__restrict__ status) {
    SOFIA_PDL_ENTRY();
    col_sort_assign_body(blockIdx.x, cond, cmask, ncols, col_start, col_atoms, zkey, cl_start, slot_orig, cl_col, atom_slot, col_fill, status);
}

// Gather the cluster-ordered records.  The position used is the build-time
// wrapped image plus the minimum-image displacement since the build, so a
// caller that wraps atoms back into the box between builds stays consistent.
__device__ __forceinline__ void pack_body(int bx, int nslots, const int *__restrict__ ncl_dev,
                       const int *__restrict__ slot_orig, const double *__restrict__ x,
                       const double *__restrict__ y, const double *__restrict__ z,
                       const double *__restrict__ rx, const double *__restrict__ ry,
                       const double *__restrict__ rz, const double *__restrict__ ix,
                       const double *__restrict__ iy, const double *__restrict__ iz,
                       const float *__restrict__ q, const int *__restrict__ type, double L,
                       AtomRec *__restrict__ rec, float *__restrict__ recf,
                       long long *__restrict__ fslot, float4 *__restrict__ bb,
                       const int *__restrict__ cond, double *__restrict__ sref) {
    const int s = bx * blockDim.x + threadIdx.x;
    // The build-time data of a slot (position and wrap shift at the last build,
    // charge, type) change only at a list build.  On a build (cond null, or its
    // build bit set) they are gathered through slot_orig and kept in slot order
    // in sref: [3][nslots] positions, [3][nslots] position + shift, then
    // [nslots] charges and [nslots] types; on the other steps they are read back
    // from there, which leaves the three current coordinates as the only
    // scattered reads.  sref holds exactly the gathered values, so both ways give
    // the same bits.
    const bool fresh = !cond || (cond[0] & 1);
    float *sq = reinterpret_cast<float *>(sref + 6 * (size_t)nslots);
    int *stype = reinterpret_cast<int *>(sq + nslots);
    // no early return: the 8 slots of a cluster (8 consecutive lanes) reduce the
    // cluster's bounding box with shuffles below
    const bool live = s < nslots && s < ncl_dev[0] * CL;
    const int o = live ? slot_orig[s] : -1;
    AtomRec r;
    if (live) {
        // the pair kernel adds into the slot-ordered accumulators: start them at zero
        fslot[s] = 0;
        fslot[nslots + s] = 0;
        fslot[2 * nslots + s] = 0;
    }
    if (o >= 0) {
        double bx0, by0, bz0, ux, uy, uz;
        if (fresh) {
            bx0 = rx[o];
            by0 = ry[o];
            bz0 = rz[o];
            ux = bx0 + ix[o];
            uy = by0 + iy[o];
            uz = bz0 + iz[o];
            r.q = q[o];
            r.type = type[o] - 1;
            sref[s] = bx0;
            sref[(size_t)nslots + s] = by0;
            sref[2 * (size_t)nslots + s] = bz0;
            sref[3 * (size_t)nslots + s] = ux;
            sref[4 * (size_t)nslots + s] = uy;
            sref[5 * (size_t)nslots + s] = uz;
            sq[s] = r.q;
            stype[s] = r.type;
        } else {
            bx0 = sref[s];
            by0 = sref[(size_t)nslots + s];
            bz0 = sref[2 * (size_t)nslots + s];
            ux = sref[3 * (size_t)nslots + s];
            uy = sref[4 * (size_t)nslots + s];
            uz = sref[5 * (size_t)nslots + s];
            r.q = sq[s];
            r.type = stype[s];
        }
        double dx = x[o] - bx0, dy = y[o] - by0, dz = z[o] - bz0;
        // minimum image with one division per thread: d * (1/L) differs from d / L
        // by an ulp at most, which could change rint only at a half box, far
        // beyond any displacement between two list builds
        const double Li = 1.0 / L;
        dx -= L * rint(dx * Li);
        dy -= L * rint(dy * Li);
        dz -= L * rint(dz * Li);
        r.x = ux + dx;
        r.y = uy + dy;
        r.z = uz + dz;
    } else {
        // padding: far away and distinct; every pair with it is masked out
        r.x = 1.0e6 + 16.0 * s;
        r.y = -1.0e6;
        r.z = 1.0e6;
        r.q = 0.0f;
        r.type = 0;
    }
    if (live) {
        rec[s] = r;
        // FP32 copy for the prune, per cluster x[8], y[8], z[8]
        float *rc = recf + (size_t)(s / CL) * (3 * CL) + (s % CL);
        rc[0] = (float)r.x;
        rc[CL] = (float)r.y;
        rc[2 * CL] = (float)r.z;
    }
    // Cluster bounding box of the real atoms (FP64 bounds rounded outward to
    // float), for the cluster-pair search and the prune; w of the low corner
    // carries the cluster's real-atom bits (padding slots clear).  min and max
    // are exact, so the shuffle order does not matter.
    double lx = o >= 0 ? r.x : 1e300, ly = o >= 0 ? r.y : 1e300, lz = o >= 0 ? r.z : 1e300;
    double hx = o >= 0 ? r.x : -1e300, hy = o >= 0 ? r.y : -1e300, hz = o >= 0 ? r.z : -1e300;
#pragma unroll
    for (int off = 1; off < CL; off <<= 1) {
        lx = fmin(lx, __shfl_xor_sync(FULL, lx, off));
        ly = fmin(ly, __shfl_xor_sync(FULL, ly, off));
        lz = fmin(lz, __shfl_xor_sync(FULL, lz, off));
        hx = fmax(hx, __shfl_xor_sync(FULL, hx, off));
        hy = fmax(hy, __shfl_xor_sync(FULL, hy, off));
        hz = fmax(hz, __shfl_xor_sync(FULL, hz, off));
    }
    const unsigned realw = __ballot_sync(FULL, o >= 0);
    if (live && (s & (CL - 1)) == 0) {
        const int c = s / CL;
        const int real = (int)((realw >> (threadIdx.x & 31)) & 0xffu);
        bb[2 * c] = make_float4(__double2float_rd(lx), __double2float_rd(ly),
                                __double2float_rd(lz), __int_as_float(real));
        bb[2 * c + 1] = make_float4(__double2float_ru(hx), __double2float_ru(hy),
                                    __double2float_ru(hz), 0.0f);
    }
}
__global__ void k_pack(int nslots, const int *__restrict__ ncl_dev,
                       const int *__restrict__ slot_orig, const double *__restrict__ x,
                       const double *__restrict__ y, const double *__restrict__ z,
                       const double *__restrict__ rx, const double *__restrict__ ry,
                       const double *__restrict__ rz, const double *__restrict__ ix,
                       const double *__restrict__ iy, const double *__restrict__ iz,
                       const float *__restrict__ q, const int *__restrict__ type, double L,
                       AtomRec *__restrict__ rec, float *__restrict__ recf,
                       long long *__restrict__ fslot, float4 *__restrict__ bb,
                       const int *__restrict__ cond, double *__restrict__ sref) {
    SOFIA_PDL_ENTRY();
    pack_body(blockIdx.x, nslots, ncl_dev, slot_orig, x, y, z, rx, ry, rz, ix, iy, iz, q, type, L,
              rec, recf, fslot, bb, cond, sref);
}

__device__ __forceinline__ float gap(float alo, float ahi, float blo, float bhi) {
    return fmaxf(0.0f, fmaxf(blo - ahi, alo - bhi));
}

struct SearchArgs {
    const int *cond;
    int cmask;
    int maxcl, ncx, reach, jcap, n;
    float L, s_col, rl, rl2, rexcl2;
    const int *ncl_dev, *cl_start, *cl_col, *slot_orig, *specbond, *num3bond, *atom_slot;
    const float4 *bb;
    int *jlist, *jcount;
    unsigned long long *jmask;
    int *status;
};

// Half list: the cluster pair (ci, cj, image) and its mirror (cj, ci, -image)
// are the same atom pairs, so exactly one of them is kept.  Distinct clusters
// split by index parity (each row keeps about half of its partners, which
// balances the rows); a cluster with its own image keeps the positive image;
// a cluster with itself (no image) keeps one entry with the upper-triangle
// mask.
__device__ __forceinline__ bool half_keep(int ci, int cj, int img) {
    if (ci != cj) return (ci < cj) != (((ci + cj) & 1) != 0);
    return img >= 13;
}

// z window of one column segment.  The clusters of a column are z-sorted, so
// their bounding-box bounds are non-decreasing along the column (up to a few
// ulp where float sort keys tie); the clusters whose z gap to the i box is at
// least rw (rl plus a slack far above those ulp) form a prefix and a suffix of
// [j0, j0 + len), found by binary search and cut off.  Each cut cluster has a
// z gap >= rl, so the bounding-box test would reject it: the list is unchanged.
__device__ __forceinline__ void z_window(const float4 *__restrict__ bb, float ilo_z, float ihi_z,
                                         float sz, float rw, int &j0, int &len) {
    int lo = 0, hi = len;
    while (lo < hi) {  // first cluster with ilo.z - (hi.z + sz) < rw
        const int mid = (lo + hi) >> 1;
        if (ilo_z - (__ldg(&bb[2 * (j0 + mid) + 1].z) + sz) >= rw)
            lo = mid + 1;
        else
            hi = mid;
    }
    const int first = lo;
    hi = len;
    while (lo < hi) {  // first cluster with (lo.z + sz) - ihi.z >= rw
        const int mid = (lo + hi) >> 1;
        if ((__ldg(&bb[2 * (j0 + mid)].z) + sz) - ihi_z >= rw)
            hi = mid;
        else
            lo = mid + 1;
    }
    j0 += first;
    len = lo - first;
}

// One warp per i-cluster: visit the xy columns within reach (periodic images
// included) in three z images, cut each column image to its z window, test the
// remaining clusters' bounding boxes, compact the accepted (cluster, image)
// pairs of the half list in visiting order and attach the pair mask.
__device__ __forceinline__ void search_body(int bx, const SearchArgs &a) {
    if (a.cond && !(a.cond[0] & a.cmask)) return;
    const int lane = threadIdx.x & 31;
    const int icl = (bx * blockDim.x + threadIdx.x) >> 5;
    if (icl >= a.maxcl || icl >= a.ncl_dev[0]) return;
    const float4 ilo = a.bb[2 * icl], ihi = a.bb[2 * icl + 1];
    const int col = a.cl_col[icl];
    const int cxi = col % a.ncx, cyi = col / a.ncx;
    // i-cluster atoms: real-atom bits and orig ids (lanes 0..7 hold one each)
    const unsigned ireal = (unsigned)__float_as_int(ilo.w) & 0xffu;
    // byte ii of iexp is 0xff when i atom ii is real
    unsigned long long iexp = 0ull;
#pragma unroll
    for (int ii = 0; ii < CL; ++ii)
        if ((ireal >> ii) & 1u) iexp |= 0xffull << (ii * CL);
    // the exclusion partners of the 8 i atoms as cluster slots, 96 items
    // (i atom b / 12, partner b % 12) spread 3 per lane
    int ex_slot[3], ex_bit[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int b = lane + 32 * t;
        const int ii = b / 12, l = b - 12 * (b / 12);
        const int io = a.slot_orig[icl * CL + ii];
        int ps = -1;
        if (io >= 0 && l < min(a.num3bond[io], 12)) {
            const int po = a.specbond[io * 12 + l] - 1;
            if (po >= 0 && po < a.n) ps = a.atom_slot[po];
        }
        ex_slot[t] = ps;
        ex_bit[t] = ii * CL + (ps & (CL - 1));
    }
    int count = 0;
    int *row = a.jlist + (size_t)icl * a.jcap;
    unsigned long long *mrow = a.jmask + (size_t)icl * a.jcap;
    // Candidates: the clusters of every (column, z image) within reach, in the
    // order column row dy, column dx, image z.  32 such segments are gathered at
    // a time (one per lane) and their clusters are then streamed over the lanes
    // as one flat sequence, so short segments do not leave lanes idle.
    __shared__ int s_seg[8][3][32];  // per warp: first cluster, flat offset, image code
    int *sj0 = s_seg[threadIdx.x >> 5][0], *scum = s_seg[threadIdx.x >> 5][1],
        *simg = s_seg[threadIdx.x >> 5][2];
    const int side = 2 * a.reach + 1;
    const int ncombo = side * side * 3;
    for (int cbase = 0; cbase < ncombo; cbase += 32) {
        const int k = cbase + lane;
        int len = 0, j0 = 0, imgk = 13;
        if (k < ncombo) {
            const int iz = k % 3, kk = k / 3;
            const int dx = kk % side - a.reach, dy = kk / side - a.reach;
            int cy = cyi + dy;
            const int imy = (cy < 0) ? -1 : (cy >= a.ncx ? 1 : 0);
            cy -= imy * a.ncx;
            int cx = cxi + dx;
            const int imx = (cx < 0) ? -1 : (cx >= a.ncx ? 1 : 0);
            cx -= imx * a.ncx;
            const int imz = iz - 1;
            const float sx = imx * a.L, sy = imy * a.L, sz = imz * a.L;
            const float gx = gap(ilo.x, ihi.x, cx * a.s_col + sx, (cx + 1) * a.s_col + sx);
            const float gy = gap(ilo.y, ihi.y, cy * a.s_col + sy, (cy + 1) * a.s_col + sy);
            // the column image spans z in [sz, sz + L)
            const float gz = gap(ilo.z, ihi.z, sz, sz + a.L);
            if (gx * gx + gy * gy + gz * gz < a.rl2) {
                j0 = a.cl_start[cx + cy * a.ncx];
                len = a.cl_start[cx + cy * a.ncx + 1] - j0;
                imgk = (imx + 1) + 3 * (imy + 1) + 9 * (imz + 1);
                if (SOFIA_SEARCH_ZWIN) z_window(a.bb, ilo.z, ihi.z, sz, a.rl + 1e-3f, j0, len);
            }
        }
        const bool has = len > 0;
        const unsigned hb = __ballot_sync(FULL, has);
        if (!hb) continue;
        const int nseg = __popc(hb);
        int incl = len;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        if (has) {
            const int at = __popc(hb & ((1u << lane) - 1u));
            sj0[at] = j0;
            scum[at] = incl - len;
            simg[at] = imgk;
        }
        __syncwarp();
        int seg = 0;
        for (int base = 0; base < total; base += 32) {
            const int t = base + lane;
            const bool act = t < total;
            int jc = 0, img = 13;
            if (act) {
                while (seg + 1 < nseg && scum[seg + 1] <= t) ++seg;
                jc = sj0[seg] + (t - scum[seg]);
                img = simg[seg];
            }
            const float sx = (float)(img % 3 - 1) * a.L, sy = (float)((img / 3) % 3 - 1) * a.L,
                        sz = (float)(img / 9 - 1) * a.L;
            bool acc = false, need_excl = false;
            unsigned long long mask = 0ull;
            if (act) {
                const float4 jlo = a.bb[2 * jc], jhi = a.bb[2 * jc + 1];
                const float ex = gap(ilo.x, ihi.x, jlo.x + sx, jhi.x + sx);
                const float ey = gap(ilo.y, ihi.y, jlo.y + sy, jhi.y + sy);
                const float ez = gap(ilo.z, ihi.z, jlo.z + sz, jhi.z + sz);
                const float d2 = ex * ex + ey * ey + ez * ez;
                acc = d2 < a.rl2 && half_keep(icl, jc, img);
                if (acc) {
                    need_excl = d2 < a.rexcl2;
                    const unsigned long long jreal =
                        (unsigned long long)((unsigned)__float_as_int(jlo.w) & 0xffu);
                    mask = (jreal * 0x0101010101010101ull) & iexp;
                    if (jc == icl && img == 13) {
                        // the cluster with itself: pairs ii < jj only
#pragma unroll
                        for (int ii = 0; ii < CL; ++ii)
                            mask &= ~(((2ull << ii) - 1ull) << (ii * CL));
                    }
                }
            }
            const unsigned ballot = __ballot_sync(FULL, acc);
            // exclusions: for each nearby accepted entry the warp ORs the bits of
            // the i atoms' partners that sit in that j-cluster
            unsigned todo = __ballot_sync(FULL, need_excl);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const int jsrc = __shfl_sync(FULL, jc, src);
                unsigned long long m = 0ull;
#pragma unroll
                for (int tt = 0; tt < 3; ++tt)
                    if (ex_slot[tt] >= 0 && (ex_slot[tt] >> 3) == jsrc) m |= 1ull << ex_bit[tt];
                const unsigned lo = __reduce_or_sync(FULL, (unsigned)m);
                const unsigned hi = __reduce_or_sync(FULL, (unsigned)(m >> 32));
                if (lane == src) mask &= ~((unsigned long long)lo | ((unsigned long long)hi << 32));
            }
            if (acc) {
                const int at = count + __popc(ballot & ((1u << lane) - 1u));
                if (at < a.jcap) {
                    row[at] = jc | (img << IMG_SHIFT);
                    mrow[at] = mask;
                }
            }
            count += __popc(ballot);
        }
        __syncwarp();
    }
    if (lane == 0) {
        a.jcount[icl] = min(count, a.jcap);
        atomicMax(&a.status[ST_NCLUSTER], count);
    }
}
__global__ void __launch_bounds__(256) k_search(SearchArgs a) {
    SOFIA_PDL_ENTRY();
    search_body(blockIdx.x, a);
}

// Displacement trigger: flag a rebuild when any atom moved more than skin/2
// (minimum image) since the last build.
// Displacement triggers: bit 0 = some atom moved more than skin/2 since the
// list build, bit 1 = more than margin/2 since the last prune.
__global__ void k_disp_check(int n, const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, const double *__restrict__ rx,
                             const double *__restrict__ ry, const double *__restrict__ rz,
                             const double *__restrict__ px, const double *__restrict__ py,
                             const double *__restrict__ pz, double L, double lim2,
                             double plim2, int *__restrict__ flag) {
    SOFIA_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool far = false, pfar = false;
    if (i < n) {
        far = disp2(x[i], y[i], z[i], rx[i], ry[i], rz[i], L) > lim2;
        pfar = disp2(x[i], y[i], z[i], px[i], py[i], pz[i], L) > plim2;
    }
    const bool a = __any_sync(FULL, far), b = __any_sync(FULL, pfar);
    if ((threadIdx.x & 31) == 0 && (a || b)) atomicOr(flag, (a ? 1 : 0) | (b ? 2 : 0));
}


struct PairConst {
    float rcut2, cut_coulsq, kexp, pa, c2a, e_shift, f_shift, coulpre;
    float A1, A2, A3, A4, A5;
    // the same FP32 constants duplicated as {c, c} operands of packed FP32x2 math
    float2 kexp2, pa2, c2a2, e_shift2, f_shift2, A1_2, A2_2, A3_2, A4_2, A5_2;
    // optional LJ energy shift: each in-range pair's energy minus its value at
    // the cut-off, ljs6 = rc^-6 (0 = no shift: the energies are unchanged bit for bit)
    float ljs6;
    float2 ljs6_2;
    double ljs6d;
    double rcut2d, cut_coulsqd, alphad, e_shiftd, f_shiftd, coulpred, MY_PIS_INV;
    double A1d, A2d, A3d, A4d, A5d, EWALD_Pd;
    double L;
    int ntypes;
};

// Single-instruction MUFU approximations (hand-written PTX).
__device__ __forceinline__ float rsqrt_a(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_a(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_a(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Separately rounded operations.  Every product, sum and fused multiply-add of
// the pair arithmetic is written out, so the compiler cannot fuse a product
// into a later addition in one template instance and not in another: the
// force-only and energy kernels then give bit-identical forces.
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fmar(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmar(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
struct PairMath;

// FP32 pair: LJ 12-6 + DSF with the reference's polynomial erfc
// (mod_force_nonbond.f90:152-175), using
//   F*r = pref * (erfc + (2 alpha/sqrt(pi)) r exp(-alpha^2 r^2) + f_shift r^2).
// exp(-alpha^2 r^2) = 2^(kexp r^2) with kexp = -alpha^2 log2(e).
template <>
struct PairMath<float> {
    // SAME: the LJ and Coulomb cut-offs are equal, so one test gates both terms
    template <bool EN, bool SAME>
    __device__ __forceinline__ static float eval(float dx, float dy, float dz, float qiq,
                                                 float4 lj, bool on, const PairConst &k,
                                                 float &elj, float &ec) {
        const float r2 = fmar(dx, dx, fmar(dy, dy, mulr(dz, dz)));
        const float rinv = rsqrt_a(r2);
        const float r2inv = mulr(rinv, rinv);
        const float r = mulr(r2, rinv);
        const float dr6i = mulr(mulr(r2inv, r2inv), r2inv);
        const bool lj_on = on && r2 <= k.rcut2;
        const bool c_on = SAME ? lj_on : (on && r2 <= k.cut_coulsq);
        const float flj = mulr(dr6i, fmar(lj.x, dr6i, -lj.y));
        const float pref = mulr(qiq, rinv);
        const float ex = ex2_a(mulr(k.kexp, r2));
        const float t = rcp_a(fmar(k.pa, r, 1.0f));
        const float poly = fmar(t, fmar(t, fmar(t, fmar(t, k.A5, k.A4), k.A3), k.A2), k.A1);
        const float erfcc = mulr(mulr(t, poly), ex);
        const float fc = mulr(pref, fmar(k.f_shift, r2, fmar(mulr(k.c2a, ex), r, erfcc)));
        if (EN) {
            // selects, not products: masked pairs may hold inf/NaN (r = 0)
            const float esh = mulr(k.ljs6, fmar(k.ljs6, lj.z, -lj.w));
            elj = lj_on ? addr(mulr(dr6i, fmar(dr6i, lj.z, -lj.w)), -esh) : 0.0f;
            ec = c_on ? mulr(pref, fmar(fmar(r, k.e_shift, mulr(r2, k.f_shift)), -1.0f, erfcc))
                      : 0.0f;
        }
        if (SAME) return lj_on ? mulr(addr(fc, flj), r2inv) : 0.0f;
        const float fs = mulr(addr(c_on ? fc : 0.0f, lj_on ? flj : 0.0f), r2inv);
        return on ? fs : 0.0f;
    }
};

template <>
struct PairMath<double> {
    template <bool EN, bool SAME>
    __device__ __forceinline__ static double eval(double dx, double dy, double dz, double qiq,
                                                  float4 lj, bool on, const PairConst &k,
                                                  double &elj, double &ec) {
        // the reference's expressions and order, each operation rounded on its own
        const double r2 = addr(addr(mulr(dx, dx), mulr(dy, dy)), mulr(dz, dz));
        const double r = sqrt(r2);
        const double rinv = 1.0 / r;
        const double r2inv = 1.0 / r2;
        const double dr6i = mulr(mulr(r2inv, r2inv), r2inv);
        const bool lj_on = on && r2 <= k.rcut2d;
        const bool c_on = on && r2 <= k.cut_coulsqd;
        const double flj = mulr(dr6i, addr(mulr((double)lj.x, dr6i), -(double)lj.y));
        const double pref = mulr(qiq, rinv);
        const double ex = exp(-mulr(mulr(mulr(k.alphad, k.alphad), r), r));
        const double t = 1.0 / addr(1.0, mulr(mulr(k.EWALD_Pd, k.alphad), r));
        const double poly = addr(k.A1d, mulr(t, addr(k.A2d, mulr(t, addr(k.A3d,
                            mulr(t, addr(k.A4d, mulr(t, k.A5d))))))));
        const double erfcc = mulr(mulr(t, poly), ex);
        const double c2a = mulr(mulr(2.0, k.alphad), k.MY_PIS_INV);
        const double fc = mulr(mulr(pref, addr(addr(mulr(erfcc, rinv), mulr(c2a, ex)),
                                               mulr(r, k.f_shiftd))), r);
        if (EN) {
            const double esh = mulr(k.ljs6d, addr(mulr(k.ljs6d, (double)lj.z), -(double)lj.w));
            elj = lj_on ? addr(mulr(dr6i, addr(mulr(dr6i, (double)lj.z), -(double)lj.w)), -esh)
                        : 0.0;
            ec = c_on ? mulr(pref, addr(addr(erfcc, -mulr(r, k.e_shiftd)),
                                        -mulr(r2, k.f_shiftd)))
                      : 0.0;
        }
        const double fs = mulr(addr(c_on ? fc : 0.0, lj_on ? flj : 0.0), r2inv);
        return on ? fs : 0.0;
    }
};

// Packed FP32x2 form of PairMath<float> for the two pairs a lane owns in one
// list entry (component x: j atom lj, component y: j atom lj + 4).  sm_100
// issues one FFMA2 / FMUL2 / FADD2 instruction for both components, so the
// pair arithmetic takes half the issue slots; only the MUFU operations, the
// range tests and the selects stay per component.  Each component goes
// through the same operations, in the same order and rounding, as
// PairMath<float>::eval.  The LJ operands arrive packed over the two pairs:
// l1 = {lj1, lj1'}, l2n = {-lj2, -lj2'}, l3 = {lj3, lj3'}, l4n = {-lj4, -lj4'}
// (l3, l4n read only for energies).
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    return __ffma2_rn(a, b, c);
}

struct PairMath2 {
    template <bool EN, bool SAME>
    __device__ __forceinline__ static float2 eval(float2 dx, float2 dy, float2 dz, float2 qq,
                                                  float2 l1, float2 l2n, float2 l3, float2 l4n,
                                                  bool on0, bool on1,
                                                  const PairConst &k, float2 &elj, float2 &ec) {
        const float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
        const float2 rinv = make_float2(rsqrt_a(r2.x), rsqrt_a(r2.y));
        const float2 r2inv = mul2(rinv, rinv);
        const float2 r = mul2(r2, rinv);
        const float2 dr6i = mul2(mul2(r2inv, r2inv), r2inv);
        const bool lj0_on = on0 && r2.x <= k.rcut2, lj1_on = on1 && r2.y <= k.rcut2;
        const bool c0_on = SAME ? lj0_on : (on0 && r2.x <= k.cut_coulsq);
        const bool c1_on = SAME ? lj1_on : (on1 && r2.y <= k.cut_coulsq);
        const float2 flj = mul2(dr6i, fma2(l1, dr6i, l2n));
        const float2 pref = mul2(qq, rinv);
        const float2 kr = mul2(k.kexp2, r2);
        const float2 ex = make_float2(ex2_a(kr.x), ex2_a(kr.y));
        const float2 u = fma2(k.pa2, r, make_float2(1.0f, 1.0f));
        const float2 t = make_float2(rcp_a(u.x), rcp_a(u.y));
        const float2 poly =
            fma2(t, fma2(t, fma2(t, fma2(t, k.A5_2, k.A4_2), k.A3_2), k.A2_2), k.A1_2);
        const float2 erfcc = mul2(mul2(t, poly), ex);
        const float2 fc = mul2(pref, fma2(k.f_shift2, r2, fma2(mul2(k.c2a2, ex), r, erfcc)));
        if (EN) {
            const float2 esh = mul2(k.ljs6_2, fma2(k.ljs6_2, l3, l4n));
            const float2 e6 = fma2(esh, make_float2(-1.0f, -1.0f), mul2(dr6i, fma2(dr6i, l3, l4n)));
            const float2 sh = fma2(r, k.e_shift2, mul2(r2, k.f_shift2));
            const float2 e1 = mul2(pref, fma2(sh, make_float2(-1.0f, -1.0f), erfcc));
            elj = make_float2(lj0_on ? e6.x : 0.0f, lj1_on ? e6.y : 0.0f);
            ec = make_float2(c0_on ? e1.x : 0.0f, c1_on ? e1.y : 0.0f);
        }
        if (SAME) {
            const float2 fs = mul2(add2(fc, flj), r2inv);
            return make_float2(lj0_on ? fs.x : 0.0f, lj1_on ? fs.y : 0.0f);
        }
        const float2 fcm = make_float2(c0_on ? fc.x : 0.0f, c1_on ? fc.y : 0.0f);
        const float2 fljm = make_float2(lj0_on ? flj.x : 0.0f, lj1_on ? flj.y : 0.0f);
        return mul2(add2(fcm, fljm), r2inv);
    }
};

template <typename T>
__device__ __forceinline__ long long to_fix(T v);
template <>
__device__ __forceinline__ long long to_fix<float>(float v) {
    return __float2ll_rn(v * 4294967296.0f);  // exact power-of-two scaling
}
template <>
__device__ __forceinline__ long long to_fix<double>(double v) {
    return __double2ll_rn(v * FIX_SCALE);
}

// The j force of one entry, (v0, v1, v2) on each of the 4 lanes that share a j
// atom (lane bits 3 and 4), summed over those lanes by reduce-scatter: afterwards
// lane bits (4, 3) = (0, 0) hold component x, (0, 1) y, (1, 0) z, (1, 1) none.
// Three shuffles.
template <typename T>
__device__ __forceinline__ T reduce_j4(T v0, T v1, T v2, int lane) {
    const bool u4 = lane & 16, u3 = lane & 8;
    const T k0 = u4 ? v2 : v0, k1 = u4 ? (T)0 : v1;
    const T o0 = u4 ? v0 : v2, o1 = u4 ? v1 : (T)0;
    const T s0 = k0 + __shfl_xor_sync(FULL, o0, 16);
    const T s1 = k1 + __shfl_xor_sync(FULL, o1, 16);
    const T k = u3 ? s1 : s0, o = u3 ? s0 : s1;
    return k + __shfl_xor_sync(FULL, o, 8);
}

// i-force partial sums of one lane (i atoms q and q + 4) -> the lane's own 64-bit
// fixed-point sums in shared memory, fi[c * 32 + lane] for component c of i atom
// q (c = 0..2) and q + 4 (c = 3..5): no atomics, no bank conflicts.
template <typename T>
__device__ __forceinline__ void flush_i(long long *__restrict__ fi, int lane, T x0, T y0, T z0,
                                        T x1, T y1, T z1) {
    fi[0 * 32 + lane] += to_fix<T>(x0);
    fi[1 * 32 + lane] += to_fix<T>(y0);
    fi[2 * 32 + lane] += to_fix<T>(z0);
    fi[3 * 32 + lane] += to_fix<T>(x1);
    fi[4 * 32 + lane] += to_fix<T>(y1);
    fi[5 * 32 + lane] += to_fix<T>(z1);
}

// Pair kernel on the half cluster-pair list (each atom pair once, Newton's
// third law).  One warp per i-cluster; lane = jj + 8 q (jj = j atom 0..7,
// q = 0..3): for every listed j-cluster the lane evaluates the pairs of j atom
// jj with i atoms q and q + 4, both in one stream of packed FP32x2
// instructions (component x: i atom q, y: i atom q + 4).  List rows are read 32
// entries at a time with coalesced loads and broadcast by shuffles.  Pruned
// mask bit 8 ii + jj (i atom ii, j atom jj) is bit 32 h + lane of the lane that
// evaluates it (ii = q + 4 h).
//   * a lane loads one j record per entry;
//   * the j force of an entry (the sum of the lane's two pairs) is reduced over
//     the 4 lanes of its j atom (reduce_j4) and added to the slot-ordered
//     fixed-point accumulators, 24 lanes x one 64-bit atomic add into one
//     j-cluster's contiguous slots;
//   * i forces are summed per lane in FP32 and flushed every FLUSH entries into
//     the lane's 64-bit fixed-point sums in shared memory; at the end of the row
//     they are summed over the 8 lanes of an i atom and added to the slot
//     accumulators.
// Integer addition makes every sum independent of the order of the atomics, so
// results stay bit-reproducible.  EN adds the LJ and Coulomb energies, VIR the
// diagonal virial (each pair once).
template <typename T, bool EN, bool VIR, bool SAME, bool TRI>
__device__ __forceinline__ void pair_body(
    int bx, int maxcl, const int *__restrict__ ncl_dev, const AtomRec *__restrict__ rec,
    const int *__restrict__ jlist, const unsigned long long *__restrict__ jmask,
    const int *__restrict__ jcount, int jcap, const float4 *__restrict__ ljtab,
    const PairConst &k, double L, unsigned long long *__restrict__ fslot,
    double *__restrict__ energy) {
    extern __shared__ float4 s_lj[];
    // FP32 path: the same bytes as two float2 tables, {lj1, -lj2} and {lj3, -lj4},
    // so a force-only lookup reads 8 bytes (fewer shared-memory wavefronts)
    float2 *s_lja = reinterpret_cast<float2 *>(s_lj);
    float2 *s_ljb = s_lja + k.ntypes * k.ntypes;
    // TRI: entry (a nt + b) nt + c = {lj1(a,c), lj1(b,c), -lj2(a,c), -lj2(b,c)} and,
    // for energies, the same of lj3 / lj4 nt^3 entries further on
    float4 *s_lj3 = reinterpret_cast<float4 *>(s_ljb + k.ntypes * k.ntypes);
    const int nt3 = k.ntypes * k.ntypes * k.ntypes;

    __shared__ double s_sh[27 * 3];
    __shared__ long long s_fi[8][6 * 32];  // per warp and lane: i-force sums (see flush_i)
    // FP32x2 path: lj2 and lj4 enter the packed FMAs as addends, stored negated
    constexpr bool PACK = sizeof(T) == 4;
    for (int t = threadIdx.x; t < k.ntypes * k.ntypes; t += blockDim.x) {
        const float4 l = ljtab[t];
        if (PACK) {
            s_lja[t] = make_float2(l.x, -l.y);
            s_ljb[t] = make_float2(l.z, -l.w);
        } else {
            s_lj[t] = l;
        }
    }
    if (TRI) {
        const int nt = k.ntypes;
        for (int t = threadIdx.x; t < nt3; t += blockDim.x) {
            const int a = t / (nt * nt), b = (t / nt) % nt, c = t % nt;
            const float4 la = ljtab[a * nt + c], lb = ljtab[b * nt + c];
            s_lj3[t] = make_float4(la.x, lb.x, -la.y, -lb.y);
            if (EN) s_lj3[nt3 + t] = make_float4(la.z, lb.z, -la.w, -lb.w);
        }
    }
    if (threadIdx.x < 27) {
        const int im = threadIdx.x;
        s_sh[im * 3 + 0] = (double)(im % 3 - 1) * L;
        s_sh[im * 3 + 1] = (double)((im / 3) % 3 - 1) * L;
        s_sh[im * 3 + 2] = (double)(im / 9 - 1) * L;
    }
    const int lane = threadIdx.x & 31;
    long long *fi = s_fi[threadIdx.x >> 5];
#pragma unroll
    for (int c = 0; c < 6; ++c) fi[c * 32 + lane] = 0;
    __syncthreads();
    const int jj = lane & 7, q = lane >> 3;
    const int icl = (bx * blockDim.x + threadIdx.x) >> 5;
    if (icl >= maxcl || icl >= ncl_dev[0]) return;
    const size_t stride = (size_t)maxcl * CL;
    // this lane's share of the reduced j force: component q (3 = none) of j atom jj
    unsigned long long *jdst = fslot + (size_t)(q < 3 ? q : 0) * stride;
    const AtomRec ri0 = rec[icl * CL + q], ri1 = rec[icl * CL + q + 4];
    const T qiq0 = (T)k.coulpre * (T)ri0.q, qiq1 = (T)k.coulpre * (T)ri1.q;
    const int ti0 = ri0.type * k.ntypes, ti1 = ri1.type * k.ntypes;
    const int t3 = (ri0.type * k.ntypes + ri1.type) * k.ntypes;  // this lane's TRI row
    const int n = jcount[icl];
    const int *row = jlist + (size_t)icl * jcap;
    const unsigned long long *mrow = jmask + (size_t)icl * jcap;
    // i-force partial sums: i atom q (x0..) and q + 4 (x1..)
    T ax0 = 0, ay0 = 0, az0 = 0, ax1 = 0, ay1 = 0, az1 = 0;
    T a_lj = 0, a_c = 0, a_xx = 0, a_yy = 0, a_zz = 0;
    // packed accumulators of the FP32x2 path (component per i atom)
    const float2 z2 = make_float2(0.0f, 0.0f);
    float2 ax2 = z2, ay2 = z2, az2 = z2, alj2 = z2, ac2 = z2, axx2 = z2, ayy2 = z2, azz2 = z2;
    const float2 qiq2 = make_float2((float)qiq0, (float)qiq1);
    double e_lj = 0.0, e_c = 0.0, vxx = 0.0, vyy = 0.0, vzz = 0.0;
    for (int base = 0; base < n; base += 32) {
        const int cnt = min(32, n - base);
        const int myw = (lane < cnt) ? row[base + lane] : 0;
        const unsigned long long mym = (lane < cnt) ? mrow[base + lane] : 0ull;
        // chunks of FLUSH entries (FLUSH divides 32), each followed by a flush of
        // the lane's FP32 i-force partials
        for (int e0 = 0; e0 < cnt; e0 += FLUSH) {
            const int e1 = min(e0 + FLUSH, cnt);
            for (int e = e0; e < e1; ++e) {
                const int w = __shfl_sync(FULL, myw, e);
                const unsigned long long mm = __shfl_sync(FULL, mym, e);
                const int jc = w & ((1 << IMG_SHIFT) - 1);
                const int img = w >> IMG_SHIFT;
                const AtomRec rj = rec[jc * CL + jj];
                // j position in the image the entry pairs with
                const double xj = rj.x + s_sh[img * 3 + 0];
                const double yj = rj.y + s_sh[img * 3 + 1];
                const double zj = rj.z + s_sh[img * 3 + 2];
                T v0 = 0, v1 = 0, v2 = 0;  // the entry's force on j atom jj (negated)
                const unsigned m0 = (unsigned)mm, m1 = (unsigned)(mm >> 32);
                // the lane's two i positions {q, q + 4} per component
                const double2 pix = make_double2(ri0.x, ri1.x), piy = make_double2(ri0.y, ri1.y),
                              piz = make_double2(ri0.z, ri1.z);
                if (PACK && SOFIA_PAIR_HYBRID && (m0 == 0u || m1 == 0u)) {
                    // one i half without pairs in range: scalar evaluation of the other
                    // (a warp-uniform branch per half, so no selects of i data)
                    const bool h1 = m0 == 0u;
                    const double xi = h1 ? pix.y : pix.x, yi = h1 ? piy.y : piy.x,
                                 zi = h1 ? piz.y : piz.x;
                    const float dx = (float)(xi - xj);
                    const float dy = (float)(yi - yj);
                    const float dz = (float)(zi - zj);
                    const int ti = h1 ? ti1 : ti0;
                    const float2 la = s_lja[ti + rj.type];
                    const float2 lb = EN ? s_ljb[ti + rj.type] : make_float2(0.0f, 0.0f);
                    float elj = 0.0f, ec = 0.0f;
                    const float fs = PairMath<float>::template eval<EN, SAME>(
                        dx, dy, dz, mulr(h1 ? qiq2.y : qiq2.x, rj.q),
                        make_float4(la.x, -la.y, lb.x, -lb.y), ((m0 | m1) >> lane) & 1u, k, elj, ec);
                    const float px = mulr(dx, fs), py = mulr(dy, fs), pz = mulr(dz, fs);
                    if (h1) {
                        ax2.y = addr(ax2.y, px);
                        ay2.y = addr(ay2.y, py);
                        az2.y = addr(az2.y, pz);
                    } else {
                        ax2.x = addr(ax2.x, px);
                        ay2.x = addr(ay2.x, py);
                        az2.x = addr(az2.x, pz);
                    }
                    v0 = px;
                    v1 = py;
                    v2 = pz;
                    if (EN) {
                        alj2.x = addr(alj2.x, elj);
                        ac2.x = addr(ac2.x, ec);
                    }
                    if (VIR) {
                        axx2.x = fmar(dx, px, axx2.x);
                        ayy2.x = fmar(dy, py, ayy2.x);
                        azz2.x = fmar(dz, pz, azz2.x);
                    }
                } else if constexpr (PACK) {
                    // both i halves at once; a half without pairs in range is computed
                    // and masked (the packed instructions cost the same for one or two)
                    const float2 dx = make_float2((float)(pix.x - xj), (float)(pix.y - xj));
                    const float2 dy = make_float2((float)(piy.x - yj), (float)(piy.y - yj));
                    const float2 dz = make_float2((float)(piz.x - zj), (float)(piz.y - zj));
                    const float2 qq = mul2(qiq2, make_float2(rj.q, rj.q));
                    const bool on0 = (m0 >> lane) & 1u;
                    const bool on1 = (m1 >> lane) & 1u;
                    float2 l1, l2n, l3 = z2, l4n = z2;
                    if constexpr (TRI) {
                        const float4 u = s_lj3[t3 + rj.type];
                        l1 = make_float2(u.x, u.y);
                        l2n = make_float2(u.z, u.w);
                        if (EN) {
                            const float4 v = s_lj3[nt3 + t3 + rj.type];
                            l3 = make_float2(v.x, v.y);
                            l4n = make_float2(v.z, v.w);
                        }
                    } else {
                        const float2 a0 = s_lja[ti0 + rj.type], a1 = s_lja[ti1 + rj.type];
                        l1 = make_float2(a0.x, a1.x);
                        l2n = make_float2(a0.y, a1.y);
                        if (EN) {
                            const float2 b0 = s_ljb[ti0 + rj.type], b1 = s_ljb[ti1 + rj.type];
                            l3 = make_float2(b0.x, b1.x);
                            l4n = make_float2(b0.y, b1.y);
                        }
                    }
                    float2 elj = z2, ec = z2;
                    const float2 fs = PairMath2::template eval<EN, SAME>(
                        dx, dy, dz, qq, l1, l2n, l3, l4n, on0, on1, k, elj, ec);
                    const float2 px = mul2(dx, fs), py = mul2(dy, fs), pz = mul2(dz, fs);
                    ax2 = add2(ax2, px);
                    ay2 = add2(ay2, py);
                    az2 = add2(az2, pz);
                    v0 = addr(px.x, px.y);
                    v1 = addr(py.x, py.y);
                    v2 = addr(pz.x, pz.y);
                    if (EN) {
                        alj2 = add2(alj2, elj);
                        ac2 = add2(ac2, ec);
                    }
                    if (VIR) {
                        axx2 = fma2(dx, px, axx2);
                        ayy2 = fma2(dy, py, ayy2);
                        azz2 = fma2(dz, pz, azz2);
                    }
                } else {
                    // FP64 twin: the two i halves one after the other; a half with no
                    // pair in range is skipped by the whole warp
    #pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const unsigned mh = h ? m1 : m0;
                        if (mh == 0u) continue;
                        const AtomRec &ri = h ? ri1 : ri0;
                        const T dx = (T)(ri.x - xj);
                        const T dy = (T)(ri.y - yj);
                        const T dz = (T)(ri.z - zj);
                        const bool on = (mh >> lane) & 1u;
                        const float4 ljp = s_lj[(h ? ti1 : ti0) + rj.type];
                        T elj = 0, ec = 0;
                        const T fs = PairMath<T>::template eval<EN, SAME>(
                            dx, dy, dz, mulr(h ? qiq1 : qiq0, (T)rj.q), ljp, on, k, elj, ec);
                        const T px = mulr(dx, fs), py = mulr(dy, fs), pz = mulr(dz, fs);
                        if (h) {
                            ax1 = addr(ax1, px);
                            ay1 = addr(ay1, py);
                            az1 = addr(az1, pz);
                        } else {
                            ax0 = addr(ax0, px);
                            ay0 = addr(ay0, py);
                            az0 = addr(az0, pz);
                        }
                        v0 = addr(v0, px);
                        v1 = addr(v1, py);
                        v2 = addr(v2, pz);
                        if (EN) {
                            a_lj = addr(a_lj, elj);
                            a_c = addr(a_c, ec);
                        }
                        if (VIR) {
                            a_xx = fmar(dx, px, a_xx);
                            a_yy = fmar(dy, py, a_yy);
                            a_zz = fmar(dz, pz, a_zz);
                        }
                    }
                }
                const T fj = reduce_j4<T>(v0, v1, v2, lane);
                if (q < 3 && fj != (T)0)
                    atomicAdd(jdst + jc * CL + jj, (unsigned long long)to_fix<T>(-fj));
            }
            if constexpr (PACK) {
                flush_i<float>(fi, lane, ax2.x, ay2.x, az2.x, ax2.y, ay2.y, az2.y);
                ax2 = ay2 = az2 = z2;
                if (EN) {
                    e_lj += (double)alj2.x + (double)alj2.y;
                    e_c += (double)ac2.x + (double)ac2.y;
                    alj2 = ac2 = z2;
                }
                if (VIR) {
                    vxx += (double)axx2.x + (double)axx2.y;
                    vyy += (double)ayy2.x + (double)ayy2.y;
                    vzz += (double)azz2.x + (double)azz2.y;
                    axx2 = ayy2 = azz2 = z2;
                }
            } else {
                flush_i<T>(fi, lane, ax0, ay0, az0, ax1, ay1, az1);
                ax0 = ay0 = az0 = ax1 = ay1 = az1 = 0;
                if (EN) {
                    e_lj += (double)a_lj;
                    e_c += (double)a_c;
                    a_lj = a_c = 0;
                }
                if (VIR) {
                    vxx += (double)a_xx;
                    vyy += (double)a_yy;
                    vzz += (double)a_zz;
                    a_xx = a_yy = a_zz = 0;
                }
            }
        }
    }
    // sum each i atom's partials over its 8 lanes (lane bits 0-2), then lane
    // jj = 0 of each quarter adds the totals of i atoms q and q + 4
    long long fsum[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        long long v = fi[c * 32 + lane];
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) v += __shfl_xor_sync(FULL, v, off);
        fsum[c] = v;
    }
    if (jj == 0) {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const int atom = q + 4 * (c / 3);
            if (fsum[c])
                atomicAdd(fslot + (size_t)(c % 3) * stride + (size_t)icl * CL + atom,
                          (unsigned long long)fsum[c]);
        }
    }
    if (EN || VIR) {
        e_lj += (double)a_lj;
        e_c += (double)a_c;
        vxx += (double)a_xx;
        vyy += (double)a_yy;
        vzz += (double)a_zz;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            e_lj += __shfl_xor_sync(FULL, e_lj, off);
            e_c += __shfl_xor_sync(FULL, e_c, off);
            vxx += __shfl_xor_sync(FULL, vxx, off);
            vyy += __shfl_xor_sync(FULL, vyy, off);
            vzz += __shfl_xor_sync(FULL, vzz, off);
        }
        if (lane == 0) {
            double *o = energy + (size_t)icl * 5;
            o[0] = e_lj;
            o[1] = e_c;
            o[2] = vxx;
            o[3] = vyy;
            o[4] = vzz;
        }
    }
}
template <typename T, bool EN, bool VIR, bool SAME, bool TRI = false>
__global__ void __launch_bounds__((pair_block<T, EN>()), (pair_minb<T, EN>())) k_pair(
    int maxcl, const int *__restrict__ ncl_dev, const AtomRec *__restrict__ rec,
    const int *__restrict__ jlist, const unsigned long long *__restrict__ jmask,
    const int *__restrict__ jcount, int jcap, const float4 *__restrict__ ljtab, PairConst k,
    unsigned long long *__restrict__ fslot, double *__restrict__ energy) {
    SOFIA_PDL_ENTRY();
    pair_body<T, EN, VIR, SAME, TRI>(blockIdx.x, maxcl, ncl_dev, rec, jlist, jmask, jcount, jcap,
                                ljtab, k, k.L, fslot, energy);
}

// Dynamic shared memory of the pair kernels: the two-index LJ table (nt^2
// float4) and, with the three-index table, nt^3 float4 (twice for energies).
inline bool pair_tri(int nt) { return nt >= 1 && nt <= SOFIA_PAIR_TRI_MAX; }
inline size_t pair_smem(int nt, bool tri, bool energy) {
    const size_t n2 = (size_t)nt * nt, n3 = n2 * nt;
    return sizeof(float4) * (n2 + (tri ? (energy ? 2 : 1) * n3 : 0));
}

// Types up to the documented maximum (48) need more than the default 48 KB of
// shared memory per block for the two-index table plus the kernels' static
// arrays: raise the pair kernels' dynamic limit to what nt needs (once, on the
// host, outside any stream capture).
inline cudaError_t pair_smem_optin(int nt) {
    static size_t done = 0;
    const size_t need = pair_smem(nt, false, true);
    if (need <= done || need <= 32768) return cudaSuccess;
    const int v = (int)need;
    cudaError_t e = cudaSuccess;
    auto set = [&](const void *f) {
        const cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
        if (r != cudaSuccess) e = r;
    };
    set((const void *)k_pair<double, true, true, true>);
    set((const void *)k_pair<double, true, false, true>);
    set((const void *)k_pair<double, false, false, true>);
    set((const void *)k_pair<float, true, true, true>);
    set((const void *)k_pair<float, true, false, true>);
    set((const void *)k_pair<float, false, false, true>);
    if (e == cudaSuccess) done = need;
    return e;
}

// Slot-ordered fixed-point pair forces -> the caller's atom order (sets the
// force arrays; bonded terms add to them afterwards).  Flags sums outside the
// fixed-point range.
// With flag != NULL, thread 0 also counts this step's list build and prune in
// cnt and clears the trigger word for the next step's displacement check (only
// bits are ORed into it).  With lg.on, each atom's Langevin force is added.
__device__ __forceinline__ void unpack_body(int bx, int nslots, const int *__restrict__ ncl_dev,
                         const int *__restrict__ slot_orig, const long long *__restrict__ fslot,
                         long long *__restrict__ fx, long long *__restrict__ fy,
                         long long *__restrict__ fz, int *__restrict__ status,
                         int *__restrict__ flag, long long *__restrict__ cnt, LangevinArgs lg,
                         float *__restrict__ ffo) {
    const int s = bx * blockDim.x + threadIdx.x;
    if (flag && s == 0) {
        const int f = flag[0];
        if (f & 1) cnt[0] += 1;
        if (f & 3) cnt[1] += 1;
        flag[0] = 0;
    }
    if (s >= nslots || s >= ncl_dev[0] * CL) return;
    const int o = slot_orig[s];
    if (o < 0) return;
    long long a = fslot[s], b = fslot[nslots + s], c = fslot[2 * (size_t)nslots + s];
    if (lg.on) {
        long long la, lb, lc;
        langevin_force(lg, o, la, lb, lc);
        a += la;
        b += lb;
        c += lc;
    }
    fx[o] = a;
    fy[o] = b;
    fz[o] = c;
    if (ffo) {
        ffo[3 * o + 0] = (float)((double)a * FIX_INV);
        ffo[3 * o + 1] = (float)((double)b * FIX_INV);
        ffo[3 * o + 2] = (float)((double)c * FIX_INV);
    }
    const long long lim = 1ll << 62;
    if (a > lim || a < -lim || b > lim || b < -lim || c > lim || c < -lim)
        atomicAdd(&status[ST_FIXED_OVF], 1);
}
__global__ void k_unpack(int nslots, const int *__restrict__ ncl_dev,
                         const int *__restrict__ slot_orig, const long long *__restrict__ fslot,
                         long long *__restrict__ fx, long long *__restrict__ fy,
                         long long *__restrict__ fz, int *__restrict__ status,
                         int *__restrict__ flag, long long *__restrict__ cnt, LangevinArgs lg,
                         float *__restrict__ ffo) {
    SOFIA_PDL_ENTRY();
    unpack_body(blockIdx.x, nslots, ncl_dev, slot_orig, fslot, fx, fy, fz, status, flag, cnt, lg, ffo);
}


// Dynamic pruning: keep the outer-list entries that have at least one unmasked
// atom pair within r_in = rc + margin at the current positions, and replace
// their pair mask by the in-range bits (bit 8*ii + jj = pair (i atom ii, j atom
// jj), the outer list's layout, which is also the pair kernel's lane layout:
// bit h*32 + lane is the pair (i atom (lane >> 3) + 4h, j atom lane & 7)).  Valid until an atom moves more than margin/2
// (checked like the rebuild trigger): a pair out of range now cannot come
// within rc before the next prune.  One warp per i-cluster, one lane per list
// entry: the i atoms sit in registers and every lane checks its entry's 64
// pairs (two i atoms per packed FP32x2 operation), so entries need no shuffles
// or ballots.  Distances here only select
// pairs, so FP32 copies of the positions suffice (the squared radius carries a
// 1e-3 A^2 safety margin).
__device__ __forceinline__ void prune_body(int bx, 
    const int *__restrict__ cond, int cmask, int maxcl, const int *__restrict__ ncl_dev,
    const float *__restrict__ recf,
    const int *__restrict__ jlist, const unsigned long long *__restrict__ jmask,
    const int *__restrict__ jcount, int jcap, float L, float rin2, float rfar2,
    const float4 *__restrict__ bb, int *__restrict__ ilist,
    unsigned long long *__restrict__ imask, int *__restrict__ icount,
    const int *__restrict__ slot_orig, const double *__restrict__ x,
    const double *__restrict__ y, const double *__restrict__ z, double *__restrict__ px,
    double *__restrict__ py, double *__restrict__ pz) {
    SOFIA_COND_RETURN;
    __shared__ float s_shf[27 * 3];
    if (threadIdx.x < 27) {
        const int im = threadIdx.x;
        s_shf[im * 3 + 0] = (float)(im % 3 - 1) * L;
        s_shf[im * 3 + 1] = (float)((im / 3) % 3 - 1) * L;
        s_shf[im * 3 + 2] = (float)(im / 9 - 1) * L;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int icl = (bx * blockDim.x + threadIdx.x) >> 5;
    if (icl >= maxcl || icl >= ncl_dev[0]) return;
    // the positions this prune is valid for (the prune trigger measures from them)
    if (lane < CL) {
        const int o = slot_orig[icl * CL + lane];
        if (o >= 0) {
            px[o] = x[o];
            py[o] = y[o];
            pz[o] = z[o];
        }
    }
    // i atoms 2p and 2p + 1 as the two components of packed FP32x2 operands,
    // read straight from the cluster's x[8], y[8], z[8]
    float2 xi[CL / 2], yi[CL / 2], zi[CL / 2];
    const float2 *ci = reinterpret_cast<const float2 *>(recf + (size_t)icl * 3 * CL);
#pragma unroll
    for (int pp = 0; pp < CL / 2; ++pp) {
        xi[pp] = ci[pp];
        yi[pp] = ci[CL / 2 + pp];
        zi[pp] = ci[CL + pp];
    }
    const float4 ilo = bb[2 * icl], ihi = bb[2 * icl + 1];
    const int n = jcount[icl];
    const int *row = jlist + (size_t)icl * jcap;
    const unsigned long long *mrow = jmask + (size_t)icl * jcap;
    int *orow = ilist + (size_t)icl * jcap;
    unsigned long long *omrow = imask + (size_t)icl * jcap;
    int kept = 0;
    for (int base = 0; base < n; base += 32) {
        const int e = base + lane;
        const bool active = e < n;
        const int w = active ? row[e] : 0;
        const unsigned long long m = active ? mrow[e] : 0ull;
        unsigned lo = 0u, hi = 0u;  // in-range bits 8*ii + jj: i atoms 0-3 in lo, 4-7 in hi
        if (active) {
            const int jc = w & ((1 << IMG_SHIFT) - 1);
            const int img = w >> IMG_SHIFT;
            const float sx = s_shf[img * 3 + 0], sy = s_shf[img * 3 + 1], sz = s_shf[img * 3 + 2];
            // bounding boxes at the current positions: an entry whose boxes are
            // farther apart than rfar (above r_in by far more than rounding) has
            // no pair in range, and its atoms are not loaded
            const float4 jlo = bb[2 * jc], jhi = bb[2 * jc + 1];
            const float gx = gap(ilo.x, ihi.x, jlo.x + sx, jhi.x + sx);
            const float gy = gap(ilo.y, ihi.y, jlo.y + sy, jhi.y + sy);
            const float gz = gap(ilo.z, ihi.z, jlo.z + sz, jhi.z + sz);
            if (gx * gx + gy * gy + gz * gz <= rfar2) {
                // the j cluster's x[8], y[8], z[8]: three 16-byte loads per 4 atoms
                // (one half at a time keeps the kernel within 64 registers)
                const float4 *cj = reinterpret_cast<const float4 *>(recf + (size_t)jc * 3 * CL);
                // The sign bit of dz^2 - rin2 + dy^2 + dx^2 (rin2 folded into the
                // first FMA of the chain) is the in-range bit, and one funnel shift
                // appends it.  Its rounding differs from that of r2 by a few ulp of
                // r2, far inside the 1e-3 A^2 that rin2 carries above (rc + margin)^2.
                // Appended for j atoms 7 down to 0 and, within one, i atoms 3 down
                // to 0 (7 down to 4 in hi), bit (jj, ii) ends at 4 jj + ii; the
                // final transpose moves it to 8 ii + jj.
                const float2 nrin2 = make_float2(-rin2, -rin2);
#pragma unroll 1
                for (int hh = 1; hh >= 0; --hh) {
                    const float4 jx = __ldg(&cj[hh]), jy = __ldg(&cj[2 + hh]),
                                 jz = __ldg(&cj[4 + hh]);
#pragma unroll
                    for (int q = 3; q >= 0; --q) {
                        const float nx = -((&jx.x)[q] + sx), ny = -((&jy.x)[q] + sy),
                                    nz = -((&jz.x)[q] + sz);
                        const float2 nx2 = make_float2(nx, nx), ny2 = make_float2(ny, ny),
                                     nz2 = make_float2(nz, nz);
#pragma unroll
                        for (int pp = CL / 2 - 1; pp >= 0; --pp) {
                            // i atoms 2pp (component x) and 2pp + 1 (component y)
                            const float2 dx = add2(xi[pp], nx2), dy = add2(yi[pp], ny2),
                                         dz = add2(zi[pp], nz2);
                            const float2 dd = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, nrin2)));
                            unsigned &acc = (pp >= 2) ? hi : lo;
                            acc = __funnelshift_l(__float_as_uint(dd.y), acc, 1);
                            acc = __funnelshift_l(__float_as_uint(dd.x), acc, 1);
                        }
                    }
                }
                lo = transpose_8x4(lo);
                hi = transpose_8x4(hi);
            }
        }
        const unsigned long long newm = (((unsigned long long)hi << 32) | lo) & m;
        const bool keep = newm != 0ull;
        const unsigned kb = __ballot_sync(FULL, keep);
        if (keep) {
            const int at = kept + __popc(kb & ((1u << lane) - 1u));
            orow[at] = w;
            omrow[at] = newm;
        }
        kept += __popc(kb);
    }
    if (lane == 0) icount[icl] = kept;
}
__global__ void __launch_bounds__(256, SOFIA_PRUNE_MINB) k_prune(
    const int *__restrict__ cond, int cmask, int maxcl, const int *__restrict__ ncl_dev,
    const float *__restrict__ recf,
    const int *__restrict__ jlist, const unsigned long long *__restrict__ jmask,
    const int *__restrict__ jcount, int jcap, float L, float rin2, float rfar2,
    const float4 *__restrict__ bb, int *__restrict__ ilist,
    unsigned long long *__restrict__ imask, int *__restrict__ icount,
    const int *__restrict__ slot_orig, const double *__restrict__ x,
    const double *__restrict__ y, const double *__restrict__ z, double *__restrict__ px,
    double *__restrict__ py, double *__restrict__ pz) {
    SOFIA_PDL_ENTRY();
    prune_body(blockIdx.x, cond, cmask, maxcl, ncl_dev, recf, jlist, jmask, jcount, jcap, L, rin2, rfar2, bb, ilist, imask, icount, slot_orig, x, y, z, px, py, pz);
}



__global__ void k_set_flag(int *__restrict__ flag, int v) {
    SOFIA_PDL_ENTRY();
    if (threadIdx.x == 0 && blockIdx.x == 0) flag[0] = v;
}

// Two-stage deterministic column sums: stage 1 = fixed grid of blocks over
// contiguous ranges (coalesced), stage 2 = one block over the partials.
__device__ __forceinline__ void red_stage1_body(int bx, int n, int w, const int *__restrict__ ncl_dev,
                             const double *__restrict__ in, double *__restrict__ part, int nblk) {
    __shared__ double s[256];
    const int nn = ncl_dev ? min(n, ncl_dev[0]) : n;
    const int chunk = (nn + nblk - 1) / nblk;
    const int b0 = bx * chunk, b1 = min(nn, b0 + chunk);
    for (int c = 0; c < w; ++c) {
        double acc = 0.0;
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += in[(size_t)i * w + c];
        s[threadIdx.x] = acc;
        __syncthreads();
        for (int off = 128; off > 0; off >>= 1) {
            if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[bx * w + c] = s[0];
        __syncthreads();
    }
}
__global__ void k_red_stage1(int n, int w, const int *__restrict__ ncl_dev,
                             const double *__restrict__ in, double *__restrict__ part) {
    SOFIA_PDL_ENTRY();
    red_stage1_body(blockIdx.x, n, w, ncl_dev, in, part, (int)gridDim.x);
}
__device__ __forceinline__ void red_stage2_body(int bx, int nblk, int w, const double *__restrict__ part,
                             double *__restrict__ out, double scale) {
    __shared__ double s[256];
    for (int c = 0; c < w; ++c) {
        s[threadIdx.x] = (threadIdx.x < nblk) ? part[threadIdx.x * w + c] : 0.0;
        __syncthreads();
        for (int off = 128; off > 0; off >>= 1) {
            if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = scale * s[0];
        __syncthreads();
    }
}
__global__ void k_red_stage2(int nblk, int w, const double *__restrict__ part,
                             double *__restrict__ out, double scale) {
    SOFIA_PDL_ENTRY();
    red_stage2_body(blockIdx.x, nblk, w, part, out, scale);
}

// Ballistic drift x += dt*v (FP64), used to move a system between
// evaluations without forces (list maintenance and throughput checks).
__global__ void k_drift(int n, double dt, double *__restrict__ x, double *__restrict__ y,
                        double *__restrict__ z, const double *__restrict__ vx,
                        const double *__restrict__ vy, const double *__restrict__ vz) {
    SOFIA_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += dt * vx[i];
    y[i] += dt * vy[i];
    z[i] += dt * vz[i];
}

__global__ void k_aos_to_soa(int n, const float4 *__restrict__ pos, double *__restrict__ x,
                             double *__restrict__ y, double *__restrict__ z) {
    SOFIA_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    x[i] = (double)p.x;
    y[i] = (double)p.y;
    z[i] = (double)p.z;
}

__global__ void k_fix_to_float(int n, const long long *__restrict__ fx,
                               const long long *__restrict__ fy,
                               const long long *__restrict__ fz, float *__restrict__ ff) {
    SOFIA_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ff[3 * i + 0] = (float)((double)fx[i] * FIX_INV);
    ff[3 * i + 1] = (float)((double)fy[i] * FIX_INV);
    ff[3 * i + 2] = (float)((double)fz[i] * FIX_INV);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side

static int sys_alloc(Sys *s) {
    sofia_nb_ctx *ctx = s->ctx;
    const size_t n = (size_t)s->n;
    for (int d = 0; d < 3; ++d) {
        SOFIA_CUDA(ctx, s->x[d].ensure(sizeof(double) * n));
        SOFIA_CUDA(ctx, s->v[d].ensure(sizeof(double) * n));
        SOFIA_CUDA(ctx, s->f[d].ensure(sizeof(long long) * n));
        SOFIA_CUDA(ctx, s->xref[d].ensure(sizeof(double) * n));
        SOFIA_CUDA(ctx, s->img[d].ensure(sizeof(double) * n));
    }
    SOFIA_CUDA(ctx, s->col_count.ensure(sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, s->col_start.ensure(sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, s->col_fill.ensure(sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, cudaMemset(s->col_count.p, 0, sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, cudaMemset(s->col_fill.p, 0, sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, s->cl_start.ensure(sizeof(int) * (s->ncols + 1)));
    SOFIA_CUDA(ctx, s->col_atoms.ensure(sizeof(int) * n * 2));  // atoms + column of atom
    SOFIA_CUDA(ctx, s->col_key.ensure(sizeof(float) * n));
    const size_t maxcl = (size_t)s->max_clusters;
    SOFIA_CUDA(ctx, s->slot_orig.ensure(sizeof(int) * maxcl * CL + sizeof(int) * maxcl));
    SOFIA_CUDA(ctx, s->rec.ensure(sizeof(AtomRec) * maxcl * CL));
    SOFIA_CUDA(ctx, s->sref.ensure((6 * sizeof(double) + sizeof(float) + sizeof(int)) * maxcl * CL));
    SOFIA_CUDA(ctx, s->recf.ensure(sizeof(float) * 3 * maxcl * CL));
    SOFIA_CUDA(ctx, s->fslot.ensure(sizeof(long long) * 3 * maxcl * CL));
    SOFIA_CUDA(ctx, s->atom_slot.ensure(sizeof(int) * n));
    SOFIA_CUDA(ctx, s->bb.ensure(sizeof(float4) * 2 * maxcl));
    SOFIA_CUDA(ctx, s->jcount.ensure(sizeof(int) * maxcl));
    SOFIA_CUDA(ctx, s->nclusters.ensure(sizeof(int) * 4));
    SOFIA_CUDA(ctx, s->energy.ensure(sizeof(double) * 5 * maxcl));
    SOFIA_CUDA(ctx, s->red.ensure(sizeof(double) * 8));
    SOFIA_CUDA(ctx, s->flag.ensure(sizeof(int) * 4));
    SOFIA_CUDA(ctx, s->status_local.ensure(sizeof(int) * ST_NSLOTS));
    for (int d = 0; d < 3; ++d) SOFIA_CUDA(ctx, s->xprn[d].ensure(sizeof(double) * n));
    SOFIA_CUDA(ctx, s->icount.ensure(sizeof(int) * maxcl));
    SOFIA_CUDA(ctx, s->part.ensure(sizeof(double) * 8 * RED_BLOCKS));
    SOFIA_CUDA(ctx, s->dcount.ensure(sizeof(long long) * 4));
    SOFIA_CUDA(ctx, cudaMemset(s->dcount.p, 0, sizeof(long long) * 4));
    SOFIA_CUDA(ctx, cudaMemset(s->status_local.p, 0, sizeof(int) * ST_NSLOTS));
    // no clusters and empty rows until the first build (host queries may come first)
    SOFIA_CUDA(ctx, cudaMemset(s->nclusters.p, 0, sizeof(int) * 4));
    SOFIA_CUDA(ctx, cudaMemset(s->jcount.p, 0, sizeof(int) * maxcl));
    SOFIA_CUDA(ctx, cudaMemset(s->icount.p, 0, sizeof(int) * maxcl));
    return SOFIA_OK;
}

// Column grid and list capacities.  aspect scales the xy column width from the
// cube side of 8 atoms (aspect 1: clusters about as tall as wide; < 1: narrower
// columns and taller clusters; > 1: wider and flatter ones).  False if the box is
// too small for the grid.
bool sys_geometry(Sys *s, double aspect) {
    const double rho = (double)s->n / (s->L * s->L * s->L);
    const double s_target = aspect * cbrt((double)CL / rho);
    const int ncx = (int)fmax(1.0, floor(s->L / s_target));
    const double s_col = s->L / ncx;
    const int reach = (int)ceil(s->rlist / s_col);
    if (reach >= ncx) return false;
    s->ncx = ncx;
    s->s_col = s_col;
    s->ncols = ncx * ncx;
    s->ncol_reach = reach;
    s->aspect = aspect;
    s->max_clusters = s->n / CL + s->ncols + 1;
    // expected j-clusters per row: bounding-box volume around rlist, plus headroom
    const double zext = (double)CL / (rho * s_col * s_col);  // cluster height
    const double reach_d = s->rlist + 1.5 * fmax(s_col, zext);
    s->jcap = (int)(4.19 * reach_d * reach_d * reach_d * rho / CL * 1.3) + 32;
    return true;
}

void dropin_drop(Sys *s) {
    for (auto &g : s->dropin)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

static int sys_alloc_list(Sys *s) {
    dropin_drop(s);  // captured drop-in graphs hold the old list pointers
    const size_t maxcl = (size_t)s->max_clusters;
    SOFIA_CUDA(s->ctx, s->jlist.ensure(sizeof(int) * maxcl * s->jcap));
    SOFIA_CUDA(s->ctx, s->jmask.ensure(sizeof(unsigned long long) * maxcl * s->jcap));
    SOFIA_CUDA(s->ctx, s->ilist.ensure(sizeof(int) * maxcl * s->jcap));
    SOFIA_CUDA(s->ctx, s->imask.ensure(sizeof(unsigned long long) * maxcl * s->jcap));
    return SOFIA_OK;
}

static void sys_pack(Sys *s, const int *cond) {
    cudaStream_t st = s->ctx->stream;
    const int nslots = s->max_clusters * CL;
    sofia::launch_pdl(k_pack, grid_for(nslots, 256), 256, 0, st,
        nslots, s->nclusters.as<int>(), s->slot_orig.as<int>(), s->x[0].as<double>(),
        s->x[1].as<double>(), s->x[2].as<double>(), s->xref[0].as<double>(),
        s->xref[1].as<double>(), s->xref[2].as<double>(), s->img[0].as<double>(),
        s->img[1].as<double>(), s->img[2].as<double>(), s->q.as<float>(), s->type.as<int>(), s->L,
        s->rec.as<AtomRec>(), s->recf.as<float>(), s->fslot.as<long long>(), s->bb.as<float4>(),
        cond, s->sref.as<double>());
    s->launches += 1;
}

// The list build, in two parts around the record pack (the bounding boxes and
// the search need current records).  With cond == nullptr the kernels always
// run; otherwise every kernel returns at once unless (cond[0] & 1).
// Part 1: bin atoms into xy columns, sort each column by z, assign cluster slots.
static void sys_build_bin(Sys *s, const int *cond) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int n = s->n;
    const int cm = 1;
    int *col_of = s->col_atoms.as<int>() + n;
    int *cl_col = s->slot_orig.as<int>() + (size_t)s->max_clusters * CL;
    // col_count and col_fill start at zero (set at creation, cleared after each
    // use); every slot of the new clusters is written by the column sort
    sofia::launch_pdl(k_wrap_bin, grid_for(n, 256), 256, 0, st,
        cond, cm, n, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(), s->L,
        s->s_col, s->ncx, s->img[0].as<double>(), s->img[1].as<double>(), s->img[2].as<double>(),
        s->xref[0].as<double>(), s->xref[1].as<double>(), s->xref[2].as<double>(), col_of,
        s->col_count.as<int>(), s->col_key.as<float>());
    sofia::launch_pdl(k_scan_cols, 1, 1024, 0, st, cond, cm, s->ncols, s->col_count.as<int>(),
                                    s->col_start.as<int>(), s->cl_start.as<int>(),
                                    s->nclusters.as<int>());
    sofia::launch_pdl(k_col_scatter, grid_for(n, 256), 256, 0, st, cond, cm, n, col_of, s->col_start.as<int>(),
                                                    s->col_fill.as<int>(),
                                                    s->col_atoms.as<int>());
    sofia::launch_pdl(k_col_sort_assign, s->ncols, 256, 0, st, cond, cm, s->ncols, s->col_start.as<int>(),
                                                s->col_atoms.as<int>(), s->col_key.as<float>(),
                                                s->cl_start.as<int>(), s->slot_orig.as<int>(),
                                                cl_col, s->atom_slot.as<int>(),
                                                s->col_fill.as<int>(), s->status_local.as<int>());
    s->launches += 4;
}

// Part 2: cluster bounding boxes and the cluster-pair search.
static int sys_build_search(Sys *s, const int *cond) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int cm = 1;
    int *cl_col = s->slot_orig.as<int>() + (size_t)s->max_clusters * CL;
    // the cluster boxes come from the record pack that precedes the search
    SearchArgs a;
    a.cond = cond;
    a.cmask = cm;
    a.maxcl = s->max_clusters;
    a.ncx = s->ncx;
    a.reach = s->ncol_reach;
    a.jcap = s->jcap;
    a.L = (float)s->L;
    a.s_col = (float)s->s_col;
    const float rl = (float)s->rlist + 1e-3f;
    a.rl = rl;
    a.rl2 = rl * rl;
    a.rexcl2 = (float)(s->r_excl * s->r_excl);
    a.ncl_dev = s->nclusters.as<int>();
    a.cl_start = s->cl_start.as<int>();
    a.cl_col = cl_col;
    a.slot_orig = s->slot_orig.as<int>();
    a.specbond = s->specbond.as<int>();
    a.num3bond = s->num3bond.as<int>();
    a.atom_slot = s->atom_slot.as<int>();
    a.n = s->n;
    a.bb = s->bb.as<float4>();
    a.jlist = s->jlist.as<int>();
    a.jcount = s->jcount.as<int>();
    a.jmask = s->jmask.as<unsigned long long>();
    a.status = s->status_local.as<int>();
    sofia::launch_pdl(k_search, grid_for((long)s->max_clusters * 32, 256), 256, 0, st, a);
    SOFIA_CUDA(ctx, cudaGetLastError());
    s->launches += 1;
    if (!cond) s->n_builds++;
    s->built = 1;
    return SOFIA_OK;
}

// The whole build; the records are current afterwards whether or not the
// list was rebuilt.
static int sys_build(Sys *s, const int *cond) {
    sys_build_bin(s, cond);
    sys_pack(s, cond);
    return sys_build_search(s, cond);
}

// Folds finished event pairs into the timers (called after a stream sync).
static void sys_collect_timers(Sys *s) {
    float ms = 0.0f;
    if (s->pending_build && cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]) == cudaSuccess) {
        s->t_build_ms += ms;
        s->n_build_timed++;
    }
    if (s->pending_pair && cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]) == cudaSuccess) {
        s->t_pair_ms += ms;
        s->n_pair++;
    }
    cudaGetLastError();
    s->pending_build = s->pending_pair = 0;
}

static PairConst make_pair_const(const Sys *s, const float *lj_dummy) {
    (void)lj_dummy;
    PairConst k;
    const double rcut2 = (double)(float)(s->rc * s->rc);
    k.rcut2d = rcut2;
    k.cut_coulsqd = rcut2;
    k.rcut2 = (float)rcut2;
    k.cut_coulsq = (float)rcut2;
    k.alphad = s->alpha;
    k.kexp = (float)(-(s->alpha * s->alpha) * 1.4426950408889634);  // -alpha^2 log2(e)
    const double EP = (double)0.3275911f;
    k.EWALD_Pd = EP;
    k.pa = (float)(EP * s->alpha);
    const double mypis = (double)1.77245385090551602729f;
    k.MY_PIS_INV = 1.0 / mypis;
    k.c2a = (float)((2.0 * s->alpha) / mypis);
    k.e_shiftd = s->e_shift;
    k.f_shiftd = s->f_shift;
    k.e_shift = (float)s->e_shift;
    k.f_shift = (float)s->f_shift;
    k.coulpre = s->coulpre;
    k.coulpred = (double)s->coulpre;
    k.A1d = (double)0.254829592f;
    k.A2d = (double)-0.284496736f;
    k.A3d = (double)1.421413741f;
    k.A4d = (double)-1.453152027f;
    k.A5d = (double)1.061405429f;
    k.A1 = 0.254829592f;
    k.A2 = -0.284496736f;
    k.A3 = 1.421413741f;
    k.A4 = -1.453152027f;
    k.A5 = 1.061405429f;
    k.kexp2 = make_float2(k.kexp, k.kexp);
    k.pa2 = make_float2(k.pa, k.pa);
    k.c2a2 = make_float2(k.c2a, k.c2a);
    k.e_shift2 = make_float2(k.e_shift, k.e_shift);
    k.f_shift2 = make_float2(k.f_shift, k.f_shift);
    k.A1_2 = make_float2(k.A1, k.A1);
    k.A2_2 = make_float2(k.A2, k.A2);
    k.A3_2 = make_float2(k.A3, k.A3);
    k.A4_2 = make_float2(k.A4, k.A4);
    k.A5_2 = make_float2(k.A5, k.A5);
    k.ljs6d = s->lj_shift ? 1.0 / (rcut2 * rcut2 * rcut2) : 0.0;
    k.ljs6 = (float)k.ljs6d;
    k.ljs6_2 = make_float2(k.ljs6, k.ljs6);
    k.L = s->L;
    k.ntypes = s->ntypes;
    return k;
}

// Launches: displacement check, conditional rebuild, pack, pair kernel.
// `force_build` rebuilds regardless of the trigger.
// The cluster boxes come from the record pack that precedes every prune.
static void sys_prune(Sys *s, const int *cond) {
    cudaStream_t st = s->ctx->stream;
    const float rin = (float)(s->rc + s->margin);
    const float rin2 = rin * rin + 1e-3f;
    const float rfar = rin + 0.01f;
    sofia::launch_pdl(k_prune, grid_for((long)s->max_clusters * 32, 256), 256, 0, st,
        cond, 3, s->max_clusters, s->nclusters.as<int>(), s->recf.as<float>(),
        s->jlist.as<int>(), s->jmask.as<unsigned long long>(), s->jcount.as<int>(), s->jcap,
        (float)s->L, rin2, rfar * rfar, s->bb.as<float4>(), s->ilist.as<int>(),
        s->imask.as<unsigned long long>(),
        s->icount.as<int>(), s->slot_orig.as<int>(), s->x[0].as<double>(), s->x[1].as<double>(),
        s->x[2].as<double>(), s->xprn[0].as<double>(), s->xprn[1].as<double>(),
        s->xprn[2].as<double>());
    s->launches += 1;
    if (!cond) s->n_prunes++;
}


// One evaluation: displacement triggers, list rebuild or prune when due, pack,
// pair kernel on the pruned list, deterministic energy reduction.
int sys_eval(Sys *s, int precision, bool energy, bool virial, bool force_build) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int n = s->n;
    bool build = force_build || !s->built;
    bool prune = build;
    if (!build) {
        const double half = 0.5 * s->skin, phalf = 0.5 * s->margin;
        SOFIA_CUDA(ctx, cudaMemsetAsync(s->flag.p, 0, sizeof(int), st));
        sofia::launch_pdl(k_disp_check, grid_for(n, 256), 256, 0, st,
            n, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(),
            s->xref[0].as<double>(), s->xref[1].as<double>(), s->xref[2].as<double>(),
            s->xprn[0].as<double>(), s->xprn[1].as<double>(), s->xprn[2].as<double>(), s->L,
            half * half, phalf * phalf, s->flag.as<int>());
        s->launches += 1;
        int h = 0;
        SOFIA_CUDA(ctx, cudaMemcpyAsync(&h, s->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
        build = (h & 1) != 0;
        prune = h != 0;
    }
    if (s->timing) sys_collect_timers(s);
    for (int attempt = 0; attempt < 4; ++attempt) {
        if (build) {
            SOFIA_CUDA(ctx, cudaMemsetAsync(s->status_local.p, 0, sizeof(int) * ST_NSLOTS, st));
            if (s->timing) cudaEventRecord(s->ev[0], st);
            int rc = sys_build(s, nullptr);
            if (rc) return rc;
            if (s->timing) {
                cudaEventRecord(s->ev[1], st);
                s->pending_build = 1;
            }
            int hs[ST_NSLOTS];
            SOFIA_CUDA(ctx, cudaMemcpyAsync(hs, s->status_local.p, sizeof(hs),
                                            cudaMemcpyDeviceToHost, st));
            SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
            if (hs[ST_CELLOVER])
                return fail(ctx, SOFIA_EINVAL, "an xy column holds more than 2048 atoms%s");
            if (hs[ST_NCLUSTER] > s->jcap) {
                // redo with a larger row capacity, like the reference's list regrow
                s->jcap = (int)(hs[ST_NCLUSTER] * 1.2) + 16;
                int r2 = sys_alloc_list(s);
                if (r2) return r2;
                continue;
            }
        } else {
            sys_pack(s, nullptr);
        }
        break;
    }
    if (prune) sys_prune(s, nullptr);
    return sys_pair(s, precision, energy, virial);
}

// Pair kernel (+ energy reduction) on the pruned list.
int sys_pair(Sys *s, int precision, bool energy, bool virial, int *count_flag,
             const LangevinArgs *lg, float *ff_out) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    PairConst k = make_pair_const(s, nullptr);
    // blocks of the force-only FP32 kernel and of the others (energies, FP64)
    const int blocks = grid_for((long)s->max_clusters * 32, SOFIA_PAIR_BLOCK);
    const int blocks_en = grid_for((long)s->max_clusters * 32, SOFIA_PAIR_BLOCK_EN);
    const size_t smem = pair_smem(s->ntypes, false, energy || virial);
    const bool tri = (energy || virial) && pair_tri(s->ntypes);
    const size_t smem3 = pair_smem(s->ntypes, tri, energy || virial);
    long long *fx = s->f[0].as<long long>(), *fy = s->f[1].as<long long>(),
              *fz = s->f[2].as<long long>();
#define SOFIA_PAIR_ARGS                                                                   \
    s->max_clusters, s->nclusters.as<int>(), s->rec.as<AtomRec>(), s->ilist.as<int>(),    \
        s->imask.as<unsigned long long>(), s->icount.as<int>(), s->jcap,                  \
        s->ljtab.as<float4>(), k, s->fslot.as<unsigned long long>(), s->energy.as<double>()
    if (s->timing) cudaEventRecord(s->ev[2], st);
    // sofia_system_create requires rcut == cut_coul: one cut-off gates both terms
    if (precision == SOFIA_PREC_FP64) {
        if (virial)
            sofia::launch_pdl(k_pair<double, true, true, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem, st, SOFIA_PAIR_ARGS);
        else if (energy)
            sofia::launch_pdl(k_pair<double, true, false, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem, st, SOFIA_PAIR_ARGS);
        else
            sofia::launch_pdl(k_pair<double, false, false, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem, st, SOFIA_PAIR_ARGS);
    } else if (tri) {
        if (virial)
            sofia::launch_pdl(k_pair<float, true, true, true, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem3, st,
                              SOFIA_PAIR_ARGS);
        else
            sofia::launch_pdl(k_pair<float, true, false, true, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem3, st,
                              SOFIA_PAIR_ARGS);
    } else {
        if (virial)
            sofia::launch_pdl(k_pair<float, true, true, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem, st, SOFIA_PAIR_ARGS);
        else if (energy)
            sofia::launch_pdl(k_pair<float, true, false, true>, blocks_en, SOFIA_PAIR_BLOCK_EN, smem, st, SOFIA_PAIR_ARGS);
        else
            sofia::launch_pdl(k_pair<float, false, false, true>, blocks, SOFIA_PAIR_BLOCK, smem, st, SOFIA_PAIR_ARGS);
    }
#undef SOFIA_PAIR_ARGS
    if (s->timing) {
        cudaEventRecord(s->ev[3], st);
        s->pending_pair = 1;
    }
    const int nslots = s->max_clusters * CL;
    LangevinArgs lgv{};
    if (lg) lgv = *lg;
    sofia::launch_pdl(k_unpack, grid_for(nslots, 256), 256, 0, st, nslots, s->nclusters.as<int>(),
                                                    s->slot_orig.as<int>(),
                                                    s->fslot.as<long long>(), fx, fy, fz,
                                                    ctx->d_status, count_flag,
                                                    s->dcount.as<long long>(), lgv, ff_out);
    s->launches += 2;
    if (energy || virial) {
        sofia::launch_pdl(k_red_stage1, RED_BLOCKS, 256, 0, st, s->max_clusters, 5, s->nclusters.as<int>(),
                                                 s->energy.as<double>(), s->part.as<double>());
        // the half list holds each pair once: no halving
        sofia::launch_pdl(k_red_stage2, 1, 256, 0, st, RED_BLOCKS, 5, s->part.as<double>(), s->red.as<double>(),
                                        1.0);
        s->launches += 2;
    }
    SOFIA_CUDA(ctx, cudaGetLastError());
    return SOFIA_OK;
}

// Device-only evaluation, no host round trip (graph-capturable): displacement
// triggers (or a forced build), conditional rebuild, pack, conditional prune,
// pair kernel.  Row-capacity overflow is recorded in status_local and checked
// by the caller after the segment (sys_list_overflow).
int sys_step_forces(Sys *s, int precision, bool energy, bool virial, bool force_build,
                    bool disp_done, const LangevinArgs *lg, float *ff_out) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int n = s->n;
    int *flag = s->flag.as<int>();
    if (force_build || !s->built) {
        sofia::launch_pdl(k_set_flag, 1, 32, 0, st, flag, 3);
    } else if (!disp_done) {
        const double half = 0.5 * s->skin, phalf = 0.5 * s->margin;
        sofia::launch_pdl(k_set_flag, 1, 32, 0, st, flag, 0);
        sofia::launch_pdl(k_disp_check, grid_for(n, 256), 256, 0, st,
            n, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(),
            s->xref[0].as<double>(), s->xref[1].as<double>(), s->xref[2].as<double>(),
            s->xprn[0].as<double>(), s->xprn[1].as<double>(), s->xprn[2].as<double>(), s->L,
            half * half, phalf * phalf, flag);
    }
    int rc = sys_build(s, flag);
    if (rc) return rc;
    sys_prune(s, flag);
    s->launches += 1;
    // the force unpack counts the build/prune events and clears the trigger word
    return sys_pair(s, precision, energy, virial, flag, lg, ff_out);
}

// After a device-only segment: SOFIA_ENEEDGROW (and a larger row capacity) if
// some list row overflowed; SOFIA_EINVAL if a column overflowed.
int sys_list_overflow(Sys *s, const int32_t *status) {
    sofia_nb_ctx *ctx = s->ctx;
    int hs[ST_NSLOTS];
    if (status) {
        memcpy(hs, status, sizeof(hs));
    } else {
        SOFIA_CUDA(ctx, cudaMemcpyAsync(hs, s->status_local.p, sizeof(hs),
                                        cudaMemcpyDeviceToHost, ctx->stream));
        SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (hs[ST_CELLOVER]) return fail(ctx, SOFIA_EINVAL, "an xy column holds more than 2048 atoms%s");
    if (hs[ST_NCLUSTER] > s->jcap) {
        s->jcap = (int)(hs[ST_NCLUSTER] * 1.2) + 16;
        int r2 = sys_alloc_list(s);
        if (r2) return r2;
        SOFIA_CUDA(ctx, cudaMemsetAsync(s->status_local.p, 0, sizeof(int) * ST_NSLOTS, ctx->stream));
        s->built = 0;
        return SOFIA_ENEEDGROW;
    }
    return SOFIA_OK;
}

// The drop-in force call as one CUDA graph: AoS positions -> FP64 SoA,
// displacement triggers, conditional rebuild and prune, pair kernel, forces ->
// real*4 AoS.  It reads stage_pos and writes stage_ff; variant e: 0 forces,
// 1 + energies, 2 + energies and virial.
static int dropin_capture(Sys *s, int e) {
    sofia_nb_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int n = s->n;
    const int timing = s->timing;
    s->timing = 0;
    const long long l0 = s->launches;
    cudaGraph_t g = nullptr;
    SOFIA_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    sofia::launch_pdl(k_aos_to_soa, grid_for(n, 256), 256, 0, st, n, s->stage_pos.as<float4>(),
                                                   s->x[0].as<double>(), s->x[1].as<double>(),
                                                   s->x[2].as<double>());
    // the force unpack also writes the real*4 forces the call returns
    const int rc = sys_step_forces(s, s->precision, e >= 1, e == 2, false, false, nullptr,
                                   s->stage_ff.as<float>());
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    s->dropin_launches[e] = s->launches - l0 + 1;
    s->launches = l0;
    s->timing = timing;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaStreamEndCapture (drop-in)");
    const cudaError_t ie = cudaGraphInstantiate(&s->dropin[e], g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return cuda_fail(ctx, ie, "cudaGraphInstantiate (drop-in)");
    return SOFIA_OK;
}

}  // namespace sofia

using sofia::Sys;

extern "C" int sofia_system_create(sofia_nb_ctx *ctx, const sofia_system_desc *d,
                                   sofia_system **out) {
    if (!ctx || !d || !out) return SOFIA_EINVAL;
    *out = nullptr;
    if (d->np <= 0 || d->ntypes <= 0 || d->ntypes > 48 || !d->type || !d->q || !d->lj1 ||
        !d->lj2 || !d->lj3 || !d->lj4 || !d->specbond || !d->num3bond || !(d->box > 0.0f) ||
        !(d->cut_coul > 0.0f) || d->neighbor_pad < 0.0f)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad system description%s");
    if (d->rcut != d->cut_coul)
        return sofia::fail(ctx, SOFIA_EINVAL, "the cluster path needs rcut == cut_coul%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, sofia::pair_smem_optin(d->ntypes));
    sofia_system *ss = new sofia_system();
    Sys *s = &ss->s;
    s->ctx = ctx;
    s->n = d->np;
    s->ntypes = d->ntypes;
    s->precision = d->precision;
    s->box = d->box;
    s->L = (double)d->box;
    s->alpha = d->alpha;
    s->rc = (double)d->cut_coul;
    s->skin = (double)d->neighbor_pad;
    s->rlist = s->rc + s->skin;
    s->coulpre = 332.06371f;
    sofia_dsf_constants(d->alpha, d->cut_coul, &s->e_shift, &s->f_shift);
    if (s->rlist > 0.5 * s->L - 1.0) {
        delete ss;
        return sofia::fail(ctx, SOFIA_EINVAL, "box too small for rc + skin%s");
    }
    if (!sofia::sys_geometry(s, 1.0)) {
        delete ss;
        return sofia::fail(ctx, SOFIA_EINVAL, "box too small for the column grid%s");
    }
    int rc = sofia::sys_alloc(s);
    if (!rc) rc = sofia::sys_alloc_list(s);
    const size_t n = (size_t)s->n;
    if (!rc) {
        // the system's stream is idle here: synchronous copies
        const cudaError_t se = cudaStreamSynchronize(ctx->stream);
        if (se != cudaSuccess) rc = sofia::cuda_fail(ctx, se, "cudaStreamSynchronize");
        if (!rc && (s->type.ensure(sizeof(int) * n) || s->q.ensure(sizeof(float) * n) ||
            s->specbond.ensure(sizeof(int) * 12 * n) || s->num3bond.ensure(sizeof(int) * n) ||
            s->ljtab.ensure(sizeof(float4) * (size_t)s->ntypes * s->ntypes) ||
            s->invm.ensure(sizeof(double) * n) || s->mass.ensure(sizeof(double) * n)))
            rc = sofia::fail(ctx, SOFIA_ECUDA, "allocation failed%s");
        if (!rc) {
            // every copy is checked; host staging lives in vectors so that an
            // early return frees it
            cudaError_t e = cudaSuccess;
            auto cp = [&](void *dst, const void *src, size_t bytes) {
                if (e == cudaSuccess) e = cudaMemcpy(dst, src, bytes, cudaMemcpyDefault);
            };
            cp(s->type.p, d->type, sizeof(int) * n);
            cp(s->q.p, d->q, sizeof(float) * n);
            cp(s->specbond.p, d->specbond, sizeof(int) * 12 * n);
            cp(s->num3bond.p, d->num3bond, sizeof(int) * n);
            const int nt2 = s->ntypes * s->ntypes;
            std::vector<float> h1(4 * (size_t)nt2);
            std::vector<float4> tab(nt2);
            cp(h1.data(), d->lj1, sizeof(float) * nt2);
            cp(h1.data() + nt2, d->lj2, sizeof(float) * nt2);
            cp(h1.data() + 2 * nt2, d->lj3, sizeof(float) * nt2);
            cp(h1.data() + 3 * nt2, d->lj4, sizeof(float) * nt2);
            for (int t = 0; t < nt2; ++t)
                tab[t] = make_float4(h1[t], h1[nt2 + t], h1[2 * nt2 + t], h1[3 * nt2 + t]);
            cp(s->ljtab.p, tab.data(), sizeof(float4) * nt2);
            std::vector<int> ht(n);
            cp(ht.data(), d->type, sizeof(int) * n);
            if (e != cudaSuccess) {
                rc = sofia::cuda_fail(ctx, e, "system upload");
            } else {
                for (size_t i = 0; i < n && !rc; ++i)
                    if (ht[i] < 1 || ht[i] > s->ntypes)
                        rc = sofia::fail(ctx, SOFIA_EINVAL, "atom type out of range%s");
            }
            if (d->mass && !rc) {
                // per-atom masses and inverses from the per-type table
                std::vector<double> hm(n), hi(n), mt(s->ntypes);
                cp(mt.data(), d->mass, sizeof(double) * s->ntypes);
                for (size_t i = 0; i < n; ++i) {
                    hm[i] = mt[ht[i] - 1];
                    hi[i] = 1.0 / hm[i];
                }
                cp(s->mass.p, hm.data(), sizeof(double) * n);
                cp(s->invm.p, hi.data(), sizeof(double) * n);
                if (e != cudaSuccess) rc = sofia::cuda_fail(ctx, e, "mass upload");
            }
        }
    }
    if (rc) {
        sofia_system_destroy(ss);
        return rc;
    }
    *out = ss;
    return SOFIA_OK;
}

extern "C" int sofia_system_destroy(sofia_system *ss) {
    if (!ss) return SOFIA_OK;
    Sys *s = &ss->s;
    if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
    sofia::dropin_drop(s);
    for (auto &e : s->ev)
        if (e) cudaEventDestroy(e);
    for (int d = 0; d < 3; ++d) s->xprn[d].release();
    s->ilist.release();
    s->imask.release();
    s->recf.release();
    s->fslot.release();
    s->sref.release();
    s->atom_slot.release();
    s->dcount.release();
    s->icount.release();
    s->part.release();
    sofia::DevBuf *bufs[] = {&s->type, &s->q, &s->invm, &s->mass, &s->specbond, &s->num3bond,
                             &s->ljtab, &s->col_count, &s->col_start, &s->col_fill, &s->col_atoms,
                             &s->col_key, &s->cl_start, &s->slot_orig, &s->rec, &s->bb, &s->jlist,
                             &s->jmask, &s->jcount, &s->nclusters, &s->status_local, &s->energy,
                             &s->red, &s->flag, &s->stage_pos, &s->stage_ff, &s->cl_pos,
                             &s->cl_gid, &s->ptta};
    for (auto *b : bufs) b->release();
    // MD state (md_setup)
    sofia::Md &md = s->md;
    for (auto &g : md.graph)
        if (g) cudaGraphExecDestroy(g);
    sofia::DevBuf *mbufs[] = {&md.bonds, &md.bcoef, &md.angles, &md.acoef, &md.diheds,
                              &md.dcoef, &md.lj14, &md.shake, &md.sbond, &md.impros,
                              &md.icoef, &md.eterm, &md.ered, &md.bpart, &md.step_dev};
    for (auto *b : mbufs) b->release();
    for (auto &b : md.snap) b.release();
    for (auto &b : md.keep) b.release();
    for (int d = 0; d < 3; ++d) {
        s->x[d].release();
        s->v[d].release();
        s->f[d].release();
        s->xref[d].release();
        s->img[d].release();
    }
    delete ss;
    return SOFIA_OK;
}

// Drop-in for lj_cut_coul_dsf_nonewton over the production list: positions in
// the reference's 16-byte AoS (host or device), real*4 forces out.
extern "C" int sofia_force_nonbond_mixed(sofia_system *ss, const sofia_ainfo *position,
                                         float *ff, double *potential, double *e_coul,
                                         double *virial_diag3) {
    if (!ss || !position || !ff) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int n = s->n;
    const size_t pbytes = sizeof(float4) * (size_t)n, fbytes = sizeof(float) * 3 * (size_t)n;
    SOFIA_CUDA(ctx, s->stage_pos.ensure(pbytes));
    SOFIA_CUDA(ctx, s->stage_ff.ensure(fbytes));
    // positions (host or device) into the fixed staging buffer the graph reads
    SOFIA_CUDA(ctx, cudaMemcpyAsync(s->stage_pos.p, position, pbytes, cudaMemcpyDefault, st));
    const bool want_e = potential || e_coul || virial_diag3;
    const bool vir = virial_diag3 != nullptr;
    const bool graph = s->built && !s->timing;
    s->md.forces_valid = 0;  // the MD's step forces are replaced
    if (graph) {
        // steady state: the whole device step is one graph launch, rebuilds and
        // prunes decided on the device
        const int e = vir ? 2 : (want_e ? 1 : 0);
        if (!s->dropin[e]) {
            const int rc = sofia::dropin_capture(s, e);
            if (rc) return rc;
        }
        SOFIA_CUDA(ctx, cudaGraphLaunch(s->dropin[e], st));
        s->launches += s->dropin_launches[e];
    } else {
        // first call after creation or set_state (or with timers on): host-driven
        sofia::launch_pdl(sofia::k_aos_to_soa, sofia::grid_for(n, 256), 256, 0, st,
            n, s->stage_pos.as<float4>(), s->x[0].as<double>(), s->x[1].as<double>(),
            s->x[2].as<double>());
        const int rc = sofia::sys_eval(s, s->precision, want_e, vir, false);
        if (rc) return rc;
        sofia::launch_pdl(sofia::k_fix_to_float, sofia::grid_for(n, 256), 256, 0, st,
            n, s->f[0].as<long long>(), s->f[1].as<long long>(), s->f[2].as<long long>(),
            s->stage_ff.as<float>());
        s->launches += 2;
    }
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ff, s->stage_ff.p, fbytes, cudaMemcpyDefault, st));
    // energies and, after a graph step, the list status words come back with the
    // forces into the context's pinned buffers: one synchronization per call
    double e[5] = {0, 0, 0, 0, 0};
    if (want_e)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_red, s->red.p, sizeof(e), cudaMemcpyDeviceToHost,
                                        st));
    if (graph)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, s->status_local.p,
                                        sizeof(int32_t) * sofia::ST_NSLOTS,
                                        cudaMemcpyDeviceToHost, st));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    if (want_e) memcpy(e, ctx->h_red, sizeof(e));
    if (graph) {
        // a list row that overflowed during a device-side rebuild: grow and redo
        const int rc = sofia::sys_list_overflow(s, ctx->h_status);
        if (rc == SOFIA_ENEEDGROW)
            return sofia_force_nonbond_mixed(ss, position, ff, potential, e_coul, virial_diag3);
        if (rc) return rc;
    }
    if (potential) *potential = e[0];
    if (e_coul) *e_coul = e[1];
    if (virial_diag3) {
        virial_diag3[0] = e[2];
        virial_diag3[1] = e[3];
        virial_diag3[2] = e[4];
    }
    return SOFIA_OK;
}

extern "C" int sofia_system_set_state(sofia_system *ss, const double *x, const double *v) {
    if (!ss || !x) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t n = (size_t)s->n;
    std::vector<double> h(3 * n), c(n);
    const double *src[2] = {x, v};
    sofia::DevBuf *dst[2] = {s->x, s->v};
    for (int k = 0; k < 2; ++k) {
        if (!src[k]) continue;
        SOFIA_CUDA(ctx, cudaMemcpy(h.data(), src[k], sizeof(double) * 3 * n, cudaMemcpyDefault));
        for (int d = 0; d < 3; ++d) {
            for (size_t i = 0; i < n; ++i) c[i] = h[3 * i + d];
            SOFIA_CUDA(ctx, cudaMemcpy(dst[k][d].p, c.data(), sizeof(double) * n,
                                       cudaMemcpyHostToDevice));
        }
    }
    s->built = 0;
    s->md.forces_valid = 0;
    return SOFIA_OK;
}

extern "C" int sofia_system_get_state(sofia_system *ss, double *x, double *v, double *f) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t n = (size_t)s->n;
    std::vector<double> c(n);
    std::vector<long long> cl(n);
    for (int d = 0; d < 3; ++d) {
        if (x) {
            SOFIA_CUDA(ctx, cudaMemcpy(c.data(), s->x[d].p, sizeof(double) * n,
                                       cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) x[3 * i + d] = c[i];
        }
        if (v) {
            SOFIA_CUDA(ctx, cudaMemcpy(c.data(), s->v[d].p, sizeof(double) * n,
                                       cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) v[3 * i + d] = c[i];
        }
        if (f) {
            SOFIA_CUDA(ctx, cudaMemcpy(cl.data(), s->f[d].p, sizeof(long long) * n,
                                       cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) f[3 * i + d] = (double)cl[i] * sofia::FIX_INV;
        }
    }
    return SOFIA_OK;
}

// Forces on the resident positions; energies[5] = potential, e_coul, virial x,y,z.
extern "C" int sofia_system_compute_forces(sofia_system *ss, int precision, int flags,
                                           double *energies) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    // the pair-only forces replace the MD's step forces: the next MD segment
    // recomputes them (with a fresh list decision)
    s->md.forces_valid = 0;
    int rc = sofia::sys_eval(s, precision, energies != nullptr,
                             energies != nullptr && (flags & SOFIA_EVAL_VIRIAL),
                             (flags & SOFIA_EVAL_REBUILD) != 0);
    if (rc) return rc;
    if (energies) {
        SOFIA_CUDA(ctx, cudaMemcpyAsync(energies, s->red.p, sizeof(double) * 5,
                                        cudaMemcpyDeviceToHost, ctx->stream));
    }
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SOFIA_OK;
}

extern "C" int sofia_system_stats(sofia_system *ss, int64_t *stats, int nstats) {
    if (!ss || !stats || nstats <= 0) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int ncl = 0;
    if (s->built)
        SOFIA_CUDA(ctx, cudaMemcpy(&ncl, s->nclusters.p, sizeof(int), cudaMemcpyDeviceToHost));
    ncl = std::min(std::max(ncl, 0), s->max_clusters);
    long long entries = 0, inner = 0;
    if (ncl > 0) {
        std::vector<int> jc(ncl), ic(ncl);
        SOFIA_CUDA(ctx, cudaMemcpy(jc.data(), s->jcount.p, sizeof(int) * ncl,
                                   cudaMemcpyDeviceToHost));
        SOFIA_CUDA(ctx, cudaMemcpy(ic.data(), s->icount.p, sizeof(int) * ncl,
                                   cudaMemcpyDeviceToHost));
        for (int i = 0; i < ncl; ++i) {
            entries += jc[i];
            inner += ic[i];
        }
    }
    long long dc[2] = {0, 0};
    SOFIA_CUDA(ctx, cudaMemcpy(dc, s->dcount.p, sizeof(dc), cudaMemcpyDeviceToHost));
    const int64_t vals[11] = {s->n_builds + dc[0], ncl, entries, s->jcap, s->ncx,
                              s->max_clusters, s->ncol_reach, s->launches, s->n_prunes + dc[1],
                              inner, s->shake_nc};
    for (int i = 0; i < nstats && i < 11; ++i) stats[i] = vals[i];
    return SOFIA_OK;
}

extern "C" int sofia_system_drift(sofia_system *ss, double dt, int nsteps) {
    if (!ss || nsteps < 0) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    for (int k = 0; k < nsteps; ++k) {
        sofia::launch_pdl(sofia::k_drift, sofia::grid_for(s->n, 256), 256, 0, ctx->stream,
            s->n, dt, s->x[0].as<double>(), s->x[1].as<double>(), s->x[2].as<double>(),
            s->v[0].as<double>(), s->v[1].as<double>(), s->v[2].as<double>());
        s->launches += 1;
    }
    SOFIA_CUDA(ctx, cudaGetLastError());
    return SOFIA_OK;
}

// timers[0..3] = list-build ms, builds timed, pair-kernel ms, pair launches timed.
extern "C" int sofia_system_timers(sofia_system *ss, int enable, double *timers) {
    if (!ss) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    if (enable && !s->ev[0])
        for (int k = 0; k < 4; ++k) SOFIA_CUDA(ctx, cudaEventCreate(&s->ev[k]));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (s->timing) sofia::sys_collect_timers(s);
    if (timers) {
        timers[0] = s->t_build_ms;
        timers[1] = (double)s->n_build_timed;
        timers[2] = s->t_pair_ms;
        timers[3] = (double)s->n_pair;
    }
    s->t_build_ms = s->t_pair_ms = 0.0;
    s->n_build_timed = s->n_pair = 0;
    s->timing = enable ? 1 : 0;
    return SOFIA_OK;
}

// The cluster-pair list expanded into atom pairs on the host (a diagnostic
// query, not a hot path): which = 0 the outer list (rc + skin, made at the
// last build), 1 the pruned list (rc + margin, made at the last prune); both
// masks hold pair (i atom ii, j atom jj) at bit 8*ii + jj.
extern "C" int sofia_system_list_pairs(sofia_system *ss, int which, int64_t capacity,
                                       int32_t *pairs, int64_t *npairs, double *xlist) {
    if (!ss || !npairs || (which != 0 && which != 1) || capacity < 0 || (capacity > 0 && !pairs))
        return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *npairs = 0;
    if (!s->built) return sofia::fail(ctx, SOFIA_ESTATE, "list_pairs: no list built yet%s");
    int ncl = 0;
    SOFIA_CUDA(ctx, cudaMemcpy(&ncl, s->nclusters.p, sizeof(int), cudaMemcpyDeviceToHost));
    ncl = std::min(std::max(ncl, 0), s->max_clusters);
    const size_t cap = (size_t)s->jcap;
    std::vector<int> cnt(ncl), lst((size_t)ncl * cap), orig((size_t)ncl * sofia::CL);
    std::vector<unsigned long long> msk((size_t)ncl * cap);
    const sofia::DevBuf &L = which ? s->ilist : s->jlist;
    const sofia::DevBuf &Mk = which ? s->imask : s->jmask;
    const sofia::DevBuf &Cn = which ? s->icount : s->jcount;
    if (ncl > 0) {
        SOFIA_CUDA(ctx, cudaMemcpy(cnt.data(), Cn.p, sizeof(int) * ncl, cudaMemcpyDeviceToHost));
        SOFIA_CUDA(ctx, cudaMemcpy(lst.data(), L.p, sizeof(int) * ncl * cap,
                                   cudaMemcpyDeviceToHost));
        SOFIA_CUDA(ctx, cudaMemcpy(msk.data(), Mk.p, sizeof(unsigned long long) * ncl * cap,
                                   cudaMemcpyDeviceToHost));
        SOFIA_CUDA(ctx, cudaMemcpy(orig.data(), s->slot_orig.p, sizeof(int) * ncl * sofia::CL,
                                   cudaMemcpyDeviceToHost));
    }
    int64_t k = 0;
    for (int ic = 0; ic < ncl; ++ic) {
        const int c = std::min(std::max(cnt[ic], 0), (int)cap);
        for (int e = 0; e < c; ++e) {
            const int w = lst[(size_t)ic * cap + e];
            const int jc = w & ((1 << sofia::IMG_SHIFT) - 1);
            if (jc < 0 || jc >= ncl)
                return sofia::fail(ctx, SOFIA_ESTATE, "list_pairs: j cluster out of range%s");
            unsigned long long m = msk[(size_t)ic * cap + e];
            while (m) {
                const int b = __builtin_ctzll(m);
                m &= m - 1;
                const int ii = b >> 3, jj = b & 7;
                const int a = orig[(size_t)ic * sofia::CL + ii];
                const int o = orig[(size_t)jc * sofia::CL + jj];
                if (a < 0 || o < 0)
                    return sofia::fail(ctx, SOFIA_ESTATE, "list_pairs: a padding slot is listed%s");
                if (k < capacity) {
                    pairs[2 * k] = a;
                    pairs[2 * k + 1] = o;
                }
                ++k;
            }
        }
    }
    *npairs = k;
    if (xlist) {
        const size_t n = (size_t)s->n;
        std::vector<double> h(n);
        const sofia::DevBuf *src = which ? s->xprn : s->xref;
        for (int d = 0; d < 3; ++d) {
            SOFIA_CUDA(ctx, cudaMemcpy(h.data(), src[d].p, sizeof(double) * n,
                                       cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) xlist[3 * i + d] = h[i];
        }
    }
    if (k > capacity) return SOFIA_ENEEDGROW;
    return SOFIA_OK;
}

// ---------------------------------------------------------------------------
// Batched replicas (see BatchDev in system.cuh): the nonbonded part of an MD
// step for every replica of a batch, one launch per kernel.  Each launch walks
// its virtual blocks in a grid-stride loop and runs the single-system kernel
// body on the owning replica's buffers, so a replica's results are bit-identical
// to the same replica stepped alone.
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

__global__ void k_wrap_bin_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_A256, BA_BUILD)
    wrap_bin_body(lb, d.flag, 1, d.n, d.x, d.y, d.z, d.L, d.s_col, d.ncx, d.ix, d.iy, d.iz, d.rx,
                  d.ry, d.rz, d.col_of, d.col_count, d.col_key);
    SOFIA_BATCH_END
}

__global__ void __launch_bounds__(1024) k_scan_cols_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_SCAN, BA_BUILD)
    scan_cols_body(lb, d.flag, 1, d.ncols, d.col_count, d.col_start, d.cl_start, d.ncl);
    __syncthreads();
    SOFIA_BATCH_END
}

__global__ void k_col_scatter_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_A256, BA_BUILD)
    col_scatter_body(lb, d.flag, 1, d.n, d.col_of, d.col_start, d.col_fill, d.col_atoms);
    SOFIA_BATCH_END
}

__global__ void k_col_sort_assign_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_COLS, BA_BUILD)
    col_sort_assign_body(lb, d.flag, 1, d.ncols, d.col_start, d.col_atoms, d.col_key, d.cl_start,
                         d.slot_orig, d.cl_col, d.atom_slot, d.col_fill, d.status);
    __syncthreads();
    SOFIA_BATCH_END
}

__global__ void __launch_bounds__(256, SOFIA_BATCH_STREAM_MINB) k_pack_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_S256)
    pack_body(lb, d.nslots, d.ncl, d.slot_orig, d.x, d.y, d.z, d.rx, d.ry, d.rz, d.ix, d.iy, d.iz,
              d.q, d.type, d.L, d.rec, d.recf, reinterpret_cast<long long *>(d.fslot), d.bb,
              d.flag, d.sref);
    SOFIA_BATCH_END
}


// 4 resident blocks per SM (64 registers, a few spills) instead of the 80
// registers the replica arguments would take (64 replicas: 383.5 -> 389 M
// atom-steps/s)
#ifndef SOFIA_BATCH_SEARCH_MINB
#define SOFIA_BATCH_SEARCH_MINB 4
#endif
__global__ void __launch_bounds__(256, SOFIA_BATCH_SEARCH_MINB) k_search_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_W256, BA_BUILD)
    SearchArgs a;
    a.cond = d.flag;
    a.cmask = 1;
    a.maxcl = d.maxcl;
    a.ncx = d.ncx;
    a.reach = d.reach;
    a.jcap = d.jcap;
    a.n = d.n;
    a.L = (float)d.L;
    a.s_col = (float)d.s_col;
    a.rl = d.rl;
    a.rl2 = d.rl2;
    a.rexcl2 = d.rexcl2;
    a.ncl_dev = d.ncl;
    a.cl_start = d.cl_start;
    a.cl_col = d.cl_col;
    a.slot_orig = d.slot_orig;
    a.specbond = d.specbond;
    a.num3bond = d.num3bond;
    a.atom_slot = d.atom_slot;
    a.bb = d.bb;
    a.jlist = d.jlist;
    a.jcount = d.jcount;
    a.jmask = d.jmask;
    a.status = d.status;
    search_body(lb, a);
    SOFIA_BATCH_END
}

__global__ void __launch_bounds__(256, SOFIA_PRUNE_MINB) k_prune_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_ACTIVE_LOOP(BK_W256, BA_PRUNE)
    prune_body(lb, d.flag, 3, d.maxcl, d.ncl, d.recf, d.jlist, d.jmask, d.jcount, d.jcap,
               (float)d.L, d.rin2, d.rfar2, d.bb, d.ilist, d.imask, d.icount, d.slot_orig, d.x,
               d.y, d.z, d.px, d.py, d.pz);
    __syncthreads();
    SOFIA_BATCH_END
}

template <typename T, bool EN, bool VIR, bool SAME, bool TRI = false>
__global__ void __launch_bounds__(256, (sizeof(T) == 4) ? (EN ? SOFIA_PAIR_MINB_EN : SOFIA_PAIR_MINB) : 2)
    k_pair_b(BatchDev *__restrict__ tab, PairConst k) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_W256)
    pair_body<T, EN, VIR, SAME, TRI>(lb, d.maxcl, d.ncl, d.rec, d.ilist, d.imask, d.icount, d.jcap,
                                d.ljtab, k, d.L, d.fslot, d.energy);
    __syncthreads();
    SOFIA_BATCH_END
}

__global__ void __launch_bounds__(256, SOFIA_BATCH_STREAM_MINB) k_unpack_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_S256)
    unpack_body(lb, d.nslots, d.ncl, d.slot_orig, reinterpret_cast<const long long *>(d.fslot),
                d.fx, d.fy, d.fz, d.ctx_status, d.flag, d.dcount, d.lg, nullptr);
    SOFIA_BATCH_END
}

__global__ void k_red_stage1_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_RED)
    red_stage1_body(lb, d.maxcl, 5, d.ncl, d.energy, d.part, RED_BLOCKS);
    __syncthreads();
    SOFIA_BATCH_END
}

__global__ void k_red_stage2_b(const BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    SOFIA_BATCH_LOOP(BK_REP)
    red_stage2_body(lb, RED_BLOCKS, 5, d.part, d.red, 1.0);
    __syncthreads();
    SOFIA_BATCH_END
}

// One block: the replicas whose trigger word has a bit of mask 1 (rebuild) or 3
// (rebuild or prune) this step, and the prefixes of their virtual blocks per
// kind, so the conditional kernels walk only blocks with work.  Runs after the
// step's first kernel has set the trigger words.  Thread t is replica t; all
// 2 x (1 + BK_N) prefix sums are taken at once (warp shuffles, then the warp
// totals through shared memory).
__global__ void __launch_bounds__(MAXREP) k_batch_active_b(BatchDev *__restrict__ tab) {
    SOFIA_PDL_ENTRY();
    constexpr int NK = BK_N + 1;       // per mask: the active count, then one per kind
    constexpr int NV = BA_N * NK;
    constexpr int NW = MAXREP / 32;
    __shared__ int s_w[NW][NV];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int nrep = tab->nrep;
    const int f = (t < nrep) ? tab->rep[t].flag[0] : 0;
    int cnt[BK_N];
#pragma unroll
    for (int k = 0; k < BK_N; ++k)
        cnt[k] = (t < nrep) ? tab->pre[k][t + 1] - tab->pre[k][t] : 0;
    bool on[BA_N];
    int v[NV];
#pragma unroll
    for (int m = 0; m < BA_N; ++m) {
        on[m] = (f & (m == BA_BUILD ? 1 : 3)) != 0;
        v[m * NK] = on[m] ? 1 : 0;
#pragma unroll
        for (int k = 0; k < BK_N; ++k) v[m * NK + 1 + k] = on[m] ? cnt[k] : 0;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const int x = __shfl_up_sync(FULL, v[i], off);
            if (lane >= off) v[i] += x;
        }
    }
    if (lane == 31) {
#pragma unroll
        for (int i = 0; i < NV; ++i) s_w[w][i] = v[i];
    }
    __syncthreads();
    for (int ww = 0; ww < w; ++ww) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += s_w[ww][i];
    }
    // v[] now holds inclusive prefixes over replicas 0..t
#pragma unroll
    for (int m = 0; m < BA_N; ++m) {
        const int rank = v[m * NK] - (on[m] ? 1 : 0);
        if (on[m]) {
            tab->act[m][rank] = t;
#pragma unroll
            for (int k = 0; k < BK_N; ++k) tab->apre[m][k][rank + 1] = v[m * NK + 1 + k];
        }
        if (t == 0) {
#pragma unroll
            for (int k = 0; k < BK_N; ++k) tab->apre[m][k][0] = 0;
        }
        if (t == MAXREP - 1) tab->nact[m] = v[m * NK];
    }
}

#undef SOFIA_BATCH_LOOP
#undef SOFIA_BATCH_END

}  // namespace

void repdev_fill_pair(const Sys *s, RepDev *d) {
    d->n = s->n;
    d->ncols = s->ncols;
    d->ncx = s->ncx;
    d->maxcl = s->max_clusters;
    d->jcap = s->jcap;
    d->reach = s->ncol_reach;
    d->nslots = s->max_clusters * CL;
    d->L = s->L;
    d->s_col = s->s_col;
    const float rl = (float)s->rlist + 1e-3f;
    d->rl = rl;
    d->rl2 = rl * rl;
    d->rexcl2 = (float)(s->r_excl * s->r_excl);
    const float rin = (float)(s->rc + s->margin);
    d->rin2 = rin * rin + 1e-3f;
    const float rfar = rin + 0.01f;
    d->rfar2 = rfar * rfar;
    d->lim2 = (0.5 * s->skin) * (0.5 * s->skin);
    d->plim2 = (0.5 * s->margin) * (0.5 * s->margin);
    d->x = s->x[0].as<double>();
    d->y = s->x[1].as<double>();
    d->z = s->x[2].as<double>();
    d->vx = s->v[0].as<double>();
    d->vy = s->v[1].as<double>();
    d->vz = s->v[2].as<double>();
    d->fx = s->f[0].as<long long>();
    d->fy = s->f[1].as<long long>();
    d->fz = s->f[2].as<long long>();
    d->rx = s->xref[0].as<double>();
    d->ry = s->xref[1].as<double>();
    d->rz = s->xref[2].as<double>();
    d->ix = s->img[0].as<double>();
    d->iy = s->img[1].as<double>();
    d->iz = s->img[2].as<double>();
    d->px = s->xprn[0].as<double>();
    d->py = s->xprn[1].as<double>();
    d->pz = s->xprn[2].as<double>();
    d->invm = s->invm.as<double>();
    d->mass = s->mass.as<double>();
    d->q = s->q.as<float>();
    d->type = s->type.as<int>();
    d->specbond = s->specbond.as<int>();
    d->num3bond = s->num3bond.as<int>();
    d->col_count = s->col_count.as<int>();
    d->col_start = s->col_start.as<int>();
    d->col_fill = s->col_fill.as<int>();
    d->col_atoms = s->col_atoms.as<int>();
    d->col_of = s->col_atoms.as<int>() + s->n;
    d->cl_start = s->cl_start.as<int>();
    d->slot_orig = s->slot_orig.as<int>();
    d->cl_col = s->slot_orig.as<int>() + (size_t)s->max_clusters * CL;
    d->atom_slot = s->atom_slot.as<int>();
    d->col_key = s->col_key.as<float>();
    d->rec = s->rec.as<AtomRec>();
    d->sref = s->sref.as<double>();
    d->recf = s->recf.as<float>();
    d->bb = s->bb.as<float4>();
    d->jlist = s->jlist.as<int>();
    d->jcount = s->jcount.as<int>();
    d->ilist = s->ilist.as<int>();
    d->icount = s->icount.as<int>();
    d->jmask = s->jmask.as<unsigned long long>();
    d->imask = s->imask.as<unsigned long long>();
    d->fslot = s->fslot.as<unsigned long long>();
    d->ncl = s->nclusters.as<int>();
    d->flag = s->flag.as<int>();
    d->status = s->status_local.as<int>();
    d->ctx_status = s->ctx->d_status;
    d->dcount = s->dcount.as<long long>();
    d->ljtab = s->ljtab.as<float4>();
    d->energy = s->energy.as<double>();
    d->part = s->part.as<double>();
    d->red = s->red.as<double>();
}

cudaError_t batch_pair_smem_optin(int nt) {
    static size_t done = 0;
    const size_t need = pair_smem(nt, false, true);
    if (need <= done || need <= 32768) return cudaSuccess;
    const int v = (int)need;
    cudaError_t e = cudaSuccess;
    auto set = [&](const void *f) {
        const cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
        if (r != cudaSuccess) e = r;
    };
    set((const void *)k_pair_b<double, true, false, true>);
    set((const void *)k_pair_b<double, false, false, true>);
    set((const void *)k_pair_b<float, true, false, true>);
    set((const void *)k_pair_b<float, false, false, true>);
    if (e == cudaSuccess) done = need;
    return e;
}

void batch_pair_path(BatchDev *tab, const Sys *s0, int precision, bool energy,
                     cudaStream_t st, int nsm, int pair_blocks) {
    const int g256 = nsm * 8, g128 = nsm * 16;
    launch_pdl(k_batch_active_b, 1, MAXREP, 0, st, tab);
    launch_pdl(k_wrap_bin_b, g256, 256, 0, st, tab);
    launch_pdl(k_scan_cols_b, nsm * 2, 1024, 0, st, tab);
    launch_pdl(k_col_scatter_b, g256, 256, 0, st, tab);
    launch_pdl(k_col_sort_assign_b, nsm * 4, 256, 0, st, tab);
    launch_pdl(k_pack_b, g256, 256, 0, st, tab);
    // one block per warp-per-cluster virtual block of all members (blocks past the
    // replicas whose trigger fired return at once)
    const int gw = pair_blocks > 0 ? pair_blocks : 1;
    launch_pdl(k_search_b, gw, 256, 0, st, tab);
    launch_pdl(k_prune_b, gw, 256, 0, st, tab);
    const PairConst k = make_pair_const(s0, nullptr);
    const size_t smem = pair_smem(s0->ntypes, false, energy);
    const bool tri = energy && pair_tri(s0->ntypes);
    const size_t smem3 = pair_smem(s0->ntypes, tri, energy);
    if (precision == SOFIA_PREC_FP64) {
        if (energy)
            launch_pdl(k_pair_b<double, true, false, true>, gw, 256, smem, st, tab, k);
        else
            launch_pdl(k_pair_b<double, false, false, true>, gw, 256, smem, st, tab, k);
    } else if (tri) {
        launch_pdl(k_pair_b<float, true, false, true, true>, gw, 256, smem3, st, tab, k);
    } else {
        if (energy)
            launch_pdl(k_pair_b<float, true, false, true>, gw, 256, smem, st, tab, k);
        else
            launch_pdl(k_pair_b<float, false, false, true>, gw, 256, smem, st, tab, k);
    }
    launch_pdl(k_unpack_b, g256, 256, 0, st, tab);
    if (energy) {
        launch_pdl(k_red_stage1_b, g256, 256, 0, st, tab);
        launch_pdl(k_red_stage2_b, nsm * 2, 256, 0, st, tab);
    }
}

}  // namespace sofia

// Cluster shape (the autotuner's geometry knob): the xy column width as a
// multiple of the cube side of 8 atoms.  Reallocates the column and list
// buffers; the next evaluation rebuilds the lists.
extern "C" int sofia_system_set_cluster_shape(sofia_system *ss, double aspect) {
    if (!ss || !(aspect >= 0.5) || !(aspect <= 2.0)) return SOFIA_EINVAL;
    Sys *s = &ss->s;
    sofia_nb_ctx *ctx = s->ctx;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const Sys keep_geom = *s;
    if (!sofia::sys_geometry(s, aspect)) {
        s->ncx = keep_geom.ncx;
        s->s_col = keep_geom.s_col;
        s->ncols = keep_geom.ncols;
        s->ncol_reach = keep_geom.ncol_reach;
        s->max_clusters = keep_geom.max_clusters;
        s->jcap = keep_geom.jcap;
        s->aspect = keep_geom.aspect;
        return sofia::fail(ctx, SOFIA_EINVAL, "box too small for that column grid%s");
    }
    if (s->jcap < keep_geom.jcap) s->jcap = keep_geom.jcap;
    int rc = sofia::sys_alloc(s);
    if (!rc) rc = sofia::sys_alloc_list(s);
    if (rc) return rc;
    sofia::md_invalidate(s);
    return SOFIA_OK;
}
