// ref_kernels.cu -- reference-semantics cell list, full Verlet list and FP64
// LJ + DSF pair kernel, 1-4 pairs and exclusion corrections.
//
// This translation unit is compiled with -fmad=false: every real*4 and real*8
// operation is rounded on its own, in the Fortran evaluation order, so the
// neighbour sets are bit-identical to the reference and the FP64 sums agree to
// the last bits up to summation order.
//
// Layout in HBM: positions as float4 {x,y,z,type-bits} (the reference's 16 B
// ainfo record, loaded with one 128-bit access), cell-sorted copies for the
// candidate sweep, neighbour rows of neigh_alloc int32 per atom (Fortran
// nlist(neigh_alloc*(i-1)+j)).
#include <climits>
#include <mutex>

#include "common.cuh"
#include "improper.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAX_CELL_SORT = 4096;  // atoms per cell handled by the in-cell sort

// xyz2bin, Source/mod_neighbor.f90:1381-1424 (binning in double from real*4).
__device__ __forceinline__ int bin_axis(float x, double boxd, double irn, int D, int *bad) {
    double xd = (double)x;
    int ix = (xd < boxd) ? (int)(xd * irn) : D - 1;
    if (ix == D) ix = D - 1;
    if (ix < 0 || ix >= D) {
        *bad = 1;
        ix = ix < 0 ? 0 : D - 1;
    }
    return ix;
}

__global__ void k_bin_atoms(int np, const float4 *__restrict__ pos, double boxd, double irn,
                            int D, int *__restrict__ cell_of, int *__restrict__ cell_count,
                            int *__restrict__ status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    float4 p = pos[i];
    int bad = 0;
    int ix = bin_axis(p.x, boxd, irn, D, &bad);
    int iy = bin_axis(p.y, boxd, irn, D, &bad);
    int iz = bin_axis(p.z, boxd, irn, D, &bad);
    int c = ix + iy * D + iz * D * D;
    cell_of[i] = c;
    atomicAdd(&cell_count[c], 1);
    if (bad) atomicAdd(&status[sofia::ST_BADBIN], 1);
}

// Exclusive scan of n counts into start[0..n] by one block (cells are few).
__global__ void k_scan_block(int n, const int *__restrict__ in, int *__restrict__ out) {
    __shared__ int s[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        int t = threadIdx.x;
        int v = (base + t < n) ? in[base + t] : 0;
        s[t] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int a = (t >= off) ? s[t - off] : 0;
            __syncthreads();
            s[t] += a;
            __syncthreads();
        }
        if (base + t < n) out[base + t] = carry + s[t] - v;
        __syncthreads();
        if (t == 1023) carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_scatter(int np, const int *__restrict__ cell_of, const int *__restrict__ start,
                          int *__restrict__ fill, int *__restrict__ sorted) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    int c = cell_of[i];
    int slot = atomicAdd(&fill[c], 1);
    sorted[start[c] + slot] = i;
}

// Orders every cell's atoms by input index (ascending, or descending = the
// reference's head-of-chain order, mod_neighbor.f90:933-941 + :956-980).
__global__ void k_sort_cells(int ncell, const int *__restrict__ start, int *__restrict__ sorted,
                             int descending, int *__restrict__ status) {
    __shared__ int s[MAX_CELL_SORT];
    int c = blockIdx.x;
    if (c >= ncell) return;
    int b = start[c], n = start[c + 1] - b;
    if (n <= 1) return;
    if (n > MAX_CELL_SORT) {
        if (threadIdx.x == 0) atomicAdd(&status[sofia::ST_CELLOVER], 1);
        return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        int v = (t < n) ? sorted[b + t] : INT_MAX;
        s[t] = descending ? ((t < n) ? -v : INT_MAX) : v;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < m; t += blockDim.x) {
                int ix = t ^ j;
                if (ix > t) {
                    bool up = ((t & k) == 0);
                    int a = s[t], bb = s[ix];
                    if ((a > bb) == up) {
                        s[t] = bb;
                        s[ix] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) sorted[b + t] = descending ? -s[t] : s[t];
}

__global__ void k_gather_sorted(int np, const int *__restrict__ sorted,
                                const float4 *__restrict__ pos, const int *__restrict__ cell_of,
                                float4 *__restrict__ ps, int *__restrict__ bin_sorted) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    int i = sorted[k];
    ps[k] = pos[i];
    bin_sorted[k] = cell_of[i];
}

// neighcell_nonewton, mod_neighbor.f90:1309-1378.
__global__ void k_stencil(int ncellT, int D, int *__restrict__ cnum) {
    int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if (ic >= ncellT) return;
    int icz = ic / (D * D);
    int icy = (ic - icz * D * D) / D;
    int icx = ic - icy * D - icz * D * D;
    int *out = cnum + 27 * ic;
    out[0] = ic;
    int k = 1;
    for (int iz = -1; iz <= 1; ++iz)
        for (int iy = -1; iy <= 1; ++iy)
            for (int ix = -1; ix <= 1; ++ix) {
                if (iz == 0 && iy == 0 && ix == 0) continue;
                int zc = icz + iz, yc = icy + iy, xc = icx + ix;
                zc = zc < 0 ? zc + D : (zc >= D ? zc - D : zc);
                yc = yc < 0 ? yc + D : (yc >= D ? yc - D : yc);
                xc = xc < 0 ? xc + D : (xc >= D ? xc - D : xc);
                out[k++] = xc + yc * D + zc * D * D;
            }
}

// build_neighbor_nonewton_nomic, mod_neighbor.f90:622-809.  One warp per atom
// (taken in cell order so warps in flight share stencils in L1/L2); lanes
// sweep 32 candidates at a time and ballot-compact the survivors in candidate
// order, so each row is written coalesced and in the reference's order.
__global__ void __launch_bounds__(256) k_build_ref_list(
    int np, const float4 *__restrict__ ps, const int *__restrict__ sorted,
    const int *__restrict__ bin_sorted, const int *__restrict__ start,
    const int *__restrict__ cnum, const int *__restrict__ specbond,
    const int *__restrict__ num3bond, float box, float ibox, double rv2, int *__restrict__ nlist,
    int *__restrict__ numneigh, int neigh_alloc, int *__restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= np) return;
    const int i = sorted[s];
    const float4 pi = ps[s];
    const int bin = bin_sorted[s];
    const int n3 = num3bond[i];
    int bonds[12];
#pragma unroll
    for (int l = 0; l < 12; ++l) bonds[l] = specbond[i * 12 + l];
    int *row = nlist + (size_t)i * (size_t)neigh_alloc;
    int count = 0;
    for (int k = 0; k < 27; ++k) {
        const int c = cnum[bin * 27 + k];
        const int cs = start[c], ce = start[c + 1];
        for (int base = cs; base < ce; base += 32) {
            const int z = base + lane;
            bool keep = false;
            int zi = -1;
            if (z < ce) {
                const float4 pz = ps[z];
                zi = sorted[z];
                float dx = pi.x - pz.x, dy = pi.y - pz.y, dz = pi.z - pz.z;
                // (b + sign(2^23,b)) - sign(2^23,dx) of :694-697 is rint(b) for |b| < 2^22
                const float bx = rintf(dx * ibox), by = rintf(dy * ibox), bz = rintf(dz * ibox);
                dx = dx - bx * box;
                dy = dy - by * box;
                dz = dz - bz * box;
                const float dr2 = dx * dx + dy * dy + dz * dz;
                keep = (zi != i) && ((double)dr2 < rv2);
                if (keep) {
#pragma unroll
                    for (int l = 0; l < 12; ++l)
                        if (l < n3 && bonds[l] == zi + 1) keep = false;
                }
            }
            const unsigned m = __ballot_sync(FULL, keep);
            if (keep) {
                const int at = count + __popc(m & ((1u << lane) - 1u));
                if (at < neigh_alloc) row[at] = zi + 1;
            }
            count += __popc(m);
        }
    }
    if (lane == 0) {
        numneigh[i] = count;
        atomicMax(&status[sofia::ST_MAXCOUNT], count);
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
    return v;
}

struct DsfConst {
    double box, ibox, rcut2, cut_coulsq, alpha, e_shift, f_shift, coulpre;
    float boxf, iboxf, coulpref;  // real*4 copies for the real*4 real-space kernel
    double gewald;
    double EWALD_P, A1, A2, A3, A4, A5, MY_PIS, MY_PIS_INV, EWALD_F;
};

__host__ DsfConst make_const(float box, float ibox, double rcut2, double cut_coulsq, double alpha,
                             double e_shift, double f_shift, float coulpre) {
    DsfConst c;
    c.box = (double)box;
    c.ibox = (double)ibox;
    c.rcut2 = rcut2;
    c.cut_coulsq = cut_coulsq;
    c.alpha = alpha;
    c.e_shift = e_shift;
    c.f_shift = f_shift;
    c.coulpre = (double)coulpre;
    c.boxf = box;
    c.iboxf = ibox;
    c.coulpref = coulpre;
    c.gewald = 0.0;
    c.EWALD_F = (double)1.12837917f;
    c.EWALD_P = (double)0.3275911f;
    c.A1 = (double)0.254829592f;
    c.A2 = (double)-0.284496736f;
    c.A3 = (double)1.421413741f;
    c.A4 = (double)-1.453152027f;
    c.A5 = (double)1.061405429f;
    c.MY_PIS = (double)1.77245385090551602729f;
    c.MY_PIS_INV = 1.0 / c.MY_PIS;
    return c;
}

// lj_cut_coul_dsf_nonewton_NOMIC, mod_force_nonbond.f90:105-196.  One warp per
// atom i; lane l takes neighbours l, l+32, ... of the row (coalesced index
// loads), keeps FP64 partial sums and the warp combines them with a fixed
// butterfly, so results are bit-reproducible run to run.
__global__ void __launch_bounds__(256) k_force_ref(
    int np, const float4 *__restrict__ pos, const float *__restrict__ q,
    const float *__restrict__ lj1, const float *__restrict__ lj2, const float *__restrict__ lj3,
    const float *__restrict__ lj4, int ntypes, const int *__restrict__ nlist,
    const int *__restrict__ numneigh, int neigh_alloc, DsfConst k, float *__restrict__ ff,
    double *__restrict__ pe) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= np) return;
    const float4 pi = pos[i];
    const double x1 = pi.x, y1 = pi.y, z1 = pi.z;
    const int itype = __float_as_int(pi.w);
    const double qtmp = (double)q[i];
    const int ioffset = (itype - 1) * ntypes;
    const int num = min(numneigh[i], neigh_alloc);
    const int *row = nlist + (size_t)i * (size_t)neigh_alloc;
    const bool itype_ok = (unsigned)(itype - 1) < (unsigned)ntypes;
    const double TWO_ALPHA_PI = (2.0 * k.alpha) * k.MY_PIS_INV;
    const double EPA = k.EWALD_P * k.alpha;
    const double AA = k.alpha * k.alpha;
    double ffx = 0.0, ffy = 0.0, ffz = 0.0, pot = 0.0, ec = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
    for (int j = lane; j < num; j += 32) {
        const int neigh = row[j] - 1;
        if ((unsigned)neigh >= (unsigned)np) continue;
        const float4 pj = pos[neigh];
        double dx = x1 - (double)pj.x, dy = y1 - (double)pj.y, dz = z1 - (double)pj.z;
        const int jtype = __float_as_int(pj.w);
        if (!itype_ok || (unsigned)(jtype - 1) >= (unsigned)ntypes) continue;
        // (b + sign(2^52,b)) - sign(2^52,dx) of :144-147 is rint(b) for |b| < 2^51
        const double bx = rint(dx * k.ibox), by = rint(dy * k.ibox), bz = rint(dz * k.ibox);
        dx = dx - k.box * bx;
        dy = dy - k.box * by;
        dz = dz - k.box * bz;
        const double dr2 = dx * dx + dy * dy + dz * dz;
        const double dr2i = 1.0 / dr2;
        double dr6i = dr2i * dr2i * dr2i;
        if (dr2 > k.rcut2) dr6i = 0.0;
        const int off = ioffset + jtype - 1;
        const double forcelj = dr6i * ((double)lj1[off] * dr6i - (double)lj2[off]);
        pot = pot + dr6i * (dr6i * (double)lj3[off] - (double)lj4[off]);
        const double r = sqrt(dr2);
        const double dri = 1.0 / r;
        double prefactor = k.coulpre * qtmp * (double)q[neigh] * dri;
        if (dr2 > k.cut_coulsq) prefactor = 0.0;
        const double erfcd = exp(-((AA * r) * r));
        const double t = 1.0 / (1.0 + EPA * r);
        const double erfcc = t * (k.A1 + t * (k.A2 + t * (k.A3 + t * (k.A4 + t * k.A5)))) * erfcd;
        const double forcecoul =
            prefactor * (erfcc * dri + TWO_ALPHA_PI * erfcd + r * k.f_shift) * r;
        ec = ec + prefactor * ((erfcc - r * k.e_shift) - dr2 * k.f_shift);
        const double force = (forcecoul + forcelj) * dr2i;
        ffx = ffx + dx * force;
        ffy = ffy + dy * force;
        ffz = ffz + dz * force;
        vx = vx + dx * dx * force;
        vy = vy + dy * dy * force;
        vz = vz + dz * dz * force;
    }
    ffx = warp_sum(ffx);
    ffy = warp_sum(ffy);
    ffz = warp_sum(ffz);
    pot = warp_sum(pot);
    ec = warp_sum(ec);
    vx = warp_sum(vx);
    vy = warp_sum(vy);
    vz = warp_sum(vz);
    if (lane == 0) {
        ff[(size_t)i * 3 + 0] = (float)ffx;
        ff[(size_t)i * 3 + 1] = (float)ffy;
        ff[(size_t)i * 3 + 2] = (float)ffz;
        double *o = pe + (size_t)i * 5;
        o[0] = pot;
        o[1] = ec;
        o[2] = vx;
        o[3] = vy;
        o[4] = vz;
    }
}

// lj_cut_coul_long_nonewton_NOMIC / _MIC (mod_force_nonbond.f90:300-400, :201-298):
// the real-space Ewald term of the PME path.  Same warp-per-atom layout as
// k_force_ref, but every pair quantity is real*4 as in the reference; the
// mixed-mode statements are promoted to double where Fortran promotes them
// (dr2i = 1.0d0/dr2, grij = gewald*r, t, the erfc polynomial, forcecoul) and
// force/virial products are added into double sums.  This unit is compiled
// without FMA contraction, so each float operation rounds as written.  The
// real*4 exp is the correctly rounded single-precision value obtained by
// rounding the double-precision exp.
__global__ void __launch_bounds__(256) k_force_long_ref(
    int np, const float4 *__restrict__ pos, const float *__restrict__ q,
    const float *__restrict__ lj1, const float *__restrict__ lj2, const float *__restrict__ lj3,
    const float *__restrict__ lj4, int ntypes, const int *__restrict__ nlist,
    const int *__restrict__ numneigh, int neigh_alloc, DsfConst k, float *__restrict__ ff,
    double *__restrict__ pe) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= np) return;
    const float4 pi = pos[i];
    const int itype = __float_as_int(pi.w);
    const float qtmp = q[i];
    const int ioffset = (itype - 1) * ntypes;
    const int num = min(numneigh[i], neigh_alloc);
    const int *row = nlist + (size_t)i * (size_t)neigh_alloc;
    const bool itype_ok = (unsigned)(itype - 1) < (unsigned)ntypes;
    const float box = k.boxf, ibox = k.iboxf, coulpre = k.coulpref;
    double ffx = 0.0, ffy = 0.0, ffz = 0.0, pot = 0.0, ec = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
    for (int j = lane; j < num; j += 32) {
        const int neigh = row[j] - 1;
        if ((unsigned)neigh >= (unsigned)np) continue;
        const float4 pj = pos[neigh];
        const int jtype = __float_as_int(pj.w);
        if (!itype_ok || (unsigned)(jtype - 1) >= (unsigned)ntypes) continue;
        float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        // (b + sign(2^23,b)) - sign(2^23,dx) is rint(b) in real*4 for |b| < 2^22
        dx = dx - box * rintf(dx * ibox);
        dy = dy - box * rintf(dy * ibox);
        dz = dz - box * rintf(dz * ibox);
        const float dr2 = dx * dx + dy * dy + dz * dz;
        const float dr2i = (float)(1.0 / (double)dr2);
        float dr6i = dr2i * dr2i * dr2i;
        if ((double)dr2 > k.rcut2) dr6i = 0.0f;
        const int off = ioffset + jtype - 1;
        const float forcelj = dr6i * (lj1[off] * dr6i - lj2[off]);
        pot = pot + (double)(dr6i * (dr6i * lj3[off] - lj4[off]));
        const float r = sqrtf(dr2);
        float prefactor = coulpre * qtmp * q[neigh] / r;
        const float grij = (float)(k.gewald * (double)r);
        const float expm2 = (float)exp((double)(-(grij * grij)));
        const double t = (double)(float)(1.0 / (1.0 + k.EWALD_P * (double)grij));
        const float erfc_ =
            (float)(t * (k.A1 + t * (k.A2 + t * (k.A3 + t * (k.A4 + t * k.A5)))) * (double)expm2);
        if ((double)dr2 > k.cut_coulsq) prefactor = 0.0f;
        const float forcecoul =
            (float)((double)prefactor * ((double)erfc_ + k.EWALD_F * (double)grij * (double)expm2));
        ec = ec + (double)(prefactor * erfc_);
        const float force = (forcecoul + forcelj) * dr2i;
        ffx = ffx + (double)(dx * force);
        ffy = ffy + (double)(dy * force);
        ffz = ffz + (double)(dz * force);
        vx = vx + (double)(dx * dx * force);
        vy = vy + (double)(dy * dy * force);
        vz = vz + (double)(dz * dz * force);
    }
    ffx = warp_sum(ffx);
    ffy = warp_sum(ffy);
    ffz = warp_sum(ffz);
    pot = warp_sum(pot);
    ec = warp_sum(ec);
    vx = warp_sum(vx);
    vy = warp_sum(vy);
    vz = warp_sum(vz);
    if (lane == 0) {
        ff[(size_t)i * 3 + 0] = (float)ffx;
        ff[(size_t)i * 3 + 1] = (float)ffy;
        ff[(size_t)i * 3 + 2] = (float)ffz;
        double *o = pe + (size_t)i * 5;
        o[0] = pot;
        o[1] = ec;
        o[2] = vx;
        o[3] = vy;
        o[4] = vz;
    }
}

// Fixed-order reduction of per-item partials pe[n][w] -> out[w]: a fixed grid
// of blocks sums contiguous ranges (coalesced), then one block sums the
// partials, so the result does not depend on scheduling.
constexpr int RED_BLOCKS = 128;
__global__ void k_red1(int n, int w, const double *__restrict__ pe, double *__restrict__ part) {
    __shared__ double s[256];
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
    for (int c = 0; c < w; ++c) {
        double acc = 0.0;
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += pe[(size_t)i * w + c];
        s[threadIdx.x] = acc;
        __syncthreads();
        for (int off = 128; off > 0; off >>= 1) {
            if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[blockIdx.x * w + c] = s[0];
        __syncthreads();
    }
}
__global__ void k_red2(int w, const double *__restrict__ part, double *__restrict__ out,
                       double scale) {
    __shared__ double s[256];
    for (int c = 0; c < w; ++c) {
        s[threadIdx.x] = (threadIdx.x < RED_BLOCKS) ? part[threadIdx.x * w + c] : 0.0;
        __syncthreads();
        for (int off = 128; off > 0; off >>= 1) {
            if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = scale * s[0];
        __syncthreads();
    }
}

// pe[n][w] -> out[w] (out = red_out, partials after it)
inline void reduce_cols(cudaStream_t st, int n, int w, const double *pe, double *out,
                        double scale) {
    double *part = out + 16;
    k_red1<<<RED_BLOCKS, 256, 0, st>>>(n, w, pe, part);
    k_red2<<<1, 256, 0, st>>>(w, part, out, scale);
}

// Minimum image of mod_minimg.f90:5-15: d - box*nint(ibox*d), box*nint() in real*4.
__device__ __forceinline__ double minimg1(double d, float box, float ibox) {
    const double n = round((double)ibox * d);  // NINT: nearest, half away from zero
    const float s = box * (float)(int)n;
    return d - (double)s;
}

// dihedral_opls_DSF, mod_force_dihed.f90:849-1068: torsion + 1-4 pair per dihedral.
__global__ void k_dihedral_dsf(int ndihed, int np, const float4 *__restrict__ pos,
                               const float *__restrict__ q, int ntypes,
                               const double *__restrict__ lj14, const int *__restrict__ dl,
                               const double *__restrict__ dc, int ndtypes, DsfConst k, float box,
                               float ibox, double *__restrict__ acc, double *__restrict__ pe,
                               int *__restrict__ status) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ndihed) return;
    const int i1 = dl[n * 5] - 1, i2 = dl[n * 5 + 1] - 1, i3 = dl[n * 5 + 2] - 1,
              i4 = dl[n * 5 + 3] - 1, type = dl[n * 5 + 4];
    pe[(size_t)n * 3 + 0] = 0.0;
    pe[(size_t)n * 3 + 1] = 0.0;
    pe[(size_t)n * 3 + 2] = 0.0;
    if ((unsigned)i1 >= (unsigned)np || (unsigned)i2 >= (unsigned)np ||
        (unsigned)i3 >= (unsigned)np || (unsigned)i4 >= (unsigned)np ||
        (unsigned)(type - 1) >= (unsigned)ndtypes) {
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        return;
    }
    const float4 p1 = pos[i1], p2 = pos[i2], p3 = pos[i3], p4 = pos[i4];
    const double vb1x = minimg1((double)(p1.x - p2.x), box, ibox);
    const double vb1y = minimg1((double)(p1.y - p2.y), box, ibox);
    const double vb1z = minimg1((double)(p1.z - p2.z), box, ibox);
    const double vb2x = minimg1((double)(p3.x - p2.x), box, ibox);
    const double vb2y = minimg1((double)(p3.y - p2.y), box, ibox);
    const double vb2z = minimg1((double)(p3.z - p2.z), box, ibox);
    const double vb2xm = minimg1(-vb2x, box, ibox);
    const double vb2ym = minimg1(-vb2y, box, ibox);
    const double vb2zm = minimg1(-vb2z, box, ibox);
    const double vb3x = minimg1((double)(p4.x - p3.x), box, ibox);
    const double vb3y = minimg1((double)(p4.y - p3.y), box, ibox);
    const double vb3z = minimg1((double)(p4.z - p3.z), box, ibox);
    const double ddx = minimg1((double)(p1.x - p4.x), box, ibox);
    const double ddy = minimg1((double)(p1.y - p4.y), box, ibox);
    const double ddz = minimg1((double)(p1.z - p4.z), box, ibox);
    const double dr2 = ddx * ddx + ddy * ddy + ddz * ddz;
    const int itype = __float_as_int(p1.w), jtype = __float_as_int(p4.w);
    const double SMALL = (double)0.001f, SMALLER = (double)0.0001f;
    const double sb1 = 1.0 / (vb1x * vb1x + vb1y * vb1y + vb1z * vb1z);
    const double sb2 = 1.0 / (vb2x * vb2x + vb2y * vb2y + vb2z * vb2z);
    const double sb3 = 1.0 / (vb3x * vb3x + vb3y * vb3y + vb3z * vb3z);
    const double rb1 = sqrt(sb1), rb3 = sqrt(sb3);
    const double c0 = (vb1x * vb3x + vb1y * vb3y + vb1z * vb3z) * rb1 * rb3;
    const double b1mag = sqrt(vb1x * vb1x + vb1y * vb1y + vb1z * vb1z);
    const double b2mag = sqrt(vb2x * vb2x + vb2y * vb2y + vb2z * vb2z);
    const double b3mag = sqrt(vb3x * vb3x + vb3y * vb3y + vb3z * vb3z);
    double ctmp = vb1x * vb2x + vb1y * vb2y + vb1z * vb2z;
    const double r12c1 = 1.0 / (b1mag * b2mag);
    const double c1mag = ctmp * r12c1;
    ctmp = vb2xm * vb3x + vb2ym * vb3y + vb2zm * vb3z;
    const double r12c2 = 1.0 / (b2mag * b3mag);
    const double c2mag = ctmp * r12c2;
    double sc1 = sqrt(fmax(1.0 - c1mag * c1mag, 0.0));
    if (sc1 < SMALL) sc1 = SMALL;
    sc1 = 1.0 / sc1;
    double sc2 = sqrt(fmax(1.0 - c2mag * c2mag, 0.0));
    if (sc2 < SMALL) sc2 = SMALL;
    sc2 = 1.0 / sc2;
    const double s1 = sc1 * sc1, s2 = sc2 * sc2;
    double s12 = sc1 * sc2;
    double c = (c0 + c1mag * c2mag) * s12;
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    const double phi = acos(c);
    double si = sin(phi);
    if (fabs(si) < SMALLER) si = SMALLER;
    const double siinv = 1.0 / si;
    const double k1 = dc[(type - 1) * 4], k2 = dc[(type - 1) * 4 + 1], k3 = dc[(type - 1) * 4 + 2],
                 k4 = dc[(type - 1) * 4 + 3];
    const double pp = k1 * (1.0 + c) + k2 * (1.0 - cos(2.0 * phi)) + k3 * (1.0 + cos(3.0 * phi)) +
                      k4 * (1.0 - cos(4.0 * phi));
    const double pd = k1 - 2.0 * k2 * sin(2.0 * phi) * siinv + 3.0 * k3 * sin(3.0 * phi) * siinv -
                      4.0 * k4 * sin(4.0 * phi) * siinv;
    c = c * pd;
    s12 = s12 * pd;
    const double a11 = c * sb1 * s1;
    const double a22 = -sb2 * (2.0 * c0 * s12 - c * (s1 + s2));
    const double a33 = c * sb3 * s2;
    const double a12 = -r12c1 * (c1mag * c * s1 + c2mag * s12);
    const double a13 = -rb1 * rb3 * s12;
    const double a23 = r12c2 * (c2mag * c * s2 + c1mag * s12);
    const double sx2 = a12 * vb1x + a22 * vb2x + a23 * vb3x;
    const double sy2 = a12 * vb1y + a22 * vb2y + a23 * vb3y;
    const double sz2 = a12 * vb1z + a22 * vb2z + a23 * vb3z;
    double f1x = a11 * vb1x + a12 * vb2x + a13 * vb3x;
    double f1y = a11 * vb1y + a12 * vb2y + a13 * vb3y;
    double f1z = a11 * vb1z + a12 * vb2z + a13 * vb3z;
    const double f2x = -sx2 - f1x, f2y = -sy2 - f1y, f2z = -sz2 - f1z;
    double f4x = a13 * vb1x + a23 * vb2x + a33 * vb3x;
    double f4y = a13 * vb1y + a23 * vb2y + a33 * vb3y;
    double f4z = a13 * vb1z + a23 * vb2z + a33 * vb3z;
    const double f3x = sx2 - f4x, f3y = sy2 - f4y, f3z = sz2 - f4z;
    double force = 0.0, ec14 = 0.0, p14 = 0.0;
    if (dr2 < k.cut_coulsq) {
        const double r = sqrt(dr2);
        const double dr2i = 1.0 / dr2;
        const double prefactor = (double)(((float)k.coulpre * q[i1]) * q[i4]) / r;
        const double erfcd = exp(-(((k.alpha * k.alpha) * r) * r));
        const double t = 1.0 / (1.0 + (k.EWALD_P * k.alpha) * r);
        const double erfcc = t * (k.A1 + t * (k.A2 + t * (k.A3 + t * (k.A4 + t * k.A5)))) * erfcd;
        const double forcecoul =
            (0.50 * prefactor) * ((erfcc / r + ((2.0 * k.alpha) / k.MY_PIS) * erfcd) + r * k.f_shift) * r;
        ec14 = (0.50 * prefactor) * ((erfcc - r * k.e_shift) - dr2 * k.f_shift);
        double forcelj = 0.0;
        if (dr2 < k.rcut2 && (unsigned)(itype - 1) < (unsigned)ntypes &&
            (unsigned)(jtype - 1) < (unsigned)ntypes) {
            const double dr6i = dr2i * dr2i * dr2i;
            const size_t o = (size_t)(itype - 1) * ntypes + (size_t)(jtype - 1);
            const size_t tn = (size_t)ntypes * ntypes;
            forcelj = dr6i * (lj14[o] * dr6i - lj14[tn + o]);
            p14 = dr6i * (dr6i * lj14[2 * tn + o] - lj14[3 * tn + o]);
        }
        force = (forcecoul + forcelj) * dr2i;
    }
    f1x += ddx * force;
    f1y += ddy * force;
    f1z += ddz * force;
    f4x -= ddx * force;
    f4y -= ddy * force;
    f4z -= ddz * force;
    atomicAdd(&acc[i1 * 3 + 0], f1x);
    atomicAdd(&acc[i1 * 3 + 1], f1y);
    atomicAdd(&acc[i1 * 3 + 2], f1z);
    atomicAdd(&acc[i2 * 3 + 0], f2x);
    atomicAdd(&acc[i2 * 3 + 1], f2y);
    atomicAdd(&acc[i2 * 3 + 2], f2z);
    atomicAdd(&acc[i3 * 3 + 0], f3x);
    atomicAdd(&acc[i3 * 3 + 1], f3y);
    atomicAdd(&acc[i3 * 3 + 2], f3z);
    atomicAdd(&acc[i4 * 3 + 0], f4x);
    atomicAdd(&acc[i4 * 3 + 1], f4y);
    atomicAdd(&acc[i4 * 3 + 2], f4z);
    pe[(size_t)n * 3 + 0] = pp;
    pe[(size_t)n * 3 + 1] = ec14;
    pe[(size_t)n * 3 + 2] = p14;
}

// correct_1x_bonds, mod_force_correction.f90:23-86 (and :111-178, :204-270).
__global__ void k_correct_pairs(int npairs, int np, const float4 *__restrict__ pos,
                                const float *__restrict__ q, const int *__restrict__ list,
                                int stride, int ca, int cb, DsfConst k, double gewald,
                                double fudge, float coulpre, double *__restrict__ acc,
                                double *__restrict__ pe, int *__restrict__ status) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= npairs) return;
    const int i1 = list[(size_t)m * stride + ca] - 1, i2 = list[(size_t)m * stride + cb] - 1;
    double *o = pe + (size_t)m * 4;
    if ((unsigned)i1 >= (unsigned)np || (unsigned)i2 >= (unsigned)np) {
        o[0] = o[1] = o[2] = o[3] = 0.0;
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        return;
    }
    const float4 a = pos[i1], b = pos[i2];
    double dx = (double)(a.x - b.x), dy = (double)(a.y - b.y), dz = (double)(a.z - b.z);
    const double bx = rint(dx * k.ibox), by = rint(dy * k.ibox), bz = rint(dz * k.ibox);
    dx = dx - k.box * bx;
    dy = dy - k.box * by;
    dz = dz - k.box * bz;
    const double dr2 = dx * dx + dy * dy + dz * dz;
    const double dr2i = 1.0 / dr2;
    const double r = sqrt(dr2);
    double prefactor = (double)((coulpre * q[i1]) * q[i2]) / r;
    const double grij = gewald * r;
    const double expm2 = exp(-(grij * grij));
    const double t = 1.0 / (1.0 + k.EWALD_P * grij);
    const double erfcv = t * (k.A1 + t * (k.A2 + t * (k.A3 + t * (k.A4 + t * k.A5)))) * expm2;
    if (dr2 > k.cut_coulsq) prefactor = 0.0;
    double forcecoul = prefactor * (erfcv + (k.EWALD_F * grij) * expm2);
    forcecoul = forcecoul - (1.0 - fudge) * prefactor;
    double e = prefactor * erfcv;
    e = e - (1.0 - fudge) * prefactor;
    const double force = forcecoul * dr2i;
    atomicAdd(&acc[i1 * 3 + 0], dx * force);
    atomicAdd(&acc[i1 * 3 + 1], dy * force);
    atomicAdd(&acc[i1 * 3 + 2], dz * force);
    atomicAdd(&acc[i2 * 3 + 0], -dx * force);
    atomicAdd(&acc[i2 * 3 + 1], -dy * force);
    atomicAdd(&acc[i2 * 3 + 2], -dz * force);
    o[0] = e;
    o[1] = dx * dx * force;
    o[2] = dy * dy * force;
    o[3] = dz * dz * force;
}

// out[i] = (float)((double)in[i] + acc[i]) for the float force arrays the reference adds into.
__global__ void k_add_to_float(long n, const double *__restrict__ acc, float *__restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (float)((double)out[i] + acc[i]);
}

int check_status(sofia_nb_ctx *ctx) {
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status,
                                    sizeof(int32_t) * sofia::ST_NSLOTS, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SOFIA_OK;
}

// Bin + sort + stencil shared by sofia_cell_sort and sofia_neighbor_build.
int cell_prepare(sofia_nb_ctx *ctx, int np, const float4 *dpos, float box, float cut_coul,
                 float rcut, int descending, int *ncellT_out, int *ncellD_out) {
    float rn;
    int nt, nd;
    sofia::cell_grid(box, cut_coul, rcut, &rn, &nt, &nd);
    if (nt < 1 || nd < 1 || (long)nd * nd * nd != nt)
        return sofia::fail(ctx, SOFIA_EINVAL, "invalid cell grid (ncellD^3 != ncellT)%s");
    SOFIA_CUDA(ctx, ctx->cell_of.ensure(sizeof(int) * (size_t)np));
    SOFIA_CUDA(ctx, ctx->cell_count.ensure(sizeof(int) * (size_t)(nt + 1)));
    SOFIA_CUDA(ctx, ctx->cell_fill.ensure(sizeof(int) * (size_t)(nt + 1)));
    SOFIA_CUDA(ctx, ctx->cell_start.ensure(sizeof(int) * (size_t)(nt + 1)));
    SOFIA_CUDA(ctx, ctx->sorted_idx.ensure(sizeof(int) * (size_t)np * 2));
    SOFIA_CUDA(ctx, ctx->pos_sorted.ensure(sizeof(float4) * (size_t)np));
    SOFIA_CUDA(ctx, ctx->cnum.ensure(sizeof(int) * 27 * (size_t)nt));
    cudaStream_t st = ctx->stream;
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->cell_count.p, 0, sizeof(int) * (size_t)(nt + 1), st));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->cell_fill.p, 0, sizeof(int) * (size_t)(nt + 1), st));
    const double irn = 1.0 / (double)rn;
    k_bin_atoms<<<sofia::grid_for(np, 256), 256, 0, st>>>(np, dpos, (double)box, irn, nd,
                                                          ctx->cell_of.as<int>(),
                                                          ctx->cell_count.as<int>(), ctx->d_status);
    k_scan_block<<<1, 1024, 0, st>>>(nt, ctx->cell_count.as<int>(), ctx->cell_start.as<int>());
    int *sorted = ctx->sorted_idx.as<int>();
    k_scatter<<<sofia::grid_for(np, 256), 256, 0, st>>>(np, ctx->cell_of.as<int>(),
                                                        ctx->cell_start.as<int>(),
                                                        ctx->cell_fill.as<int>(), sorted);
    k_sort_cells<<<nt, 256, 0, st>>>(nt, ctx->cell_start.as<int>(), sorted, descending,
                                     ctx->d_status);
    int *bin_sorted = sorted + np;
    k_gather_sorted<<<sofia::grid_for(np, 256), 256, 0, st>>>(
        np, sorted, dpos, ctx->cell_of.as<int>(), ctx->pos_sorted.as<float4>(), bin_sorted);
    k_stencil<<<sofia::grid_for(nt, 128), 128, 0, st>>>(nt, nd, ctx->cnum.as<int>());
    SOFIA_CUDA(ctx, cudaGetLastError());
    *ncellT_out = nt;
    *ncellD_out = nd;
    return SOFIA_OK;
}

__global__ void k_sort_outputs(int np, int nt, const int *__restrict__ sorted,
                               const int *__restrict__ bin_sorted, const int *__restrict__ start,
                               int *__restrict__ tt, int *__restrict__ ttb, int *__restrict__ st,
                               int *__restrict__ en, int *__restrict__ atombin) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < np) {
        int i = sorted[k];
        if (tt) tt[i] = k + 1;
        if (ttb) ttb[k] = i + 1;
        if (atombin) atombin[k] = bin_sorted[k];
    }
    if (k < nt) {
        if (st) st[k] = start[k] + 1;
        if (en) en[k] = start[k + 1];
    }
}

}  // namespace

extern "C" int sofia_cell_sort(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position, float box,
                               float cut_coul, float rcut, int32_t *tt, int32_t *ttb,
                               int32_t *start, int32_t *endposit, int32_t *atombin,
                               sofia_ainfo *position_sorted) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !(box > 0.0f)) return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    const void *dpos;
    int rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos);
    if (rc) return rc;
    int nt, nd;
    rc = cell_prepare(ctx, np, (const float4 *)dpos, box, cut_coul, rcut, 1, &nt, &nd);
    if (rc) return rc;
    sofia::OutArg o_tt, o_ttb, o_st, o_en, o_ab, o_ps;
    if ((rc = sofia::stage_out(ctx, tt, sizeof(int) * (size_t)np, 1, &o_tt))) return rc;
    if ((rc = sofia::stage_out(ctx, ttb, sizeof(int) * (size_t)np, 2, &o_ttb))) return rc;
    if ((rc = sofia::stage_out(ctx, start, sizeof(int) * (size_t)nt, 3, &o_st))) return rc;
    if ((rc = sofia::stage_out(ctx, endposit, sizeof(int) * (size_t)nt, 4, &o_en))) return rc;
    if ((rc = sofia::stage_out(ctx, atombin, sizeof(int) * (size_t)np, 5, &o_ab))) return rc;
    if ((rc = sofia::stage_out(ctx, position_sorted, sizeof(float4) * (size_t)np, 6, &o_ps)))
        return rc;
    const int *sorted = ctx->sorted_idx.as<int>();
    int n = np > nt ? np : nt;
    k_sort_outputs<<<sofia::grid_for(n, 256), 256, 0, ctx->stream>>>(
        np, nt, sorted, sorted + np, ctx->cell_start.as<int>(), (int *)o_tt.dev, (int *)o_ttb.dev,
        (int *)o_st.dev, (int *)o_en.dev, (int *)o_ab.dev);
    if (o_ps.dev)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(o_ps.dev, ctx->pos_sorted.p, sizeof(float4) * (size_t)np,
                                        cudaMemcpyDeviceToDevice, ctx->stream));
    SOFIA_CUDA(ctx, cudaGetLastError());
    for (auto *o : {&o_tt, &o_ttb, &o_st, &o_en, &o_ab, &o_ps})
        if ((rc = sofia::finish_out(ctx, *o))) return rc;
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_CELLOVER])
        return sofia::fail(ctx, SOFIA_EINVAL, "a cell holds more than 4096 atoms%s");
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "positions outside [0, box]%s");
    return SOFIA_OK;
}

extern "C" int sofia_neighbor_build(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                    const int32_t *specbond, const int32_t *num3bond, float box,
                                    double rv2, float cut_coul, float rcut, int32_t *nlist,
                                    int32_t *numneigh, int32_t neigh_alloc,
                                    int32_t *needed_alloc) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !specbond || !num3bond || neigh_alloc <= 0 || !(box > 0.0f))
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const void *dpos, *dsb, *dn3;
    int rc;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, specbond, sizeof(int) * 12 * (size_t)np, 1, &dsb))) return rc;
    if ((rc = sofia::stage_in(ctx, num3bond, sizeof(int) * (size_t)np, 2, &dn3))) return rc;
    int nt, nd;
    if ((rc = cell_prepare(ctx, np, (const float4 *)dpos, box, cut_coul, rcut, 0, &nt, &nd)))
        return rc;
    // the list lands in the caller's device buffer, or in the resident buffer
    int32_t *dlist;
    int32_t *dnum;
    const size_t list_bytes = sizeof(int) * (size_t)np * (size_t)neigh_alloc;
    if (nlist && sofia::is_device_ptr(nlist)) {
        dlist = nlist;
    } else {
        SOFIA_CUDA(ctx, ctx->res_nlist.ensure(list_bytes));
        dlist = ctx->res_nlist.as<int32_t>();
    }
    if (numneigh && sofia::is_device_ptr(numneigh)) {
        dnum = numneigh;
    } else {
        SOFIA_CUDA(ctx, ctx->res_numneigh.ensure(sizeof(int) * (size_t)np));
        dnum = ctx->res_numneigh.as<int32_t>();
    }
    const int *sorted = ctx->sorted_idx.as<int>();
    const long threads = (long)np * 32;
    k_build_ref_list<<<sofia::grid_for(threads, 256), 256, 0, st>>>(
        np, ctx->pos_sorted.as<float4>(), sorted, sorted + np, ctx->cell_start.as<int>(),
        ctx->cnum.as<int>(), (const int *)dsb, (const int *)dn3, box,
        (float)(1.0 / (double)box), rv2, dlist, dnum, neigh_alloc, ctx->d_status);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_CELLOVER])
        return sofia::fail(ctx, SOFIA_EINVAL, "a cell holds more than 4096 atoms%s");
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "positions outside [0, box]%s");
    const int mx = ctx->h_status[sofia::ST_MAXCOUNT];
    ctx->res_np = np;
    ctx->res_neigh_alloc = neigh_alloc;
    if (mx > neigh_alloc) {
        long grow = (long)(mx * 1.2);
        while (grow % 16) ++grow;
        if (needed_alloc) *needed_alloc = (int32_t)grow;
        ctx->res_np = 0;
        return sofia::fail(ctx, SOFIA_ENEEDGROW, "neighbour row exceeds neigh_alloc%s");
    }
    if (needed_alloc) *needed_alloc = neigh_alloc;
    if (nlist && dlist != nlist)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(nlist, dlist, list_bytes, cudaMemcpyDeviceToHost, st));
    if (numneigh && dnum != numneigh)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(numneigh, dnum, sizeof(int) * (size_t)np,
                                        cudaMemcpyDeviceToHost, st));
    // keep the resident copy coherent when the caller's buffers were device memory
    if (dlist == nlist) {
        SOFIA_CUDA(ctx, ctx->res_nlist.ensure(list_bytes));
        SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->res_nlist.p, dlist, list_bytes,
                                        cudaMemcpyDeviceToDevice, st));
    }
    if (dnum == numneigh) {
        SOFIA_CUDA(ctx, ctx->res_numneigh.ensure(sizeof(int) * (size_t)np));
        SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->res_numneigh.p, dnum, sizeof(int) * (size_t)np,
                                        cudaMemcpyDeviceToDevice, st));
    }
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    return SOFIA_OK;
}

// Shared body of the two reference-semantics force entry points: stage the
// module arrays, run the pair kernel (DSF in FP64 or real-space Ewald in
// real*4), reduce the per-atom partials in fixed order and halve them.
static int force_ref_run(sofia_nb_ctx *ctx, bool long_range, int np,
                         const sofia_ainfo *position, const float *q, const float *lj1,
                         const float *lj2, const float *lj3, const float *lj4, int ntypes,
                         const int32_t *nlist, const int32_t *numneigh, int32_t neigh_alloc,
                         const DsfConst &k, float *ff, double *potential, double *e_coul,
                         double *virial_diag3) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !q || !lj1 || !lj2 || !lj3 || !lj4 || ntypes <= 0 || !ff)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dpos, *dq, *d1, *d2, *d3, *d4, *dl, *dn;
    const size_t tsz = sizeof(float) * (size_t)ntypes * (size_t)ntypes;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, q, sizeof(float) * (size_t)np, 1, &dq))) return rc;
    if ((rc = sofia::stage_in(ctx, lj1, tsz, 2, &d1))) return rc;
    if ((rc = sofia::stage_in(ctx, lj2, tsz, 3, &d2))) return rc;
    if ((rc = sofia::stage_in(ctx, lj3, tsz, 4, &d3))) return rc;
    if ((rc = sofia::stage_in(ctx, lj4, tsz, 5, &d4))) return rc;
    if (nlist) {
        if (!numneigh || neigh_alloc <= 0) return sofia::fail(ctx, SOFIA_EINVAL, "bad list%s");
        if ((rc = sofia::stage_in(ctx, nlist, sizeof(int) * (size_t)np * (size_t)neigh_alloc, 6,
                                  &dl)))
            return rc;
        if ((rc = sofia::stage_in(ctx, numneigh, sizeof(int) * (size_t)np, 7, &dn))) return rc;
    } else {
        if (ctx->res_np != np)
            return sofia::fail(ctx, SOFIA_EINVAL, "no resident neighbour list for this np%s");
        dl = ctx->res_nlist.p;
        dn = ctx->res_numneigh.p;
        neigh_alloc = ctx->res_neigh_alloc;
    }
    sofia::OutArg o_ff;
    if ((rc = sofia::stage_out(ctx, ff, sizeof(float) * 3 * (size_t)np, 8, &o_ff))) return rc;
    SOFIA_CUDA(ctx, ctx->pe_atom.ensure(sizeof(double) * 5 * (size_t)np));
    SOFIA_CUDA(ctx, ctx->red_out.ensure(sizeof(double) * (16 + 8 * RED_BLOCKS)));
    const long threads = (long)np * 32;
    if (long_range)
        k_force_long_ref<<<sofia::grid_for(threads, 256), 256, 0, st>>>(
            np, (const float4 *)dpos, (const float *)dq, (const float *)d1, (const float *)d2,
            (const float *)d3, (const float *)d4, ntypes, (const int *)dl, (const int *)dn,
            neigh_alloc, k, (float *)o_ff.dev, ctx->pe_atom.as<double>());
    else
        k_force_ref<<<sofia::grid_for(threads, 256), 256, 0, st>>>(
            np, (const float4 *)dpos, (const float *)dq, (const float *)d1, (const float *)d2,
            (const float *)d3, (const float *)d4, ntypes, (const int *)dl, (const int *)dn,
            neigh_alloc, k, (float *)o_ff.dev, ctx->pe_atom.as<double>());
    reduce_cols(st, np, 5, ctx->pe_atom.as<double>(), ctx->red_out.as<double>(), 0.5);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o_ff))) return rc;
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_red, ctx->red_out.p, sizeof(double) * 5,
                                    cudaMemcpyDeviceToHost, st));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    if (potential) *potential = ctx->h_red[0];
    if (e_coul) *e_coul = ctx->h_red[1];
    if (virial_diag3) {
        virial_diag3[0] = ctx->h_red[2];
        virial_diag3[1] = ctx->h_red[3];
        virial_diag3[2] = ctx->h_red[4];
    }
    return SOFIA_OK;
}

extern "C" int sofia_force_nonbond_dsf(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                       const float *q, const float *lj1, const float *lj2,
                                       const float *lj3, const float *lj4, int ntypes,
                                       const int32_t *nlist, const int32_t *numneigh,
                                       int32_t neigh_alloc, float box, float ibox, double rcut2,
                                       double cut_coulsq, double alpha, double e_shift,
                                       double f_shift, float coulpre, float *ff,
                                       double *potential, double *e_coul,
                                       double *virial_diag3) {
    const DsfConst k = make_const(box, ibox, rcut2, cut_coulsq, alpha, e_shift, f_shift, coulpre);
    return force_ref_run(ctx, false, np, position, q, lj1, lj2, lj3, lj4, ntypes, nlist,
                         numneigh, neigh_alloc, k, ff, potential, e_coul, virial_diag3);
}

extern "C" int sofia_force_nonbond_long(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                        const float *q, const float *lj1, const float *lj2,
                                        const float *lj3, const float *lj4, int ntypes,
                                        const int32_t *nlist, const int32_t *numneigh,
                                        int32_t neigh_alloc, float box, float ibox, double rcut2,
                                        double cut_coulsq, double gewald, float coulpre,
                                        float *ff, double *potential, double *e_coul,
                                        double *virial_diag3) {
    if (ctx && !(gewald > 0.0)) return sofia::fail(ctx, SOFIA_EINVAL, "gewald must be > 0%s");
    DsfConst k = make_const(box, ibox, rcut2, cut_coulsq, 0.0, 0.0, 0.0, coulpre);
    k.gewald = gewald;
    return force_ref_run(ctx, true, np, position, q, lj1, lj2, lj3, lj4, ntypes, nlist,
                         numneigh, neigh_alloc, k, ff, potential, e_coul, virial_diag3);
}

extern "C" int sofia_pair14_dsf(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                const float *q, int ntypes, const double *lj14, int ndihed,
                                const int32_t *dihedlist, const double *dihedcoeff,
                                int ndihedtypes, float box, float ibox, double rcut2,
                                double cut_coulsq, double alpha, double e_shift, double f_shift,
                                float coulpre, float *ffh, double *e_dihedral, double *e_coul_14,
                                double *pot_14) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !q || !lj14 || ntypes <= 0 || ndihed < 0 ||
        (ndihed > 0 && !dihedlist) || !dihedcoeff || ndihedtypes <= 0 || !ffh)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    if (ndihed == 0) return SOFIA_OK;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dpos, *dq, *dlj, *ddl, *ddc;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, q, sizeof(float) * (size_t)np, 1, &dq))) return rc;
    if ((rc = sofia::stage_in(ctx, lj14, sizeof(double) * 4 * (size_t)ntypes * ntypes, 2, &dlj)))
        return rc;
    if ((rc = sofia::stage_in(ctx, dihedlist, sizeof(int) * 5 * (size_t)ndihed, 3, &ddl))) return rc;
    if ((rc = sofia::stage_in(ctx, dihedcoeff, sizeof(double) * 4 * (size_t)ndihedtypes, 4, &ddc)))
        return rc;
    sofia::OutArg o_ff;
    if ((rc = sofia::stage_out(ctx, ffh, sizeof(float) * 3 * (size_t)np, 5, &o_ff, true))) return rc;
    SOFIA_CUDA(ctx, ctx->acc64.ensure(sizeof(double) * 3 * (size_t)np));
    SOFIA_CUDA(ctx, ctx->pe_atom.ensure(sizeof(double) * 3 * (size_t)ndihed));
    SOFIA_CUDA(ctx, ctx->red_out.ensure(sizeof(double) * (16 + 8 * RED_BLOCKS)));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->acc64.p, 0, sizeof(double) * 3 * (size_t)np, st));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    DsfConst k = make_const(box, ibox, rcut2, cut_coulsq, alpha, e_shift, f_shift, coulpre);
    k_dihedral_dsf<<<sofia::grid_for(ndihed, 128), 128, 0, st>>>(
        ndihed, np, (const float4 *)dpos, (const float *)dq, ntypes, (const double *)dlj,
        (const int *)ddl, (const double *)ddc, ndihedtypes, k, box, ibox,
        ctx->acc64.as<double>(), ctx->pe_atom.as<double>(), ctx->d_status);
    reduce_cols(st, ndihed, 3, ctx->pe_atom.as<double>(), ctx->red_out.as<double>(), 1.0);
    k_add_to_float<<<sofia::grid_for(3L * np, 256), 256, 0, st>>>(3L * np, ctx->acc64.as<double>(),
                                                                  (float *)o_ff.dev);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o_ff))) return rc;
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_red, ctx->red_out.p, sizeof(double) * 3,
                                    cudaMemcpyDeviceToHost, st));
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "dihedral atom index or type out of range%s");
    if (e_dihedral) *e_dihedral += ctx->h_red[0];
    if (e_coul_14) *e_coul_14 += ctx->h_red[1];
    if (pot_14) *pot_14 += ctx->h_red[2];
    return SOFIA_OK;
}

// improper_harmonic_lammps14 (mod_force_dihed.f90:1546-1724), one thread per
// improper: real*4 coordinate differences with the NINT minimum image, FP64
// angle math (sofia::improper_harmonic); forces into FP64 accumulators,
// energy and virial per improper for a fixed-order reduction.
__global__ void k_improper_ref(int nimpro, int np, const float4 *__restrict__ pos,
                               const int *__restrict__ il, const double *__restrict__ ic,
                               int nimprotypes, float box, float ibox, double *__restrict__ acc,
                               double *__restrict__ pe, int *__restrict__ status) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nimpro) return;
    const int i1 = il[5 * m] - 1, i2 = il[5 * m + 1] - 1, i3 = il[5 * m + 2] - 1,
              i4 = il[5 * m + 3] - 1, t = il[5 * m + 4] - 1;
    double *o = pe + (size_t)m * 4;
    if ((unsigned)i1 >= (unsigned)np || (unsigned)i2 >= (unsigned)np ||
        (unsigned)i3 >= (unsigned)np || (unsigned)i4 >= (unsigned)np ||
        (unsigned)t >= (unsigned)nimprotypes) {
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        o[0] = o[1] = o[2] = o[3] = 0.0;
        return;
    }
    const float4 p1 = pos[i1], p2 = pos[i2], p3 = pos[i3], p4 = pos[i4];
    const double v1[3] = {minimg1((double)(p1.x - p2.x), box, ibox),
                          minimg1((double)(p1.y - p2.y), box, ibox),
                          minimg1((double)(p1.z - p2.z), box, ibox)};
    const double v2[3] = {minimg1((double)(p3.x - p2.x), box, ibox),
                          minimg1((double)(p3.y - p2.y), box, ibox),
                          minimg1((double)(p3.z - p2.z), box, ibox)};
    const double v3[3] = {minimg1((double)(p4.x - p3.x), box, ibox),
                          minimg1((double)(p4.y - p3.y), box, ibox),
                          minimg1((double)(p4.z - p3.z), box, ibox)};
    const sofia::ImproperOut r = sofia::improper_harmonic(v1, v2, v3, ic[2 * t], ic[2 * t + 1]);
    for (int d = 0; d < 3; ++d) {
        atomicAdd(&acc[3 * i1 + d], r.f1[d]);
        atomicAdd(&acc[3 * i2 + d], r.f2[d]);
        atomicAdd(&acc[3 * i3 + d], r.f3[d]);
        atomicAdd(&acc[3 * i4 + d], r.f4[d]);
    }
    o[0] = r.e;
    o[1] = r.vir[0];
    o[2] = r.vir[1];
    o[3] = r.vir[2];
}

extern "C" int sofia_improper_harmonic(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                       int nimpro, const int32_t *improlist,
                                       const double *improcoeff, int nimprotypes, float box,
                                       float ibox, float *ff_impro, double *e_improper,
                                       double *virial3) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || nimpro < 0 || (nimpro > 0 && !improlist) || !improcoeff ||
        nimprotypes <= 0 || !ff_impro)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    if (nimpro == 0) return SOFIA_OK;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dpos, *dil, *dic;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, improlist, sizeof(int) * 5 * (size_t)nimpro, 1, &dil))) return rc;
    if ((rc = sofia::stage_in(ctx, improcoeff, sizeof(double) * 2 * (size_t)nimprotypes, 2, &dic)))
        return rc;
    sofia::OutArg o_ff;
    if ((rc = sofia::stage_out(ctx, ff_impro, sizeof(float) * 3 * (size_t)np, 5, &o_ff, true)))
        return rc;
    SOFIA_CUDA(ctx, ctx->acc64.ensure(sizeof(double) * 3 * (size_t)np));
    SOFIA_CUDA(ctx, ctx->pe_atom.ensure(sizeof(double) * 4 * (size_t)nimpro));
    SOFIA_CUDA(ctx, ctx->red_out.ensure(sizeof(double) * (16 + 8 * RED_BLOCKS)));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->acc64.p, 0, sizeof(double) * 3 * (size_t)np, st));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_improper_ref<<<sofia::grid_for(nimpro, 128), 128, 0, st>>>(
        nimpro, np, (const float4 *)dpos, (const int *)dil, (const double *)dic, nimprotypes, box,
        ibox, ctx->acc64.as<double>(), ctx->pe_atom.as<double>(), ctx->d_status);
    reduce_cols(st, nimpro, 4, ctx->pe_atom.as<double>(), ctx->red_out.as<double>(), 1.0);
    k_add_to_float<<<sofia::grid_for(3L * np, 256), 256, 0, st>>>(3L * np, ctx->acc64.as<double>(),
                                                                  (float *)o_ff.dev);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o_ff))) return rc;
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_red, ctx->red_out.p, sizeof(double) * 4,
                                    cudaMemcpyDeviceToHost, st));
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "improper atom index or type out of range%s");
    if (e_improper) *e_improper += ctx->h_red[0];
    if (virial3) {
        virial3[0] += ctx->h_red[1];
        virial3[1] += ctx->h_red[2];
        virial3[2] += ctx->h_red[3];
    }
    return SOFIA_OK;
}

// ---------------------------------------------------------------------------
// The permutations that follow a cell sort (sort_posit_charge,
// sort_specbond_numbond, sort_*list; Source/mod_neighbor.f90:946-1168) and the
// periodic wrap (pbc, Source/mod_pbc.f90:6-39).

// out[new] = in[ttb[new] - 1], rows of `words` 32-bit words.
__global__ void k_sort_gather(int np, int words, const int *__restrict__ ttb,
                              const unsigned *__restrict__ in, unsigned *__restrict__ out,
                              int *__restrict__ status) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)np * words) return;
    const int i = (int)(t / words), w = (int)(t - (long)i * words);
    const int o = ttb[i] - 1;
    if ((unsigned)o >= (unsigned)np) {
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        return;
    }
    out[t] = in[(long)o * words + w];
}

// sort_specbond_numbond: row i moves to tt(i); its first num3bond entries are
// mapped through tt; entries past num3bond are zero.
__global__ void k_sort_specbond(int np, const int *__restrict__ tt, const int *__restrict__ sb,
                                const int *__restrict__ n1, const int *__restrict__ n2,
                                const int *__restrict__ n3, int *__restrict__ sb_out,
                                int *__restrict__ n1_out, int *__restrict__ n2_out,
                                int *__restrict__ n3_out, int *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int dst = tt[i] - 1;
    const int k3 = n3[i];
    if ((unsigned)dst >= (unsigned)np || k3 < 0 || k3 > 12) {
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        return;
    }
    n1_out[dst] = n1[i];
    n2_out[dst] = n2[i];
    n3_out[dst] = k3;
    for (int l = 0; l < 12; ++l) {
        int v = 0;
        if (l < k3) {
            const int old = sb[i * 12 + l] - 1;
            if ((unsigned)old < (unsigned)np) v = tt[old];
            else atomicAdd(&status[sofia::ST_BADBIN], 1);
        }
        sb_out[dst * 12 + l] = v;
    }
}

// sort_bondlist / sort_anglelist / ...: ids in the first ncols columns of each
// row (1-based, 0 = unused) are mapped through tt.
__global__ void k_remap_ids(int nrows, int stride, int ncols, int np, const int *__restrict__ tt,
                            int *__restrict__ list, int *__restrict__ status) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nrows * ncols) return;
    const int r = (int)(t / ncols), c = (int)(t - (long)r * ncols);
    int *v = list + (long)r * stride + c;
    const int id = *v;
    if (id == 0) return;
    if (id < 1 || id > np) {
        atomicAdd(&status[sofia::ST_BADBIN], 1);
        return;
    }
    *v = tt[id - 1];
}

// pbc: while x > box: x -= box; while x <= 0: x += box (real*4), per coordinate.
// Each loop is bounded; a coordinate still outside after PBC_MAX_WRAPS steps
// (a position more than that many boxes away) is flagged instead.
constexpr int PBC_MAX_WRAPS = 64;
__device__ __forceinline__ float pbc1(float x, float box, int *bad) {
    int k = 0;
    while (x > box && k < PBC_MAX_WRAPS) {
        x = x - box;
        ++k;
    }
    while (x <= 0.0f && k < PBC_MAX_WRAPS) {
        x = x + box;
        ++k;
    }
    if (!(x > 0.0f && x <= box)) *bad = 1;
    return x;
}
__global__ void k_pbc(int np, float4 *__restrict__ pos, float box, int *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    float4 p = pos[i];
    int bad = 0;
    p.x = pbc1(p.x, box, &bad);
    p.y = pbc1(p.y, box, &bad);
    p.z = pbc1(p.z, box, &bad);
    pos[i] = p;
    if (bad) atomicAdd(&status[sofia::ST_NONFINITE], 1);
}

extern "C" int sofia_sort_gather(sofia_nb_ctx *ctx, int np, int elem_bytes, const int32_t *ttb,
                                 const void *in, void *out) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !ttb || !in || !out || elem_bytes <= 0 || elem_bytes % 4 || elem_bytes > 256 ||
        in == out)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args (elem_bytes a multiple of 4, at most 256; in != out)%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const size_t bytes = (size_t)np * elem_bytes;
    const void *dt, *din;
    if ((rc = sofia::stage_in(ctx, ttb, sizeof(int) * (size_t)np, 0, &dt))) return rc;
    if ((rc = sofia::stage_in(ctx, in, bytes, 1, &din))) return rc;
    sofia::OutArg o;
    if ((rc = sofia::stage_out(ctx, out, bytes, 5, &o))) return rc;
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    const int words = elem_bytes / 4;
    k_sort_gather<<<sofia::grid_for((long)np * words, 256), 256, 0, st>>>(
        np, words, (const int *)dt, (const unsigned *)din, (unsigned *)o.dev, ctx->d_status);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o))) return rc;
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "ttb is not a permutation of 1..np%s");
    return SOFIA_OK;
}

extern "C" int sofia_sort_specbond(sofia_nb_ctx *ctx, int np, const int32_t *tt, int32_t *specbond,
                                   int32_t *num1bond, int32_t *num2bond, int32_t *num3bond) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !tt || !specbond || !num1bond || !num2bond || !num3bond)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dt;
    if ((rc = sofia::stage_in(ctx, tt, sizeof(int) * (size_t)np, 0, &dt))) return rc;
    sofia::OutArg osb, o1, o2, o3;
    if ((rc = sofia::stage_out(ctx, specbond, sizeof(int) * 12 * (size_t)np, 5, &osb, true))) return rc;
    if ((rc = sofia::stage_out(ctx, num1bond, sizeof(int) * (size_t)np, 6, &o1, true))) return rc;
    if ((rc = sofia::stage_out(ctx, num2bond, sizeof(int) * (size_t)np, 7, &o2, true))) return rc;
    if ((rc = sofia::stage_out(ctx, num3bond, sizeof(int) * (size_t)np, 8, &o3, true))) return rc;
    // sorted copies are built in scratch, then copied over the inputs
    SOFIA_CUDA(ctx, ctx->acc64.ensure(sizeof(int) * 15 * (size_t)np));
    int *scr = ctx->acc64.as<int>();
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_sort_specbond<<<sofia::grid_for(np, 256), 256, 0, st>>>(
        np, (const int *)dt, (const int *)osb.dev, (const int *)o1.dev, (const int *)o2.dev,
        (const int *)o3.dev, scr, scr + 12 * (size_t)np, scr + 13 * (size_t)np,
        scr + 14 * (size_t)np, ctx->d_status);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "tt is not a permutation or specbond holds an id outside 1..np%s");
    SOFIA_CUDA(ctx, cudaMemcpyAsync(osb.dev, scr, sizeof(int) * 12 * (size_t)np, cudaMemcpyDeviceToDevice, st));
    SOFIA_CUDA(ctx, cudaMemcpyAsync(o1.dev, scr + 12 * (size_t)np, sizeof(int) * (size_t)np, cudaMemcpyDeviceToDevice, st));
    SOFIA_CUDA(ctx, cudaMemcpyAsync(o2.dev, scr + 13 * (size_t)np, sizeof(int) * (size_t)np, cudaMemcpyDeviceToDevice, st));
    SOFIA_CUDA(ctx, cudaMemcpyAsync(o3.dev, scr + 14 * (size_t)np, sizeof(int) * (size_t)np, cudaMemcpyDeviceToDevice, st));
    if ((rc = sofia::finish_out(ctx, osb))) return rc;
    if ((rc = sofia::finish_out(ctx, o1))) return rc;
    if ((rc = sofia::finish_out(ctx, o2))) return rc;
    if ((rc = sofia::finish_out(ctx, o3))) return rc;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    return SOFIA_OK;
}

extern "C" int sofia_remap_ids(sofia_nb_ctx *ctx, int np, const int32_t *tt, int nrows, int stride,
                               int ncols, int32_t *list) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !tt || nrows < 0 || (nrows > 0 && !list) || stride <= 0 || ncols < 0 ||
        ncols > stride)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    if (nrows == 0 || ncols == 0) return SOFIA_OK;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dt;
    if ((rc = sofia::stage_in(ctx, tt, sizeof(int) * (size_t)np, 0, &dt))) return rc;
    sofia::OutArg o;
    if ((rc = sofia::stage_out(ctx, list, sizeof(int) * (size_t)nrows * stride, 5, &o, true)))
        return rc;
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_remap_ids<<<sofia::grid_for((long)nrows * ncols, 256), 256, 0, st>>>(
        nrows, stride, ncols, np, (const int *)dt, (int *)o.dev, ctx->d_status);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o))) return rc;
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "list holds an id outside 1..np%s");
    return SOFIA_OK;
}

extern "C" int sofia_pbc(sofia_nb_ctx *ctx, int np, sofia_ainfo *position, float box) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !(box > 0.0f)) return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    sofia::OutArg o;
    if ((rc = sofia::stage_out(ctx, position, sizeof(float4) * (size_t)np, 5, &o, true))) return rc;
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_pbc<<<sofia::grid_for(np, 256), 256, 0, st>>>(np, (float4 *)o.dev, box, ctx->d_status);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o))) return rc;
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_NONFINITE])
        return sofia::fail(ctx, SOFIA_ESTATE, "a coordinate is non-finite or more than 64 boxes outside%s");
    return SOFIA_OK;
}

extern "C" int sofia_correct_1x(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                const float *q, int npairs, const int32_t *list, int stride,
                                int col_a, int col_b, float box, float ibox, double cut_coulsq,
                                double gewald, double fudge, float coulpre, float *ffc,
                                double *e_corr, double *virial3) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !q || npairs < 0 || (npairs > 0 && !list) || stride <= 0 ||
        col_a < 0 || col_b < 0 || col_a >= stride || col_b >= stride || !ffc)
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    if (npairs == 0) return SOFIA_OK;
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dpos, *dq, *dlist;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, q, sizeof(float) * (size_t)np, 1, &dq))) return rc;
    if ((rc = sofia::stage_in(ctx, list, sizeof(int) * (size_t)stride * npairs, 2, &dlist)))
        return rc;
    sofia::OutArg o_ff;
    if ((rc = sofia::stage_out(ctx, ffc, sizeof(float) * 3 * (size_t)np, 3, &o_ff, true))) return rc;
    SOFIA_CUDA(ctx, ctx->acc64.ensure(sizeof(double) * 3 * (size_t)np));
    SOFIA_CUDA(ctx, ctx->pe_atom.ensure(sizeof(double) * 4 * (size_t)npairs));
    SOFIA_CUDA(ctx, ctx->red_out.ensure(sizeof(double) * (16 + 8 * RED_BLOCKS)));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->acc64.p, 0, sizeof(double) * 3 * (size_t)np, st));
    DsfConst k = make_const(box, ibox, 0.0, cut_coulsq, 0.0, 0.0, 0.0, coulpre);
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_correct_pairs<<<sofia::grid_for(npairs, 128), 128, 0, st>>>(
        npairs, np, (const float4 *)dpos, (const float *)dq, (const int *)dlist, stride, col_a,
        col_b, k, gewald, fudge, coulpre, ctx->acc64.as<double>(), ctx->pe_atom.as<double>(),
        ctx->d_status);
    reduce_cols(st, npairs, 4, ctx->pe_atom.as<double>(), ctx->red_out.as<double>(), 1.0);
    k_add_to_float<<<sofia::grid_for(3L * np, 256), 256, 0, st>>>(3L * np, ctx->acc64.as<double>(),
                                                                  (float *)o_ff.dev);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o_ff))) return rc;
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_red, ctx->red_out.p, sizeof(double) * 4,
                                    cudaMemcpyDeviceToHost, st));
    if ((rc = check_status(ctx))) return rc;
    if (ctx->h_status[sofia::ST_BADBIN])
        return sofia::fail(ctx, SOFIA_EINVAL, "pair atom index out of range%s");
    if (e_corr) *e_corr += ctx->h_red[0];
    if (virial3) {
        virial3[0] += ctx->h_red[1];
        virial3[1] += ctx->h_red[2];
        virial3[2] += ctx->h_red[3];
    }
    return SOFIA_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of sofia_force_nonbond_dsf.
//
// Some callers cannot allocate device memory at the time they need forces:
// hosts that hand the library a fixed device arena or run under a memory budget
// enforced outside the library, and Fortran drivers that keep every device
// array in their own module and never expect a library to allocate behind
// their back.  For them this entry point takes only caller-owned
// device buffers and keeps its per-atom energy partials in a fixed array that
// lives in the library image.
//
// The scratch array below is defined at file scope in device memory, so every
// GPU that loads this library holds it until the process exits.  Its host-side
// name is only a stand-in for the device symbol: host code must never pass it
// to a kernel; the device address is looked up once per device with
// cudaGetSymbolAddress and cached.
namespace {

constexpr size_t NOALLOC_DOUBLES = (size_t)SOFIA_NOALLOC_MAX_ATOMS * 5 + 16 + 8 * RED_BLOCKS;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (looked up once).
int noalloc_scratch(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return SOFIA_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return SOFIA_ECUDA;
        }
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
    return SOFIA_OK;
}

// Device memory on the current device (the one the scratch address and the
// launches belong to), or managed memory.  A buffer on another GPU would be
// read without peer access: rejected here instead of faulting in the kernel.
bool noalloc_buffer_ok(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    int dev = -1;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int sofia_force_nonbond_dsf_noalloc(
    void *stream, int np, const sofia_ainfo *position, const float *q, const float *lj1,
    const float *lj2, const float *lj3, const float *lj4, int ntypes, const int32_t *nlist,
    const int32_t *numneigh, int32_t neigh_alloc, float box, float ibox, double rcut2,
    double cut_coulsq, double alpha, double e_shift, double f_shift, float coulpre, float *ff,
    double *potential, double *e_coul, double *virial_diag3) {
    if (np <= 0 || ntypes <= 0 || neigh_alloc <= 0 || !position || !q || !lj1 || !lj2 || !lj3 ||
        !lj4 || !nlist || !numneigh || !ff)
        return SOFIA_EINVAL;
    if (np > SOFIA_NOALLOC_MAX_ATOMS) return SOFIA_ETOOBIG;
    // every array must already be in the current device's memory: staging would
    // need an allocation
    const void *ptrs[] = {position, q, lj1, lj2, lj3, lj4, nlist, numneigh, ff};
    for (const void *p : ptrs)
        if (!noalloc_buffer_ok(p)) return SOFIA_EINVAL;
    double *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double *pe = scratch;
    double *out = scratch + (size_t)SOFIA_NOALLOC_MAX_ATOMS * 5;
    // every scratch element this call reads is first written by this call
    // (k_force_ref fills pe[0..5*np), the reduction fills its partials and out),
    // so nothing needs clearing between calls
    DsfConst k = make_const(box, ibox, rcut2, cut_coulsq, alpha, e_shift, f_shift, coulpre);
    const long threads = (long)np * 32;
    k_force_ref<<<sofia::grid_for(threads, 256), 256, 0, st>>>(
        np, (const float4 *)position, q, lj1, lj2, lj3, lj4, ntypes, nlist, numneigh, neigh_alloc,
        k, ff, pe);
    reduce_cols(st, np, 5, pe, out, 0.5);
    double h[5];
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SOFIA_ECUDA;
    }
    if (potential) *potential = h[0];
    if (e_coul) *e_coul = h[1];
    if (virial_diag3) {
        virial_diag3[0] = h[2];
        virial_diag3[1] = h[3];
        virial_diag3[2] = h[4];
    }
    return SOFIA_OK;
}

// check_neighbor (Source/mod_neighbor.f90:895-913): rebuild flag when any atom's
// accumulated real*4 displacement satisfies drx^2+dry^2+drz^2 >= rvrc2.
namespace {
__global__ void k_check_neighbor(int np, const float *__restrict__ drx,
                                 const float *__restrict__ dry, const float *__restrict__ drz,
                                 double rvrc2, int *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool far = false;
    if (i < np) {
        const float d2 = drx[i] * drx[i] + dry[i] * dry[i] + drz[i] * drz[i];
        far = (double)d2 >= rvrc2;
    }
    if (__any_sync(FULL, far) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
}  // namespace

extern "C" int sofia_check_neighbor(sofia_nb_ctx *ctx, int np, const float *drx,
                                    const float *dry, const float *drz, double rvrc2,
                                    int32_t *nflag) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !drx || !dry || !drz || !nflag) return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dx, *dy, *dz;
    if ((rc = sofia::stage_in(ctx, drx, sizeof(float) * (size_t)np, 0, &dx))) return rc;
    if ((rc = sofia::stage_in(ctx, dry, sizeof(float) * (size_t)np, 1, &dy))) return rc;
    if ((rc = sofia::stage_in(ctx, drz, sizeof(float) * (size_t)np, 2, &dz))) return rc;
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    k_check_neighbor<<<sofia::grid_for(np, 256), 256, 0, st>>>(np, (const float *)dx, (const float *)dy,
                                                               (const float *)dz, rvrc2,
                                                               ctx->d_status + sofia::ST_REBUILD);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = check_status(ctx))) return rc;
    *nflag = ctx->h_status[sofia::ST_REBUILD] ? 1 : 0;
    return SOFIA_OK;
}
