// cluster.cu -- largest solid-glycine cluster (get_greatestCluster) on the GPU.
//
// The reference (Source/mod_cluster.f90:15-83) builds per-molecule centres,
// a centre cell list, a density list within denscut, a recursive flood fill
// over "solid" molecules (denstrack >= densmin), a histogram, the largest
// cluster by strict '>' in discovery order, and appends adjacent non-solid
// molecules.  The partition into clusters is independent of the visiting
// order, so the flood fill is replaced by a min-label propagation whose labels
// are the smallest molecule index of each component; ranking the roots in
// ascending order gives exactly the reference's discovery numbering.  The
// integer result is therefore bit-identical.
//
// Compiled with -fmad=false like the other reference-semantics kernels.
#include "common.cuh"

namespace {

constexpr int DCAP = 256;  // density-list entries per molecule

// build_ptta_wrap_cluster2, Source/mod_build_ptta.f90:116-132: the atom whose
// global id equals n_gly*apg is never refreshed (`id.lt.flag`).
__global__ void k_ptta_refresh(int np, const float4 *__restrict__ pos,
                               const int *__restrict__ gid, int flag,
                               double *__restrict__ ptta) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    int id = gid[i];
    if (id >= 1 && id < flag) {
        float4 p = pos[i];
        ptta[(size_t)(id - 1) * 3 + 0] = (double)p.x;
        ptta[(size_t)(id - 1) * 3 + 1] = (double)p.y;
        ptta[(size_t)(id - 1) * 3 + 2] = (double)p.z;
    }
}

__device__ __forceinline__ double shift_real4(double d, float box, float ibox) {
    // box*nint(d*ibox) with the product in real*4 (mod_build_ptta.f90:158-160,
    // mod_neighbor_cluster.f90:104-106)
    int n = (int)round(d * (double)ibox);
    return (double)(box * (float)n);
}

struct ClusterArgs {
    int n_gly, apg, densmin, mncellD, mncellT;
    float box, ibox;
    double mrcut2, denscut2, imrn;
    double *ptta;
    double *com;
    int *mcell, *cell_count, *cell_start, *cell_fill, *cell_list;
    int *denstrack, *densvl, *label, *rank, *csize, *surf;
    int *status;
    int *result;  // [0] size, [1] greatest_belongsto (in/out)
};

// One block does the molecule-level work; the molecule counts of the
// workloads here are a few thousand.
__global__ void __launch_bounds__(1024) k_cluster(ClusterArgs a) {
    const int t = threadIdx.x, nt = blockDim.x;
    const int n = a.n_gly;
    const double boxd = (double)a.box;
    // unwrap about the first atom + unweighted centre + wrap to [0, box]
    // (mod_build_ptta.f90:135-163, mod_cluster.f90:803-884)
    for (int m = t; m < n; m += nt) {
        double *base = a.ptta + (size_t)m * a.apg * 3;
        const double x1 = base[0], y1 = base[1], z1 = base[2];
        double xc = x1, yc = y1, zc = z1;
        for (int j = 1; j < a.apg; ++j) {
            double *pj = base + (size_t)j * 3;
            const double x2 = pj[0], y2 = pj[1], z2 = pj[2];
            pj[0] = x2 - shift_real4(x2 - x1, a.box, a.ibox);
            pj[1] = y2 - shift_real4(y2 - y1, a.box, a.ibox);
            pj[2] = z2 - shift_real4(z2 - z1, a.box, a.ibox);
        }
        xc = 0.0;
        yc = 0.0;
        zc = 0.0;
        for (int j = 0; j < a.apg; ++j) {
            xc += base[(size_t)j * 3 + 0];
            yc += base[(size_t)j * 3 + 1];
            zc += base[(size_t)j * 3 + 2];
        }
        const double na = (double)(float)a.apg;
        double c[3] = {xc / na, yc / na, zc / na};
        for (int d = 0; d < 3; ++d) {
            int guard = 0;
            while (c[d] > boxd && guard++ < 64) c[d] = c[d] - boxd;
            while (c[d] < 0.0 && guard++ < 128) c[d] = c[d] + boxd;
            a.com[(size_t)m * 3 + d] = c[d];
        }
        // mol_xyz2bin, mod_neighbor_cluster.f90:668-709
        const int D = a.mncellD;
        int ix = (c[0] < boxd) ? (int)(c[0] * a.imrn) : D - 1;
        int iy = (c[1] < boxd) ? (int)(c[1] * a.imrn) : D - 1;
        int iz = (c[2] < boxd) ? (int)(c[2] * a.imrn) : D - 1;
        if (ix >= D) ix = D - 1;
        if (iy >= D) iy = D - 1;
        if (iz >= D) iz = D - 1;
        if (ix < 0) ix = 0;
        if (iy < 0) iy = 0;
        if (iz < 0) iz = 0;
        a.mcell[m] = ix + iy * D + iz * D * D;
    }
    for (int c = t; c <= a.mncellT; c += nt) {
        a.cell_count[c] = 0;
        a.cell_fill[c] = 0;
    }
    __syncthreads();
    for (int m = t; m < n; m += nt) atomicAdd(&a.cell_count[a.mcell[m]], 1);
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int c = 0; c < a.mncellT; ++c) {
            a.cell_start[c] = acc;
            acc += a.cell_count[c];
        }
        a.cell_start[a.mncellT] = acc;
    }
    __syncthreads();
    for (int m = t; m < n; m += nt) {
        int c = a.mcell[m];
        int s = atomicAdd(&a.cell_fill[c], 1);
        a.cell_list[a.cell_start[c] + s] = m;
    }
    __syncthreads();
    // mol_build_neighbor_nosort (mod_neighbor_cluster.f90:57-176): 26 stencil
    // cells (mol_neigh order, :578-650) with minimum image, then the own cell
    // without it.  Counts include repeated cells when mncellD < 3, as there.
    for (int p1 = t; p1 < n; p1 += nt) {
        const double x1 = a.com[(size_t)p1 * 3], y1 = a.com[(size_t)p1 * 3 + 1],
                     z1 = a.com[(size_t)p1 * 3 + 2];
        const int D = a.mncellD;
        const int cell = a.mcell[p1];
        const int icz = cell / (D * D);
        const int icy = (cell - icz * D * D) / D;
        const int icx = cell - icy * D - icz * D * D;
        int cnt = 0;
        int *dv = a.densvl + (size_t)p1 * DCAP;
        for (int iz = -1; iz <= 1; ++iz)
            for (int iy = -1; iy <= 1; ++iy)
                for (int ix = -1; ix <= 1; ++ix) {
                    if (iz == 0 && iy == 0 && ix == 0) continue;
                    int zc = icz + iz, yc = icy + iy, xc = icx + ix;
                    zc = zc < 0 ? zc + D : (zc >= D ? zc - D : zc);
                    yc = yc < 0 ? yc + D : (yc >= D ? yc - D : yc);
                    xc = xc < 0 ? xc + D : (xc >= D ? xc - D : xc);
                    const int cn = xc + yc * D + zc * D * D;
                    for (int k = a.cell_start[cn]; k < a.cell_start[cn + 1]; ++k) {
                        const int p2 = a.cell_list[k];
                        double dx = x1 - a.com[(size_t)p2 * 3];
                        double dy = y1 - a.com[(size_t)p2 * 3 + 1];
                        double dz = z1 - a.com[(size_t)p2 * 3 + 2];
                        dx = dx + (-shift_real4(dx, a.box, a.ibox));
                        dy = dy + (-shift_real4(dy, a.box, a.ibox));
                        dz = dz + (-shift_real4(dz, a.box, a.ibox));
                        const double dr2 = dx * dx + dy * dy + dz * dz;
                        if (dr2 < a.mrcut2 && dr2 < a.denscut2) {
                            if (cnt < DCAP) dv[cnt] = p2;
                            cnt++;
                        }
                    }
                }
        for (int k = a.cell_start[cell]; k < a.cell_start[cell + 1]; ++k) {
            const int p2 = a.cell_list[k];
            if (p2 == p1) continue;
            const double dx = x1 - a.com[(size_t)p2 * 3];
            const double dy = y1 - a.com[(size_t)p2 * 3 + 1];
            const double dz = z1 - a.com[(size_t)p2 * 3 + 2];
            const double dr2 = dx * dx + dy * dy + dz * dz;
            if (dr2 < a.mrcut2 && dr2 < a.denscut2) {
                if (cnt < DCAP) dv[cnt] = p2;
                cnt++;
            }
        }
        if (cnt > DCAP) atomicAdd(&a.status[sofia::ST_DENSOVER], 1);
        a.denstrack[p1] = cnt;
        a.label[p1] = p1;
    }
    __syncthreads();
    // connected components of solids: min-label propagation + pointer jumping
    __shared__ int changed;
    for (int iter = 0; iter <= n + 1; ++iter) {
        if (t == 0) changed = 0;
        __syncthreads();
        for (int u = t; u < n; u += nt) {
            if (a.denstrack[u] < a.densmin) continue;
            int lu = a.label[u];
            const int cnt = min(a.denstrack[u], DCAP);
            const int *dv = a.densvl + (size_t)u * DCAP;
            for (int l = 0; l < cnt; ++l) {
                const int v = dv[l];
                if (a.denstrack[v] < a.densmin) continue;
                const int lv = a.label[v];
                if (lv < lu) lu = lv;
            }
            if (lu < a.label[u]) {
                atomicMin(&a.label[u], lu);
                changed = 1;
            }
        }
        __syncthreads();
        for (int u = t; u < n; u += nt) {
            int l = a.label[u];
            int ll = a.label[l];
            if (ll < l) {
                atomicMin(&a.label[u], ll);
                changed = 1;
            }
        }
        __syncthreads();
        if (!changed) break;
        __syncthreads();
    }
    // rank roots in ascending index = buildClusters discovery numbering (:228-246)
    if (t == 0) {
        int r = 0;
        for (int u = 0; u < n; ++u) {
            const bool solid = a.denstrack[u] >= a.densmin;
            a.rank[u] = (solid && a.label[u] == u) ? ++r : 0;
            a.csize[u] = 0;
        }
        a.csize[n] = r;  // number of clusters
    }
    __syncthreads();
    for (int u = t; u < n; u += nt) {
        const bool solid = a.denstrack[u] >= a.densmin;
        const int b = solid ? a.rank[a.label[u]] : 0;
        a.rank[u] = a.rank[u];  // root ranks stay
        a.label[u] = b;         // label now holds belongsto
        a.surf[u] = 0;
    }
    __syncthreads();
    for (int u = t; u < n; u += nt)
        if (a.label[u] > 0) atomicAdd(&a.csize[a.label[u] - 1], 1);
    __syncthreads();
    __shared__ int s_cluster, s_greatest;
    if (t == 0) {
        const int nclus = a.csize[n];
        int greatest = 0;
        int gb = a.result[1];
        for (int c = 1; c <= nclus; ++c)
            if (a.csize[c - 1] > greatest) {
                greatest = a.csize[c - 1];
                gb = c;
            }
        s_greatest = greatest;
        s_cluster = gb;
        a.result[1] = gb;
    }
    __syncthreads();
    // append_surface_molecules (mod_cluster.f90:163-194)
    const int cluster = s_cluster;
    for (int u = t; u < n; u += nt) {
        if (a.label[u] != cluster) continue;
        const int cnt = min(a.denstrack[u], DCAP);
        const int *dv = a.densvl + (size_t)u * DCAP;
        for (int l = 0; l < cnt; ++l) {
            const int v = dv[l];
            if (a.denstrack[v] < a.densmin) a.surf[v] = 1;
        }
    }
    __syncthreads();
    __shared__ int s_surface;
    if (t == 0) s_surface = 0;
    __syncthreads();
    int mine = 0;
    for (int u = t; u < n; u += nt)
        if (a.surf[u]) {
            mine++;
            a.label[u] = cluster;
        }
    atomicAdd(&s_surface, mine);
    __syncthreads();
    if (t == 0) a.result[0] = s_greatest + s_surface;
}

}  // namespace

extern "C" int sofia_greatest_cluster(sofia_nb_ctx *ctx, int np, const sofia_ainfo *position,
                                      const int32_t *global_id, int n_gly, int atoms_per_gly,
                                      float box, double mrcut, double denscut, int densmin,
                                      double *ptta_full, int32_t *greatest_belongsto,
                                      int32_t *size_out, int32_t *denstrack,
                                      int32_t *belongsto) {
    if (!ctx) return SOFIA_EINVAL;
    if (np <= 0 || !position || !global_id || n_gly < 0 || atoms_per_gly <= 0 || !ptta_full ||
        !greatest_belongsto || !size_out || !(box > 0.0f) || !(mrcut > 0.0) || !(denscut > 0.0))
        return sofia::fail(ctx, SOFIA_EINVAL, "bad args%s");
    if (n_gly == 0) {
        *size_out = 0;
        return SOFIA_OK;
    }
    SOFIA_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc;
    const void *dpos, *dgid;
    if ((rc = sofia::stage_in(ctx, position, sizeof(float4) * (size_t)np, 0, &dpos))) return rc;
    if ((rc = sofia::stage_in(ctx, global_id, sizeof(int) * (size_t)np, 1, &dgid))) return rc;
    sofia::OutArg o_ptta;
    const size_t ptta_bytes = sizeof(double) * 3 * (size_t)n_gly * atoms_per_gly;
    if ((rc = sofia::stage_out(ctx, ptta_full, ptta_bytes, 2, &o_ptta, true))) return rc;
    // cell grid of check_allocation_cluster (mod_neighbor_cluster.f90:546-548)
    const float ibox = (float)(1.0 / (double)box);
    volatile float vb2 = box * box;
    volatile float vol = vb2 * box;
    const int nside = (int)((double)box / mrcut);
    if (nside < 1) return sofia::fail(ctx, SOFIA_EINVAL, "box smaller than mrcut%s");
    volatile float mrn_f = box / (float)nside;
    const double mrn = (double)mrn_f;
    const int mncellT = (int)lround((double)vol / ((mrn * mrn) * mrn));
    const int mncellD = (int)lround(pow((double)mncellT, 1.0 / 3.0));
    if ((long)mncellD * mncellD * mncellD != mncellT)
        return sofia::fail(ctx, SOFIA_EINVAL, "invalid cluster cell grid%s");
    const size_t n = (size_t)n_gly;
    SOFIA_CUDA(ctx, ctx->cl_buf[0].ensure(sizeof(double) * 3 * n));
    SOFIA_CUDA(ctx, ctx->cl_buf[1].ensure(sizeof(int) * n * 4));
    SOFIA_CUDA(ctx, ctx->cl_buf[2].ensure(sizeof(int) * ((size_t)mncellT + 1) * 3));
    SOFIA_CUDA(ctx, ctx->cl_buf[3].ensure(sizeof(int) * n * DCAP));
    SOFIA_CUDA(ctx, ctx->cl_buf[4].ensure(sizeof(int) * (n + 1) * 4));
    SOFIA_CUDA(ctx, ctx->cl_buf[5].ensure(sizeof(int) * 4));
    ClusterArgs a;
    a.n_gly = n_gly;
    a.apg = atoms_per_gly;
    a.densmin = densmin;
    a.mncellD = mncellD;
    a.mncellT = mncellT;
    a.box = box;
    a.ibox = ibox;
    a.mrcut2 = mrcut * mrcut;
    a.denscut2 = denscut * denscut;
    a.imrn = 1.0 / mrn;
    a.ptta = (double *)o_ptta.dev;
    a.com = ctx->cl_buf[0].as<double>();
    int *b1 = ctx->cl_buf[1].as<int>();
    a.mcell = b1;
    a.cell_list = b1 + n;
    a.denstrack = b1 + 2 * n;
    int *b2 = ctx->cl_buf[2].as<int>();
    a.cell_count = b2;
    a.cell_start = b2 + (mncellT + 1);
    a.cell_fill = b2 + 2 * (mncellT + 1);
    a.densvl = ctx->cl_buf[3].as<int>();
    int *b4 = ctx->cl_buf[4].as<int>();
    a.label = b4;
    a.rank = b4 + (n + 1);
    a.csize = b4 + 2 * (n + 1);
    a.surf = b4 + 3 * (n + 1);
    a.status = ctx->d_status;
    a.result = ctx->cl_buf[5].as<int>();
    const int32_t res_init[2] = {0, *greatest_belongsto};
    SOFIA_CUDA(ctx, cudaMemcpyAsync(a.result, res_init, sizeof(res_init), cudaMemcpyHostToDevice, st));
    SOFIA_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS, st));
    const int flag = n_gly * atoms_per_gly;
    k_ptta_refresh<<<sofia::grid_for(np, 256), 256, 0, st>>>(np, (const float4 *)dpos,
                                                            (const int *)dgid, flag, a.ptta);
    k_cluster<<<1, 1024, 0, st>>>(a);
    SOFIA_CUDA(ctx, cudaGetLastError());
    if ((rc = sofia::finish_out(ctx, o_ptta))) return rc;
    int32_t res[2];
    SOFIA_CUDA(ctx, cudaMemcpyAsync(res, a.result, sizeof(res), cudaMemcpyDeviceToHost, st));
    if (denstrack)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(denstrack, a.denstrack, sizeof(int) * n,
                                        sofia::is_device_ptr(denstrack) ? cudaMemcpyDeviceToDevice
                                                                        : cudaMemcpyDeviceToHost,
                                        st));
    if (belongsto)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(belongsto, a.label, sizeof(int) * n,
                                        sofia::is_device_ptr(belongsto) ? cudaMemcpyDeviceToDevice
                                                                        : cudaMemcpyDeviceToHost,
                                        st));
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status,
                                    sizeof(int32_t) * sofia::ST_NSLOTS, cudaMemcpyDeviceToHost, st));
    SOFIA_CUDA(ctx, cudaStreamSynchronize(st));
    if (ctx->h_status[sofia::ST_DENSOVER])
        return sofia::fail(ctx, SOFIA_EINVAL, "density list overflow (more than 256 entries)%s");
    *size_out = res[0];
    *greatest_belongsto = res[1];
    return SOFIA_OK;
}
