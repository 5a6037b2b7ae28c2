// api_ctx.cu -- context lifetime and small host helpers of the C ABI.
#include <cmath>
#include <new>

#include "common.cuh"

extern "C" int sofia_nb_create(const sofia_nb_params *params, sofia_nb_ctx **out) {
    if (!out) return SOFIA_EINVAL;
    *out = nullptr;
    int dev = params ? params->device : 0;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SOFIA_ECUDA;
    }
    if (dev < 0 || dev >= ndev) return SOFIA_EINVAL;
    sofia_nb_ctx *ctx = new (std::nothrow) sofia_nb_ctx();
    if (!ctx) return SOFIA_ECUDA;
    ctx->device = dev;
    if (cudaSetDevice(dev) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_status, sizeof(int32_t) * sofia::ST_NSLOTS) != cudaSuccess ||
        cudaMallocHost(&ctx->h_status, sizeof(int32_t) * sofia::ST_NSLOTS) != cudaSuccess ||
        cudaMallocHost(&ctx->h_red, sizeof(double) * 16) != cudaSuccess) {
        cudaGetLastError();
        sofia_nb_destroy(ctx);
        return SOFIA_ECUDA;
    }
    if (cudaMemset(ctx->d_status, 0, sizeof(int32_t) * sofia::ST_NSLOTS) != cudaSuccess) {
        cudaGetLastError();
        sofia_nb_destroy(ctx);
        return SOFIA_ECUDA;
    }
    *out = ctx;
    return SOFIA_OK;
}

extern "C" int sofia_nb_destroy(sofia_nb_ctx *ctx) {
    if (!ctx) return SOFIA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &b : ctx->stage) b.release();
    ctx->cell_of.release();
    ctx->cell_count.release();
    ctx->cell_start.release();
    ctx->cell_fill.release();
    ctx->sorted_idx.release();
    ctx->pos_sorted.release();
    ctx->cnum.release();
    ctx->pe_atom.release();
    ctx->red_out.release();
    ctx->res_nlist.release();
    ctx->res_numneigh.release();
    ctx->acc64.release();
    for (auto &b : ctx->cl_buf) b.release();
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_red) cudaFreeHost(ctx->h_red);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SOFIA_OK;
}

extern "C" const char *sofia_last_error(const sofia_nb_ctx *ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

extern "C" int sofia_wait(sofia_nb_ctx *ctx) {
    if (!ctx) return SOFIA_EINVAL;
    SOFIA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SOFIA_OK;
}

extern "C" void *sofia_stream(sofia_nb_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// init, Source/get_started.f90:101-117: f_shift and e_shift in double with the
// single-precision literal MY_PIS (:109) and libm erfc/exp.
extern "C" int sofia_dsf_constants(double alpha, float cut_coul, double *e_shift,
                                   double *f_shift) {
    if (!e_shift || !f_shift || !(cut_coul > 0.0f)) return SOFIA_EINVAL;
    const double my_pis = (double)1.77245385090551602729f;
    const double cc = (double)cut_coul;
    const double cut_coulsq = (double)(cut_coul * cut_coul);
    const double erfcc = erfc(alpha * cc);
    const double erfcd = exp(-(((alpha * alpha) * cc) * cc));
    const double fs = -(erfcc / cut_coulsq + (((2.0 / my_pis) * alpha) * erfcd) / cc);
    *f_shift = fs;
    *e_shift = erfcc / cc - fs * cc;
    return SOFIA_OK;
}

extern "C" int sofia_cell_grid(float box, float cut_coul, float rcut, float *rn,
                               int32_t *ncellT, int32_t *ncellD) {
    if (!rn || !ncellT || !ncellD || !(box > 0.0f) || !(cut_coul > 0.0f || rcut > 0.0f))
        return SOFIA_EINVAL;
    int nt, nd;
    sofia::cell_grid(box, cut_coul, rcut, rn, &nt, &nd);
    *ncellT = nt;
    *ncellD = nd;
    return (nt >= 1 && nd >= 1) ? SOFIA_OK : SOFIA_EINVAL;
}
