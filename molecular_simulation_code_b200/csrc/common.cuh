// common.cuh -- shared context, buffers and launch helpers of libsofia_nb.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <utility>

#include "../../include/sofia_nb.h"

namespace sofia {

// Grow-only device buffer owned by a context.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t sz = need ? need : 16;
        cudaError_t e = cudaMalloc(&p, sz);
        if (e == cudaSuccess) bytes = sz;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T *as() const { return reinterpret_cast<T *>(p); }
};

// Slots of the device status word array (per context).
enum StatusSlot {
    ST_MAXCOUNT = 0,     // largest neighbour row / list fill seen
    ST_BADBIN = 1,       // atoms binned outside [0,ncellD)
    ST_CELLOVER = 2,     // cell holds more atoms than the in-cell sort supports
    ST_SHAKE = 3,        // SHAKE determinant / convergence failures
    ST_NONFINITE = 4,    // non-finite force or position seen
    ST_EXCL_FAR = 5,     // excluded pair farther apart than the exclusion radius
    ST_DENSOVER = 6,     // cluster density-list overflow
    ST_REBUILD = 7,      // rebuild flag set by the displacement check
    ST_NCLUSTER = 8,     // cluster-pair list fill
    ST_FIXED_OVF = 9,    // fixed-point force range exceeded
    ST_SHAKE_NC = 10,    // SHAKE groups that hit maxiter (warning, as the reference prints)
    ST_NSLOTS = 16
};

// Bit transpose of an 8 x 4 bit matrix held in one word: the bit at position
// 4 j + i (j = 0..7, i = 0..3) moves to position 8 i + j.  The permutation of
// the five index bits (j2 j1 j0 i1 i0) -> (i1 i0 j2 j1 j0) is done as four
// exchanges of index-bit pairs, (1,0), (2,0), (3,1), (4,2), each one delta swap
// (bits at positions p with index bit a clear and b set trade places with p + d,
// d = 2^a - 2^b).
__host__ __device__ inline uint32_t delta_swap(uint32_t x, uint32_t m, int d) {
    const uint32_t t = ((x >> d) ^ x) & m;
    return x ^ t ^ (t << d);
}
__host__ __device__ inline uint32_t transpose_8x4(uint32_t x) {
    x = delta_swap(x, 0x22222222u, 1);
    x = delta_swap(x, 0x0a0a0a0au, 3);
    x = delta_swap(x, 0x00cc00ccu, 6);
    return delta_swap(x, 0x0000f0f0u, 12);
}

}  // namespace sofia

struct sofia_nb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    // status words: device array + pinned host mirror
    int32_t *d_status = nullptr;
    int32_t *h_status = nullptr;
    // staging buffers for host-pointer arguments
    sofia::DevBuf stage[12];
    // reference-semantics cell grid / list scratch
    sofia::DevBuf cell_of, cell_count, cell_start, cell_fill, sorted_idx, pos_sorted, cnum;
    sofia::DevBuf pe_atom;   // per-atom energy partials
    sofia::DevBuf red_out;   // reduction output
    // resident reference list (kept when the caller passes nlist == NULL to the force call)
    sofia::DevBuf res_nlist, res_numneigh;
    int res_np = 0;
    int res_neigh_alloc = 0;
    // pair14 / correction accumulators
    sofia::DevBuf acc64;
    // cluster analysis scratch
    sofia::DevBuf cl_buf[10];
    double *h_red = nullptr;  // pinned reduction results
};

namespace sofia {

inline int fail(sofia_nb_ctx *ctx, int code, const char *fmt, const char *a = "") {
    char buf[512];
    snprintf(buf, sizeof(buf), fmt, a);
    if (ctx) ctx->last_error = buf;
    return code;
}

inline int cuda_fail(sofia_nb_ctx *ctx, cudaError_t e, const char *where,
                     const char *file = nullptr, int line = 0) {
    char buf[512];
    if (file) {
        const char *base = strrchr(file, '/');
        snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", where, cudaGetErrorString(e),
                 base ? base + 1 : file, line);
    } else {
        snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    }
    if (ctx) ctx->last_error = buf;
    return SOFIA_ECUDA;
}

#define SOFIA_CUDA(ctx, call)                                                                \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess) return sofia::cuda_fail((ctx), _e, #call, __FILE__, __LINE__); \
    } while (0)

// True when p is device (or managed) memory; host pointers are staged.
inline bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Returns a device pointer holding `bytes` of input; host data is copied into stage[slot].
inline int stage_in(sofia_nb_ctx *ctx, const void *p, size_t bytes, int slot, const void **out) {
    if (!p || bytes == 0) {
        *out = p;
        return SOFIA_OK;
    }
    if (is_device_ptr(p)) {
        *out = p;
        return SOFIA_OK;
    }
    SOFIA_CUDA(ctx, ctx->stage[slot].ensure(bytes));
    SOFIA_CUDA(ctx, cudaMemcpyAsync(ctx->stage[slot].p, p, bytes, cudaMemcpyHostToDevice,
                                    ctx->stream));
    *out = ctx->stage[slot].p;
    return SOFIA_OK;
}

// Output helper: returns a device pointer to write to; `host` is set when a copy-back is due.
struct OutArg {
    void *dev = nullptr;
    void *host = nullptr;
    size_t bytes = 0;
};
inline int stage_out(sofia_nb_ctx *ctx, void *p, size_t bytes, int slot, OutArg *o,
                     bool copy_in_first = false) {
    o->bytes = bytes;
    if (!p || bytes == 0) {
        o->dev = p;
        return SOFIA_OK;
    }
    if (is_device_ptr(p)) {
        o->dev = p;
        return SOFIA_OK;
    }
    SOFIA_CUDA(ctx, ctx->stage[slot].ensure(bytes));
    o->dev = ctx->stage[slot].p;
    o->host = p;
    if (copy_in_first)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(o->dev, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return SOFIA_OK;
}
inline int finish_out(sofia_nb_ctx *ctx, const OutArg &o) {
    if (o.host && o.bytes)
        SOFIA_CUDA(ctx, cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost,
                                        ctx->stream));
    return SOFIA_OK;
}

inline int grid_for(long n, int block) { return (int)((n + block - 1) / block); }

// Cell grid of check_allocation (mod_neighbor.f90:1446-1452), real*4 arithmetic.
inline void cell_grid(float box, float cut_coul, float rcut, float *rn, int *ncellT,
                      int *ncellD) {
    float c = (cut_coul > rcut) ? cut_coul : rcut;
    volatile float bq = box / c;
    int nside = (int)bq;
    volatile float r = box / (float)nside;
    volatile float vb = box * box;
    volatile float vol = vb * box;
    volatile float r2 = r * r;
    volatile float r3 = r2 * r;
    volatile float ratio = vol / r3;
    *rn = r;
    *ncellT = (int)lroundf(ratio);
    *ncellD = (int)lround(pow((double)(*ncellT), 1.0 / 3.0));
}

}  // namespace sofia

// Programmatic dependent launch.  launch_pdl starts a kernel with the
// programmatic-serialization attribute, so it may be scheduled while its
// predecessor in the stream drains; every kernel so launched begins with
// SOFIA_PDL_ENTRY(), which waits until the predecessor grid has completed and
// its memory is visible (griddepcontrol.wait) before any other statement, then
// lets its own dependents be scheduled.  Results are those of plain stream
// order; only the launch gaps shrink.
#define SOFIA_PDL_ENTRY() \
    asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory")

namespace sofia {
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, A &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}
}  // namespace sofia
