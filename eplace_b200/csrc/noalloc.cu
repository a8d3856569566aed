// noalloc.cu -- the density scatter for callers that cannot allocate device
// memory.
//
// Some hosts of this library own every byte of device memory: a placement
// tool whose allocator reserves its pool up front and forbids plugins from
// calling cudaMalloc, or a caller that must not introduce the device-wide
// synchronisation a cudaMalloc / cudaFree pair can bring into the middle of
// its stream work.  ep_density_scatter_noalloc serves them: the caller
// passes device inputs and outputs, and the int64 fixed-point accumulation
// maps the scatter needs live in g_noalloc_scratch, a file-scope __device__
// array that every GPU loading this library holds until the process exits.
//
// Host code must not pass g_noalloc_scratch itself to a kernel: on the host
// that name is a stand-in, not a device address.  The first call in each
// CUDA context of a device (with that device current) looks up the array's
// device address with cudaGetSymbolAddress and keeps it for later calls; the
// cache is keyed by the context's id, so a call after cudaDeviceReset (a new
// primary context, the module loaded again) looks the address up again.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "engine.h"

namespace ep {
namespace {

// Largest grid the fixed-size scratch holds: 512 x 512 bins, two int64 maps
// (node, filler) = 4 MiB.
constexpr int kNoallocMaxBins = 512 * 512;
// Objects whose bin footprint may exceed this many bins are scattered by the
// whole block instead of one thread (a macro can cover most of the grid).
constexpr int kNoallocSmallBins = 16;
constexpr int kNoallocThreads = 256;

__device__ __align__(256) unsigned long long g_noalloc_scratch[2 * kNoallocMaxBins];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct ScratchAddr {
    unsigned long long ctx_id = 0;  // 0: not looked up yet
    unsigned long long *addr = nullptr;
};
ScratchAddr g_addr[kMaxDevices];

// Driver entry points for the context id (through the runtime, so the library
// does not link libcuda itself).
typedef CUresult (*PFN_ctx_get_current)(CUcontext *);
typedef CUresult (*PFN_ctx_get_id)(CUcontext, unsigned long long *);

bool current_context_id(unsigned long long &id) {
    static PFN_ctx_get_current get_current = nullptr;
    static PFN_ctx_get_id get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            return false;
        get_current = (PFN_ctx_get_current)a;
        get_id = (PFN_ctx_get_id)b;
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, &id) == CUDA_SUCCESS;
}

__global__ void k_noalloc_clear(unsigned long long *__restrict__ s, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s[k] = 0ull;
}

__device__ __forceinline__ void noalloc_add(const Grid &g, const Rect &r, float s, int i, int j, double qscale,
                                            unsigned long long *__restrict__ map) {
    float ovl = (float)rect_bin_overlap(g, r, i, j);
    if (ovl == 0.0f) return;
    long long q = __double2ll_rn(__dmul_rn((double)__fmul_rn(s, ovl), qscale));
    atomicAdd(&map[(size_t)i * g.ny + j], (unsigned long long)q);
}

// Same contributions as the engine's scatter (EPlace/eplace.cpp:1029-1133).
// A thread takes its object's bins when the footprint is small; objects that
// may cover more than kNoallocSmallBins bins are queued in shared memory and
// each is then scattered by the whole block, its bins strided over the threads.
__global__ void __launch_bounds__(kNoallocThreads)
k_noalloc_scatter(Grid g, int n, const float *__restrict__ cx, const float *__restrict__ cy,
                  const float *__restrict__ w, const float *__restrict__ h,
                  const uint8_t *__restrict__ flags, double qscale,
                  unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q) {
    __shared__ int big[kNoallocThreads];
    __shared__ int n_big;
    if (threadIdx.x == 0) n_big = 0;
    __syncthreads();
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n) {
        const uint8_t f = flags ? flags[o] : 0;
        const Rect r = object_rect(g, cx[o], cy[o], w[o], h[o]);
        int i0, i1, j0, j1;
        bin_range(g, r, i0, i1, j0, j1);
        if ((long long)max(i1 - i0 + 1, 0) * max(j1 - j0 + 1, 0) > kNoallocSmallBins) {
            big[atomicAdd(&n_big, 1)] = o;
        } else {
            float s = __fmul_rn(r.sx, r.sy);
            if (f & kMacro) s = __fmul_rn(s, g.td);
            unsigned long long *map = (f & kFiller) ? filler_q : node_q;
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++) noalloc_add(g, r, s, i, j, qscale, map);
        }
    }
    __syncthreads();
    for (int k = 0; k < n_big; k++) {
        const int b = big[k];
        const uint8_t f = flags ? flags[b] : 0;
        const Rect r = object_rect(g, cx[b], cy[b], w[b], h[b]);
        int i0, i1, j0, j1;
        bin_range(g, r, i0, i1, j0, j1);
        float s = __fmul_rn(r.sx, r.sy);
        if (f & kMacro) s = __fmul_rn(s, g.td);
        unsigned long long *map = (f & kFiller) ? filler_q : node_q;
        const int wy = j1 - j0 + 1, nbins = (i1 - i0 + 1) * wy;
        for (int t = threadIdx.x; t < nbins; t += blockDim.x) noalloc_add(g, r, s, i0 + t / wy, j0 + t % wy, qscale, map);
    }
}

__global__ void k_noalloc_emit(int nb, const unsigned long long *__restrict__ node_q,
                               const unsigned long long *__restrict__ filler_q, double inv_qscale,
                               float *__restrict__ node_out, float *__restrict__ filler_out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        node_out[k] = (float)((double)(long long)node_q[k] * inv_qscale);
        if (filler_out) filler_out[k] = (float)((double)(long long)filler_q[k] * inv_qscale);
    }
}

void set_msg(char *err, int32_t len, const char *msg) {
    if (err && len > 0) std::snprintf(err, (size_t)len, "%s", msg);
}

}  // namespace
}  // namespace ep

using namespace ep;

extern "C" ep_status ep_density_scatter_noalloc(const ep_scatter_grid *grid, int32_t num_objects,
                                                const float *cx, const float *cy, const float *w,
                                                const float *h, const uint8_t *flags,
                                                float *node_out, float *filler_out, void *stream,
                                                char *err, int32_t err_len) {
    if (!grid || num_objects < 0 || (num_objects > 0 && (!cx || !cy || !w || !h)) || !node_out) {
        set_msg(err, err_len, "ep_density_scatter_noalloc: null argument");
        return EP_ERR_ARG;
    }
    const long long nb = (long long)grid->bins_x * grid->bins_y;
    if (grid->bins_x < 1 || grid->bins_y < 1 || nb > kNoallocMaxBins) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "ep_density_scatter_noalloc: %d x %d bins exceeds the fixed scratch of %d bins "
                      "(512 x 512); use the engine's allocating path",
                      grid->bins_x, grid->bins_y, kNoallocMaxBins);
        set_msg(err, err_len, msg);
        return EP_ERR_ARG;
    }
    if (!(grid->bin_step_x > 0) || !(grid->bin_step_y > 0)) {
        set_msg(err, err_len, "ep_density_scatter_noalloc: bin steps must be positive");
        return EP_ERR_ARG;
    }
    if (!(grid->target_density > 0) || grid->target_density > 1.0f) {
        set_msg(err, err_len, "ep_density_scatter_noalloc: target_density must be in (0, 1]");
        return EP_ERR_ARG;
    }
    // Fixed-point scale 2^k: one contribution is at most a bin's area (the
    // smoothing scale sx*sy and the target density are <= 1), so no bin sum
    // exceeds num_objects * bin area; k keeps 1.05 times that below 2^62.
    const double bin_area = (double)grid->bin_step_x * (double)grid->bin_step_y;
    const int qbits = std::min(40, (int)std::floor(62.0 - std::log2(1.05 * (double)num_objects * bin_area + 1.0)));
    if (!std::isfinite(bin_area) || qbits < 8) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "ep_density_scatter_noalloc: %d objects on bins of area %g can sum past the int64 "
                      "fixed point of the scratch maps (needs 2^8 units per area unit at least)",
                      num_objects, bin_area);
        set_msg(err, err_len, msg);
        return EP_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_msg(err, err_len, "ep_density_scatter_noalloc: no usable current CUDA device");
        return EP_ERR_CUDA;
    }
    unsigned long long *scratch;
    {
        // set-up, once per device context, with that device current
        // (cudaGetSymbolAddress makes the device's primary context current
        // when there is none yet, so the id is read again after it)
        unsigned long long ctx = 0;
        const bool known = current_context_id(ctx);
        std::lock_guard<std::mutex> lock(g_mu);
        if (!known || g_addr[dev].ctx_id != ctx || !g_addr[dev].addr) {
            void *p = nullptr;
            cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (rc != cudaSuccess || !p) {
                set_msg(err, err_len, cudaGetErrorString(rc));
                return EP_ERR_CUDA;
            }
            if (!known && !current_context_id(ctx)) {
                set_msg(err, err_len, "ep_density_scatter_noalloc: no current CUDA context");
                return EP_ERR_CUDA;
            }
            g_addr[dev].addr = (unsigned long long *)p;
            g_addr[dev].ctx_id = ctx;
        }
        scratch = g_addr[dev].addr;
    }
    cudaStream_t st = (cudaStream_t)stream;
    Grid g{};
    g.nx = grid->bins_x;
    g.ny = grid->bins_y;
    g.llx = grid->core_llx;
    g.lly = grid->core_lly;
    g.sx = grid->bin_step_x;
    g.sy = grid->bin_step_y;
    g.urx = grid->core_llx + grid->bin_step_x * grid->bins_x;
    g.ury = grid->core_lly + grid->bin_step_y * grid->bins_y;
    g.td = grid->target_density;
    const double qscale = std::ldexp(1.0, qbits), inv_qscale = std::ldexp(1.0, -qbits);
    unsigned long long *node_q = scratch, *filler_q = scratch + nb;
    int blocks = (int)std::min<long long>((2 * nb + 255) / 256, 148 * 8);
    k_noalloc_clear<<<blocks, 256, 0, st>>>(scratch, (int)(2 * nb));
    if (num_objects > 0)
        k_noalloc_scatter<<<(num_objects + kNoallocThreads - 1) / kNoallocThreads, kNoallocThreads, 0, st>>>(
            g, num_objects, cx, cy, w, h, flags, qscale, node_q, filler_q);
    k_noalloc_emit<<<blocks, 256, 0, st>>>((int)nb, node_q, filler_q, inv_qscale, node_out, filler_out);
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess) {
        set_msg(err, err_len, cudaGetErrorString(rc));
        return EP_ERR_CUDA;
    }
    return EP_OK;
}
