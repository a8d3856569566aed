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
// that name is a stand-in, not a device address.  The first call on each
// device (with that device current) looks up the array's device address with
// cudaGetSymbolAddress and keeps it for later calls.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "engine.h"

namespace ep {
namespace {

// Largest grid the fixed-size scratch holds: 512 x 512 bins, two int64 maps
// (node, filler) = 4 MiB.
constexpr int kNoallocMaxBins = 512 * 512;
// Fixed-point scale of the scratch maps: 2^32 units per unit area, so the
// total object area must stay below 2^30 for every partial sum to fit.
constexpr double kNoallocScale = 4294967296.0;

__device__ __align__(256) unsigned long long g_noalloc_scratch[2 * kNoallocMaxBins];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned long long *g_addr[kMaxDevices] = {nullptr};

__global__ void k_noalloc_clear(unsigned long long *__restrict__ s, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s[k] = 0ull;
}

// Same contributions as the engine's scatter (EPlace/eplace.cpp:1029-1133),
// one thread per object looping over every bin it covers.
__global__ void k_noalloc_scatter(Grid g, int n, const float *__restrict__ cx,
                                  const float *__restrict__ cy, const float *__restrict__ w,
                                  const float *__restrict__ h, const uint8_t *__restrict__ flags,
                                  unsigned long long *__restrict__ node_q,
                                  unsigned long long *__restrict__ filler_q) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    uint8_t f = flags ? flags[o] : 0;
    Rect r = object_rect(g, cx[o], cy[o], w[o], h[o]);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    float s = __fmul_rn(r.sx, r.sy);
    if (f & kMacro) s = __fmul_rn(s, g.td);
    unsigned long long *map = (f & kFiller) ? filler_q : node_q;
    for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++) {
            float ovl = (float)rect_bin_overlap(g, r, i, j);
            if (ovl == 0.0f) continue;
            long long q = __double2ll_rn(__dmul_rn((double)__fmul_rn(s, ovl), kNoallocScale));
            atomicAdd(&map[(size_t)i * g.ny + j], (unsigned long long)q);
        }
}

__global__ void k_noalloc_emit(int nb, const unsigned long long *__restrict__ node_q,
                               const unsigned long long *__restrict__ filler_q,
                               float *__restrict__ node_out, float *__restrict__ filler_out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        node_out[k] = (float)((double)(long long)node_q[k] / kNoallocScale);
        if (filler_out) filler_out[k] = (float)((double)(long long)filler_q[k] / kNoallocScale);
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
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_msg(err, err_len, "ep_density_scatter_noalloc: no usable current CUDA device");
        return EP_ERR_CUDA;
    }
    unsigned long long *scratch;
    {
        // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void *p = nullptr;
            cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (rc != cudaSuccess || !p) {
                set_msg(err, err_len, cudaGetErrorString(rc));
                return EP_ERR_CUDA;
            }
            g_addr[dev] = (unsigned long long *)p;
        }
        scratch = g_addr[dev];
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
    unsigned long long *node_q = scratch, *filler_q = scratch + nb;
    int blocks = (int)std::min<long long>((2 * nb + 255) / 256, 148 * 8);
    k_noalloc_clear<<<blocks, 256, 0, st>>>(scratch, (int)(2 * nb));
    if (num_objects > 0)
        k_noalloc_scatter<<<(num_objects + 255) / 256, 256, 0, st>>>(g, num_objects, cx, cy, w, h, flags,
                                                                     node_q, filler_q);
    k_noalloc_emit<<<blocks, 256, 0, st>>>((int)nb, node_q, filler_q, node_out, filler_out);
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess) {
        set_msg(err, err_len, cudaGetErrorString(rc));
        return EP_ERR_CUDA;
    }
    return EP_OK;
}
