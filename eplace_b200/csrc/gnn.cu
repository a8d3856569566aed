// gnn.cu -- the learned warm start: a small message-passing network over the
// cell-net incidence that proposes the initial placement in place of the
// quadratic placement (QPPlacer::quadraticPlacement, QPlace/qplace.cpp:20-103),
// which stays the fallback and the judge.  No counterpart in the reference.
//
// Graph: the movable nodes (0..nn-1) and the terminals (nn..nn+nt-1) of an
// engine, read from the engine's device arrays (nets contiguous in device
// pin order, each object's pins through its object -> pin map); a net joins
// the nodes of its pins.  Two mean aggregations:
//   net_mean   a[n] = mean over the pins of net n of h[node(pin)]
//   node_mean  m[c] = mean over the pins of movable node c of a[net(pin)]
//                     (terminals receive nothing: m = 0)
//
// Features (kF per node, from the netlist alone, computed on the device):
// log(1 + area) / 4, log(1 + pins) / 3, terminal flag, and the node's
// coordinates (normalised to the core) after 8, 32 and 128 steps of
// pad-anchored diffusion: every movable node starts at the core centre,
// terminals sit at their own centres, and a step replaces each movable node
// by node_mean(net_mean(.)).  These are the fixed-pin distances the network
// reads: a node's diffused coordinate says how its pads pull it, at three
// ranges; d, the 128-step coordinates, is the base of the predictions.
//
// Network (hidden 64, weights stored BF16 for the forward pass, FP32
// accumulate, FP32 master weights for training):
//   h0 = relu(W0 x + b0)
//   h_l = relu(W_l [h_{l-1} ; node_mean(net_mean(h_{l-1}))] + b_l),  l = 1..3
//   q = d + 0.25 tanh(W4[0:2] h3 + b4[0:2])   the engine's quadratic placement
//   f = d + 0.25 tanh(W4[2:4] h3 + b4[2:4])   the engine's final mGP placement
// (normalised core coordinates).  Training: the mean squared error of both
// heads against the engine's own quadratic placement and final placement of
// the design, Adam; every reduction (weight gradients, loss) is a per-block
// partial summed in a fixed order, so a training step is bitwise repeatable.
// A proposal moves the movable nodes to q + alpha (f - q), mapped to the
// core: the quadratic placement's compact layout moved part of the way to
// where the optimizer ends.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "engine.h"
#include "tc_ptx.cuh"

namespace ep {
namespace {

constexpr int kH = 64;      // hidden width
constexpr int kF = 9;       // input features
constexpr int kOut = 4;     // q (x, y), f (x, y)
constexpr int kLayers = 3;  // message-passing layers
constexpr int kDiffSteps[3] = {8, 32, 128};
constexpr float kCorr = 0.25f;  // bound of a head's correction, in core sizes

// Parameter layout (floats): W0[kH][kF], b0[kH], per layer W[kH][2kH], b[kH],
// then W4[kOut][kH], b4[kOut].
constexpr int kOffW0 = 0, kOffB0 = kOffW0 + kH * kF, kOffL = kOffB0 + kH;
constexpr int kLayerParams = kH * 2 * kH + kH;
constexpr int kOffW4 = kOffL + kLayers * kLayerParams, kOffB4 = kOffW4 + kOut * kH;
constexpr int kParams = kOffB4 + kOut;
inline int off_w(int l) { return kOffL + (l - 1) * kLayerParams; }
inline int off_b(int l) { return off_w(l) + kH * 2 * kH; }

constexpr int kT = 256;
constexpr int kRowsPerBlock = 512;  // rows of one partial weight gradient
inline int nblk(long long n, int t = kT) { return (int)((n + t - 1) / t); }

// Device view of the bound netlist.
struct Net {
    int nn, n_obj, N, nnet;
    const int32_t *owner, *net_first, *net_deg, *pin_net, *obj_pin_start, *obj_pin_dev;
    const int32_t *net_order;            // nets in device pin order (neighbouring nets of equal degree)
    int n_big;                           // nets above kWarpPins pins: the head of net_order
    const int32_t *pad_start, *pad_net;  // terminals' pins (training only; may be null)
    // flattened indices, built once per bound netlist (k_graph_index):
    const int4 *kinfo;        // [nnet] per net in device order: first pin, degree, 1/degree (bits), net
    const int32_t *pin_node;  // [np] node (0..N-1) of each device pin
    const int32_t *q_net;     // [pins of movable nodes] net of each pin, in object pin order
};

__device__ __forceinline__ int node_of(int o, int nn, int n_obj) { return o < nn ? o : nn + (o - n_obj); }
__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// ------------------------------------------------------------ features ----
template <typename R>
__global__ void k_init(Net g, const float *__restrict__ area, const float *__restrict__ npins,
                       const vec2<R> *__restrict__ pos, Grid gr, float *__restrict__ X, float2 *__restrict__ v,
                       float *__restrict__ inv_pins) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    float *x = X + (size_t)c * kF;
#pragma unroll
    for (int k = 0; k < kF; k++) x[k] = 0.f;
    if (c < g.nn) {
        x[0] = log1pf(area[c]) * 0.25f;
        x[1] = log1pf(npins[c]) * (1.f / 3.f);
        v[c] = make_float2(0.5f, 0.5f);
        inv_pins[c] = npins[c] > 0.f ? 1.f / npins[c] : 0.f;
    } else {
        const vec2<R> t = pos[g.n_obj + (c - g.nn)];
        x[2] = 1.f;
        v[c] = make_float2((float)(((double)t.x - gr.llx) / ((double)gr.urx - gr.llx)),
                           (float)(((double)t.y - gr.lly) / ((double)gr.ury - gr.lly)));
        inv_pins[c] = 0.f;
    }
}

__global__ void k_pad_pins(int np, Net g, int *__restrict__ cnt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np && g.owner[p] >= g.n_obj) atomicAdd(&cnt[g.owner[p] - g.n_obj], 1);
}

__global__ void k_pad_feature(int nt, int nn, const int *__restrict__ cnt, float *__restrict__ X) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nt) X[(size_t)(nn + t) * kF + 1] = log1pf((float)cnt[t]) * (1.f / 3.f);
}

__global__ void k_inv_deg(int nnet, const int32_t *__restrict__ deg, float *__restrict__ inv) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nnet) inv[n] = deg[n] > 0 ? 1.f / deg[n] : 0.f;
}

// The aggregations' index arrays, one level of indirection shallower than
// the engine's: kinfo[k] for the k-th net of the device order (its first
// pin, degree, 1/degree as in k_inv_deg, id), the node of every pin, and the
// net of every pin of a movable node in object pin order.  Launched with
// max(nnet, np) threads.
__global__ void k_graph_index(Net g, int np, int4 *__restrict__ kinfo, int32_t *__restrict__ pin_node,
                              int32_t *__restrict__ q_net) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < g.nnet) {
        const int n = g.net_order[t], d = g.net_deg[n];
        kinfo[t] = make_int4(g.net_first[n], d, __float_as_int(d > 0 ? 1.f / d : 0.f), n);
    }
    if (t < np) pin_node[t] = node_of(g.owner[t], g.nn, g.n_obj);
    if (t < g.obj_pin_start[g.nn]) q_net[t] = g.pin_net[g.obj_pin_dev[t]];
}

// The nets above kWarpPins pins (the head of the device order) take a warp
// each: lane l sums pins l, l + 32, ... and a fixed xor tree adds the lanes.
// Every other net takes a thread, in device order, so a warp's nets have the
// same degree.  Launched with 32 n_big + (nnet - n_big) threads.
__global__ void k_diff_net(Net g, const float2 *__restrict__ v, float2 *__restrict__ a) {
    pdl_begin();
    const int t = blockIdx.x * blockDim.x + threadIdx.x, big = g.n_big * 32;
    if (t < big) {  // whole warps
        const int4 r = g.kinfo[t >> 5];
        const int lane = t & 31;
        float sx = 0.f, sy = 0.f;
        for (int p = r.x + lane, e = r.x + r.y; p < e; p += 32) {
            const float2 q = v[g.pin_node[p]];
            sx += q.x;
            sy += q.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        const float inv = __int_as_float(r.z);
        if (lane == 0) a[r.w] = make_float2(sx * inv, sy * inv);
        return;
    }
    const int k = g.n_big + (t - big);
    if (k >= g.nnet) return;
    const int4 r = g.kinfo[k];
    float sx = 0.f, sy = 0.f;
#pragma unroll 4
    for (int p = r.x, e = r.x + r.y; p < e; p++) {
        const float2 q = v[g.pin_node[p]];
        sx += q.x;
        sy += q.y;
    }
    const float inv = __int_as_float(r.z);
    a[r.w] = make_float2(sx * inv, sy * inv);
}

__global__ void k_diff_node(Net g, const float *__restrict__ inv_pins, const float2 *__restrict__ a,
                            float2 *__restrict__ v) {
    pdl_begin();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nn) return;
    const int q0 = g.obj_pin_start[c], q1 = g.obj_pin_start[c + 1];
    if (q1 == q0) return;
    float sx = 0.f, sy = 0.f;
#pragma unroll 4
    for (int q = q0; q < q1; q++) {
        const float2 t = a[g.q_net[q]];
        sx += t.x;
        sy += t.y;
    }
    v[c] = make_float2(sx * inv_pins[c], sy * inv_pins[c]);
}

__global__ void k_store_feature(int N, const float2 *__restrict__ v, float *__restrict__ X, int col) {
    pdl_begin();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    X[(size_t)c * kF + col] = v[c].x;
    X[(size_t)c * kF + col + 1] = v[c].y;
}

// ------------------------------------------------------ aggregations ------
// One warp per row, a float2 of channels per lane.  k_net_mean: the first
// n_big blocks take the nets above kWarpPins pins, a block each (warp w sums
// pins w, w + 8, ..., the 8 warp sums are added in warp order); the other
// nets take a warp each.
constexpr int kBigWarps = kT / 32;
__global__ void __launch_bounds__(kT) k_net_mean(Net g, const float2 *__restrict__ h,
                                                 float2 *__restrict__ a) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if ((int)blockIdx.x < g.n_big) {
        __shared__ float2 part[kBigWarps][32];
        const int4 r = g.kinfo[blockIdx.x];
        const int n = r.w;
        float2 s = make_float2(0.f, 0.f);
        for (int p = r.x + w, e = r.x + r.y; p < e; p += kBigWarps) {
            const float2 q = h[(size_t)g.pin_node[p] * 32 + lane];
            s.x += q.x;
            s.y += q.y;
        }
        part[w][lane] = s;
        __syncthreads();
        if (w == 0) {
            float2 t = part[0][lane];
            for (int k = 1; k < kBigWarps; k++) {
                t.x += part[k][lane].x;
                t.y += part[k][lane].y;
            }
            const float inv = __int_as_float(r.z);
            a[(size_t)n * 32 + lane] = make_float2(t.x * inv, t.y * inv);
        }
        return;
    }
    const int k = g.n_big + ((int)(blockIdx.x - g.n_big) * kBigWarps + w);
    if (k >= g.nnet) return;
    const int4 r = g.kinfo[k];
    const int n = r.w;
    float2 s = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int p = r.x, e = r.x + r.y; p < e; p++) {
        const float2 q = h[(size_t)g.pin_node[p] * 32 + lane];
        s.x += q.x;
        s.y += q.y;
    }
    const float inv = __int_as_float(r.z);
    a[(size_t)n * 32 + lane] = make_float2(s.x * inv, s.y * inv);
}

__global__ void k_node_mean(Net g, const float *__restrict__ inv_pins, const float2 *__restrict__ a,
                            float2 *__restrict__ m) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= g.N) return;
    float2 s = make_float2(0.f, 0.f);
    if (c < g.nn) {
        for (int q = g.obj_pin_start[c]; q < g.obj_pin_start[c + 1]; q++) {
            const float2 t = a[(size_t)g.q_net[q] * 32 + lane];
            s.x += t.x;
            s.y += t.y;
        }
        s.x *= inv_pins[c];
        s.y *= inv_pins[c];
    }
    m[(size_t)c * 32 + lane] = s;
}

// transpose of node_mean: da[n] = sum over the pins of n on movable nodes c of dm[c] / pins(c)
__global__ void k_node_mean_t(Net g, const float *__restrict__ inv_pins, const float2 *__restrict__ dm,
                              float2 *__restrict__ da) {
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (n >= g.nnet) return;
    float2 s = make_float2(0.f, 0.f);
    for (int p = g.net_first[n], e = p + g.net_deg[n]; p < e; p++) {
        const int c = g.pin_node[p];
        if (c >= g.nn) continue;
        const float2 t = dm[(size_t)c * 32 + lane];
        s.x += t.x * inv_pins[c];
        s.y += t.y * inv_pins[c];
    }
    da[(size_t)n * 32 + lane] = s;
}

// transpose of net_mean, added: dh[c] += sum over the pins of node c of da[net] / deg(net)
__global__ void k_net_mean_t_add(Net g, const float *__restrict__ inv_deg, const float2 *__restrict__ da,
                                 float2 *__restrict__ dh) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= g.N) return;
    float2 s = make_float2(0.f, 0.f);
    if (c < g.nn) {
        for (int q = g.obj_pin_start[c]; q < g.obj_pin_start[c + 1]; q++) {
            const int n = g.q_net[q];
            const float2 t = da[(size_t)n * 32 + lane];
            s.x += t.x * inv_deg[n];
            s.y += t.y * inv_deg[n];
        }
    } else {
        const int t0 = c - g.nn;
        for (int q = g.pad_start[t0]; q < g.pad_start[t0 + 1]; q++) {
            const int n = g.pad_net[q];
            const float2 t = da[(size_t)n * 32 + lane];
            s.x += t.x * inv_deg[n];
            s.y += t.y * inv_deg[n];
        }
    }
    float2 &o = dh[(size_t)c * 32 + lane];
    o.x += s.x;
    o.y += s.y;
}

// ------------------------------------------------------------ dense -------
// Y[r][o] = relu(b[o] + sum_k X[r][k] W[o][k]) with X = [XA (KA cols) | XB
// (KB cols)], W the BF16 weights, read here from their FP32 transposed copy
// Wt[k][o] (k_transpose_w).  kDenseRows rows per 256-thread block: Wt and
// the block's rows (row-major, padded to K + 1) staged in shared memory;
// thread (tx, ty) accumulates rows 4 ty .. 4 ty + 3 x outputs 8 tx .. 8 tx + 7
// in registers, k in order (two 16-byte weight loads and four row loads per
// 32 FMAs, without bank conflicts), so each output is the same sum as a
// plain loop over k.
constexpr int kDenseRows = 128;
template <int KA, int KB>
__global__ void __launch_bounds__(kT) k_dense(int N, const float *__restrict__ XA, const float *__restrict__ XB,
                                              const float *__restrict__ Wt, const float *__restrict__ b,
                                              float *__restrict__ Y) {
    constexpr int K = KA + KB, XP = K + 1;
    extern __shared__ float sm[];
    float *Ws = sm;            // [K][kH]
    float *Xs = sm + K * kH;   // [kDenseRows][XP]
    for (int i = threadIdx.x; i < K * kH / 4; i += kT)
        reinterpret_cast<float4 *>(Ws)[i] = reinterpret_cast<const float4 *>(Wt)[i];
    const int r0 = blockIdx.x * kDenseRows;
    for (int i = threadIdx.x; i < kDenseRows * K; i += kT) {
        const int r = i / K, k = i - r * K, row = r0 + r;
        float v = 0.f;
        if (row < N) v = k < KA ? XA[(size_t)row * KA + k] : XB[(size_t)row * KB + (k - KA)];
        Xs[r * XP + k] = v;
    }
    __syncthreads();
    const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;
    const float4 *W4 = reinterpret_cast<const float4 *>(Ws);
    float acc[4][8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float bj = b[tx * 8 + j];
#pragma unroll
        for (int i = 0; i < 4; i++) acc[i][j] = bj;
    }
#pragma unroll 4
    for (int k = 0; k < K; k++) {
        float x[4];
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] = Xs[(ty * 4 + i) * XP + k];
        const float4 wa = W4[k * (kH / 4) + tx * 2], wb = W4[k * (kH / 4) + tx * 2 + 1];
        const float w[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = fmaf(x[i], w[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int row = r0 + ty * 4 + i;
        if (row >= N) continue;
        float4 *y = reinterpret_cast<float4 *>(Y + (size_t)row * kH + tx * 8);
        y[0] = make_float4(fmaxf(acc[i][0], 0.f), fmaxf(acc[i][1], 0.f), fmaxf(acc[i][2], 0.f), fmaxf(acc[i][3], 0.f));
        y[1] = make_float4(fmaxf(acc[i][4], 0.f), fmaxf(acc[i][5], 0.f), fmaxf(acc[i][6], 0.f), fmaxf(acc[i][7], 0.f));
    }
}

// The input layer's BF16 weights as FP32, transposed to [k][o], for k_dense.
constexpr int kWtSize = kF * kH;
__global__ void k_transpose_w(const __nv_bfloat16 *__restrict__ wb, float *__restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWtSize) return;
    const int k = i / kH, o = i % kH;
    wt[i] = bf(wb[kOffW0 + o * kF + k]);
}

// ------------------------------------------------------ dense, tcgen05 ----
// The hidden layers (K = 2 kH = 128 inputs [XA | XB], kH = 64 outputs) on
// the tensor cores: Y = relu(b + [XA | XB] W^T).  Each FP32 input is split
// into two BF16 planes, hi = bf16(x) and lo = bf16(x - hi) (hi + lo holds x
// to 2^-17 relative), and both are multiplied by the BF16 weights (exact in
// BF16) with tcgen05.mma.kind::f16, FP32 accumulators in tensor memory.  A
// persistent CTA of 256 threads (two per SM) takes 128-row tiles in turn:
//   all threads  load the tile's rows (coalesced float4), split them and
//                store both planes in shared memory in the K-major,
//                128-byte-swizzled layout of the MMA descriptors;
//   thread 0     issues 16 MMAs (2 K blocks x 4 steps of 16 x 2 planes) and
//                commits them to an mbarrier;
//   all threads  wait (bounded), read the accumulators (warp w: TMEM lanes
//                32 (w % 4) .. + 31 = tile rows, columns 32 (w / 4) .. + 31),
//                add the bias, relu, stage the tile in shared memory (over the
//                consumed planes) and store it row-major with coalesced float4
//                stores.
// The next tile's loads are in flight during a tile's MMAs and epilogue.  The
// weights (64 x 128 BF16) are staged once per CTA.  A wait that gives up sets
// its flag in *status (and EP_ERR_TIMEOUT in the engine's word); the CTA
// waits for its own MMAs (bounded) before it frees its tensor memory.
constexpr int kTcRows = 128, kTcThreads = 256, kTcKB = 2;
constexpr int kTcWBlock = kH * 128;                 // one K block of W: 64 rows x 128 B
constexpr int kTcABlock = kTcRows * 128;            // one K block of one input plane
constexpr int kTcW = kTcKB * kTcWBlock;             // 16 KB
constexpr int kTcA = 2 * kTcKB * kTcABlock;         // hi and lo planes, 64 KB
constexpr int kTcLd = kH + 4;                       // staging row stride, floats
constexpr int kTcLoads = kTcRows * 32 / kTcThreads;  // float4 loads per thread and tile
constexpr int kTcCols = 64;                         // TMEM columns
static_assert(kTcRows * kTcLd * 4 <= kTcA, "the staged tile fits over the input planes");
constexpr size_t kTcSmem = 1024 + kTcW + kTcA + 64;

// Byte offset of element k (0..63) of row r in a K-major block with the
// 128-byte swizzle: 8-row x 128-byte atoms 1024 bytes apart, the 16-byte
// chunk index XOR-ed with the row inside the atom.
__device__ __forceinline__ uint32_t sw128(int r, int k) {
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + (((k >> 3) ^ (r & 7)) << 4) + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t pack_bf16(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

__global__ void __launch_bounds__(kTcThreads, 2)
k_dense_tc(int N, const float *__restrict__ XA, const float *__restrict__ XB, const __nv_bfloat16 *__restrict__ W,
           const float *__restrict__ b, float *__restrict__ Y, int *__restrict__ status, int *__restrict__ engine_status,
           unsigned wait_limit) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *Ws = smem, *As = smem + kTcW;
    float *stage = (float *)As;
    uint64_t *bar = (uint64_t *)(As + kTcA);
    volatile uint32_t *tmem_slot = (volatile uint32_t *)(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(tc::smem_u32((const void *)tmem_slot)), "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // weights: row o, K block kb, 16-byte chunk j (8 BF16)
    for (int i = tid; i < kH * kTcKB * 8; i += kTcThreads) {
        const int o = i >> 4, kb = (i >> 3) & 1, j = i & 7;
        const uint4 v = *reinterpret_cast<const uint4 *>(W + (size_t)o * 2 * kH + kb * 64 + j * 8);
        *reinterpret_cast<uint4 *>(Ws + kb * kTcWBlock + sw128(o, j * 8)) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int ntiles = (N + kTcRows - 1) / kTcRows;
    const int kb_l = lane >> 4, k_l = (lane & 15) * 4;  // this lane's K block and first K of its float4
    const float *src = kb_l ? XB : XA;
    uint32_t phase = 0;
    bool ok = true;
    // warp w, load i: row 8 i + w of a tile (a warp reads one row: XA's 64
    // floats in lanes 0-15, XB's in lanes 16-31); rows past N (and tiles past
    // the last) read as zeros
    float4 v[kTcLoads];
    auto load_tile = [&](int t) {
#pragma unroll
        for (int i = 0; i < kTcLoads; i++) {
            const int gr = t * kTcRows + i * 8 + warp;
            v[i] = gr < N ? __ldg(reinterpret_cast<const float4 *>(src + (size_t)gr * kH + k_l))
                          : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    load_tile(blockIdx.x);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int r0 = tile * kTcRows;
#pragma unroll
        for (int i = 0; i < kTcLoads; i++) {
            const int row = i * 8 + warp;
            uint16_t h[4], l[4];
            tc::bf16_split(v[i].x, h[0], l[0]);
            tc::bf16_split(v[i].y, h[1], l[1]);
            tc::bf16_split(v[i].z, h[2], l[2]);
            tc::bf16_split(v[i].w, h[3], l[3]);
            const uint32_t off = kb_l * kTcABlock + sw128(row, k_l);
            *reinterpret_cast<uint2 *>(As + off) = make_uint2(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]));
            *reinterpret_cast<uint2 *>(As + kTcKB * kTcABlock + off) =
                make_uint2(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t idesc = tc::umma_idesc(kTcRows, kH);
            const uint32_t a = tc::smem_u32(As), w = tc::smem_u32(Ws);
#pragma unroll
            for (int kb = 0; kb < kTcKB; kb++)
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t ao = kb * kTcABlock + k * 32, wo = kb * kTcWBlock + k * 32;
                    tc::umma_bf16(tmem, tc::umma_desc(a + ao), tc::umma_desc(w + wo), idesc, (kb | k) != 0);
                    tc::umma_bf16(tmem, tc::umma_desc(a + kTcKB * kTcABlock + ao), tc::umma_desc(w + wo), idesc, 1);
                }
            tc::umma_commit(bar);
        }
        load_tile(tile + gridDim.x);  // the next tile's rows in flight during the MMAs and the epilogue
        // lane 0 of each warp waits; the CTA goes on only if every warp saw
        // the commit (a uniform decision, so no barrier is left half-reached)
        int got = 1;
        if (lane == 0) {
            got = 0;
            for (unsigned it = 0; it < wait_limit; it++)
                if (tc::mbar_try_wait(bar, phase)) {
                    got = 1;
                    break;
                }
        }
        got = __shfl_sync(0xffffffffu, got, 0);
        ok = __syncthreads_and(got) != 0;
        if (!ok) break;
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        {
            const int q = warp & 3, ch = warp >> 2, row = q * 32 + lane;
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ch * 32);
#pragma unroll
            for (int c0 = 0; c0 < 32; c0 += 16) {
                uint32_t r[16];
                tc::tmem_ld16(taddr + (uint32_t)c0, r);
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    const int col = ch * 32 + c0 + j;
                    float4 o;
                    o.x = fmaxf(__uint_as_float(r[j]) + __ldg(b + col), 0.f);
                    o.y = fmaxf(__uint_as_float(r[j + 1]) + __ldg(b + col + 1), 0.f);
                    o.z = fmaxf(__uint_as_float(r[j + 2]) + __ldg(b + col + 2), 0.f);
                    o.w = fmaxf(__uint_as_float(r[j + 3]) + __ldg(b + col + 3), 0.f);
                    *reinterpret_cast<float4 *>(stage + row * kTcLd + col) = o;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kTcRows * 16 / kTcThreads; i++) {
            const int u = i * kTcThreads + tid, row = u >> 4, c4 = u & 15, gr = r0 + row;
            if (gr < N)
                *reinterpret_cast<float4 *>(Y + (size_t)gr * kH + c4 * 4) =
                    *reinterpret_cast<const float4 *>(stage + row * kTcLd + c4 * 4);
        }
        __syncthreads();  // the staged rows are read before the next tile's planes overwrite them
    }
    if (!ok && tid == 0) {
        // the MMAs of the tile in flight complete before the tensor memory is freed
        for (unsigned it = 0; it < tc::kWaitLimit && !tc::mbar_try_wait(bar, phase); it++) {
        }
        *(volatile int *)status = 1;  // mapped host memory: a plain store
        if (engine_status) atomicOr(engine_status, 1 << EP_ERR_TIMEOUT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
    }
}

// Launched as clusters of one CTA, like the tensor-core Poisson GEMMs.
void launch_dense_tc(int grid, cudaStream_t st, int N, const float *XA, const float *XB, const __nv_bfloat16 *W,
                     const float *b, float *Y, int *status, int *engine_status, unsigned wait_limit) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = kTcSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_dense_tc, N, XA, XB, W, b, Y, status, engine_status, wait_limit);
}

// dX = (dY .* (Y > 0)) W, split into dXA (KA cols) and dXB (KB cols).
template <int KA, int KB>
__global__ void __launch_bounds__(kT) k_dense_dx(int N, const float *__restrict__ dY, const float *__restrict__ Y,
                                                 const __nv_bfloat16 *__restrict__ W, float *__restrict__ dXA,
                                                 float *__restrict__ dXB) {
    constexpr int K = KA + KB, PER = (K + 3) / 4;
    extern __shared__ float sm[];
    float *Ws = sm;           // [kH][K]
    float *Zs = sm + kH * K;  // [64][kH + 1]
    for (int i = threadIdx.x; i < kH * K; i += kT) Ws[i] = bf(W[i]);
    const int r0 = blockIdx.x * 64;
    for (int i = threadIdx.x; i < 64 * kH; i += kT) {
        const int r = i / kH, o = i - r * kH, row = r0 + r;
        float z = 0.f;
        if (row < N) {
            const size_t at = (size_t)row * kH + o;
            z = Y[at] > 0.f ? dY[at] : 0.f;
        }
        Zs[r * (kH + 1) + o] = z;
    }
    __syncthreads();
    const int r = threadIdx.x >> 2, k0 = (threadIdx.x & 3) * PER;
    float acc[PER];
#pragma unroll
    for (int j = 0; j < PER; j++) acc[j] = 0.f;
    for (int o = 0; o < kH; o++) {
        const float z = Zs[r * (kH + 1) + o];
#pragma unroll
        for (int j = 0; j < PER; j++)
            if (k0 + j < K) acc[j] = fmaf(z, Ws[o * K + k0 + j], acc[j]);
    }
    const int row = r0 + r;
    if (row >= N) return;
#pragma unroll
    for (int j = 0; j < PER; j++) {
        const int k = k0 + j;
        if (k < KA)
            dXA[(size_t)row * KA + k] = acc[j];
        else if (k < K && dXB)
            dXB[(size_t)row * KB + (k - KA)] = acc[j];
    }
}

// Per-block partial weight gradient: P[o][k] = sum_r Z[r][o] X[r][k] and
// P[O*K + o] = sum_r Z[r][o] over the block's rows, Z = dY .* (Y > 0) when Y
// is given (ReLU layers) else dY.  Rows are read in 32-row tiles.
template <int O, int KA, int KB>
__global__ void __launch_bounds__(kT) k_dweight(int N, int rows_per_block, const float *__restrict__ dY,
                                                const float *__restrict__ Y, const float *__restrict__ XA,
                                                const float *__restrict__ XB, float *__restrict__ partial) {
    constexpr int K = KA + KB, OK = O * K, PER = (OK + kT - 1) / kT, TR = 32;
    __shared__ float Zs[TR][O + 1];
    __shared__ float Xs[TR][K + 1];
    float acc[PER], bacc = 0.f;
#pragma unroll
    for (int j = 0; j < PER; j++) acc[j] = 0.f;
    const int rb = blockIdx.x * rows_per_block, re = min(N, rb + rows_per_block);
    for (int t0 = rb; t0 < re; t0 += TR) {
        __syncthreads();
        for (int i = threadIdx.x; i < TR * O; i += kT) {
            const int r = i / O, o = i - r * O, row = t0 + r;
            float z = 0.f;
            if (row < re) {
                const size_t at = (size_t)row * O + o;
                z = (!Y || Y[at] > 0.f) ? dY[at] : 0.f;
            }
            Zs[r][o] = z;
        }
        for (int i = threadIdx.x; i < TR * K; i += kT) {
            const int r = i / K, k = i - r * K, row = t0 + r;
            float v = 0.f;
            if (row < re) v = k < KA ? XA[(size_t)row * KA + k] : XB[(size_t)row * KB + (k - KA)];
            Xs[r][k] = v;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const int i = threadIdx.x + j * kT;
            if (i >= OK) break;
            const int o = i / K, k = i - o * K;
            float s = acc[j];
            for (int r = 0; r < TR; r++) s = fmaf(Zs[r][o], Xs[r][k], s);
            acc[j] = s;
        }
        if (threadIdx.x < O)
            for (int r = 0; r < TR; r++) bacc += Zs[r][threadIdx.x];
    }
    float *P = partial + (size_t)blockIdx.x * (OK + O);
#pragma unroll
    for (int j = 0; j < PER; j++) {
        const int i = threadIdx.x + j * kT;
        if (i < OK) P[i] = acc[j];
    }
    if (threadIdx.x < O) P[OK + threadIdx.x] = bacc;
}

// grad[w_off + i] = sum over blocks of partial[blk][i] (weights), then biases.
__global__ void k_reduce_partials(int blocks, int OK, int O, const float *__restrict__ partial, float *__restrict__ grad,
                                  int w_off, int b_off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= OK + O) return;
    float s = 0.f;
    for (int b = 0; b < blocks; b++) s += partial[(size_t)b * (OK + O) + i];
    if (i < OK)
        grad[w_off + i] = s;
    else
        grad[b_off + (i - OK)] = s;
}

// ------------------------------------------------------------ output ------
// raw = W4 h + b4; pred = d + 0.25 tanh(raw) for both heads.
__global__ void k_output(int N, const float *__restrict__ h, const __nv_bfloat16 *__restrict__ W4,
                         const float *__restrict__ b4, const float2 *__restrict__ base, float4 *__restrict__ raw,
                         float4 *__restrict__ pred) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    float r[kOut];
#pragma unroll
    for (int j = 0; j < kOut; j++) r[j] = b4[j];
    const float4 *hc = reinterpret_cast<const float4 *>(h + (size_t)c * kH);
    float4 x4[kH / 4];
#pragma unroll
    for (int k4 = 0; k4 < kH / 4; k4++) x4[k4] = __ldg(hc + k4);  // the whole row in flight
#pragma unroll
    for (int k4 = 0; k4 < kH / 4; k4++) {
        const float x[4] = {x4[k4].x, x4[k4].y, x4[k4].z, x4[k4].w};
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < kOut; j++) r[j] = fmaf(x[i], bf(W4[j * kH + 4 * k4 + i]), r[j]);
    }
    raw[c] = make_float4(r[0], r[1], r[2], r[3]);
    const float2 b = base[c];
    pred[c] = make_float4(b.x + kCorr * tanhf(r[0]), b.y + kCorr * tanhf(r[1]), b.x + kCorr * tanhf(r[2]),
                          b.y + kCorr * tanhf(r[3]));
}

// Loss: the squared errors of both heads over the movable nodes, divided by
// 2 nn (per-block partials), and d loss / d raw.
__global__ void k_loss(int N, int nn, const float4 *__restrict__ raw, const float4 *__restrict__ pred,
                       const float4 *__restrict__ target, float4 *__restrict__ dout, double *__restrict__ part) {
    __shared__ double sh[kT / 32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (c < N) {
        float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < nn) {
            const float4 p = pred[c], t = target[c], r = raw[c];
            const float e[4] = {p.x - t.x, p.y - t.y, p.z - t.z, p.w - t.w};
            const float rr[4] = {r.x, r.y, r.z, r.w};
            float dd[4];
            const float s = 1.f / (float)nn;  // d/dp of e^2 / (2 nn)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                l += (double)e[j] * e[j];
                const float th = tanhf(rr[j]);
                dd[j] = s * e[j] * kCorr * (1.f - th * th);
            }
            d = make_float4(dd[0], dd[1], dd[2], dd[3]);
        }
        dout[c] = d;
    }
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kT / 32; w++) s += sh[w];
        part[blockIdx.x] = s;
    }
}

__global__ void k_sum_loss(int n, const double *__restrict__ part, int nn, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; i++) s += part[i];
    out[0] = s / (2.0 * nn);
}

// dh[c][k] = sum_j dout[c][j] W4[j][k]
__global__ void k_output_dh(int N, const float4 *__restrict__ dout, const __nv_bfloat16 *__restrict__ W4,
                            float *__restrict__ dh) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)N * kH) return;
    const int c = (int)(i / kH), k = (int)(i % kH);
    const float4 d = dout[c];
    dh[i] = d.x * bf(W4[k]) + d.y * bf(W4[kH + k]) + d.z * bf(W4[2 * kH + k]) + d.w * bf(W4[3 * kH + k]);
}

// -------------------------------------------------------------- adam ------
__global__ void k_adam(int n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float c1, float c2, __nv_bfloat16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi, vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_to_bf16(int n, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// proposal: the movable nodes at q + alpha (f - q), in core units
__global__ void k_propose(int nn, const float4 *__restrict__ pred, float alpha, float llx, float lly, float w,
                          float h, float2 *__restrict__ xy) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    const float4 p = pred[c];
    const float x = fminf(fmaxf(p.x + alpha * (p.z - p.x), 0.f), 1.f);
    const float y = fminf(fmaxf(p.y + alpha * (p.w - p.y), 0.f), 1.f);
    xy[c] = make_float2(llx + x * w, lly + y * h);
}

}  // namespace
}  // namespace ep

using namespace ep;

// Workspace of the network, grown to the largest netlist bound so far, and
// the netlist it currently holds features of.
struct ep_gnn {
    int device = 0;
    std::string err;
    float *w = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16 *wb = nullptr;
    float *wt = nullptr;  // the input layer's weights as FP32 [k][o] (k_transpose_w)
    int *tc_flag_h = nullptr, *tc_flag_d = nullptr;  // mapped: EP_ERR_TIMEOUT bit of the tensor-core layers
    unsigned tc_wait_limit = tc::kWaitLimit;          // polls of their mbarrier wait (ep_gnn_set_wait_limit)
    int sms = 148;
    double *loss = nullptr;
    int64_t step = 0;
    // bound netlist
    uint64_t uid = 0;         // 0: none
    bool pads_ready = false;  // terminal pin lists uploaded (training)
    Net net{};
    EngineGraph eg{};
    // capacities and buffers
    size_t capN = 0, capNet = 0, capPad = 0, capT = 0, capP = 0;
    float *X = nullptr, *inv_pins = nullptr, *inv_deg = nullptr;
    float2 *v = nullptr, *netv = nullptr;
    int *padcnt = nullptr;
    int32_t *pad_start = nullptr, *pad_net = nullptr;
    int4 *kinfo = nullptr;
    int32_t *pin_node = nullptr, *q_net = nullptr;
    float *h[kLayers + 1] = {}, *m[kLayers + 1] = {};
    float *a = nullptr, *dh = nullptr, *dx = nullptr, *dm = nullptr, *da = nullptr, *partial = nullptr;
    float4 *raw = nullptr, *pred = nullptr, *dout = nullptr, *target = nullptr;
    float2 *xy = nullptr;
    double *loss_part = nullptr;
    std::vector<void *> ws;  // workspace allocations (freed on growth)
    ep_gnn() { err.reserve(256); }
};

namespace {

#define GK(call)                                                                  \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess) {                                                  \
            g->err = std::string(#call) + ": " + cudaGetErrorString(_e);          \
            return EP_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)

size_t smem_dense(int K) { return sizeof(float) * ((size_t)K * kH + (size_t)kDenseRows * (K + 1)); }
size_t smem_dx(int K) { return sizeof(float) * ((size_t)kH * K + 64 * (size_t)(kH + 1)); }

void set_smem_attrs() {
    static std::vector<int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    done.push_back(dev);
    cudaFuncSetAttribute(k_dense<kF, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dense(kF));
    cudaFuncSetAttribute(k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    cudaFuncSetAttribute(k_dense_dx<kH, kH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dx(2 * kH));
}

template <typename T>
bool walloc(ep_gnn *g, T *&p, size_t n) {
    if (cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
        p = nullptr;
        return false;
    }
    g->ws.push_back(p);
    return true;
}

// Grow the workspace to hold N nodes, nnet nets, nt terminals and np pins.
ep_status reserve(ep_gnn *g, size_t N, size_t nnet, size_t nt, size_t np) {
    if (N <= g->capN && nnet <= g->capNet && nt <= g->capT && np <= g->capP) return EP_OK;
    cudaDeviceSynchronize();
    for (void *p : g->ws) cudaFree(p);
    g->ws.clear();
    g->uid = 0;
    g->pads_ready = false;
    g->capPad = 0;
    g->pad_net = nullptr;
    // a quarter of headroom on every dimension, so designs of about the same
    // size do not each grow the workspace again (a growth frees and
    // reallocates all of it)
    auto grow = [](size_t want, size_t cap) { return std::max(want + want / 4, cap); };
    N = grow(N, g->capN);
    nnet = grow(nnet, g->capNet);
    nt = grow(nt, g->capT);
    np = grow(np, g->capP);
    bool ok = walloc(g, g->X, N * kF) && walloc(g, g->inv_pins, N) && walloc(g, g->inv_deg, nnet) &&
              walloc(g, g->v, N) && walloc(g, g->netv, nnet) && walloc(g, g->padcnt, nt) &&
              walloc(g, g->pad_start, nt + 1) && walloc(g, g->a, nnet * kH) && walloc(g, g->dh, N * kH) &&
              walloc(g, g->dx, N * kH) && walloc(g, g->dm, N * kH) && walloc(g, g->da, nnet * kH) &&
              walloc(g, g->partial, (size_t)nblk((long long)N, kRowsPerBlock) * (kH * 2 * kH + kH)) &&
              walloc(g, g->raw, N) && walloc(g, g->pred, N) && walloc(g, g->dout, N) && walloc(g, g->target, N) &&
              walloc(g, g->xy, N) && walloc(g, g->loss_part, nblk((long long)N)) && walloc(g, g->kinfo, nnet) &&
              walloc(g, g->pin_node, np) && walloc(g, g->q_net, np);
    for (int l = 0; l <= kLayers && ok; l++) ok = walloc(g, g->h[l], N * kH) && walloc(g, g->m[l], N * kH);
    if (!ok) {
        g->capN = g->capNet = g->capT = g->capP = 0;
        g->err = "cudaMalloc failed for the network's workspace";
        return EP_ERR_NOMEM;
    }
    g->capN = N;
    g->capNet = nnet;
    g->capT = nt;
    g->capP = np;
    return EP_OK;
}

// Bind an engine's netlist: its device arrays, the features (computed on the
// engine's stream) -- skipped when the workspace already holds them.
ep_status bind(ep_gnn *g, ep_engine *e) {
    EngineGraph eg{};
    if (engine_graph(e, &eg)) return EP_ERR_ARG;
    if (eg.nn <= 0 || eg.nnet <= 0) {
        g->err = "the network needs movable nodes and nets";
        return EP_ERR_ARG;
    }
    if (eg.device != g->device) {
        g->err = "the engine lives on another device than the network";
        return EP_ERR_ARG;
    }
    if (g->uid == eg.uid) {
        g->eg = eg;
        return EP_OK;
    }
    set_smem_attrs();
    const int N = eg.nn + eg.nt;
    ep_status s = reserve(g, N, eg.nnet, eg.nt, eg.np);
    if (s) return s;
    g->eg = eg;
    g->pads_ready = false;
    Net &n = g->net;
    n.nn = eg.nn;
    n.n_obj = eg.n_obj;
    n.N = N;
    n.nnet = eg.nnet;
    n.owner = eg.d_pin_owner;
    n.net_first = eg.d_net_first;
    n.net_deg = eg.d_net_deg;
    n.pin_net = eg.d_pin_net;
    n.obj_pin_start = eg.d_obj_pin_start;
    n.obj_pin_dev = eg.d_obj_pin_dev;
    n.net_order = eg.d_net_dev_order;
    n.n_big = eg.n_big_nets;
    n.pad_start = g->pad_start;
    n.pad_net = g->pad_net;
    n.kinfo = g->kinfo;
    n.pin_node = g->pin_node;
    n.q_net = g->q_net;
    cudaStream_t st = eg.st;
    if (eg.fp64)
        k_init<double><<<nblk(N), kT, 0, st>>>(n, eg.d_area, eg.d_npins, (const double2 *)eg.d_pos, eg.grid, g->X,
                                                g->v, g->inv_pins);
    else
        k_init<float><<<nblk(N), kT, 0, st>>>(n, eg.d_area, eg.d_npins, (const float2 *)eg.d_pos, eg.grid, g->X,
                                               g->v, g->inv_pins);
    if (eg.nt > 0) {
        GK(cudaMemsetAsync(g->padcnt, 0, sizeof(int) * eg.nt, st));
        k_pad_pins<<<nblk(eg.np), kT, 0, st>>>(eg.np, n, g->padcnt);
        k_pad_feature<<<nblk(eg.nt), kT, 0, st>>>(eg.nt, eg.nn, g->padcnt, g->X);
    }
    k_inv_deg<<<nblk(eg.nnet), kT, 0, st>>>(eg.nnet, eg.d_net_deg, g->inv_deg);
    k_graph_index<<<nblk(std::max(eg.nnet, eg.np)), kT, 0, st>>>(n, eg.np, g->kinfo, g->pin_node, g->q_net);
    int col = 3;
    for (int k = 1; k <= kDiffSteps[2]; k++) {
        // programmatic serialisation: the next pass's blocks wait resident
        launch_k(k_diff_net, nblk(31LL * n.n_big + eg.nnet), kT, 0, st, n, (const float2 *)g->v, g->netv);
        launch_k(k_diff_node, nblk(eg.nn), kT, 0, st, n, (const float *)g->inv_pins, (const float2 *)g->netv, g->v);
        if (k == kDiffSteps[0] || k == kDiffSteps[1] || k == kDiffSteps[2]) {
            launch_k(k_store_feature, nblk(N), kT, 0, st, N, (const float2 *)g->v, g->X, col);
            col += 2;
        }
    }
    GK(cudaGetLastError());
    g->uid = eg.uid;
    return EP_OK;
}

// The terminals' pin lists (the transposed aggregation into terminals needs
// them; training only), built on the host from the engine's pin owners.
ep_status bind_pads(ep_gnn *g) {
    if (g->pads_ready) return EP_OK;
    const EngineGraph &eg = g->eg;
    std::vector<int32_t> start(eg.nt + 1, 0), nets;
    for (int p = 0; p < eg.np; p++)
        if (eg.pin_owner[p] >= eg.n_obj) start[eg.pin_owner[p] - eg.n_obj + 1]++;
    for (int t = 0; t < eg.nt; t++) start[t + 1] += start[t];
    nets.resize(std::max(start[eg.nt], 1));
    {
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (int p = 0; p < eg.np; p++)
            if (eg.pin_owner[p] >= eg.n_obj) nets[fill[eg.pin_owner[p] - eg.n_obj]++] = eg.pin_net[p];
    }
    if (nets.size() > g->capPad) {
        if (g->pad_net) {
            cudaStreamSynchronize(eg.st);
            cudaFree(g->pad_net);
            g->ws.erase(std::find(g->ws.begin(), g->ws.end(), (void *)g->pad_net));
            g->pad_net = nullptr;
        }
        if (!walloc(g, g->pad_net, nets.size())) {
            g->capPad = 0;
            g->err = "cudaMalloc failed for the terminals' pin lists";
            return EP_ERR_NOMEM;
        }
        g->capPad = nets.size();
    }
    GK(cudaMemcpyAsync(g->pad_start, start.data(), sizeof(int32_t) * start.size(), cudaMemcpyHostToDevice, eg.st));
    GK(cudaMemcpyAsync(g->pad_net, nets.data(), sizeof(int32_t) * nets.size(), cudaMemcpyHostToDevice, eg.st));
    GK(cudaStreamSynchronize(eg.st));  // the host vectors go out of scope
    g->net.pad_start = g->pad_start;
    g->net.pad_net = g->pad_net;
    g->pads_ready = true;
    return EP_OK;
}

// A give-up of the tensor-core layers' wait since the last check, reported
// once (the flag is mapped host memory the kernel writes).
ep_status tc_give_up(ep_gnn *g) {
    if (!*(volatile int *)g->tc_flag_h) return EP_OK;
    *(volatile int *)g->tc_flag_h = 0;
    g->err = "a bounded wait of the tensor-core dense layers gave up";
    return EP_ERR_TIMEOUT;
}

// Forward pass on the bound netlist (activations kept for the backward pass).
ep_status forward(ep_gnn *g) {
    const Net &n = g->net;
    const int N = n.N;
    cudaStream_t st = g->eg.st;
    const float *w = g->w;
    const __nv_bfloat16 *wb = g->wb;
    if (ep_status s = tc_give_up(g)) return s;  // of an earlier (asynchronous) pass
    const int tc_grid = std::max(1, std::min((N + kTcRows - 1) / kTcRows, 2 * g->sms));
    k_dense<kF, 0><<<nblk(N, kDenseRows), kT, smem_dense(kF), st>>>(N, g->X, nullptr, g->wt, w + kOffB0,
                                                                    g->h[0]);
    for (int l = 1; l <= kLayers; l++) {
        k_net_mean<<<n.n_big + nblk(n.nnet - n.n_big, kBigWarps), kT, 0, st>>>(n, (const float2 *)g->h[l - 1],
                                                                (float2 *)g->a);
        k_node_mean<<<nblk((long long)N * 32), kT, 0, st>>>(n, g->inv_pins, (const float2 *)g->a, (float2 *)g->m[l]);
        launch_dense_tc(tc_grid, st, N, g->h[l - 1], g->m[l], wb + off_w(l), w + off_b(l), g->h[l], g->tc_flag_d,
                        g->eg.d_status, g->tc_wait_limit);
    }
    k_output<<<nblk(N), kT, 0, st>>>(N, g->h[kLayers], wb + kOffW4, w + kOffB4, g->v, g->raw, g->pred);
    GK(cudaGetLastError());
    return EP_OK;
}

// Loss against g->target and the gradient of every parameter into g->grad.
ep_status backward(ep_gnn *g) {
    const Net &n = g->net;
    const int N = n.N;
    cudaStream_t st = g->eg.st;
    const __nv_bfloat16 *wb = g->wb;
    const int lb = nblk(N);
    k_loss<<<lb, kT, 0, st>>>(N, n.nn, g->raw, g->pred, g->target, g->dout, g->loss_part);
    k_sum_loss<<<1, 32, 0, st>>>(lb, g->loss_part, n.nn, g->loss);
    const int pb = nblk(N, kRowsPerBlock);
    // output layer
    k_dweight<kOut, kH, 0><<<pb, kT, 0, st>>>(N, kRowsPerBlock, (const float *)g->dout, nullptr, g->h[kLayers],
                                             nullptr, g->partial);
    k_reduce_partials<<<nblk(kOut * kH + kOut), kT, 0, st>>>(pb, kOut * kH, kOut, g->partial, g->grad, kOffW4,
                                                             kOffB4);
    k_output_dh<<<nblk((long long)N * kH), kT, 0, st>>>(N, g->dout, wb + kOffW4, g->dh);
    // message-passing layers, last to first; dh holds d loss / d h_l
    float *dh = g->dh, *dx = g->dx;
    for (int l = kLayers; l >= 1; l--) {
        k_dweight<kH, kH, kH><<<pb, kT, 0, st>>>(N, kRowsPerBlock, dh, g->h[l], g->h[l - 1], g->m[l], g->partial);
        k_reduce_partials<<<nblk(kH * 2 * kH + kH), kT, 0, st>>>(pb, kH * 2 * kH, kH, g->partial, g->grad, off_w(l),
                                                                 off_b(l));
        // d h_{l-1} (direct part) into dx, d m_l into g->dm
        k_dense_dx<kH, kH><<<nblk(N, 64), kT, smem_dx(2 * kH), st>>>(N, dh, g->h[l], wb + off_w(l), dx, g->dm);
        k_node_mean_t<<<nblk((long long)n.nnet * 32), kT, 0, st>>>(n, g->inv_pins, (const float2 *)g->dm,
                                                                   (float2 *)g->da);
        k_net_mean_t_add<<<nblk((long long)N * 32), kT, 0, st>>>(n, g->inv_deg, (const float2 *)g->da,
                                                                 (float2 *)dx);
        std::swap(dh, dx);
    }
    // input layer
    k_dweight<kH, kF, 0><<<pb, kT, 0, st>>>(N, kRowsPerBlock, dh, g->h[0], g->X, nullptr, g->partial);
    k_reduce_partials<<<nblk(kH * kF + kH), kT, 0, st>>>(pb, kH * kF, kH, g->partial, g->grad, kOffW0, kOffB0);
    GK(cudaGetLastError());
    return EP_OK;
}

// Targets of the movable nodes: [nn][4] core coordinates (quadratic
// placement x, y, final x, y), normalised to the core.
ep_status upload_target(ep_gnn *g, const float *t4) {
    const Grid &gr = g->eg.grid;
    const float W = gr.urx - gr.llx, H = gr.ury - gr.lly;
    std::vector<float4> t(g->net.N, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int c = 0; c < g->net.nn; c++)
        t[c] = make_float4((t4[4 * c] - gr.llx) / W, (t4[4 * c + 1] - gr.lly) / H, (t4[4 * c + 2] - gr.llx) / W,
                           (t4[4 * c + 3] - gr.lly) / H);
    GK(cudaMemcpyAsync(g->target, t.data(), sizeof(float4) * t.size(), cudaMemcpyHostToDevice, g->eg.st));
    GK(cudaStreamSynchronize(g->eg.st));
    return EP_OK;
}

ep_status oom(ep_gnn *g) {
    g->err.assign("out of host memory");
    return EP_ERR_NOMEM;
}

}  // namespace

extern "C" {

int32_t ep_gnn_num_weights(void) { return kParams; }

const char *ep_gnn_last_error(const ep_gnn *g) { return g ? g->err.c_str() : "null network"; }

ep_status ep_gnn_create(int32_t device, uint64_t seed, ep_gnn **out) try {
    if (!out) return EP_ERR_ARG;
    *out = nullptr;
    ep_gnn *g = new ep_gnn();
    *out = g;
    g->device = device;
    GK(cudaSetDevice(device));
    if (cudaMalloc(&g->w, sizeof(float) * kParams) != cudaSuccess ||
        cudaMalloc(&g->grad, sizeof(float) * kParams) != cudaSuccess ||
        cudaMalloc(&g->adam_m, sizeof(float) * kParams) != cudaSuccess ||
        cudaMalloc(&g->adam_v, sizeof(float) * kParams) != cudaSuccess ||
        cudaMalloc(&g->wb, sizeof(__nv_bfloat16) * kParams) != cudaSuccess ||
        cudaMalloc(&g->wt, sizeof(float) * kWtSize) != cudaSuccess ||
        cudaMalloc(&g->loss, sizeof(double)) != cudaSuccess ||
        cudaHostAlloc(&g->tc_flag_h, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&g->tc_flag_d, g->tc_flag_h, 0) != cudaSuccess) {
        g->err = "cudaMalloc failed for the network's weights";
        return EP_ERR_NOMEM;
    }
    *g->tc_flag_h = 0;
    cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, device);
    // Glorot-uniform weights, zero biases; the output layer starts small so
    // the first predictions stay near the diffusion coordinates
    std::vector<float> w(kParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols, float gain) {
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        const float a = gain * std::sqrt(6.f / (float)(rows + cols));
        for (int i = 0; i < rows * cols; i++) w[off + i] = a * u(rng);
    };
    fill(kOffW0, kH, kF, 1.f);
    for (int l = 1; l <= kLayers; l++) fill(off_w(l), kH, 2 * kH, 1.f);
    fill(kOffW4, kOut, kH, 0.1f);
    return ep_gnn_set_weights(g, w.data());
} catch (const std::bad_alloc &) {
    return EP_ERR_NOMEM;
}

void ep_gnn_destroy(ep_gnn *g) {
    if (!g) return;
    cudaDeviceSynchronize();
    for (void *p : g->ws) cudaFree(p);
    for (void *p : {(void *)g->w, (void *)g->grad, (void *)g->adam_m, (void *)g->adam_v, (void *)g->wb,
                    (void *)g->wt, (void *)g->loss})
        if (p) cudaFree(p);
    if (g->tc_flag_h) cudaFreeHost(g->tc_flag_h);
    delete g;
}

ep_status ep_gnn_get_weights(ep_gnn *g, float *w) {
    if (!g || !w) return EP_ERR_ARG;
    GK(cudaMemcpy(w, g->w, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    return EP_OK;
}

ep_status ep_gnn_set_weights(ep_gnn *g, const float *w) {
    if (!g || !w) return EP_ERR_ARG;
    GK(cudaMemcpy(g->w, w, sizeof(float) * kParams, cudaMemcpyHostToDevice));
    GK(cudaMemset(g->adam_m, 0, sizeof(float) * kParams));
    GK(cudaMemset(g->adam_v, 0, sizeof(float) * kParams));
    k_to_bf16<<<nblk(kParams), kT>>>(kParams, g->w, g->wb);
    k_transpose_w<<<nblk(kWtSize), kT>>>(g->wb, g->wt);
    GK(cudaGetLastError());
    GK(cudaDeviceSynchronize());
    g->step = 0;
    return EP_OK;
}

ep_status ep_gnn_release(ep_gnn *g, ep_engine *e) {
    if (!g || !e) return EP_ERR_ARG;
    EngineGraph eg{};
    if (engine_graph(e, &eg)) return EP_ERR_ARG;
    if (g->uid == eg.uid) g->uid = 0;
    return EP_OK;
}

ep_status ep_gnn_features(ep_gnn *g, ep_engine *e, float *X) {
    if (!g || !e || !X) return EP_ERR_ARG;
    ep_status s = bind(g, e);
    if (s) return s;
    GK(cudaMemcpyAsync(X, g->X, sizeof(float) * (size_t)g->net.N * kF, cudaMemcpyDeviceToHost, g->eg.st));
    GK(cudaStreamSynchronize(g->eg.st));
    return EP_OK;
}

ep_status ep_gnn_forward(ep_gnn *g, ep_engine *e, float *xy4) try {
    if (!g || !e || !xy4) return EP_ERR_ARG;
    ep_status s = bind(g, e);
    if (s || (s = forward(g))) return s;
    const int nn = g->net.nn;
    std::vector<float4> p(nn);
    GK(cudaMemcpyAsync(p.data(), g->pred, sizeof(float4) * nn, cudaMemcpyDeviceToHost, g->eg.st));
    GK(cudaStreamSynchronize(g->eg.st));
    if ((s = tc_give_up(g))) return s;
    const Grid &gr = g->eg.grid;
    const float W = gr.urx - gr.llx, H = gr.ury - gr.lly;
    for (int c = 0; c < nn; c++) {
        xy4[4 * c] = gr.llx + p[c].x * W;
        xy4[4 * c + 1] = gr.lly + p[c].y * H;
        xy4[4 * c + 2] = gr.llx + p[c].z * W;
        xy4[4 * c + 3] = gr.lly + p[c].w * H;
    }
    return EP_OK;
} catch (const std::bad_alloc &) {
    return oom(g);
}

ep_status ep_gnn_loss_grad(ep_gnn *g, ep_engine *e, const float *target4, double *loss, float *grad) try {
    if (!g || !e || !target4) return EP_ERR_ARG;
    ep_status s = bind(g, e);
    if (s || (s = bind_pads(g)) || (s = upload_target(g, target4)) || (s = forward(g)) || (s = backward(g)))
        return s;
    if (loss) GK(cudaMemcpyAsync(loss, g->loss, sizeof(double), cudaMemcpyDeviceToHost, g->eg.st));
    if (grad) GK(cudaMemcpyAsync(grad, g->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, g->eg.st));
    GK(cudaStreamSynchronize(g->eg.st));
    return tc_give_up(g);
} catch (const std::bad_alloc &) {
    return oom(g);
}

ep_status ep_gnn_train_step(ep_gnn *g, ep_engine *e, const float *target4, float lr, double *loss) try {
    if (!g || !e || !target4 || !(lr > 0)) return EP_ERR_ARG;
    ep_status s = bind(g, e);
    if (s || (s = bind_pads(g)) || (s = upload_target(g, target4)) || (s = forward(g)) || (s = backward(g)))
        return s;
    g->step++;
    const float c1 = 1.f / (1.f - std::pow(0.9f, (float)g->step)), c2 = 1.f / (1.f - std::pow(0.999f, (float)g->step));
    k_adam<<<nblk(kParams), kT, 0, g->eg.st>>>(kParams, g->w, g->grad, g->adam_m, g->adam_v, lr, c1, c2, g->wb);
    k_transpose_w<<<nblk(kWtSize), kT, 0, g->eg.st>>>(g->wb, g->wt);
    GK(cudaGetLastError());
    if (loss) GK(cudaMemcpyAsync(loss, g->loss, sizeof(double), cudaMemcpyDeviceToHost, g->eg.st));
    GK(cudaStreamSynchronize(g->eg.st));
    return tc_give_up(g);
} catch (const std::bad_alloc &) {
    return oom(g);
}

ep_status ep_gnn_set_wait_limit(ep_gnn *g, int32_t polls) {
    if (!g) return EP_ERR_ARG;
    g->tc_wait_limit = polls < 0 ? tc::kWaitLimit : (unsigned)polls;
    return EP_OK;
}

ep_status ep_gnn_propose(ep_gnn *g, ep_engine *e, float alpha) {
    if (!g || !e || !(alpha >= 0.f) || alpha > 1.f) return EP_ERR_ARG;
    ep_status s = bind(g, e);
    if (s || (s = forward(g))) return s;
    const Grid &gr = g->eg.grid;
    k_propose<<<nblk(g->net.nn), kT, 0, g->eg.st>>>(g->net.nn, g->pred, alpha, gr.llx, gr.lly, gr.urx - gr.llx,
                                                    gr.ury - gr.lly, g->xy);
    GK(cudaGetLastError());
    if (engine_set_node_centres(e, g->xy)) {
        g->err = "setting the proposed positions failed";
        return EP_ERR_CUDA;
    }
    return EP_OK;
}

}  // extern "C"
