// dct_tc.cu -- the four DCT GEMMs of dct.cu on the tcgen05 tensor cores.
//
// Every operand is stored as two bf16 planes, hi = bf16(v) and
// lo = bf16(v - hi); a product is formed from three MMAs
// (hi*hi + hi*lo + lo*hi) accumulated in FP32 in tensor memory, which keeps
// ~2^-17 relative accuracy per product (3xBF16 split products).
//
// One CTA computes a 128 x BN output tile:
//   warp 0, one thread : TMA producer (cp.async.bulk.tensor, 128B swizzle)
//                        into a kStages-deep shared-memory ring
//   warp 1, one thread : MMA issuer (tcgen05.mma.cta_group::1.kind::f16,
//                        A and B from shared-memory descriptors, D in TMEM);
//                        warp 1 also allocates / frees the TMEM columns
//   warps 0-3          : epilogue, tcgen05.ld of their 32 TMEM lanes, then
//                        the GEMM's store, always transposed (lane-contiguous):
//                        bf16 hi/lo planes, optionally spectrally scaled, or
//                        the FP32 field
// Every wait on an mbarrier is bounded; a wait that gives up raises the
// EP_ERR_TIMEOUT bit in DevScalars::status, the CTA drains what it issued,
// frees its TMEM and returns.  No TMA multicast is used.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.h"
#include "tc_ptx.cuh"

namespace ep {

namespace {

constexpr int kBM = 128;            // UMMA M (TMEM lanes)
constexpr int kBN = 64;             // UMMA N (TMEM columns)
constexpr int kBK = 64;             // bf16 elements per 128-byte swizzle row
constexpr int kStages = 3;
constexpr int kATile = kBM * kBK * 2;   // 16 KiB
constexpr int kBTile = kBN * kBK * 2;   // 8 KiB
constexpr int kStageBytes = 2 * kATile + 2 * kBTile;
// split-K reduction slots, [split][kBM][kBN / split + 4] floats (largest at split 4)
constexpr int kRedBytes = 4 * kBM * (kBN / 4 + 4) * 4;
constexpr int kSmemBytes = kStages * kStageBytes + kRedBytes + 1024 /*barriers*/ + 1024 /*alignment*/;
constexpr int kThreads = 128;
using namespace tc;

enum TcEpi { kTcTransposed = 0, kTcSpectral = 1, kTcField = 2 };

struct TcGemmParams {
    CUtensorMap a_hi[3], a_lo[3], b_hi[3], b_lo[3];
    int M, N, K;
    int split;                  // CTAs per cluster sharing one tile (split-K), 1 = none
    int b_const;                // B does not depend on the previous grid (loaded before its end)
    int epi;
    uint16_t *out_hi, *out_lo;  // bf16 planes (kTcTransposed / kTcSpectral)
    int ldo;
    const float *kscale;        // spectral scale, laid out like the output
    float2 *field;              // kTcField, batches 0 (x) and 1 (y)
    float *phi;                 // kTcField, batch 2
    unsigned wait_limit;        // try_wait rounds of a pipeline wait before it gives up
};

// Output store of one accumulator value: C[m][n] -> out[n * ldo + m].
__device__ __forceinline__ void store_out(const TcGemmParams &p, int bz, int n, int m, float v) {
    const size_t o = (size_t)n * p.ldo + m;
    if (p.epi == kTcField) {
        if (bz == 0)
            p.field[o].x = v;
        else if (bz == 1)
            p.field[o].y = v;
        else
            p.phi[o] = v;
    } else {
        uint16_t hi, lo;
        bf16_split(v, hi, lo);
        p.out_hi[o] = hi;
        p.out_lo[o] = lo;
    }
}

template <int SPLIT>
__global__ void __launch_bounds__(kThreads, 1)
k_umma_nt(const __grid_constant__ TcGemmParams p, DevScalars *__restrict__ S) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // S->done is final before this grid starts: only the update kernel writes
    // it, and that grid completed before the previous grid passed its own
    // wait.  The check is uniform over the grid, so no cluster member is left
    // waiting; the early exit still waits for the previous grid first.
    if (S && S->done) {
        pdl_begin();
        return;
    }
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    float *red = (float *)(smem + kStages * kStageBytes);  // split-K reduction slots
    uint64_t *full = (uint64_t *)(smem + kStages * kStageBytes + kRedBytes);
    uint64_t *empty = full + kStages;
    uint64_t *done = empty + kStages;
    volatile uint32_t *tmem_slot = (volatile uint32_t *)(done + 1);
    volatile int *abort = (volatile int *)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bz = blockIdx.z;
    // split-K: the `split` CTAs of a cluster (consecutive in x) share one
    // output tile and take consecutive K ranges
    constexpr int split = SPLIT;
    const int part = blockIdx.x % split;
    const int m0 = blockIdx.y * kBM, n0 = (blockIdx.x / split) * kBN;
    const int nk = p.K / kBK / split, kb0 = part * nk;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32((const void *)tmem_slot)), "r"(kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // Everything above and the B tiles of the first ring stages (B is a
    // constant DCT table in all four GEMMs) overlap the previous grid; the A
    // tiles are its output, so they are loaded after the wait.
    const int pre = p.b_const ? (nk < kStages ? nk : kStages) : 0;
    if (threadIdx.x == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.a_hi[bz]) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.a_lo[bz]) : "memory");
        for (int kb = 0; kb < pre; kb++) {
            uint8_t *st = smem + kb * kStageBytes;
            const int kc = (kb0 + kb) * kBK;
            mbar_expect_tx(&full[kb], kStageBytes);
            tma_load_2d(st + 2 * kATile, &p.b_hi[bz], &full[kb], kc, n0);
            tma_load_2d(st + 2 * kATile + kBTile, &p.b_lo[bz], &full[kb], kc, n0);
        }
    }
    pdl_begin();

    int issued = pre;  // TMA stages thread 0 has issued (drained on an abort)
    if (threadIdx.x == 0) {
        // ---- TMA producer ----
        for (int kb = 0; kb < pre; kb++) {
            uint8_t *st = smem + kb * kStageBytes;
            const int kc = (kb0 + kb) * kBK;
            tma_load_2d(st, &p.a_hi[bz], &full[kb], kc, m0);
            tma_load_2d(st + kATile, &p.a_lo[bz], &full[kb], kc, m0);
        }
        for (int kb = pre; kb < nk; kb++) {
            int s = kb % kStages, use = kb / kStages;
            if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1, abort, p.wait_limit)) break;
            uint8_t *st = smem + s * kStageBytes;
            const int kc = (kb0 + kb) * kBK;
            mbar_expect_tx(&full[s], kStageBytes);
            tma_load_2d(st, &p.a_hi[bz], &full[s], kc, m0);
            tma_load_2d(st + kATile, &p.a_lo[bz], &full[s], kc, m0);
            tma_load_2d(st + 2 * kATile, &p.b_hi[bz], &full[s], kc, n0);
            tma_load_2d(st + 2 * kATile + kBTile, &p.b_lo[bz], &full[s], kc, n0);
            issued = kb + 1;
        }
    } else if (threadIdx.x == 32) {
        // ---- MMA issuer ----
        const uint32_t idesc = umma_idesc(kBM, kBN);
        bool ok = true;
        for (int kb = 0; kb < nk && ok; kb++) {
            int s = kb % kStages, use = kb / kStages;
            if (!mbar_wait(&full[s], use & 1, abort, p.wait_limit)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint8_t *st = smem + s * kStageBytes;
            uint32_t ah = smem_u32(st), al = smem_u32(st + kATile);
            uint32_t bh = smem_u32(st + 2 * kATile), bl = smem_u32(st + 2 * kATile + kBTile);
#pragma unroll
            for (int k = 0; k < kBK / 16; k++) {
                uint32_t off = k * 32;  // 16 bf16 = 32 bytes along K inside the swizzle atom
                umma_bf16(tmem, umma_desc(ah + off), umma_desc(bl + off), idesc, (kb | k) != 0);
                umma_bf16(tmem, umma_desc(al + off), umma_desc(bh + off), idesc, 1);
                umma_bf16(tmem, umma_desc(ah + off), umma_desc(bh + off), idesc, 1);
            }
            umma_commit(&empty[s]);
        }
        umma_commit(done);  // also fences the MMAs issued before an abort
    }
    __syncwarp();

    // ---- epilogue: warp w owns TMEM lanes 32w..32w+31 = tile rows ----
    // lane 0 waits, the warp follows its result (tcgen05.ld is warp-aligned).
    // Every GEMM stores its tile transposed, C[m][n] -> out[n * ldo + m], so
    // the 32 lanes of a warp (consecutive m) write consecutive addresses.
    // On an abort, `done` still completes: the issuer commits it after its
    // last MMA on every path, and the CTA waits for it before freeing TMEM.
    int ready = 0;
    if (lane == 0) {
        ready = mbar_wait(done, 0, abort, p.wait_limit) && !*abort;
        if (!ready) mbar_drain(done, 0);
    }
    ready = __shfl_sync(0xffffffffu, ready, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = warp * 32 + lane, m = m0 + row;
    const uint32_t tm_row = tmem + ((uint32_t)(warp * 32) << 16);
    if constexpr (SPLIT == 1) {
        if (ready) {
#pragma unroll 1
            for (int c0 = 0; c0 < kBN; c0 += 16) {
                // spectral scale of these 16 columns, loaded before the
                // stores so the loads do not queue behind them
                float ks[16];
                if (p.epi == kTcSpectral) {
#pragma unroll
                    for (int c = 0; c < 16; c++) ks[c] = __ldg(&p.kscale[(size_t)(n0 + c0 + c) * p.ldo + m]);
                }
                uint32_t r[16];
                tmem_ld16(tm_row + (uint32_t)c0, r);
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    float v = __uint_as_float(r[c]);
                    if (p.epi == kTcSpectral) v *= ks[c];
                    store_out(p, bz, n0 + c0 + c, m, v);
                }
            }
        }
    } else {
        // Split-K reduction.  CTA q of the cluster owns columns
        // [q * kCols, (q + 1) * kCols) of the tile.  Every CTA pushes each
        // 16-column chunk of its FP32 partial straight into the owner's slot
        // for this CTA (remote stores through distributed shared memory, no
        // round trip), one cluster barrier makes them visible, and each CTA
        // then sums its SPLIT slots in rank order (deterministic) from its own
        // shared memory and stores the result.  The slots have their own
        // region, so a peer that finishes early never writes into a stage
        // ring that is still being filled.  The barrier is reached on every
        // path.
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        constexpr int kCols = kBN / (SPLIT > 1 ? SPLIT : 1), kRedLd = kCols + 4;
        if (ready) {
#pragma unroll 1
            for (int c0 = 0; c0 < kBN; c0 += 16) {
                uint32_t r[16];
                tmem_ld16(tm_row + (uint32_t)c0, r);
                const int q = c0 / kCols;  // owner of these 16 columns
                float *dst = cl.map_shared_rank(red, q) + (part * kBM + row) * kRedLd + (c0 - q * kCols);
#pragma unroll
                for (int i = 0; i < 4; i++)
                    *(float4 *)(dst + 4 * i) =
                        make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]),
                                    __uint_as_float(r[4 * i + 2]), __uint_as_float(r[4 * i + 3]));
            }
        }
        cl.sync();
        const int cbeg = part * kCols;
        float ks[kCols];
        if (p.epi == kTcSpectral) {
#pragma unroll
            for (int j = 0; j < kCols; j++) ks[j] = __ldg(&p.kscale[(size_t)(n0 + cbeg + j) * p.ldo + m]);
        }
#pragma unroll
        for (int q4 = 0; q4 < kCols / 4; q4++) {
            float4 v = *(const float4 *)&red[row * kRedLd + 4 * q4];
#pragma unroll
            for (int r = 1; r < SPLIT; r++) {
                const float4 w = *(const float4 *)&red[(r * kBM + row) * kRedLd + 4 * q4];
                v.x += w.x;
                v.y += w.y;
                v.z += w.z;
                v.w += w.w;
            }
            const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int j = 4 * q4 + i;
                if (ready) store_out(p, bz, n0 + cbeg + j, m, p.epi == kTcSpectral ? vv[i] * ks[j] : vv[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // every role is past its last wait, so the abort flag is final: on an
    // abort the loads thread 0 issued may not all have been consumed, and the
    // last one into each stage must land before the CTA exits
    if (threadIdx.x == 0 && *abort)
        for (int kb = issued - kStages > 0 ? issued - kStages : 0; kb < issued; kb++)
            mbar_drain(&full[kb % kStages], (kb / kStages) & 1);
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
    }
    if (threadIdx.x == 0 && *abort && S) atomicOr(&S->status, 1 << EP_ERR_TIMEOUT);
}

// ---- host side ------------------------------------------------------------------
struct TcPlan {
    // bf16 planes (hi, lo contiguous: lo = hi + rows*cols)
    uint16_t *rho = nullptr, *Cy = nullptr, *Cx = nullptr, *Tt = nullptr, *P = nullptr;
    uint16_t *B3 = nullptr, *A4 = nullptr, *T3 = nullptr;
    TcGemmParams g[4];
    int sms = 148;       // SMs of the device
    int max_split = 1;   // largest cluster the GEMM can be launched with
};

// Split-K factor: double it while the grid still fits in one wave and every
// CTA keeps at least one K block.
int pick_split(const TcPlan &t, const TcGemmParams &g, int batch) {
    const int tiles = (g.M / kBM) * (g.N / kBN) * batch, nk = g.K / kBK;
    int s = 1;
    while (s * 2 <= t.max_split && tiles * s * 2 <= t.sms && nk % (s * 2) == 0) s *= 2;
    return s;
}

void launch_tc(const TcGemmParams &g, dim3 grid, DevScalars *S, cudaStream_t st) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[3];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = (unsigned)g.split;
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    attr[2].id = cudaLaunchAttributePriority;
    attr[2].val.priority = launch_priority(true);
    cfg.attrs = attr;
    cfg.numAttrs = 3;
    switch (g.split) {
        case 4: cudaLaunchKernelEx(&cfg, k_umma_nt<4>, g, S); break;
        case 2: cudaLaunchKernelEx(&cfg, k_umma_nt<2>, g, S); break;
        default: cudaLaunchKernelEx(&cfg, k_umma_nt<1>, g, S); break;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool load_encoder(std::string &err) {
    if (g_encode) return true;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        err = "cuTensorMapEncodeTiled is not available from the driver";
        return false;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return true;
}

// Row-major bf16 plane [rows][cols] (cols contiguous = K), box of box_rows x 64.
bool make_map(CUtensorMap *m, const uint16_t *base, int rows, int cols, int box_rows, std::string &err) {
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult rc = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)rc) + ")";
        return false;
    }
    return true;
}

void split_host(const std::vector<float> &v, std::vector<uint16_t> &out) {
    size_t n = v.size();
    out.resize(2 * n);
    for (size_t i = 0; i < n; i++) {
        uint32_t u;
        std::memcpy(&u, &v[i], 4);
        uint32_t r = u + 0x7fffu + ((u >> 16) & 1u);
        uint16_t hi = (uint16_t)(r >> 16);
        uint32_t hu = (uint32_t)hi << 16;
        float hf;
        std::memcpy(&hf, &hu, 4);
        float rem = v[i] - hf;
        uint32_t u2;
        std::memcpy(&u2, &rem, 4);
        out[i] = hi;
        out[n + i] = (uint16_t)((u2 + 0x7fffu + ((u2 >> 16) & 1u)) >> 16);
    }
}

bool upload_planes(uint16_t *&dst, const float *dev_src, size_t n, std::string &err) {
    std::vector<float> h(n);
    if (cudaMemcpy(h.data(), dev_src, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        err = "reading DCT tables failed";
        return false;
    }
    std::vector<uint16_t> s;
    split_host(h, s);
    if (cudaMalloc(&dst, s.size() * 2) != cudaSuccess) {
        err = "cudaMalloc failed for bf16 DCT planes";
        return false;
    }
    return cudaMemcpy(dst, s.data(), s.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace

int dct_tc_init(DctPlan &p, std::string &err) {
    const int nx = p.nx, ny = p.ny;
    if (nx % kBM || ny % kBM || nx % kBK || ny % kBK) {
        err = "tensor-core DCT needs bins_x and bins_y to be multiples of 128";
        return EP_ERR_UNSUPPORTED;
    }
    if (!load_encoder(err)) return EP_ERR_UNSUPPORTED;
    TcPlan *t = new TcPlan();
    p.tc = t;
    const size_t nb = (size_t)nx * ny;
    if (!upload_planes(t->Cy, p.Cy, (size_t)ny * ny, err) || !upload_planes(t->Cx, p.Cx, (size_t)nx * nx, err) ||
        !upload_planes(t->B3, p.B3, (size_t)2 * ny * ny, err) ||
        !upload_planes(t->A4, p.A4, (size_t)2 * nx * nx, err))
        return EP_ERR_NOMEM;
    if (cudaMalloc(&t->rho, 2 * nb * 2) != cudaSuccess || cudaMalloc(&t->Tt, 2 * nb * 2) != cudaSuccess ||
        cudaMalloc(&t->P, 2 * nb * 2) != cudaSuccess || cudaMalloc(&t->T3, 2 * 2 * nb * 2) != cudaSuccess) {
        err = "cudaMalloc failed for bf16 DCT intermediates";
        return EP_ERR_NOMEM;
    }
    auto lo = [](uint16_t *base, size_t n) { return base + n; };
    // G1: Tt[v][x] = sum_y rho[x][y] Cy[v][y]
    TcGemmParams &g1 = t->g[0];
    std::memset(&g1, 0, sizeof(g1));
    g1.M = nx; g1.N = ny; g1.K = ny; g1.epi = kTcTransposed; g1.b_const = 1;
    g1.out_hi = t->Tt; g1.out_lo = lo(t->Tt, nb); g1.ldo = nx;
    bool ok = make_map(&g1.a_hi[0], t->rho, nx, ny, kBM, err) && make_map(&g1.a_lo[0], lo(t->rho, nb), nx, ny, kBM, err) &&
              make_map(&g1.b_hi[0], t->Cy, ny, ny, kBN, err) && make_map(&g1.b_lo[0], lo(t->Cy, (size_t)ny * ny), ny, ny, kBN, err);
    // G2: P[u][v] = K[u][v] sum_x Tt[v][x] Cx[u][x], run as C[v][u] (A = Tt,
    // B = Cx) so the transposed store writes P[u][v]; K has P's layout
    TcGemmParams &g2 = t->g[1];
    std::memset(&g2, 0, sizeof(g2));
    g2.M = ny; g2.N = nx; g2.K = nx; g2.epi = kTcSpectral; g2.b_const = 1;
    g2.out_hi = t->P; g2.out_lo = lo(t->P, nb); g2.ldo = ny; g2.kscale = p.K;
    ok = ok && make_map(&g2.a_hi[0], t->Tt, ny, nx, kBM, err) && make_map(&g2.a_lo[0], lo(t->Tt, nb), ny, nx, kBM, err) &&
         make_map(&g2.b_hi[0], t->Cx, nx, nx, kBN, err) && make_map(&g2.b_lo[0], lo(t->Cx, (size_t)nx * nx), nx, nx, kBN, err);
    // G3: T3[n][u] = sum_v P[u][v] B3[n][v]
    TcGemmParams &g3 = t->g[2];
    std::memset(&g3, 0, sizeof(g3));
    g3.M = nx; g3.N = 2 * ny; g3.K = ny; g3.epi = kTcTransposed; g3.b_const = 1;
    g3.out_hi = t->T3; g3.out_lo = lo(t->T3, 2 * nb); g3.ldo = nx;
    ok = ok && make_map(&g3.a_hi[0], t->P, nx, ny, kBM, err) && make_map(&g3.a_lo[0], lo(t->P, nb), nx, ny, kBM, err) &&
         make_map(&g3.b_hi[0], t->B3, 2 * ny, ny, kBN, err) && make_map(&g3.b_lo[0], lo(t->B3, (size_t)2 * ny * ny), 2 * ny, ny, kBN, err);
    // G4: field[x][y] = sum_u {Ut,Vt}[y][u] A4{x,y}[x][u], run as C[y][x]
    // (A = Ut / Vt, B = A4x / A4y) so the transposed store writes field[x][y];
    // batch 2 = phi (Ut with A4y)
    TcGemmParams &g4 = t->g[3];
    std::memset(&g4, 0, sizeof(g4));
    g4.M = ny; g4.N = nx; g4.K = nx; g4.epi = kTcField; g4.ldo = ny; g4.b_const = 1;
    const size_t a4 = (size_t)2 * nx * nx;  // lo plane offset of A4
    const size_t t3 = (size_t)2 * nb;       // lo plane offset of T3
    uint16_t *A4x = t->A4, *A4y = t->A4 + (size_t)nx * nx;
    uint16_t *Ut = t->T3, *Vt = t->T3 + nb;
    uint16_t *As[3] = {Ut, Vt, Ut}, *Bs[3] = {A4x, A4y, A4y};
    for (int b = 0; b < 3 && ok; b++)
        ok = make_map(&g4.a_hi[b], As[b], ny, nx, kBM, err) && make_map(&g4.a_lo[b], As[b] + t3, ny, nx, kBM, err) &&
             make_map(&g4.b_hi[b], Bs[b], nx, nx, kBN, err) && make_map(&g4.b_lo[b], Bs[b] + a4, nx, nx, kBN, err);
    if (!ok) return EP_ERR_UNSUPPORTED;
    if (cudaFuncSetAttribute(k_umma_nt<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess ||
        cudaFuncSetAttribute(k_umma_nt<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess ||
        cudaFuncSetAttribute(k_umma_nt<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess) {
        err = "cannot raise the dynamic shared memory limit of the tcgen05 GEMM";
        return EP_ERR_CUDA;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&t->sms, cudaDevAttrMultiProcessorCount, dev);
    // largest cluster (<= 4) of which at least one fits on the device
    for (int c = 4; c >= 2; c /= 2) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = kSmemBytes;
        cudaLaunchAttribute a[1];
        a[0].id = cudaLaunchAttributeClusterDimension;
        a[0].val.clusterDim.x = (unsigned)c;
        a[0].val.clusterDim.y = 1;
        a[0].val.clusterDim.z = 1;
        cfg.attrs = a;
        cfg.numAttrs = 1;
        int n = 0;
        cudaError_t q = c == 4 ? cudaOccupancyMaxActiveClusters(&n, k_umma_nt<4>, &cfg)
                               : cudaOccupancyMaxActiveClusters(&n, k_umma_nt<2>, &cfg);
        if (q == cudaSuccess && n > 0) {
            t->max_split = c;
            break;
        }
    }
    cudaGetLastError();  // clear a refused query
    return EP_OK;
}

void dct_tc_free(DctPlan &p) {
    TcPlan *t = (TcPlan *)p.tc;
    if (!t) return;
    for (uint16_t *q : {t->rho, t->Cy, t->Cx, t->Tt, t->P, t->B3, t->A4, t->T3})
        if (q) cudaFree(q);
    delete t;
    p.tc = nullptr;
}

void *dct_tc_rho_planes(DctPlan &p) { return p.tc ? ((TcPlan *)p.tc)->rho : nullptr; }

int dct_tc_run(DctPlan &p, float2 *field, float *phi, const DevScalars *S, cudaStream_t st) {
    TcPlan *t = (TcPlan *)p.tc;
    DevScalars *s = const_cast<DevScalars *>(S);
    for (int i = 0; i < 4; i++) {
        TcGemmParams &g = t->g[i];
        g.wait_limit = p.wait_limit;
        int batch = 1;
        if (i == 3) {
            g.field = field;
            g.phi = phi;
            batch = phi ? 3 : 2;
        }
        g.split = pick_split(*t, g, batch);
        dim3 grid(g.N / kBN * g.split, g.M / kBM, batch);
        launch_tc(g, grid, s, st);
    }
    return EP_OK;
}

}  // namespace ep
