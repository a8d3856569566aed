// kernels.cu -- the per-iteration kernels of the ePlace inner loop.
//
//   scatter   cell/filler -> bin overlap areas as int64 fixed point with
//             atomics: order-independent, so the maps are bit-exact and
//             deterministic (EPlacer_2D::binNodeDensityUpdate,
//             EPlace/eplace.cpp:1029-1133)
//   prep      fixed point -> bin density for the Poisson solve, overflow tau
//             in FP64, the 1/gamma schedule (EPlace/eplace.cpp:438-500,
//             570-580)
//   wirelength  per-net bound pins + HPWL (FP64), WA / LSE exponentials and
//             per-pin gradients (PlaceCommon/objects.cpp:75-144,161-241,
//             248-437); the lambda update owed by the previous step
//             (EPlace/eplace.cpp:846-883)
//   combine   field gather (EPlace/eplace.cpp:599-674), per-object sum of its
//             pin gradients in pin order (:531-549), preconditioned direction
//             (:698-737), FP64 Lipschitz sums and the step / a_k update
//             (Optimization/optutils.hpp:20-35, nesterov.hpp:375-415)
//   update    x_{k+1} = y_k + s g_k, y_{k+1} = x_{k+1} + (a_k-1)/a_{k+1}
//             (x_{k+1}-x_k), clamp into the core (PlaceDB/placedb.cpp:253-288)
//
// Every kernel of the loop returns at once when S->done is set, so a captured
// multi-iteration graph stops doing work after the stop condition.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "engine.h"

namespace ep {

namespace {

constexpr int kThreads = 256;
constexpr int kPinChunk = 128;  // pin gradients a warp of the combine kernel stages per round

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------- scatter --
__device__ __forceinline__ void scatter_one(const Grid &g, const Rect &r, float scale, int i,
                                            int j, double qscale,
                                            unsigned long long *__restrict__ map) {
    float ovl = (float)rect_bin_overlap(g, r, i, j);
    if (ovl == 0.0f) return;
    float c = __fmul_rn(scale, ovl);
    long long q = __double2ll_rn(__dmul_rn((double)c, qscale));
    atomicAdd(&map[(size_t)i * g.ny + j], (unsigned long long)q);
}

// Contribution scale: sx*sy, times the target density for macros
// (EPlace/eplace.cpp:1114-1128, evaluated left to right in float).
__device__ __forceinline__ float contrib_scale(const Rect &r, uint8_t f, float td) {
    float s = __fmul_rn(r.sx, r.sy);
    return (f & kMacro) ? __fmul_rn(s, td) : s;
}

// One object of the thread-per-object path (kBig objects excluded).
__device__ __forceinline__ void scatter_small_object(const Grid &g, float2 p, float2 s, uint8_t f, double qscale,
                                                     unsigned long long *__restrict__ node_q,
                                                     unsigned long long *__restrict__ filler_q) {
    Rect r = object_rect(g, p.x, p.y, s.x, s.y);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    float scale = contrib_scale(r, f, g.td);
    unsigned long long *map = (f & kFiller) ? filler_q : node_q;
    for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++) scatter_one(g, r, scale, i, j, qscale, map);
}

// One kBig object by a whole block, its bins strided over the threads.
__device__ __forceinline__ void scatter_big_object(const Grid &g, float2 p, float2 s, uint8_t f, double qscale,
                                                   unsigned long long *__restrict__ node_q,
                                                   unsigned long long *__restrict__ filler_q) {
    Rect r = object_rect(g, p.x, p.y, s.x, s.y);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    if (i1 < i0 || j1 < j0) return;
    float scale = contrib_scale(r, f, g.td);
    unsigned long long *map = (f & kFiller) ? filler_q : node_q;
    const int wy = j1 - j0 + 1, nb = (i1 - i0 + 1) * wy;
    for (int t = threadIdx.x; t < nb; t += blockDim.x)
        scatter_one(g, r, scale, i0 + t / wy, j0 + t % wy, qscale, map);
}

// Blocks [0, small_blocks): thread per object; the blocks after them: one
// kBig object each.
__global__ void __launch_bounds__(kThreads)
k_scatter(Grid g, const float2 *__restrict__ pos, const float2 *__restrict__ size,
          const uint8_t *__restrict__ flags, int n, int small_blocks, const int32_t *__restrict__ big,
          double qscale, unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q,
          const DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    if ((int)blockIdx.x >= small_blocks) {
        const int o = big[blockIdx.x - small_blocks];
        scatter_big_object(g, pos[o], size[o], flags[o], qscale, node_q, filler_q);
        return;
    }
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const uint8_t f = flags[o];
    if (f & kBig) return;
    scatter_small_object(g, pos[o], size[o], f, qscale, node_q, filler_q);
}

// ------------------------------------------------------------------- prep --
// 1/gamma of wirelengthGradientUpdate (EPlace/eplace.cpp:475-500), in the
// reference's float sequence: 0.125f / binStep, then the tau-dependent factor.
__device__ __forceinline__ void inv_gamma(double tau_d, float sx, float sy, double &gx, double &gy) {
    float tau = (float)tau_d;
    float bx = __fdiv_rn(0.125f, sx), by = __fdiv_rn(0.125f, sy);
    if (tau > 1.0f) {
        bx = (float)((double)bx * 0.1);
        by = (float)((double)by * 0.1);
    } else if (tau < 0.1f) {
        bx = (float)((double)bx * 10.0);
        by = (float)((double)by * 10.0);
    } else {
        float t = (float)(1.0 / pow(10.0, ((double)tau - 0.1) * 20 / 9.0 - 1.0));
        bx = __fmul_rn(bx, t);
        by = __fmul_rn(by, t);
    }
    gx = bx;
    gy = by;
}

__global__ void __launch_bounds__(kThreads)
k_prep(Grid g, unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q,
       const float2 *__restrict__ stat, float *__restrict__ rho, uint16_t *__restrict__ rho_hi,
       uint16_t *__restrict__ rho_lo, float *__restrict__ node_f, float *__restrict__ filler_f,
       int zero, double inv_q, double inv_bin_area, double bin_area, double area_norm,
       double *__restrict__ partials, DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ double sh[32];
    if (S->done) return;
    int nb = g.nx * g.ny;
    double acc[1] = {0.0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        double node = (double)(long long)node_q[k] * inv_q;
        double fill = (double)(long long)filler_q[k] * inv_q;
        float2 st = stat[k];  // (terminal, base)
        // eDensity = node + base + filler + terminal (EPlace/eplace.cpp:576-577)
        double dens = (node + (double)st.y + fill + (double)st.x) * inv_bin_area;
        float d = (float)dens;
        if (rho) rho[k] = d;
        if (rho_hi) {
            // 3xBF16 operand split: hi = bf16(d), lo = bf16(d - hi)
            uint32_t u = __float_as_uint(d);
            uint32_t r = u + 0x7fffu + ((u >> 16) & 1u);
            uint16_t h = (uint16_t)(r >> 16);
            float hf = __uint_as_float((uint32_t)h << 16);
            float rem = d - hf;
            uint32_t u2 = __float_as_uint(rem);
            uint32_t r2 = u2 + 0x7fffu + ((u2 >> 16) & 1u);
            rho_hi[k] = h;
            rho_lo[k] = (uint16_t)(r2 >> 16);
        }
        // overflow counts nodes, terminals and base, not fillers (:438-453)
        double ov = (node + (double)st.x + (double)st.y) * inv_bin_area - (double)g.td;
        if (ov > 0.0) acc[0] += ov * bin_area;
        if (node_f) {
            node_f[k] = (float)node;
            filler_f[k] = (float)fill;
        }
        if (zero) {
            node_q[k] = 0ull;
            filler_q[k] = 0ull;
        }
    }
    if (grid_sum<1>(acc, sh, partials, &S->cnt_prep, gridDim.x, blockIdx.x) && threadIdx.x == 0) {
        {
            double tau = acc[0] / area_norm;
            S->tau = tau;
            if (!isfinite(tau)) S->status |= 1 << EP_ERR_NAN;
            double gx, gy;
            inv_gamma(tau, g.sx, g.sy, gx, gy);
            S->inv_gamma_x = gx;
            S->inv_gamma_y = gy;
        }
    }
}

// ------------------------------------------------------------- wirelength --
struct PinCtx {
    const int32_t *__restrict__ owner;
    const float2 *__restrict__ off;
    const float2 *__restrict__ pos;
};

// Pin::calculateAbsolutePos: centre + offset in float.
__device__ __forceinline__ float2 pin_xy(const PinCtx &c, int p) {
    float2 o = c.off[p];
    float2 q = c.pos[c.owner[p]];
    return make_float2(__fadd_rn(q.x, o.x), __fadd_rn(q.y, o.y));
}

struct NetSums {
    float nmx, dmx, nnx, dnx, nmy, dmy, nny, dny;
};

// Exponential terms of one pin (calcWirelengthWA_2D, objects.cpp:275-332):
// arguments <= -300 make the term zero.
struct PinExp {
    float emx, enx, emy, eny;
};

template <bool EXACT>
__device__ __forceinline__ float term_exp(float a) {
    if (!(a > (float)kNegMaxExp)) return 0.0f;
    return EXACT ? expf(a) : fast_exp(a);
}

template <bool EXACT>
__device__ __forceinline__ PinExp pin_exps(float2 xy, float x1, float x0, float y1, float y0, float igx,
                                           float igy) {
    PinExp e;
    e.emx = term_exp<EXACT>(__fmul_rn(__fsub_rn(xy.x, x1), igx));
    e.enx = term_exp<EXACT>(__fmul_rn(__fsub_rn(x0, xy.x), igx));
    e.emy = term_exp<EXACT>(__fmul_rn(__fsub_rn(xy.y, y1), igy));
    e.eny = term_exp<EXACT>(__fmul_rn(__fsub_rn(y0, xy.y), igy));
    return e;
}

// Add one pin's terms to a running sum set (calcWirelengthWA_2D's sums).
__device__ __forceinline__ void add_terms(float (&s)[8], const PinExp &e, float2 xy) {
    s[0] = __fadd_rn(s[0], __fmul_rn(xy.x, e.emx));
    s[1] = __fadd_rn(s[1], e.emx);
    s[2] = __fadd_rn(s[2], __fmul_rn(xy.x, e.enx));
    s[3] = __fadd_rn(s[3], e.enx);
    s[4] = __fadd_rn(s[4], __fmul_rn(xy.y, e.emy));
    s[5] = __fadd_rn(s[5], e.emy);
    s[6] = __fadd_rn(s[6], __fmul_rn(xy.y, e.eny));
    s[7] = __fadd_rn(s[7], e.eny);
}

// Per-net factors of the gradient: 1 / (sum of exponentials) and the
// exponentially weighted mean coordinate of each of the four terms.  Every
// denominator holds the bound pin's exp(0) = 1, so it is >= 1.
struct NetCoef {
    float rmx, mmx, rnx, mnx, rmy, mmy, rny, mny;
};

__device__ __forceinline__ NetCoef net_coef(const NetSums &s) {
    NetCoef c;
    c.rmx = __frcp_rn(s.dmx);
    c.rnx = __frcp_rn(s.dnx);
    c.rmy = __frcp_rn(s.dmy);
    c.rny = __frcp_rn(s.dny);
    c.mmx = s.nmx * c.rmx;
    c.mnx = s.nnx * c.rnx;
    c.mmy = s.nmy * c.rmy;
    c.mny = s.nny * c.rny;
    return c;
}

// Per-pin gradient of the WA model (objects.cpp:359-415).  The reference's
// (nd * d - dd * n) / d^2 equals e / d * (1 + (x - n / d) / gamma) for the max
// term and e / d * (1 - (x - n / d) / gamma) for the min term; this form
// subtracts the weighted mean from the coordinate before scaling, which
// avoids the cancellation of the expanded quotient (the two agree to the
// reference's own rounding).  A zero exponential (argument <= -300) gives a
// zero term as in the reference.  LSE (:423-437): e / d per term.
template <bool LSE>
__device__ __forceinline__ float2 pin_gradient(const PinExp &e, float2 xy, float igx, float igy,
                                               const NetCoef &c) {
    if (LSE)
        return make_float2(e.emx * c.rmx - e.enx * c.rnx, e.emy * c.rmy - e.eny * c.rny);
    const float gmx = e.emx * c.rmx * fmaf(igx, xy.x - c.mmx, 1.0f);
    const float gnx = e.enx * c.rnx * fmaf(-igx, xy.x - c.mnx, 1.0f);
    const float gmy = e.emy * c.rmy * fmaf(igy, xy.y - c.mmy, 1.0f);
    const float gny = e.eny * c.rny * fmaf(-igy, xy.y - c.mny, 1.0f);
    return make_float2(gmx - gnx, gmy - gny);
}

__device__ __forceinline__ double net_value(const NetSums &s, float x1, float x0, float y1,
                                            float y0, float igx, float igy, bool lse) {
    if (lse)
        return ((double)x1 - x0 + log((double)s.dmx) / igx + log((double)s.dnx) / igx) +
               ((double)y1 - y0 + log((double)s.dmy) / igy + log((double)s.dny) / igy);
    return ((double)s.nmx / s.dmx - (double)s.nnx / s.dnx) + ((double)s.nmy / s.dmy - (double)s.nny / s.dny);
}

// lambda multiplier of updatePenaltyFactor (EPlace/eplace.cpp:849-871).
__device__ __forceinline__ double lambda_multiplier(double cur, double last) {
    double delta = cur - last;
    double m = delta < 0.0 ? 1.05 : pow(1.05, -delta / 350000.0 + 1.0);
    return fmin(fmax(m, 0.95), 1.05);
}

// HPWL finaliser shared by the wirelength kernels.
__device__ void finish_wirelength(DevScalars *S, double hp, double wl) {
    S->wirelength = wl;
    S->hpwl = hp;
    // atomic: the Poisson GEMMs, running beside this pass, may raise a bit too
    if (!isfinite(hp)) atomicOr(&S->status, 1 << EP_ERR_NAN);
    if (S->lambda_pending) {
        S->lambda *= lambda_multiplier(hp, S->last_hpwl);
        S->last_hpwl = hp;
        S->lambda_pending = 0;
    }
    if (S->lambda0_mode) S->last_hpwl = hp;  // penaltyFactorInitilization: lastHPWL = calcHPWL()
}

// Finaliser of the HPWL-only pass (PlaceDB::calcHPWL): mode 0 stores it,
// mode 1 applies updatePenaltyFactor, mode 2 applies it only if one is owed.
__device__ void finish_hpwl(DevScalars *S, double hp, int mode) {
    S->hpwl_query = hp;
    if (mode == 1 || (mode == 2 && S->lambda_pending)) {
        S->lambda *= lambda_multiplier(hp, S->last_hpwl);
        S->last_hpwl = hp;
        S->lambda_pending = 0;
    }
}

// ---- the per-net pass ---------------------------------------------------------
// On the device the nets are ordered by degree and each warp runs one task
// (tasks[w] = degree D, first pin, nets, m):
//   D <= kWarpPins: the task's nets (up to floor(32 / D), all of degree D)
//       sit on lanes s*D .. s*D+D-1, one pin per lane (s = lane * m >> 16,
//       m = ceil(2^16 / D), exact for lanes < 32), and the bound pins and
//       exponential sums are segmented shuffle reductions over those lanes;
//   D >  kWarpPins: one net; the warp strides over its pins, keeping the
//       first kStagedPins of them in shared memory between the passes.
// Nets above kWarpPins pins come first (largest first), then degree 32 down
// to 1, so the long tasks start early.  The sums are FP32 as in
// Net::calcWirelengthWA_2D, added in a fixed tree order instead of pin order
// (a few ulps apart).  Pin gradients are written in device pin order
// (coalesced); the combine kernel gathers them back in each object's
// reference pin order.  WL = false computes only the HPWL with the same
// layout and reduction tree, so both passes give bitwise the same HPWL.
struct NetOut {
    double hpwl, value;
};

constexpr unsigned kFull = 0xffffffffu;

// Bound pins of each aligned segment of D lanes (segment base `base`, this
// lane's index k in it); every lane of the segment gets them.  The windows
// double cyclically, which is exact for max / min.
__device__ __forceinline__ void seg_bounds(float &x1, float &x0, float &y1, float &y0, int D,
                                           int base, int k) {
    for (int o = 1; o < D; o <<= 1) {
        const int j = k + o;
        const int src = base + (j < D ? j : j - D);
        x1 = fmaxf(x1, __shfl_sync(kFull, x1, src));
        x0 = fminf(x0, __shfl_sync(kFull, x0, src));
        y1 = fmaxf(y1, __shfl_sync(kFull, y1, src));
        y0 = fminf(y0, __shfl_sync(kFull, y0, src));
    }
}

// The eight exponential sums of each segment, every lane of the segment gets
// bitwise the same totals: a butterfly when D is a power of two, else a tree
// into the segment's first lane and a broadcast.
__device__ __forceinline__ void seg_sums(float (&s)[8], int D, int base, int k) {
    if ((D & (D - 1)) == 0) {
        for (int o = D >> 1; o > 0; o >>= 1)
#pragma unroll
            for (int i = 0; i < 8; i++) s[i] = __fadd_rn(s[i], __shfl_xor_sync(kFull, s[i], o));
        return;
    }
    for (int o = 1; o < D; o <<= 1) {
        const bool take = k + o < D;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float t = __shfl_down_sync(kFull, s[i], o);
            if (take) s[i] = __fadd_rn(s[i], t);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = __shfl_sync(kFull, s[i], base);
}

__device__ __forceinline__ NetSums net_sums(const float (&s)[8]) {
    return NetSums{s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7]};
}

// Nets of degree D <= 32 packed on the lanes of one warp.
template <bool WL, bool EXACT, bool LSE>
__device__ __forceinline__ NetOut nets_in_warp(const int4 t, int lane, const PinCtx &pc,
                                               float2 *__restrict__ out, float igx, float igy,
                                               int want_value) {
    const int D = t.x, p0 = t.y;
    const int seg = (lane * t.w) >> 16, base = seg * D, k = lane - base;
    const bool act = seg < t.z;
    const float2 xy = act ? pin_xy(pc, p0 + lane) : make_float2(0.f, 0.f);
    // bound pins (Net::calcBoundPin, PlaceCommon/objects.cpp:75-144)
    float x1 = xy.x, x0 = xy.x, y1 = xy.y, y0 = xy.y;
    seg_bounds(x1, x0, y1, y0, D, base, k);
    NetOut r{0.0, 0.0};
    if (act && k == 0) r.hpwl = ((double)x1 - (double)x0) + ((double)y1 - (double)y0);
    if (WL) {
        const PinExp e = pin_exps<EXACT>(xy, x1, x0, y1, y0, igx, igy);
        float s[8] = {__fmul_rn(xy.x, e.emx), e.emx, __fmul_rn(xy.x, e.enx), e.enx,
                      __fmul_rn(xy.y, e.emy), e.emy, __fmul_rn(xy.y, e.eny), e.eny};
        seg_sums(s, D, base, k);
        const NetSums ns = net_sums(s);
        if (act) out[p0 + lane] = pin_gradient<LSE>(e, xy, igx, igy, net_coef(ns));
        if (want_value && act && k == 0) r.value = net_value(ns, x1, x0, y1, y0, igx, igy, LSE);
    }
    return r;
}

// One net of D > 32 pins on one warp; `stage` holds kStagedPins pin positions.
template <bool WL, bool EXACT, bool LSE>
__device__ __forceinline__ NetOut net_in_warp(const int4 t, int lane, const PinCtx &pc,
                                              float2 *__restrict__ out, float igx, float igy,
                                              int want_value, float2 *__restrict__ stage) {
    const int D = t.x, p0 = t.y;
    float x1 = -3.4e38f, x0 = 3.4e38f, y1 = -3.4e38f, y0 = 3.4e38f;
#pragma unroll 4
    for (int k = lane; k < D; k += 32) {
        const float2 xy = pin_xy(pc, p0 + k);
        if (k < kStagedPins) stage[k] = xy;  // read back by this lane only
        x1 = fmaxf(x1, xy.x);
        x0 = fminf(x0, xy.x);
        y1 = fmaxf(y1, xy.y);
        y0 = fminf(y0, xy.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x1 = fmaxf(x1, __shfl_xor_sync(kFull, x1, o));
        x0 = fminf(x0, __shfl_xor_sync(kFull, x0, o));
        y1 = fmaxf(y1, __shfl_xor_sync(kFull, y1, o));
        y0 = fminf(y0, __shfl_xor_sync(kFull, y0, o));
    }
    NetOut r{lane == 0 ? ((double)x1 - (double)x0) + ((double)y1 - (double)y0) : 0.0, 0.0};
    if (WL) {
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int k = lane; k < D; k += 32) {
            const float2 xy = k < kStagedPins ? stage[k] : pin_xy(pc, p0 + k);
            add_terms(s, pin_exps<EXACT>(xy, x1, x0, y1, y0, igx, igy), xy);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int i = 0; i < 8; i++) s[i] = __fadd_rn(s[i], __shfl_xor_sync(kFull, s[i], o));
        const NetSums ns = net_sums(s);
        const NetCoef c = net_coef(ns);
        for (int k = lane; k < D; k += 32) {
            const float2 xy = k < kStagedPins ? stage[k] : pin_xy(pc, p0 + k);
            out[p0 + k] = pin_gradient<LSE>(pin_exps<EXACT>(xy, x1, x0, y1, y0, igx, igy), xy, igx, igy, c);
        }
        if (want_value && lane == 0) r.value = net_value(ns, x1, x0, y1, y0, igx, igy, LSE);
    }
    return r;
}

template <bool WL, bool EXACT, bool LSE>
__global__ void __launch_bounds__(kNetWarps * 32)
k_wl(const int4 *__restrict__ tasks, int n_tasks, PinCtx pc, float2 *__restrict__ out,
     int want_value, double *__restrict__ partials, int mode, DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ double sh[64];
    __shared__ float2 stage[WL ? kNetWarps : 1][WL ? kStagedPins : 1];
    if (WL && S->done) return;
    const float igx = (float)S->inv_gamma_x, igy = (float)S->inv_gamma_y;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = blockIdx.x * kNetWarps + wid;
    NetOut r{0.0, 0.0};
    if (w < n_tasks) {  // warp-uniform
        const int4 t = tasks[w];
        r = t.x <= kWarpPins ? nets_in_warp<WL, EXACT, LSE>(t, lane, pc, out, igx, igy, want_value)
                             : net_in_warp<WL, EXACT, LSE>(t, lane, pc, out, igx, igy, want_value,
                                                           stage[WL ? wid : 0]);
    }
    // the smooth wirelength value rides along only when asked for
    bool last;
    double acc[2] = {r.hpwl, r.value};
    if (WL && want_value) {
        last = grid_sum<2>(acc, sh, partials, &S->cnt_wl, gridDim.x, blockIdx.x);
    } else {
        double a1[1] = {r.hpwl};
        last = grid_sum<1>(a1, sh, partials, WL ? &S->cnt_wl : &S->cnt_hp, gridDim.x, blockIdx.x);
        acc[0] = a1[0];
        acc[1] = 0.0;
    }
    if (last && threadIdx.x == 0) {
        if (WL)
            finish_wirelength(S, acc[0], acc[1]);
        else
            finish_hpwl(S, acc[0], mode);
    }
}

// ---------------------------------------------------------------- gather --
// Field gather (EPlace/eplace.cpp:599-674) in FP32: the same smoothed
// rectangle and bin range as the scatter, the overlap in float, and the
// static smoothing scale sx*sy of the object.  (The scatter keeps the
// reference's exact FP64 overlap arithmetic because its maps are compared
// bit for bit; the gather is compared within tolerance.)
struct FRect {
    float l, b, r, t;
};

__device__ __forceinline__ FRect gather_rect(const Grid &g, float2 p, float2 s, uint8_t f) {
    const float hw = 0.5f * ((f & kSmoothX) ? g.sx : s.x);
    const float hh = 0.5f * ((f & kSmoothY) ? g.sy : s.y);
    return FRect{p.x - hw, p.y - hh, p.x + hw, p.y + hh};
}

__device__ __forceinline__ void gather_range(const Grid &g, const FRect &r, int &i0, int &i1, int &j0,
                                             int &j1) {
    i0 = max(0, (int)((r.l - g.llx) * g.isx));
    i1 = min(g.nx - 1, (int)((r.r - g.llx) * g.isx));
    j0 = max(0, (int)((r.b - g.lly) * g.isy));
    j1 = min(g.ny - 1, (int)((r.t - g.lly) * g.isy));
}

__device__ __forceinline__ float2 gather_bin(const Grid &g, const FRect &r, float sxy, int i, int j,
                                             const float2 *__restrict__ field) {
    const float bl = fmaf((float)i, g.sx, g.llx), bb = fmaf((float)j, g.sy, g.lly);
    const float ox = fminf(r.r, bl + g.sx) - fmaxf(r.l, bl);
    const float oy = fminf(r.t, bb + g.sy) - fmaxf(r.b, bb);
    if (ox <= 0.0f || oy <= 0.0f) return make_float2(0.f, 0.f);
    const float ov = sxy * ox * oy;
    const float2 e = field[(size_t)i * g.ny + j];
    return make_float2(ov * e.x, ov * e.y);
}

__global__ void __launch_bounds__(128)
k_gather_big(Grid g, const float2 *__restrict__ pos, const float2 *__restrict__ size,
             const uint8_t *__restrict__ flags, const float *__restrict__ sxy_of,
             const int32_t *__restrict__ big, const float2 *__restrict__ field,
             float2 *__restrict__ out, const DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ float shx[4], shy[4];
    if (S->done) return;
    const int o = big[blockIdx.x];
    const FRect r = gather_rect(g, pos[o], size[o], flags[o]);
    const float sxy = sxy_of[o];
    int i0, i1, j0, j1;
    gather_range(g, r, i0, i1, j0, j1);
    const int wy = j1 - j0 + 1;
    const int nb = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * wy : 0;
    float gx = 0.f, gy = 0.f;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        float2 v = gather_bin(g, r, sxy, i0 + t / wy, j0 + t % wy, field);
        gx += v.x;
        gy += v.y;
    }
    gx = warp_sum_f(gx);
    gy = warp_sum_f(gy);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        shx[wid] = gx;
        shy[wid] = gy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float ax = 0.f, ay = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            ax += shx[k];
            ay += shy[k];
        }
        out[blockIdx.x] = make_float2(ax, ay);
    }
}

// --------------------------------------------------------------- combine --
// stop_condition after a step (Optimization/nesterov.hpp:86-122): `it` steps
// taken in this stage, tau of the last gradient evaluation.
__device__ int stop_after_step(const DevScalars *S, double tau, int it) {
    int stop;
    if (S->stage == EP_STAGE_MGP)
        stop = tau < (double)S->target_overflow || it > S->max_iter;
    else if (S->stage == EP_STAGE_FILLERONLY)
        stop = it >= 20;
    else
        stop = tau < (double)0.07f || it > S->max_iter;
    if (S->step_cap > 0 && it >= S->step_cap) stop = 1;
    if (S->status) stop = 1;
    return stop;
}

__global__ void __launch_bounds__(kThreads)
k_combine(Grid g, DeviceNetlist d, const float2 *__restrict__ field,
          const float2 *__restrict__ gd_big, const float2 *__restrict__ pin_grad,
          float2 *__restrict__ gout, const float2 *__restrict__ g_prev,
          const float2 *__restrict__ y_prev, float2 *__restrict__ dump_gd,
          float2 *__restrict__ dump_gwl, int stepping, double *__restrict__ partials,
          DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ double sh[32 * 5];
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    float lam = S->lambda0_mode ? 0.0f : (float)S->lambda;
    int iter = S->iter;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // dg2, dy2, s.y, |gwl|, |gd|

    // Wirelength gradient of the object: its pins' gradients added in pin
    // order (EPlace/eplace.cpp:539-547).  The objects of a warp own one
    // contiguous run of pin slots, so the warp stages that run's gradients
    // in shared memory with all its loads in flight at once (kPinChunk per
    // round), then every lane adds its own pins from there in order.
    // Fillers own no pins.
    __shared__ float2 pin_sm[kThreads / 32][kPinChunk];
    float wx = 0.f, wy = 0.f;
    {
        const int lane = threadIdx.x & 31;
        float2 *sm = pin_sm[threadIdx.x >> 5];
        const bool valid = o < d.n_obj;
        const int ps = valid ? d.obj_pin_start[o] : 0, pe = valid ? d.obj_pin_start[o + 1] : 0;
        const int wbeg = __shfl_sync(0xffffffffu, ps, 0);
        const int wend = __reduce_max_sync(0xffffffffu, (unsigned)pe);
        for (int base = wbeg; base < wend; base += kPinChunk) {  // warp-uniform
            const int n = min(kPinChunk, wend - base);
            int idx[kPinChunk / 32];
#pragma unroll
            for (int u = 0; u < kPinChunk / 32; u++) {
                const int t = lane + 32 * u;
                idx[u] = t < n ? d.obj_pin_dev[base + t] : -1;
            }
#pragma unroll
            for (int u = 0; u < kPinChunk / 32; u++)
                if (idx[u] >= 0) sm[lane + 32 * u] = pin_grad[idx[u]];
            __syncwarp();
            const int k1 = min(pe, base + n);
            for (int k = max(ps, base); k < k1; k++) {
                const float2 v = sm[k - base];
                wx = __fadd_rn(wx, v.x);
                wy = __fadd_rn(wy, v.y);
            }
            __syncwarp();
        }
    }
    if (o < d.n_obj) {
        uint8_t f = d.flags[o];
        float2 p = d.pos[o];
        float gdx = 0.f, gdy = 0.f;
        if (f & kBig) {
            float2 v = gd_big[d.big_slot[o]];
            gdx = v.x;
            gdy = v.y;
        } else {
            const FRect r = gather_rect(g, p, d.size[o], f);
            const float sxy = d.sxy[o];
            int i0, i1, j0, j1;
            gather_range(g, r, i0, i1, j0, j1);
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++) {
                    float2 v = gather_bin(g, r, sxy, i, j, field);
                    gdx += v.x;
                    gdy += v.y;
                }
        }
        // preconditioner 1/max(1, #pins + lambda*area) and direction
        float den = fmaxf(1.0f, __fadd_rn(d.npins[o], __fmul_rn(lam, d.area[o])));
        float pre = __fdiv_rn(1.0f, den);
        float2 gg;
        if (f & kFiller) {
            gg.x = __fmul_rn(__fmul_rn(pre, lam), gdx);
            gg.y = __fmul_rn(__fmul_rn(pre, lam), gdy);
        } else {
            gg.x = __fmul_rn(pre, __fsub_rn(__fmul_rn(lam, gdx), wx));
            gg.y = __fmul_rn(pre, __fsub_rn(__fmul_rn(lam, gdy), wy));
        }
        gout[o] = gg;
        if (dump_gd) {
            dump_gd[o] = make_float2(gdx, gdy);
            dump_gwl[o] = make_float2(wx, wy);
        }
        // Lipschitz sums against the previous reference point: from the
        // second step on, and for every backtracking trial (stepping == 2)
        if ((stepping == 2 || (stepping && iter > 0)) && (f & kInView)) {
            float2 gp = g_prev[o], yp = y_prev[o];
            double dgx = __fsub_rn(gg.x, gp.x), dgy = __fsub_rn(gg.y, gp.y);
            double dyx = __fsub_rn(p.x, yp.x), dyy = __fsub_rn(p.y, yp.y);
            acc[0] = dgx * dgx + dgy * dgy;
            acc[1] = dyx * dyx + dyy * dyy;
            acc[2] = dyx * dgx + dyy * dgy;
        }
        if (S->lambda0_mode) {
            if (!(f & kFiller)) acc[3] = fabs((double)wx) + fabs((double)wy);
            acc[4] = fabs((double)gdx) + fabs((double)gdy);
        }
    }
    if (grid_sum<5>(acc, sh, partials, &S->cnt_comb, gridDim.x, blockIdx.x) && threadIdx.x == 0) {
        {
            double dg2 = acc[0], dy2 = acc[1], sy = acc[2];
            double l1w = acc[3], l1d = acc[4];
            if (S->lambda0_mode) {
                // penaltyFactorInitilization (EPlace/eplace.cpp:812-835)
                S->lambda = l1w / l1d;
                S->lambda0_mode = 0;
                if (!isfinite(S->lambda)) S->status |= 1 << EP_ERR_NAN;
            }
            if (stepping == 2) {
                // backtracking trial (opt_step_bktrk, Optimization/nesterov.hpp:351-364):
                // 1/L between the trial point and y_k; accepted when it is at
                // least BKTRK_EPS (0.95, nesterov.hpp:37) of the step tried
                double ns = sqrt(dy2) / sqrt(dg2);
                if (!isfinite(ns)) {
                    S->status |= 1 << EP_ERR_NAN;
                    ns = 0.0;
                }
                S->bk_accept = 0.95 * S->step <= ns;
                S->step = ns;
                S->stop_pending = stop_after_step(S, S->tau, S->iter + 1);
            } else if (stepping) {
                double step = 1.0;
                if (S->iter > 0) {
                    double lip = sqrt(dy2) / sqrt(dg2);  // 1/L
                    S->lip_step = lip;
                    step = lip;
                    if (S->step_rule == EP_STEP_BB) {
                        // BB short step s.y / y.y, else min(|s|/|y|, 1/L) (nesterov.hpp:262-274)
                        double bb = sy / dg2;
                        step = bb > 0.0 ? bb : fmin(sqrt(dy2) / sqrt(dg2), lip);
                    }
                }
                if (!isfinite(step)) {
                    S->status |= 1 << EP_ERR_NAN;
                    step = 0.0;
                }
                double a = S->a;
                double an = (1.0 + sqrt(4.0 * a * a + 1.0)) / 2.0;
                S->step = step;
                S->coef = (a - 1.0) / an;
                S->a = an;
                S->stop_pending = stop_after_step(S, S->tau, S->iter + 1);
            }
        }
    }
}

// ---------------------------------------------------------------- update --

// x_{k+1} = y_k + s g_k, y_{k+1} = x_{k+1} + c (x_{k+1} - x_k)
// (opt_step_vanilla, Optimization/nesterov.hpp:391-404); returns the clamped
// new position, which becomes the object's position.
__device__ __forceinline__ float2 nesterov_move(const Grid &g, int o, float s, float c,
                                                const float2 *__restrict__ size, float2 *__restrict__ pos,
                                                float2 *__restrict__ x, const float2 *__restrict__ gin,
                                                float2 *__restrict__ y_prev, float2 *__restrict__ g_prev) {
    float2 y = pos[o], gg = gin[o], xo = x[o];
    float2 xn = make_float2(__fadd_rn(y.x, __fmul_rn(gg.x, s)), __fadd_rn(y.y, __fmul_rn(gg.y, s)));
    float2 yn = make_float2(__fadd_rn(xn.x, __fmul_rn(__fsub_rn(xn.x, xo.x), c)),
                            __fadd_rn(xn.y, __fmul_rn(__fsub_rn(xn.y, xo.y), c)));
    y_prev[o] = y;
    g_prev[o] = gg;
    x[o] = xn;
    const float2 p = clamp_center(g, yn, size[o]);
    pos[o] = p;
    return p;
}

// The scalar side of the end of a step (last block of the update).
__device__ __forceinline__ void end_step(DevScalars *S) {
    S->iter += 1;
    S->lambda_pending = 1;
    if (S->stop_pending) {
        S->done = 1;
        if (S->stage == EP_STAGE_MGP) S->mgp_iterations = S->iter;
    }
}

__global__ void __launch_bounds__(kThreads)
k_update(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
         float2 *__restrict__ pos, float2 *__restrict__ x, const float2 *__restrict__ gin,
         float2 *__restrict__ y_prev, float2 *__restrict__ g_prev, DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView))
        nesterov_move(g, o, (float)S->step, (float)S->coef, size, pos, x, gin, y_prev, g_prev);
    if (threadIdx.x == 0 && last_block(&S->cnt_upd, gridDim.x)) end_step(S);
}

// The update of the captured loop, with the next evaluation's scatter fused
// in: every object is scattered at its new position right after its move
// (objects outside the stage view at their unchanged one).  kBig objects are
// moved and scattered by a block of their own (the blocks after
// small_blocks).  The step that ends the stage scatters nothing, so the maps
// stay clear (prep clears them after each read).
__global__ void __launch_bounds__(kThreads)
k_update_scatter(Grid g, int n, int small_blocks, const int32_t *__restrict__ big,
                 const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
                 float2 *__restrict__ pos, float2 *__restrict__ x, const float2 *__restrict__ gin,
                 float2 *__restrict__ y_prev, float2 *__restrict__ g_prev, double qscale,
                 unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q,
                 DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ float2 big_pos;
    if (S->done) return;
    const float s = (float)S->step, c = (float)S->coef;
    const bool scatter = !S->stop_pending;
    if ((int)blockIdx.x >= small_blocks) {
        const int o = big[blockIdx.x - small_blocks];
        const uint8_t f = flags[o];
        if (threadIdx.x == 0)
            big_pos = (f & kInView) ? nesterov_move(g, o, s, c, size, pos, x, gin, y_prev, g_prev) : pos[o];
        __syncthreads();
        if (scatter) scatter_big_object(g, big_pos, size[o], f, qscale, node_q, filler_q);
    } else {
        const int o = blockIdx.x * blockDim.x + threadIdx.x;
        if (o < n) {
            const uint8_t f = flags[o];
            if (!(f & kBig)) {
                const float2 p = (f & kInView) ? nesterov_move(g, o, s, c, size, pos, x, gin, y_prev, g_prev) : pos[o];
                if (scatter) scatter_small_object(g, p, size[o], f, qscale, node_q, filler_q);
            }
        }
    }
    if (threadIdx.x == 0 && last_block(&S->cnt_upd, gridDim.x)) end_step(S);
}

// Backtracking trial move (opt_step_bktrk, Optimization/nesterov.hpp:337-349):
// from y_k (kept in ysave) x_t = y_k + step g_k, y_t = x_t + coef (x_t - x_k);
// the positions become clamp(y_t) and x_t is kept in xtrial until accepted.
__global__ void __launch_bounds__(kThreads)
k_bktrk_move(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
             const float2 *__restrict__ ysave, const float2 *__restrict__ gin,
             const float2 *__restrict__ x, float2 *__restrict__ pos, float2 *__restrict__ xtrial,
             const DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    if (!(flags[o] & kInView)) {
        xtrial[o] = x[o];
        return;
    }
    float s = (float)S->step, c = (float)S->coef;
    float2 y = ysave[o], gg = gin[o], xo = x[o];
    float2 xn = make_float2(__fadd_rn(y.x, __fmul_rn(gg.x, s)), __fadd_rn(y.y, __fmul_rn(gg.y, s)));
    float2 yn = make_float2(__fadd_rn(xn.x, __fmul_rn(__fsub_rn(xn.x, xo.x), c)),
                            __fadd_rn(xn.y, __fmul_rn(__fsub_rn(xn.y, xo.y), c)));
    xtrial[o] = xn;
    pos[o] = clamp_center(g, yn, size[o]);
}

// The accepted trial ends the step: the scalar side of k_update.
__global__ void k_bktrk_commit(DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    S->iter += 1;
    S->lambda_pending = 1;
    if (S->stop_pending) {
        S->done = 1;
        if (S->stage == EP_STAGE_MGP) S->mgp_iterations = S->iter;
    }
}

// EplaceNesterovOpt::init (nesterov.hpp:207-214): x_0 = current positions.
__global__ void k_stage_begin(int n, const uint8_t *__restrict__ flags,
                              const float2 *__restrict__ pos, float2 *__restrict__ x,
                              DevScalars *__restrict__ S) {
    pdl_begin();
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n; o += gridDim.x * blockDim.x)
        if (flags[o] & kInView) x[o] = pos[o];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->a = 1.0;
        S->iter = 0;
        S->lambda_pending = 0;
        S->stop_pending = 0;
        S->status = 0;
        double tau = S->tau;
        int stop;
        if (S->stage == EP_STAGE_MGP)
            stop = tau < (double)S->target_overflow;
        else if (S->stage == EP_STAGE_FILLERONLY)
            stop = 0;
        else
            stop = tau < (double)0.07f;
        S->done = stop;
        if (stop && S->stage == EP_STAGE_MGP) S->mgp_iterations = 0;
    }
}

// wrap_up (nesterov.hpp:216-223): positions = main solution, clamped.
__global__ void k_wrap_up(Grid g, int n, const uint8_t *__restrict__ flags,
                          const float2 *__restrict__ size, float2 *__restrict__ pos,
                          const float2 *__restrict__ x) {
    pdl_begin();
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView)) pos[o] = clamp_center(g, x[o], size[o]);
}

}  // namespace

// ------------------------------------------------------------- launchers --
int launch_priority(bool high) {
    static int lo = 1, hi = 1;
    if (lo > 0) {
        int l = 0, h = 0;
        cudaDeviceGetStreamPriorityRange(&l, &h);
        hi = h;
        lo = l;
    }
    return high ? hi : lo;
}

int prep_blocks(const Grid &g) { return std::min(blocks_for(g.nx * g.ny, kThreads), 148 * 8); }

int reduction_blocks(const DeviceNetlist &d, int which) {
    switch (which) {
        case 0: return blocks_for(d.n_net_tasks, kNetWarps);
        default: return blocks_for(d.n_obj, kThreads);
    }
}

void launch_scatter(const KernelCtx &c, const DeviceNetlist &d, unsigned long long *node_q,
                    unsigned long long *filler_q, const DevScalars *S, cudaStream_t st) {
    const int sb = blocks_for(d.n_obj, kThreads);
    launch_k(k_scatter, sb + d.n_big_objs, kThreads, 0, st, c.grid, d.pos, d.size, d.flags, d.n_obj, sb,
             d.big_objs, c.qscale, node_q, filler_q, S);
}

void launch_update_scatter(const KernelCtx &c, const DeviceNetlist &d, float2 *pos, float2 *x,
                           const float2 *g, float2 *y_prev, float2 *g_prev, unsigned long long *node_q,
                           unsigned long long *filler_q, DevScalars *S, cudaStream_t st) {
    const int sb = blocks_for(d.n_obj, kThreads);
    launch_k(k_update_scatter, sb + d.n_big_objs, kThreads, 0, st, c.grid, d.n_obj, sb, d.big_objs,
             d.flags, d.size, pos, x, g, y_prev, g_prev, c.qscale, node_q, filler_q, S);
}

void launch_prep(const KernelCtx &c, unsigned long long *node_q, unsigned long long *filler_q,
                 const float2 *static_map, float *rho, void *rho_bf16, float *node_f,
                 float *filler_f, int zero_maps, DevScalars *S, cudaStream_t st) {
    int nb = c.grid.nx * c.grid.ny;
    int blocks = prep_blocks(c.grid);
    uint16_t *hi = (uint16_t *)rho_bf16;
    uint16_t *lo = hi ? hi + nb : nullptr;
    launch_k(k_prep, blocks, kThreads, 0, st, c.grid, node_q, filler_q, static_map, rho, hi, lo, node_f,
             filler_f, zero_maps, c.inv_qscale, c.inv_bin_area, c.bin_area, c.area_norm, c.part_prep, S);
}

template <bool WL, bool EXACT, bool LSE>
void launch_nets(const KernelCtx &c, const DeviceNetlist &d, float2 *pin_grad, double *partials,
                 int mode, DevScalars *S, cudaStream_t st) {
    PinCtx pc{d.pin_owner, d.pin_off, d.pos};
    if (d.n_net_tasks == 0) return;
    launch_kp(k_wl<WL, EXACT, LSE>, reduction_blocks(d, 0), kNetWarps * 32, 0, st, launch_priority(false),
              d.net_tasks, d.n_net_tasks, pc, pin_grad, c.want_wl_value, partials, mode, S);
}

void launch_wirelength(const KernelCtx &c, const DeviceNetlist &d, float2 *pin_grad,
                       DevScalars *S, cudaStream_t st) {
    if (c.exact_exp)
        c.lse ? launch_nets<true, true, true>(c, d, pin_grad, c.part_wl, 0, S, st)
              : launch_nets<true, true, false>(c, d, pin_grad, c.part_wl, 0, S, st);
    else
        c.lse ? launch_nets<true, false, true>(c, d, pin_grad, c.part_wl, 0, S, st)
              : launch_nets<true, false, false>(c, d, pin_grad, c.part_wl, 0, S, st);
}

void launch_gather_big(const KernelCtx &c, const DeviceNetlist &d, const float2 *field,
                       float2 *gd_big, const DevScalars *S, cudaStream_t st) {
    if (d.n_big_objs > 0)
        launch_k(k_gather_big, d.n_big_objs, 128, 0, st, c.grid, d.pos, d.size, d.flags, d.sxy,
                 d.big_objs, field, gd_big, S);
}

void launch_combine(const KernelCtx &c, const DeviceNetlist &d, const float2 *field,
                    const float2 *gd_big, const float2 *pin_grad, float2 *g, const float2 *g_prev,
                    const float2 *y_prev, float2 *dump_gd, float2 *dump_gwl, int stepping,
                    DevScalars *S, cudaStream_t st) {
    launch_k(k_combine, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d, field, gd_big,
             pin_grad, g, g_prev, y_prev, dump_gd, dump_gwl, stepping, c.part_comb, S);
}

void launch_update(const KernelCtx &c, const DeviceNetlist &d, float2 *pos, float2 *x,
                   const float2 *g, float2 *y_prev, float2 *g_prev, DevScalars *S,
                   cudaStream_t st) {
    launch_k(k_update, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
             pos, x, g, y_prev, g_prev, S);
}

void launch_bktrk_move(const KernelCtx &c, const DeviceNetlist &d, const float2 *ysave, const float2 *g,
                       const float2 *x, float2 *pos, float2 *xtrial, const DevScalars *S,
                       cudaStream_t st) {
    launch_k(k_bktrk_move, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags,
             d.size, ysave, g, x, pos, xtrial, S);
}

void launch_bktrk_commit(DevScalars *S, cudaStream_t st) { launch_k(k_bktrk_commit, 1, 1, 0, st, S); }

void launch_stage_begin(const DeviceNetlist &d, const float2 *pos, float2 *x, DevScalars *S,
                        cudaStream_t st) {
    launch_k(k_stage_begin, std::min(blocks_for(d.n_obj, kThreads), 148 * 4), kThreads, 0, st, d.n_obj,
             d.flags, pos, x, S);
}

void launch_wrap_up(const KernelCtx &c, const DeviceNetlist &d, float2 *pos, const float2 *x,
                    cudaStream_t st) {
    launch_k(k_wrap_up, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
             pos, x);
}

void launch_hpwl(const KernelCtx &c, const DeviceNetlist &d, int mode, DevScalars *S,
                 cudaStream_t st) {
    launch_nets<false, false, false>(c, d, nullptr, c.part_hp, mode, S, st);
}

int carveout_percent(size_t smem_bytes) {
    // shared-memory capacities of an sm_100 SM, KB; the driver maps a
    // preferred percentage of the largest to one of them, so ask for the
    // middle of the interval that rounds to the capacity wanted
    static const int kConfigs[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
    const double kb = (double)smem_bytes / 1024.0;
    for (int i = 1; i < 10; i++)
        if (kConfigs[i] >= kb) return (int)std::ceil(50.0 * (kConfigs[i - 1] + kConfigs[i]) / 228.0);
    return 100;
}

// One L1/shared split, kLoopSmemBytes of shared memory, for every kernel of
// the loop: an SM whose split has to change between consecutive kernels must
// drain first, which costs the programmatic overlap of the launches (on the
// 200k-cell solve with the FFT Poisson path: 14.5 ms per solve with one split
// against 18.3 ms with the driver's choice per kernel).  64 KB holds the
// per-net and combine kernels' staging at full occupancy and leaves 192 KB of
// L1; smaller splits cost them occupancy, larger ones L1.
// Function attributes belong to the current device: set once per device.
void set_loop_carveout() {
    static std::mutex mu;
    static std::vector<int> done_devices;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (std::find(done_devices.begin(), done_devices.end(), dev) != done_devices.end()) return;
        done_devices.push_back(dev);
    }
    const int carveout = carveout_percent(kLoopSmemBytes);
    const void *fns[] = {(const void *)k_scatter, (const void *)k_prep, (const void *)k_wl<true, false, false>,
                         (const void *)k_wl<true, true, false>, (const void *)k_wl<true, false, true>,
                         (const void *)k_wl<true, true, true>, (const void *)k_wl<false, false, false>,
                         (const void *)k_wl<false, true, false>, (const void *)k_wl<false, false, true>,
                         (const void *)k_wl<false, true, true>, (const void *)k_gather_big, (const void *)k_combine,
                         (const void *)k_update, (const void *)k_update_scatter, (const void *)k_bktrk_move,
                         (const void *)k_bktrk_commit, (const void *)k_stage_begin, (const void *)k_wrap_up};
    for (const void *f : fns) cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
    set_sgemm_carveout(carveout);
}

}  // namespace ep
