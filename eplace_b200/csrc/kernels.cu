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
// multi-iteration graph stops doing work after the stop condition.  Each is a
// template on the working precision R (float: the engine's mixed-precision
// form, whose arithmetic follows the reference's float steps; double: the
// plain FP64 form); the launchers pick the instance from KernelCtx::fp64.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iterator>
#include <mutex>
#include <vector>

#include "engine.h"

namespace ep {

namespace {

constexpr int kThreads = 256;
constexpr int kPinChunk = 128;  // pin gradients a warp of the combine kernel stages per round

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

using ull = unsigned long long;

__device__ __forceinline__ float exact_exp(float a) { return expf(a); }
__device__ __forceinline__ double exact_exp(double a) { return exp(a); }
__device__ __forceinline__ float warp_sum_r(float v) { return warp_sum_f(v); }
__device__ __forceinline__ double warp_sum_r(double v) { return warp_sum(v); }

// ---------------------------------------------------------------- scatter --
template <typename R>
__device__ __forceinline__ void scatter_one(const Grid &g, const RectT<R> &r, R scale, int i, int j, double qscale,
                                            ull *__restrict__ map) {
    R ovl = (R)rect_bin_overlap<R>(g, r, i, j);
    if (ovl == (R)0) return;
    R c = mul_rn(scale, ovl);
    long long q = __double2ll_rn(__dmul_rn((double)c, qscale));
    atomicAdd(&map[(size_t)i * g.ny + j], (ull)q);
}

// Contribution scale: sx*sy, times the target density for macros
// (EPlace/eplace.cpp:1114-1128, evaluated left to right).
template <typename R>
__device__ __forceinline__ R contrib_scale(const RectT<R> &r, uint8_t f, float td) {
    R s = mul_rn(r.sx, r.sy);
    return (f & kMacro) ? mul_rn(s, (R)td) : s;
}

// One object of the thread-per-object path (kBig objects excluded).
template <typename R>
__device__ __forceinline__ void scatter_small_object(const Grid &g, vec2<R> p, float2 s, uint8_t f, double qscale,
                                                     ull *__restrict__ node_q, ull *__restrict__ filler_q) {
    RectT<R> r = object_rect(g, p.x, p.y, (R)s.x, (R)s.y);
    int i0, i1, j0, j1;
    bin_range<R>(g, r, i0, i1, j0, j1);
    R scale = contrib_scale<R>(r, f, g.td);
    ull *map = (f & kFiller) ? filler_q : node_q;
    for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++) scatter_one<R>(g, r, scale, i, j, qscale, map);
}

// One kBig object by a whole block, its bins strided over the threads.
template <typename R>
__device__ __forceinline__ void scatter_big_object(const Grid &g, vec2<R> p, float2 s, uint8_t f, double qscale,
                                                   ull *__restrict__ node_q, ull *__restrict__ filler_q) {
    RectT<R> r = object_rect(g, p.x, p.y, (R)s.x, (R)s.y);
    int i0, i1, j0, j1;
    bin_range<R>(g, r, i0, i1, j0, j1);
    if (i1 < i0 || j1 < j0) return;
    R scale = contrib_scale<R>(r, f, g.td);
    ull *map = (f & kFiller) ? filler_q : node_q;
    const int wy = j1 - j0 + 1, nb = (i1 - i0 + 1) * wy;
    for (int t = threadIdx.x; t < nb; t += blockDim.x)
        scatter_one<R>(g, r, scale, i0 + t / wy, j0 + t % wy, qscale, map);
}

// Blocks [0, small_blocks): thread per object; the blocks after them: one
// kBig object each.
template <typename R>
__global__ void __launch_bounds__(kThreads)
k_scatter(Grid g, const vec2<R> *__restrict__ pos, const float2 *__restrict__ size,
          const uint8_t *__restrict__ flags, int n, int small_blocks, const int32_t *__restrict__ big,
          double qscale, ull *__restrict__ node_q, ull *__restrict__ filler_q, const DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    if ((int)blockIdx.x >= small_blocks) {
        const int o = big[blockIdx.x - small_blocks];
        scatter_big_object<R>(g, pos[o], size[o], flags[o], qscale, node_q, filler_q);
        return;
    }
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const uint8_t f = flags[o];
    if (f & kBig) return;
    scatter_small_object<R>(g, pos[o], size[o], f, qscale, node_q, filler_q);
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

template <typename R>
__global__ void __launch_bounds__(kThreads)
k_prep(Grid g, ull *__restrict__ node_q, ull *__restrict__ filler_q, const float2 *__restrict__ stat,
       R *__restrict__ rho, uint16_t *__restrict__ rho_hi, uint16_t *__restrict__ rho_lo, float *__restrict__ node_f,
       float *__restrict__ filler_f, int zero, double inv_q, double inv_bin_area, double bin_area, double area_norm,
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
        R d = (R)dens;
        if (rho) rho[k] = d;
        if (rho_hi) {
            // 3xBF16 operand split (FP32 path only): hi = bf16(d), lo = bf16(d - hi)
            const float df = (float)d;
            uint32_t u = __float_as_uint(df);
            uint32_t r = u + 0x7fffu + ((u >> 16) & 1u);
            uint16_t h = (uint16_t)(r >> 16);
            float hf = __uint_as_float((uint32_t)h << 16);
            float rem = df - hf;
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
template <typename R>
struct PinCtx {
    const int32_t *__restrict__ owner;
    const float2 *__restrict__ off;
    const vec2<R> *__restrict__ pos;
    const int32_t *__restrict__ slot;  // device pin -> object-major gradient slot (-1: terminal)
};

// Pin::calculateAbsolutePos: centre + offset.
template <typename R>
__device__ __forceinline__ vec2<R> pin_xy(const PinCtx<R> &c, int p) {
    float2 o = c.off[p];
    vec2<R> q = c.pos[c.owner[p]];
    return mk2<R>(add_rn(q.x, (R)o.x), add_rn(q.y, (R)o.y));
}

template <typename R>
struct NetSums {
    R nmx, dmx, nnx, dnx, nmy, dmy, nny, dny;
};

// Exponential terms of one pin (calcWirelengthWA_2D, objects.cpp:275-332):
// arguments <= -300 make the term zero.
template <typename R>
struct PinExp {
    R emx, enx, emy, eny;
};

template <bool EXACT, typename R>
__device__ __forceinline__ R term_exp(R a) {
    if (!(a > (R)kNegMaxExp)) return (R)0;
    return EXACT ? exact_exp(a) : fast_exp<R>(a);
}

template <bool EXACT, typename R>
__device__ __forceinline__ PinExp<R> pin_exps(vec2<R> xy, R x1, R x0, R y1, R y0, R igx, R igy) {
    PinExp<R> e;
    e.emx = term_exp<EXACT, R>(mul_rn(sub_rn(xy.x, x1), igx));
    e.enx = term_exp<EXACT, R>(mul_rn(sub_rn(x0, xy.x), igx));
    e.emy = term_exp<EXACT, R>(mul_rn(sub_rn(xy.y, y1), igy));
    e.eny = term_exp<EXACT, R>(mul_rn(sub_rn(y0, xy.y), igy));
    return e;
}

// Add one pin's terms to a running sum set (calcWirelengthWA_2D's sums).
template <typename R>
__device__ __forceinline__ void add_terms(R (&s)[8], const PinExp<R> &e, vec2<R> xy) {
    s[0] = add_rn(s[0], mul_rn(xy.x, e.emx));
    s[1] = add_rn(s[1], e.emx);
    s[2] = add_rn(s[2], mul_rn(xy.x, e.enx));
    s[3] = add_rn(s[3], e.enx);
    s[4] = add_rn(s[4], mul_rn(xy.y, e.emy));
    s[5] = add_rn(s[5], e.emy);
    s[6] = add_rn(s[6], mul_rn(xy.y, e.eny));
    s[7] = add_rn(s[7], e.eny);
}

// Per-net factors of the gradient: 1 / (sum of exponentials) and the
// exponentially weighted mean coordinate of each of the four terms.  Every
// denominator holds the bound pin's exp(0) = 1, so it is >= 1.
template <typename R>
struct NetCoef {
    R rmx, mmx, rnx, mnx, rmy, mmy, rny, mny;
};

template <typename R>
__device__ __forceinline__ NetCoef<R> net_coef(const NetSums<R> &s) {
    NetCoef<R> c;
    c.rmx = rcp_rn(s.dmx);
    c.rnx = rcp_rn(s.dnx);
    c.rmy = rcp_rn(s.dmy);
    c.rny = rcp_rn(s.dny);
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
template <bool LSE, typename R>
__device__ __forceinline__ vec2<R> pin_gradient(const PinExp<R> &e, vec2<R> xy, R igx, R igy, const NetCoef<R> &c) {
    if (LSE) return mk2<R>(e.emx * c.rmx - e.enx * c.rnx, e.emy * c.rmy - e.eny * c.rny);
    const R gmx = e.emx * c.rmx * fma_r(igx, xy.x - c.mmx, (R)1);
    const R gnx = e.enx * c.rnx * fma_r(-igx, xy.x - c.mnx, (R)1);
    const R gmy = e.emy * c.rmy * fma_r(igy, xy.y - c.mmy, (R)1);
    const R gny = e.eny * c.rny * fma_r(-igy, xy.y - c.mny, (R)1);
    return mk2<R>(gmx - gnx, gmy - gny);
}

template <typename R>
__device__ __forceinline__ double net_value(const NetSums<R> &s, R x1, R x0, R y1, R y0, R igx, R igy, bool lse) {
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
    // atomic: the Poisson solve, running beside this pass, may raise a bit too
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
// to 1, so the long tasks start early.  The sums are in the working precision
// as in Net::calcWirelengthWA_2D (float there), added in a fixed tree order
// instead of pin order (a few ulps apart).  Pin gradients are written in
// device pin order (coalesced); the combine kernel gathers them back in each
// object's reference pin order.  WL = false computes only the HPWL with the
// same layout and reduction tree, so both passes give bitwise the same HPWL.
struct NetOut {
    double hpwl, value;
};

constexpr unsigned kFull = 0xffffffffu;

// Bound pins of each aligned segment of D lanes (segment base `base`, this
// lane's index k in it); every lane of the segment gets them.  The windows
// double cyclically, which is exact for max / min.
template <typename R>
__device__ __forceinline__ void seg_bounds(R &x1, R &x0, R &y1, R &y0, int D, int base, int k) {
    for (int o = 1; o < D; o <<= 1) {
        const int j = k + o;
        const int src = base + (j < D ? j : j - D);
        x1 = max_r(x1, __shfl_sync(kFull, x1, src));
        x0 = min_r(x0, __shfl_sync(kFull, x0, src));
        y1 = max_r(y1, __shfl_sync(kFull, y1, src));
        y0 = min_r(y0, __shfl_sync(kFull, y0, src));
    }
}

// The eight exponential sums of each segment, every lane of the segment gets
// bitwise the same totals: a butterfly when D is a power of two, else a tree
// into the segment's first lane and a broadcast.
template <typename R>
__device__ __forceinline__ void seg_sums(R (&s)[8], int D, int base, int k) {
    if ((D & (D - 1)) == 0) {
        for (int o = D >> 1; o > 0; o >>= 1)
#pragma unroll
            for (int i = 0; i < 8; i++) s[i] = add_rn(s[i], __shfl_xor_sync(kFull, s[i], o));
        return;
    }
    for (int o = 1; o < D; o <<= 1) {
        const bool take = k + o < D;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const R t = __shfl_down_sync(kFull, s[i], o);
            if (take) s[i] = add_rn(s[i], t);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = __shfl_sync(kFull, s[i], base);
}

template <typename R>
__device__ __forceinline__ NetSums<R> net_sums(const R (&s)[8]) {
    return NetSums<R>{s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7]};
}

// Nets of degree D <= 32 packed on the lanes of one warp.
template <bool WL, bool EXACT, bool LSE, typename R>
__device__ __forceinline__ NetOut nets_in_warp(const int4 t, int lane, const PinCtx<R> &pc, vec2<R> *__restrict__ out,
                                               R igx, R igy, int want_value) {
    const int D = t.x, p0 = t.y;
    const int seg = (lane * t.w) >> 16, base = seg * D, k = lane - base;
    const bool act = seg < t.z;
    const vec2<R> xy = act ? pin_xy<R>(pc, p0 + lane) : mk2<R>((R)0, (R)0);
    // bound pins (Net::calcBoundPin, PlaceCommon/objects.cpp:75-144)
    R x1 = xy.x, x0 = xy.x, y1 = xy.y, y0 = xy.y;
    seg_bounds<R>(x1, x0, y1, y0, D, base, k);
    NetOut r{0.0, 0.0};
    if (act && k == 0) r.hpwl = ((double)x1 - (double)x0) + ((double)y1 - (double)y0);
    if (WL) {
        const PinExp<R> e = pin_exps<EXACT, R>(xy, x1, x0, y1, y0, igx, igy);
        R s[8] = {mul_rn(xy.x, e.emx), e.emx, mul_rn(xy.x, e.enx), e.enx,
                  mul_rn(xy.y, e.emy), e.emy, mul_rn(xy.y, e.eny), e.eny};
        seg_sums<R>(s, D, base, k);
        const NetSums<R> ns = net_sums<R>(s);
        const int sl = act ? pc.slot[p0 + lane] : -1;
        if (sl >= 0) out[sl] = pin_gradient<LSE, R>(e, xy, igx, igy, net_coef<R>(ns));
        if (want_value && act && k == 0) r.value = net_value<R>(ns, x1, x0, y1, y0, igx, igy, LSE);
    }
    return r;
}

// One net of D > 32 pins on one warp; `stage` holds kStagedPins pin positions.
template <bool WL, bool EXACT, bool LSE, typename R>
__device__ __forceinline__ NetOut net_in_warp(const int4 t, int lane, const PinCtx<R> &pc, vec2<R> *__restrict__ out,
                                              R igx, R igy, int want_value, vec2<R> *__restrict__ stage) {
    const int D = t.x, p0 = t.y;
    R x1 = (R)-3.4e38f, x0 = (R)3.4e38f, y1 = (R)-3.4e38f, y0 = (R)3.4e38f;
#pragma unroll 4
    for (int k = lane; k < D; k += 32) {
        const vec2<R> xy = pin_xy<R>(pc, p0 + k);
        if (k < kStagedPins) stage[k] = xy;  // read back by this lane only
        x1 = max_r(x1, xy.x);
        x0 = min_r(x0, xy.x);
        y1 = max_r(y1, xy.y);
        y0 = min_r(y0, xy.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x1 = max_r(x1, __shfl_xor_sync(kFull, x1, o));
        x0 = min_r(x0, __shfl_xor_sync(kFull, x0, o));
        y1 = max_r(y1, __shfl_xor_sync(kFull, y1, o));
        y0 = min_r(y0, __shfl_xor_sync(kFull, y0, o));
    }
    NetOut r{lane == 0 ? ((double)x1 - (double)x0) + ((double)y1 - (double)y0) : 0.0, 0.0};
    if (WL) {
        R s[8] = {(R)0, (R)0, (R)0, (R)0, (R)0, (R)0, (R)0, (R)0};
        for (int k = lane; k < D; k += 32) {
            const vec2<R> xy = k < kStagedPins ? stage[k] : pin_xy<R>(pc, p0 + k);
            add_terms<R>(s, pin_exps<EXACT, R>(xy, x1, x0, y1, y0, igx, igy), xy);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int i = 0; i < 8; i++) s[i] = add_rn(s[i], __shfl_xor_sync(kFull, s[i], o));
        const NetSums<R> ns = net_sums<R>(s);
        const NetCoef<R> c = net_coef<R>(ns);
        for (int k = lane; k < D; k += 32) {
            const vec2<R> xy = k < kStagedPins ? stage[k] : pin_xy<R>(pc, p0 + k);
            const int sl = pc.slot[p0 + k];
            if (sl >= 0)
                out[sl] = pin_gradient<LSE, R>(pin_exps<EXACT, R>(xy, x1, x0, y1, y0, igx, igy), xy, igx, igy, c);
        }
        if (want_value && lane == 0) r.value = net_value<R>(ns, x1, x0, y1, y0, igx, igy, LSE);
    }
    return r;
}

template <bool WL, bool EXACT, bool LSE, typename R>
__global__ void __launch_bounds__(kNetWarps * 32)
k_wl(const int4 *__restrict__ tasks, int n_tasks, PinCtx<R> pc, vec2<R> *__restrict__ out, int want_value,
     double *__restrict__ partials, int mode, DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ double sh[64];
    __shared__ vec2<R> stage[WL ? kNetWarps : 1][WL ? kStagedPins : 1];
    if (WL && S->done) return;
    const R igx = (R)S->inv_gamma_x, igy = (R)S->inv_gamma_y;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = blockIdx.x * kNetWarps + wid;
    NetOut r{0.0, 0.0};
    if (w < n_tasks) {  // warp-uniform
        const int4 t = tasks[w];
        r = t.x <= kWarpPins ? nets_in_warp<WL, EXACT, LSE, R>(t, lane, pc, out, igx, igy, want_value)
                             : net_in_warp<WL, EXACT, LSE, R>(t, lane, pc, out, igx, igy, want_value,
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
// Field gather (EPlace/eplace.cpp:599-674) in the working precision: the same
// smoothed rectangle and bin range as the scatter, the overlap in R, and the
// smoothing scale sx*sy of the object (the static FP32 table in the FP32
// path, formed in double from the size in the FP64 path).  (The scatter
// keeps the reference's exact FP64 overlap arithmetic because its maps are
// compared bit for bit; the gather is compared within tolerance.)
template <typename R>
struct FRect {
    R l, b, r, t;
};

template <typename R>
__device__ __forceinline__ FRect<R> gather_rect(const Grid &g, vec2<R> p, float2 s, uint8_t f) {
    const R hw = (R)0.5 * (R)((f & kSmoothX) ? g.sx : s.x);
    const R hh = (R)0.5 * (R)((f & kSmoothY) ? g.sy : s.y);
    return FRect<R>{p.x - hw, p.y - hh, p.x + hw, p.y + hh};
}

template <typename R>
__device__ __forceinline__ void gather_range(const Grid &g, const FRect<R> &r, int &i0, int &i1, int &j0, int &j1) {
    if constexpr (sizeof(R) == 4) {
        i0 = max(0, (int)((r.l - g.llx) * g.isx));
        i1 = min(g.nx - 1, (int)((r.r - g.llx) * g.isx));
        j0 = max(0, (int)((r.b - g.lly) * g.isy));
        j1 = min(g.ny - 1, (int)((r.t - g.lly) * g.isy));
    } else {
        i0 = max(0, (int)((r.l - (R)g.llx) / (R)g.sx));
        i1 = min(g.nx - 1, (int)((r.r - (R)g.llx) / (R)g.sx));
        j0 = max(0, (int)((r.b - (R)g.lly) / (R)g.sy));
        j1 = min(g.ny - 1, (int)((r.t - (R)g.lly) / (R)g.sy));
    }
}

template <typename R>
__device__ __forceinline__ R smoothing_scale(const Grid &g, float table, float2 s, uint8_t f) {
    if constexpr (sizeof(R) == 4) {
        return table;
    } else {
        const R sx = (f & kSmoothX) ? (R)s.x / (R)g.sx : (R)1;
        const R sy = (f & kSmoothY) ? (R)s.y / (R)g.sy : (R)1;
        return sx * sy;
    }
}

template <typename R>
__device__ __forceinline__ vec2<R> gather_bin(const Grid &g, const FRect<R> &r, R sxy, int i, int j,
                                              const vec2<R> *__restrict__ field) {
    const R bl = fma_r((R)i, (R)g.sx, (R)g.llx), bb = fma_r((R)j, (R)g.sy, (R)g.lly);
    const R ox = min_r(r.r, bl + (R)g.sx) - max_r(r.l, bl);
    const R oy = min_r(r.t, bb + (R)g.sy) - max_r(r.b, bb);
    if (ox <= (R)0 || oy <= (R)0) return mk2<R>((R)0, (R)0);
    const R ov = sxy * ox * oy;
    const vec2<R> e = field[(size_t)i * g.ny + j];
    return mk2<R>(ov * e.x, ov * e.y);
}

template <typename R>
__global__ void __launch_bounds__(128)
k_gather_big(Grid g, const vec2<R> *__restrict__ pos, const float2 *__restrict__ size,
             const uint8_t *__restrict__ flags, const float *__restrict__ sxy_of, const int32_t *__restrict__ big,
             const vec2<R> *__restrict__ field, vec2<R> *__restrict__ out, const DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ R shx[4], shy[4];
    if (S->done) return;
    const int o = big[blockIdx.x];
    const uint8_t f = flags[o];
    const FRect<R> r = gather_rect<R>(g, pos[o], size[o], f);
    const R sxy = smoothing_scale<R>(g, sxy_of[o], size[o], f);
    int i0, i1, j0, j1;
    gather_range<R>(g, r, i0, i1, j0, j1);
    const int wy = j1 - j0 + 1;
    const int nb = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * wy : 0;
    R gx = (R)0, gy = (R)0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        vec2<R> v = gather_bin<R>(g, r, sxy, i0 + t / wy, j0 + t % wy, field);
        gx += v.x;
        gy += v.y;
    }
    gx = warp_sum_r(gx);
    gy = warp_sum_r(gy);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        shx[wid] = gx;
        shy[wid] = gy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        R ax = (R)0, ay = (R)0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            ax += shx[k];
            ay += shy[k];
        }
        out[blockIdx.x] = mk2<R>(ax, ay);
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

template <typename R>
__global__ void __launch_bounds__(kThreads)
k_combine(Grid g, DeviceNetlist d, const vec2<R> *__restrict__ field, const vec2<R> *__restrict__ gd_big,
          const vec2<R> *__restrict__ pin_grad, vec2<R> *__restrict__ gout, const vec2<R> *__restrict__ g_prev,
          const vec2<R> *__restrict__ y_prev, vec2<R> *__restrict__ dump_gd, vec2<R> *__restrict__ dump_gwl,
          int stepping, double *__restrict__ partials, DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ double sh[32 * 5];
    if (S->done) return;
    const vec2<R> *__restrict__ pos = (const vec2<R> *)d.pos;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    R lam = S->lambda0_mode ? (R)0 : (R)S->lambda;
    int iter = S->iter;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // dg2, dy2, s.y, |gwl|, |gd|

    // Wirelength gradient of the object: its pins' gradients added in pin
    // order (EPlace/eplace.cpp:539-547).  The per-net pass wrote them in
    // object-major order, so the objects of a warp own one contiguous run of
    // gradient slots: the warp stages that run in shared memory with
    // coalesced loads all in flight at once (kPinChunk per round), then
    // every lane adds its own pins from there in order.  Fillers own no pins.
    __shared__ vec2<R> pin_sm[kThreads / 32][kPinChunk];
    R wx = (R)0, wy = (R)0;
    {
        const int lane = threadIdx.x & 31;
        vec2<R> *sm = pin_sm[threadIdx.x >> 5];
        const bool valid = o < d.n_obj;
        const int ps = valid ? d.obj_pin_start[o] : 0, pe = valid ? d.obj_pin_start[o + 1] : 0;
        const int wbeg = __shfl_sync(0xffffffffu, ps, 0);
        const int wend = __reduce_max_sync(0xffffffffu, (unsigned)pe);
        for (int base = wbeg; base < wend; base += kPinChunk) {  // warp-uniform
            const int n = min(kPinChunk, wend - base);
#pragma unroll
            for (int u = 0; u < kPinChunk / 32; u++) {
                const int t = lane + 32 * u;
                if (t < n) sm[t] = pin_grad[base + t];
            }
            __syncwarp();
            const int k1 = min(pe, base + n);
            for (int k = max(ps, base); k < k1; k++) {
                const vec2<R> v = sm[k - base];
                wx = add_rn(wx, v.x);
                wy = add_rn(wy, v.y);
            }
            __syncwarp();
        }
    }
    if (o < d.n_obj) {
        uint8_t f = d.flags[o];
        vec2<R> p = pos[o];
        R gdx = (R)0, gdy = (R)0;
        if (f & kBig) {
            vec2<R> v = gd_big[d.big_slot[o]];
            gdx = v.x;
            gdy = v.y;
        } else {
            const float2 sz = d.size[o];
            const FRect<R> r = gather_rect<R>(g, p, sz, f);
            const R sxy = smoothing_scale<R>(g, d.sxy[o], sz, f);
            int i0, i1, j0, j1;
            gather_range<R>(g, r, i0, i1, j0, j1);
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++) {
                    vec2<R> v = gather_bin<R>(g, r, sxy, i, j, field);
                    gdx += v.x;
                    gdy += v.y;
                }
        }
        // preconditioner 1/max(1, #pins + lambda*area) and direction
        R den = max_r((R)1, add_rn((R)d.npins[o], mul_rn(lam, (R)d.area[o])));
        R pre = div_rn((R)1, den);
        vec2<R> gg;
        if (f & kFiller) {
            gg.x = mul_rn(mul_rn(pre, lam), gdx);
            gg.y = mul_rn(mul_rn(pre, lam), gdy);
        } else {
            gg.x = mul_rn(pre, sub_rn(mul_rn(lam, gdx), wx));
            gg.y = mul_rn(pre, sub_rn(mul_rn(lam, gdy), wy));
        }
        gout[o] = gg;
        if (dump_gd) {
            dump_gd[o] = mk2<R>(gdx, gdy);
            dump_gwl[o] = mk2<R>(wx, wy);
        }
        // Lipschitz sums against the previous reference point: from the
        // second step on, and for every backtracking trial (stepping == 2)
        if ((stepping == 2 || (stepping && iter > 0)) && (f & kInView)) {
            vec2<R> gp = g_prev[o], yp = y_prev[o];
            double dgx = sub_rn(gg.x, gp.x), dgy = sub_rn(gg.y, gp.y);
            double dyx = sub_rn(p.x, yp.x), dyy = sub_rn(p.y, yp.y);
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
                // least BKTRK_EPS (0.95, nesterov.hpp:37; ep_limits) of the step tried
                double ns = sqrt(dy2) / sqrt(dg2);
                if (!isfinite(ns)) {
                    S->status |= 1 << EP_ERR_NAN;
                    ns = 0.0;
                }
                S->bk_accept = S->bk_ratio * S->step <= ns;
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
template <typename R>
__device__ __forceinline__ vec2<R> nesterov_move(const Grid &g, int o, R s, R c, const float2 *__restrict__ size,
                                                 vec2<R> *__restrict__ pos, vec2<R> *__restrict__ x,
                                                 const vec2<R> *__restrict__ gin, vec2<R> *__restrict__ y_prev,
                                                 vec2<R> *__restrict__ g_prev) {
    vec2<R> y = pos[o], gg = gin[o], xo = x[o];
    vec2<R> xn = mk2<R>(add_rn(y.x, mul_rn(gg.x, s)), add_rn(y.y, mul_rn(gg.y, s)));
    vec2<R> yn = mk2<R>(add_rn(xn.x, mul_rn(sub_rn(xn.x, xo.x), c)), add_rn(xn.y, mul_rn(sub_rn(xn.y, xo.y), c)));
    y_prev[o] = y;
    g_prev[o] = gg;
    x[o] = xn;
    const vec2<R> p = clamp_center<R>(g, yn, size[o]);
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

template <typename R>
__global__ void __launch_bounds__(kThreads)
k_update(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size, vec2<R> *__restrict__ pos,
         vec2<R> *__restrict__ x, const vec2<R> *__restrict__ gin, vec2<R> *__restrict__ y_prev,
         vec2<R> *__restrict__ g_prev, DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView))
        nesterov_move<R>(g, o, (R)S->step, (R)S->coef, size, pos, x, gin, y_prev, g_prev);
    if (threadIdx.x == 0 && last_block(&S->cnt_upd, gridDim.x)) end_step(S);
}

// The update of the captured loop, with the next evaluation's scatter fused
// in: every object is scattered at its new position right after its move
// (objects outside the stage view at their unchanged one).  kBig objects are
// moved and scattered by a block of their own (the blocks after
// small_blocks).  The step that ends the stage scatters nothing, so the maps
// stay clear (prep clears them after each read).
template <typename R>
__global__ void __launch_bounds__(kThreads)
k_update_scatter(Grid g, int n, int small_blocks, const int32_t *__restrict__ big, const uint8_t *__restrict__ flags,
                 const float2 *__restrict__ size, vec2<R> *__restrict__ pos, vec2<R> *__restrict__ x,
                 const vec2<R> *__restrict__ gin, vec2<R> *__restrict__ y_prev, vec2<R> *__restrict__ g_prev,
                 double qscale, ull *__restrict__ node_q, ull *__restrict__ filler_q, DevScalars *__restrict__ S) {
    pdl_begin();
    __shared__ vec2<R> big_pos;
    if (S->done) return;
    const R s = (R)S->step, c = (R)S->coef;
    const bool scatter = !S->stop_pending;
    if ((int)blockIdx.x >= small_blocks) {
        const int o = big[blockIdx.x - small_blocks];
        const uint8_t f = flags[o];
        if (threadIdx.x == 0)
            big_pos = (f & kInView) ? nesterov_move<R>(g, o, s, c, size, pos, x, gin, y_prev, g_prev) : pos[o];
        __syncthreads();
        if (scatter) scatter_big_object<R>(g, big_pos, size[o], f, qscale, node_q, filler_q);
    } else {
        const int o = blockIdx.x * blockDim.x + threadIdx.x;
        if (o < n) {
            const uint8_t f = flags[o];
            if (!(f & kBig)) {
                const vec2<R> p =
                    (f & kInView) ? nesterov_move<R>(g, o, s, c, size, pos, x, gin, y_prev, g_prev) : pos[o];
                if (scatter) scatter_small_object<R>(g, p, size[o], f, qscale, node_q, filler_q);
            }
        }
    }
    if (threadIdx.x == 0 && last_block(&S->cnt_upd, gridDim.x)) end_step(S);
}

// Backtracking trial move (opt_step_bktrk, Optimization/nesterov.hpp:337-349):
// from y_k (kept in ysave) x_t = y_k + step g_k, y_t = x_t + coef (x_t - x_k);
// the positions become clamp(y_t) and x_t is kept in xtrial until accepted.
template <typename R>
__global__ void __launch_bounds__(kThreads)
k_bktrk_move(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
             const vec2<R> *__restrict__ ysave, const vec2<R> *__restrict__ gin, const vec2<R> *__restrict__ x,
             vec2<R> *__restrict__ pos, vec2<R> *__restrict__ xtrial, const DevScalars *__restrict__ S) {
    pdl_begin();
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    if (!(flags[o] & kInView)) {
        xtrial[o] = x[o];
        return;
    }
    R s = (R)S->step, c = (R)S->coef;
    vec2<R> y = ysave[o], gg = gin[o], xo = x[o];
    vec2<R> xn = mk2<R>(add_rn(y.x, mul_rn(gg.x, s)), add_rn(y.y, mul_rn(gg.y, s)));
    vec2<R> yn = mk2<R>(add_rn(xn.x, mul_rn(sub_rn(xn.x, xo.x), c)), add_rn(xn.y, mul_rn(sub_rn(xn.y, xo.y), c)));
    xtrial[o] = xn;
    pos[o] = clamp_center<R>(g, yn, size[o]);
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
template <typename R>
__global__ void k_stage_begin(int n, const uint8_t *__restrict__ flags, const vec2<R> *__restrict__ pos,
                              vec2<R> *__restrict__ x, DevScalars *__restrict__ S) {
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
template <typename R>
__global__ void k_wrap_up(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
                          vec2<R> *__restrict__ pos, const vec2<R> *__restrict__ x) {
    pdl_begin();
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView)) pos[o] = clamp_center<R>(g, x[o], size[o]);
}

}  // namespace

// ------------------------------------------------------------- launchers --
int launch_priority(bool high) {
    // the range is the same on every device; a function-local static is
    // initialised once even when engines are created on several threads
    static const int2 range = [] {
        int l = 0, h = 0;
        cudaDeviceGetStreamPriorityRange(&l, &h);
        return make_int2(l, h);
    }();
    return high ? range.y : range.x;
}

int prep_blocks(const Grid &g) { return std::min(blocks_for(g.nx * g.ny, kThreads), 148 * 8); }

int reduction_blocks(const DeviceNetlist &d, int which) {
    switch (which) {
        case 0: return blocks_for(d.n_net_tasks, kNetWarps);
        default: return blocks_for(d.n_obj, kThreads);
    }
}

namespace {
template <typename R>
inline vec2<R> *V(void *p) {
    return static_cast<vec2<R> *>(p);
}
template <typename R>
inline const vec2<R> *V(const void *p) {
    return static_cast<const vec2<R> *>(p);
}
}  // namespace

template <typename R>
static void scatter_t(const KernelCtx &c, const DeviceNetlist &d, ull *node_q, ull *filler_q, const DevScalars *S,
                      cudaStream_t st) {
    const int sb = blocks_for(d.n_obj, kThreads);
    launch_k(k_scatter<R>, sb + d.n_big_objs, kThreads, 0, st, c.grid, V<R>(d.pos), d.size, d.flags, d.n_obj, sb,
             d.big_objs, c.qscale, node_q, filler_q, S);
}

void launch_scatter(const KernelCtx &c, const DeviceNetlist &d, ull *node_q, ull *filler_q, const DevScalars *S,
                    cudaStream_t st) {
    c.fp64 ? scatter_t<double>(c, d, node_q, filler_q, S, st) : scatter_t<float>(c, d, node_q, filler_q, S, st);
}

template <typename R>
static void update_scatter_t(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g,
                             void *y_prev, void *g_prev, ull *node_q, ull *filler_q, DevScalars *S, cudaStream_t st) {
    const int sb = blocks_for(d.n_obj, kThreads);
    launch_k(k_update_scatter<R>, sb + d.n_big_objs, kThreads, 0, st, c.grid, d.n_obj, sb, d.big_objs, d.flags,
             d.size, V<R>(pos), V<R>(x), V<R>(g), V<R>(y_prev), V<R>(g_prev), c.qscale, node_q, filler_q, S);
}

void launch_update_scatter(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g,
                           void *y_prev, void *g_prev, ull *node_q, ull *filler_q, DevScalars *S, cudaStream_t st) {
    c.fp64 ? update_scatter_t<double>(c, d, pos, x, g, y_prev, g_prev, node_q, filler_q, S, st)
           : update_scatter_t<float>(c, d, pos, x, g, y_prev, g_prev, node_q, filler_q, S, st);
}

void launch_prep(const KernelCtx &c, ull *node_q, ull *filler_q, const float2 *static_map, void *rho,
                 void *rho_bf16, float *node_f, float *filler_f, int zero_maps, DevScalars *S, cudaStream_t st) {
    int nb = c.grid.nx * c.grid.ny;
    int blocks = prep_blocks(c.grid);
    uint16_t *hi = (uint16_t *)rho_bf16;
    uint16_t *lo = hi ? hi + nb : nullptr;
    if (c.fp64)
        launch_k(k_prep<double>, blocks, kThreads, 0, st, c.grid, node_q, filler_q, static_map, (double *)rho,
                 (uint16_t *)nullptr, (uint16_t *)nullptr, node_f, filler_f, zero_maps, c.inv_qscale,
                 c.inv_bin_area, c.bin_area, c.area_norm, c.part_prep, S);
    else
        launch_k(k_prep<float>, blocks, kThreads, 0, st, c.grid, node_q, filler_q, static_map, (float *)rho, hi, lo,
                 node_f, filler_f, zero_maps, c.inv_qscale, c.inv_bin_area, c.bin_area, c.area_norm, c.part_prep,
                 S);
}

template <bool WL, bool EXACT, bool LSE, typename R>
static void launch_nets(const KernelCtx &c, const DeviceNetlist &d, void *pin_grad, double *partials, int mode,
                        DevScalars *S, cudaStream_t st) {
    PinCtx<R> pc{d.pin_owner, d.pin_off, V<R>(d.pos), d.pin_obj_slot};
    if (d.n_net_tasks == 0) return;
    launch_kp(k_wl<WL, EXACT, LSE, R>, reduction_blocks(d, 0), kNetWarps * 32, 0, st, launch_priority(false),
              d.net_tasks, d.n_net_tasks, pc, V<R>(pin_grad), c.want_wl_value, partials, mode, S);
}

template <typename R>
static void wirelength_t(const KernelCtx &c, const DeviceNetlist &d, void *pin_grad, DevScalars *S, cudaStream_t st) {
    if (c.exact_exp)
        c.lse ? launch_nets<true, true, true, R>(c, d, pin_grad, c.part_wl, 0, S, st)
              : launch_nets<true, true, false, R>(c, d, pin_grad, c.part_wl, 0, S, st);
    else
        c.lse ? launch_nets<true, false, true, R>(c, d, pin_grad, c.part_wl, 0, S, st)
              : launch_nets<true, false, false, R>(c, d, pin_grad, c.part_wl, 0, S, st);
}

void launch_wirelength(const KernelCtx &c, const DeviceNetlist &d, void *pin_grad, DevScalars *S, cudaStream_t st) {
    c.fp64 ? wirelength_t<double>(c, d, pin_grad, S, st) : wirelength_t<float>(c, d, pin_grad, S, st);
}

void launch_gather_big(const KernelCtx &c, const DeviceNetlist &d, const void *field, void *gd_big,
                       const DevScalars *S, cudaStream_t st) {
    if (d.n_big_objs == 0) return;
    if (c.fp64)
        launch_k(k_gather_big<double>, d.n_big_objs, 128, 0, st, c.grid, V<double>(d.pos), d.size, d.flags, d.sxy,
                 d.big_objs, V<double>(field), V<double>(gd_big), S);
    else
        launch_k(k_gather_big<float>, d.n_big_objs, 128, 0, st, c.grid, V<float>(d.pos), d.size, d.flags, d.sxy,
                 d.big_objs, V<float>(field), V<float>(gd_big), S);
}

void launch_combine(const KernelCtx &c, const DeviceNetlist &d, const void *field, const void *gd_big,
                    const void *pin_grad, void *g, const void *g_prev, const void *y_prev, void *dump_gd,
                    void *dump_gwl, int stepping, DevScalars *S, cudaStream_t st) {
    if (c.fp64)
        launch_k(k_combine<double>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d, V<double>(field),
                 V<double>(gd_big), V<double>(pin_grad), V<double>(g), V<double>(g_prev), V<double>(y_prev),
                 V<double>(dump_gd), V<double>(dump_gwl), stepping, c.part_comb, S);
    else
        launch_k(k_combine<float>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d, V<float>(field),
                 V<float>(gd_big), V<float>(pin_grad), V<float>(g), V<float>(g_prev), V<float>(y_prev),
                 V<float>(dump_gd), V<float>(dump_gwl), stepping, c.part_comb, S);
}

template <typename R>
static void update_t(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g, void *y_prev,
                     void *g_prev, DevScalars *S, cudaStream_t st) {
    launch_k(k_update<R>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
             V<R>(pos), V<R>(x), V<R>(g), V<R>(y_prev), V<R>(g_prev), S);
}

void launch_update(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g, void *y_prev,
                   void *g_prev, DevScalars *S, cudaStream_t st) {
    c.fp64 ? update_t<double>(c, d, pos, x, g, y_prev, g_prev, S, st)
           : update_t<float>(c, d, pos, x, g, y_prev, g_prev, S, st);
}

template <typename R>
static void bktrk_move_t(const KernelCtx &c, const DeviceNetlist &d, const void *ysave, const void *g,
                         const void *x, void *pos, void *xtrial, const DevScalars *S, cudaStream_t st) {
    launch_k(k_bktrk_move<R>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
             V<R>(ysave), V<R>(g), V<R>(x), V<R>(pos), V<R>(xtrial), S);
}

void launch_bktrk_move(const KernelCtx &c, const DeviceNetlist &d, const void *ysave, const void *g, const void *x,
                       void *pos, void *xtrial, const DevScalars *S, cudaStream_t st) {
    c.fp64 ? bktrk_move_t<double>(c, d, ysave, g, x, pos, xtrial, S, st)
           : bktrk_move_t<float>(c, d, ysave, g, x, pos, xtrial, S, st);
}

void launch_bktrk_commit(DevScalars *S, cudaStream_t st) { launch_k(k_bktrk_commit, 1, 1, 0, st, S); }

void launch_stage_begin(const KernelCtx &c, const DeviceNetlist &d, const void *pos, void *x, DevScalars *S,
                        cudaStream_t st) {
    const int blocks = std::min(blocks_for(d.n_obj, kThreads), 148 * 4);
    if (c.fp64)
        launch_k(k_stage_begin<double>, blocks, kThreads, 0, st, d.n_obj, d.flags, V<double>(pos), V<double>(x), S);
    else
        launch_k(k_stage_begin<float>, blocks, kThreads, 0, st, d.n_obj, d.flags, V<float>(pos), V<float>(x), S);
}

void launch_wrap_up(const KernelCtx &c, const DeviceNetlist &d, void *pos, const void *x, cudaStream_t st) {
    if (c.fp64)
        launch_k(k_wrap_up<double>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
                 V<double>(pos), V<double>(x));
    else
        launch_k(k_wrap_up<float>, blocks_for(d.n_obj, kThreads), kThreads, 0, st, c.grid, d.n_obj, d.flags, d.size,
                 V<float>(pos), V<float>(x));
}

void launch_hpwl(const KernelCtx &c, const DeviceNetlist &d, int mode, DevScalars *S, cudaStream_t st) {
    c.fp64 ? launch_nets<false, false, false, double>(c, d, nullptr, c.part_hp, mode, S, st)
           : launch_nets<false, false, false, float>(c, d, nullptr, c.part_hp, mode, S, st);
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

template <typename R>
static void loop_kernels(std::vector<const void *> &fns) {
    const void *f[] = {(const void *)k_scatter<R>, (const void *)k_prep<R>, (const void *)k_wl<true, false, false, R>,
                       (const void *)k_wl<true, true, false, R>, (const void *)k_wl<true, false, true, R>,
                       (const void *)k_wl<true, true, true, R>, (const void *)k_wl<false, false, false, R>,
                       (const void *)k_gather_big<R>, (const void *)k_combine<R>, (const void *)k_update<R>,
                       (const void *)k_update_scatter<R>, (const void *)k_bktrk_move<R>,
                       (const void *)k_stage_begin<R>, (const void *)k_wrap_up<R>};
    fns.insert(fns.end(), std::begin(f), std::end(f));
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
    std::vector<const void *> fns = {(const void *)k_bktrk_commit};
    loop_kernels<float>(fns);
    loop_kernels<double>(fns);
    for (const void *f : fns) cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
    set_sgemm_carveout(carveout);
}

}  // namespace ep
