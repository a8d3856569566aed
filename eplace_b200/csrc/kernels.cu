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
#include <cstdio>

#include "engine.h"

namespace ep {

namespace {

constexpr int kThreads = 256;

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

__global__ void __launch_bounds__(kThreads)
k_scatter_small(Grid g, const float2 *__restrict__ pos, const float2 *__restrict__ size,
                const uint8_t *__restrict__ flags, int n, double qscale,
                unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q,
                const DevScalars *__restrict__ S) {
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    uint8_t f = flags[o];
    if (f & kBig) return;
    float2 p = pos[o], s = size[o];
    Rect r = object_rect(g, p.x, p.y, s.x, s.y);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    float scale = contrib_scale(r, f, g.td);
    unsigned long long *map = (f & kFiller) ? filler_q : node_q;
    for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++) scatter_one(g, r, scale, i, j, qscale, map);
}

__global__ void __launch_bounds__(128)
k_scatter_big(Grid g, const float2 *__restrict__ pos, const float2 *__restrict__ size,
              const uint8_t *__restrict__ flags, const int32_t *__restrict__ big, double qscale,
              unsigned long long *__restrict__ node_q, unsigned long long *__restrict__ filler_q,
              const DevScalars *__restrict__ S) {
    if (S->done) return;
    int o = big[blockIdx.x];
    uint8_t f = flags[o];
    float2 p = pos[o], s = size[o];
    Rect r = object_rect(g, p.x, p.y, s.x, s.y);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    float scale = contrib_scale(r, f, g.td);
    unsigned long long *map = (f & kFiller) ? filler_q : node_q;
    int wy = j1 - j0 + 1;
    int nb = (i1 - i0 + 1) * wy;
    if (i1 < i0 || j1 < j0) return;
    for (int t = threadIdx.x; t < nb; t += blockDim.x)
        scatter_one(g, r, scale, i0 + t / wy, j0 + t % wy, qscale, map);
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

// Per-pin gradient of the WA model (objects.cpp:359-415) or LSE (:423-437).
__device__ __forceinline__ float2 pin_gradient(float2 xy, float x1, float x0, float y1, float y0,
                                               float igx, float igy, const NetSums &s, int exact,
                                               int lse) {
    float amx = __fmul_rn(__fsub_rn(xy.x, x1), igx);
    float anx = __fmul_rn(__fsub_rn(x0, xy.x), igx);
    float amy = __fmul_rn(__fsub_rn(xy.y, y1), igy);
    float any = __fmul_rn(__fsub_rn(y0, xy.y), igy);
    bool fmx = amx > (float)kNegMaxExp, fnx = anx > (float)kNegMaxExp;
    bool fmy = amy > (float)kNegMaxExp, fny = any > (float)kNegMaxExp;
    float emx = fmx ? wl_exp(amx, exact) : 0.0f;
    float enx = fnx ? wl_exp(anx, exact) : 0.0f;
    float emy = fmy ? wl_exp(amy, exact) : 0.0f;
    float eny = fny ? wl_exp(any, exact) : 0.0f;
    float2 gr;
    if (lse) {
        gr.x = __fsub_rn(__fdiv_rn(emx, s.dmx), __fdiv_rn(enx, s.dnx));
        gr.y = __fsub_rn(__fdiv_rn(emy, s.dmy), __fdiv_rn(eny, s.dny));
        return gr;
    }
    float gmx = 0.f, gnx = 0.f, gmy = 0.f, gny = 0.f;
    if (fmx) {
        float dd = __fmul_rn(igx, emx);
        float nd = __fadd_rn(emx, __fmul_rn(xy.x, dd));
        gmx = __fdiv_rn(__fsub_rn(__fmul_rn(nd, s.dmx), __fmul_rn(dd, s.nmx)), __fmul_rn(s.dmx, s.dmx));
    }
    if (fmy) {
        float dd = __fmul_rn(igy, emy);
        float nd = __fadd_rn(emy, __fmul_rn(xy.y, dd));
        gmy = __fdiv_rn(__fsub_rn(__fmul_rn(nd, s.dmy), __fmul_rn(dd, s.nmy)), __fmul_rn(s.dmy, s.dmy));
    }
    if (fnx) {
        float dd = __fmul_rn(igx, enx);
        float nd = __fsub_rn(enx, __fmul_rn(xy.x, dd));
        gnx = __fdiv_rn(__fadd_rn(__fmul_rn(nd, s.dnx), __fmul_rn(dd, s.nnx)), __fmul_rn(s.dnx, s.dnx));
    }
    if (fny) {
        float dd = __fmul_rn(igy, eny);
        float nd = __fsub_rn(eny, __fmul_rn(xy.y, dd));
        gny = __fdiv_rn(__fadd_rn(__fmul_rn(nd, s.dny), __fmul_rn(dd, s.nny)), __fmul_rn(s.dny, s.dny));
    }
    gr.x = __fsub_rn(gmx, gnx);
    gr.y = __fsub_rn(gmy, gny);
    return gr;
}

// Accumulate one pin into the net sums (calcWirelengthWA_2D order).
__device__ __forceinline__ void add_pin(NetSums &s, float2 xy, float x1, float x0, float y1,
                                        float y0, float igx, float igy, int exact) {
    float amx = __fmul_rn(__fsub_rn(xy.x, x1), igx);
    float anx = __fmul_rn(__fsub_rn(x0, xy.x), igx);
    float amy = __fmul_rn(__fsub_rn(xy.y, y1), igy);
    float any = __fmul_rn(__fsub_rn(y0, xy.y), igy);
    if (amx > (float)kNegMaxExp) {
        float e = wl_exp(amx, exact);
        s.nmx = __fadd_rn(s.nmx, __fmul_rn(xy.x, e));
        s.dmx = __fadd_rn(s.dmx, e);
    }
    if (anx > (float)kNegMaxExp) {
        float e = wl_exp(anx, exact);
        s.nnx = __fadd_rn(s.nnx, __fmul_rn(xy.x, e));
        s.dnx = __fadd_rn(s.dnx, e);
    }
    if (amy > (float)kNegMaxExp) {
        float e = wl_exp(amy, exact);
        s.nmy = __fadd_rn(s.nmy, __fmul_rn(xy.y, e));
        s.dmy = __fadd_rn(s.dmy, e);
    }
    if (any > (float)kNegMaxExp) {
        float e = wl_exp(any, exact);
        s.nny = __fadd_rn(s.nny, __fmul_rn(xy.y, e));
        s.dny = __fadd_rn(s.dny, e);
    }
}

__device__ __forceinline__ double net_value(const NetSums &s, float x1, float x0, float y1,
                                            float y0, float igx, float igy, int lse) {
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
    if (!isfinite(hp)) S->status |= 1 << EP_ERR_NAN;
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

// Thread per net (sequential float sums in pin order, as the reference).
// WL = false computes only the HPWL, with the same thread layout and
// reduction tree, so both passes give bitwise the same HPWL.
template <bool WL>
__global__ void __launch_bounds__(kThreads)
k_wl_small(const int32_t *__restrict__ nets, int n_list, const int32_t *__restrict__ net_start,
           PinCtx pc, float2 *__restrict__ pin_grad, int exact, int lse, unsigned total_blocks,
           unsigned block_base, double *__restrict__ partials, int mode, DevScalars *__restrict__ S) {
    __shared__ double sh[64];
    if (WL && S->done) return;
    float igx = (float)S->inv_gamma_x, igy = (float)S->inv_gamma_y;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (t < n_list) {
        int n = nets[t];
        int a = net_start[n], b = net_start[n + 1];
        // bound pins (Net::calcBoundPin): strict compares keep the first pin
        float x0 = 3.4e38f, x1 = -3.4e38f, y0 = 3.4e38f, y1 = -3.4e38f;
        for (int p = a; p < b; p++) {
            float2 xy = pin_xy(pc, p);
            if (xy.x < x0) x0 = xy.x;
            if (xy.x > x1) x1 = xy.x;
            if (xy.y < y0) y0 = xy.y;
            if (xy.y > y1) y1 = xy.y;
        }
        acc[0] = ((double)x1 - (double)x0) + ((double)y1 - (double)y0);
        if (WL) {
            NetSums s = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int p = a; p < b; p++) add_pin(s, pin_xy(pc, p), x1, x0, y1, y0, igx, igy, exact);
            acc[1] = net_value(s, x1, x0, y1, y0, igx, igy, lse);
            for (int p = a; p < b; p++)
                pin_grad[p] = pin_gradient(pin_xy(pc, p), x1, x0, y1, y0, igx, igy, s, exact, lse);
        }
    }
    if (grid_sum<2>(acc, sh, partials, WL ? &S->cnt_wl : &S->cnt_hp, total_blocks,
                    block_base + blockIdx.x) &&
        threadIdx.x == 0) {
        if (WL)
            finish_wirelength(S, acc[0], acc[1]);
        else
            finish_hpwl(S, acc[0], mode);
    }
}

// Warp per net for high-degree nets (lane-strided pins, tree reductions).
template <bool WL>
__global__ void __launch_bounds__(kThreads)
k_wl_big(const int32_t *__restrict__ nets, int n_list, const int32_t *__restrict__ net_start,
         PinCtx pc, float2 *__restrict__ pin_grad, int exact, int lse, unsigned total_blocks,
         unsigned block_base, double *__restrict__ partials, int mode, DevScalars *__restrict__ S) {
    __shared__ double sh[64];
    if (WL && S->done) return;
    float igx = (float)S->inv_gamma_x, igy = (float)S->inv_gamma_y;
    int lane = threadIdx.x & 31;
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double acc[2] = {0.0, 0.0};
    if (w < n_list) {
        int n = nets[w];
        int a = net_start[n], b = net_start[n + 1];
        float x0 = 3.4e38f, x1 = -3.4e38f, y0 = 3.4e38f, y1 = -3.4e38f;
        for (int p = a + lane; p < b; p += 32) {
            float2 xy = pin_xy(pc, p);
            x0 = fminf(x0, xy.x);
            x1 = fmaxf(x1, xy.x);
            y0 = fminf(y0, xy.y);
            y1 = fmaxf(y1, xy.y);
        }
        x0 = warp_min(x0);
        x1 = warp_max(x1);
        y0 = warp_min(y0);
        y1 = warp_max(y1);
        NetSums s = {0, 0, 0, 0, 0, 0, 0, 0};
        if (WL) {
            for (int p = a + lane; p < b; p += 32) add_pin(s, pin_xy(pc, p), x1, x0, y1, y0, igx, igy, exact);
            s.nmx = warp_sum_f(s.nmx);
            s.dmx = warp_sum_f(s.dmx);
            s.nnx = warp_sum_f(s.nnx);
            s.dnx = warp_sum_f(s.dnx);
            s.nmy = warp_sum_f(s.nmy);
            s.dmy = warp_sum_f(s.dmy);
            s.nny = warp_sum_f(s.nny);
            s.dny = warp_sum_f(s.dny);
            for (int p = a + lane; p < b; p += 32)
                pin_grad[p] = pin_gradient(pin_xy(pc, p), x1, x0, y1, y0, igx, igy, s, exact, lse);
        }
        if (lane == 0) {
            acc[0] = ((double)x1 - (double)x0) + ((double)y1 - (double)y0);
            if (WL) acc[1] = net_value(s, x1, x0, y1, y0, igx, igy, lse);
        }
    }
    if (grid_sum<2>(acc, sh, partials, WL ? &S->cnt_wl : &S->cnt_hp, total_blocks,
                    block_base + blockIdx.x) &&
        threadIdx.x == 0) {
        if (WL)
            finish_wirelength(S, acc[0], acc[1]);
        else
            finish_hpwl(S, acc[0], mode);
    }
}

// ---------------------------------------------------------------- gather --
__device__ __forceinline__ float2 gather_bin(const Grid &g, const Rect &r, float sxy, int i, int j,
                                             const float2 *__restrict__ field) {
    // overlapArea = (sx*sy) * getOverlapArea (double) stored to float
    double ovd = rect_bin_overlap(g, r, i, j);
    float ov = (float)__dmul_rn((double)sxy, ovd);
    float2 e = field[(size_t)i * g.ny + j];
    return make_float2(__fmul_rn(ov, e.x), __fmul_rn(ov, e.y));
}

__global__ void __launch_bounds__(128)
k_gather_big(Grid g, const float2 *__restrict__ pos, const float2 *__restrict__ size,
             const int32_t *__restrict__ big, const float2 *__restrict__ field,
             float2 *__restrict__ out, const DevScalars *__restrict__ S) {
    __shared__ float shx[4], shy[4];
    if (S->done) return;
    int o = big[blockIdx.x];
    float2 p = pos[o], s = size[o];
    Rect r = object_rect(g, p.x, p.y, s.x, s.y);
    int i0, i1, j0, j1;
    bin_range(g, r, i0, i1, j0, j1);
    float sxy = __fmul_rn(r.sx, r.sy);
    int wy = j1 - j0 + 1;
    int nb = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * wy : 0;
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
__global__ void __launch_bounds__(kThreads)
k_combine(Grid g, DeviceNetlist d, const float2 *__restrict__ field,
          const float2 *__restrict__ gd_big, const float2 *__restrict__ pin_grad,
          float2 *__restrict__ gout, const float2 *__restrict__ g_prev,
          const float2 *__restrict__ y_prev, float2 *__restrict__ dump_gd,
          float2 *__restrict__ dump_gwl, int stepping, double *__restrict__ partials,
          DevScalars *__restrict__ S) {
    __shared__ double sh[32 * 5];
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    float lam = S->lambda0_mode ? 0.0f : (float)S->lambda;
    int iter = S->iter;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // dg2, dy2, s.y, |gwl|, |gd|
    if (o < d.n_obj) {
        uint8_t f = d.flags[o];
        float2 p = d.pos[o];
        float gdx = 0.f, gdy = 0.f;
        if (f & kBig) {
            float2 v = gd_big[d.big_slot[o]];
            gdx = v.x;
            gdy = v.y;
        } else {
            float2 s = d.size[o];
            Rect r = object_rect(g, p.x, p.y, s.x, s.y);
            int i0, i1, j0, j1;
            bin_range(g, r, i0, i1, j0, j1);
            float sxy = __fmul_rn(r.sx, r.sy);
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++) {
                    float2 v = gather_bin(g, r, sxy, i, j, field);
                    gdx = __fadd_rn(gdx, v.x);
                    gdy = __fadd_rn(gdy, v.y);
                }
        }
        // wirelength gradient: the module's pins in pin order (eplace.cpp:539-547)
        float wx = 0.f, wy = 0.f;
        if (!(f & kFiller)) {
            for (int k = d.obj_pin_start[o]; k < d.obj_pin_start[o + 1]; k++) {
                float2 v = pin_grad[d.obj_pins[k]];
                wx = __fadd_rn(wx, v.x);
                wy = __fadd_rn(wy, v.y);
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
        if (stepping && iter > 0 && (f & kInView)) {
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
            if (stepping) {
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
                // stop_condition after this step (nesterov.hpp:86-122)
                int it = S->iter + 1;
                double tau = S->tau;
                int stop;
                if (S->stage == EP_STAGE_MGP)
                    stop = tau < (double)S->target_overflow || it > S->max_iter;
                else if (S->stage == EP_STAGE_FILLERONLY)
                    stop = it >= 20;
                else
                    stop = tau < (double)0.07f || it > S->max_iter;
                if (S->step_cap > 0 && it >= S->step_cap) stop = 1;
                if (S->status) stop = 1;
                S->stop_pending = stop;
            }
        }
    }
}

// ---------------------------------------------------------------- update --
// PlaceDB::setModuleCenter_2D clamp (PlaceDB/placedb.cpp:257-281), double
// compares and double sums stored to float, as the reference evaluates them.
__device__ __forceinline__ float2 clamp_center(const Grid &g, float2 c, float2 s) {
    double hw = 0.5 * (double)s.x, hh = 0.5 * (double)s.y;
    float x = c.x, y = c.y;
    if ((double)x - hw < (double)g.llx) x = (float)((double)g.llx + hw + kEps);
    if ((double)x + hw > (double)g.urx) x = (float)((double)g.urx - hw - kEps);
    if ((double)y - hh < (double)g.lly) y = (float)((double)g.lly + hh + kEps);
    if ((double)y + hh > (double)g.ury) y = (float)((double)g.ury - hh - kEps);
    return make_float2(x, y);
}

__global__ void __launch_bounds__(kThreads)
k_update(Grid g, int n, const uint8_t *__restrict__ flags, const float2 *__restrict__ size,
         float2 *__restrict__ pos, float2 *__restrict__ x, const float2 *__restrict__ gin,
         float2 *__restrict__ y_prev, float2 *__restrict__ g_prev, DevScalars *__restrict__ S) {
    if (S->done) return;
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView)) {
        float s = (float)S->step, c = (float)S->coef;
        float2 y = pos[o], gg = gin[o], xo = x[o];
        float2 xn = make_float2(__fadd_rn(y.x, __fmul_rn(gg.x, s)), __fadd_rn(y.y, __fmul_rn(gg.y, s)));
        float2 yn = make_float2(__fadd_rn(xn.x, __fmul_rn(__fsub_rn(xn.x, xo.x), c)),
                                __fadd_rn(xn.y, __fmul_rn(__fsub_rn(xn.y, xo.y), c)));
        y_prev[o] = y;
        g_prev[o] = gg;
        x[o] = xn;
        pos[o] = clamp_center(g, yn, size[o]);
    }
    if (threadIdx.x == 0 && last_block(&S->cnt_upd, gridDim.x)) {
        S->iter += 1;
        S->lambda_pending = 1;
        if (S->stop_pending) {
            S->done = 1;
            if (S->stage == EP_STAGE_MGP) S->mgp_iterations = S->iter;
        }
    }
}

// EplaceNesterovOpt::init (nesterov.hpp:207-214): x_0 = current positions.
__global__ void k_stage_begin(int n, const uint8_t *__restrict__ flags,
                              const float2 *__restrict__ pos, float2 *__restrict__ x,
                              DevScalars *__restrict__ S) {
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
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n && (flags[o] & kInView)) pos[o] = clamp_center(g, x[o], size[o]);
}

}  // namespace

// ------------------------------------------------------------- launchers --
int prep_blocks(const Grid &g) { return std::min(blocks_for(g.nx * g.ny, kThreads), 148 * 8); }

int reduction_blocks(const DeviceNetlist &d, int which) {
    switch (which) {
        case 0: return blocks_for(d.n_small_nets, kThreads) + blocks_for(d.n_big_nets * 32, kThreads);
        default: return blocks_for(d.n_obj, kThreads);
    }
}

void launch_scatter(const KernelCtx &c, const DeviceNetlist &d, unsigned long long *node_q,
                    unsigned long long *filler_q, const DevScalars *S, cudaStream_t st) {
    k_scatter_small<<<blocks_for(d.n_obj, kThreads), kThreads, 0, st>>>(
        c.grid, d.pos, d.size, d.flags, d.n_obj, c.qscale, node_q, filler_q, S);
    if (d.n_big_objs > 0)
        k_scatter_big<<<d.n_big_objs, 128, 0, st>>>(c.grid, d.pos, d.size, d.flags, d.big_objs,
                                                    c.qscale, node_q, filler_q, S);
}

void launch_prep(const KernelCtx &c, unsigned long long *node_q, unsigned long long *filler_q,
                 const float2 *static_map, float *rho, void *rho_bf16, float *node_f,
                 float *filler_f, int zero_maps, DevScalars *S, cudaStream_t st) {
    int nb = c.grid.nx * c.grid.ny;
    int blocks = prep_blocks(c.grid);
    uint16_t *hi = (uint16_t *)rho_bf16;
    uint16_t *lo = hi ? hi + nb : nullptr;
    k_prep<<<blocks, kThreads, 0, st>>>(c.grid, node_q, filler_q, static_map, rho, hi, lo, node_f,
                                        filler_f, zero_maps, c.inv_qscale, c.inv_bin_area,
                                        c.bin_area, c.area_norm, c.part_prep, S);
}

template <bool WL>
void launch_nets(const KernelCtx &c, const DeviceNetlist &d, float2 *pin_grad, double *partials,
                 int mode, DevScalars *S, cudaStream_t st) {
    PinCtx pc{d.pin_owner, d.pin_off, d.pos};
    int bs = blocks_for(d.n_small_nets, kThreads);
    int bb = blocks_for(d.n_big_nets * 32, kThreads);
    unsigned total = (unsigned)(bs + bb);
    if (total == 0) return;
    if (bb > 0)
        k_wl_big<WL><<<bb, kThreads, 0, st>>>(d.big_nets, d.n_big_nets, d.net_start, pc, pin_grad,
                                              c.exact_exp, c.lse, total, 0u, partials, mode, S);
    if (bs > 0)
        k_wl_small<WL><<<bs, kThreads, 0, st>>>(d.small_nets, d.n_small_nets, d.net_start, pc,
                                                pin_grad, c.exact_exp, c.lse, total, (unsigned)bb,
                                                partials, mode, S);
}

void launch_wirelength(const KernelCtx &c, const DeviceNetlist &d, float2 *pin_grad,
                       DevScalars *S, cudaStream_t st) {
    launch_nets<true>(c, d, pin_grad, c.part_wl, 0, S, st);
}

void launch_gather_big(const KernelCtx &c, const DeviceNetlist &d, const float2 *field,
                       float2 *gd_big, const DevScalars *S, cudaStream_t st) {
    if (d.n_big_objs > 0)
        k_gather_big<<<d.n_big_objs, 128, 0, st>>>(c.grid, d.pos, d.size, d.big_objs, field,
                                                   gd_big, S);
}

void launch_combine(const KernelCtx &c, const DeviceNetlist &d, const float2 *field,
                    const float2 *gd_big, const float2 *pin_grad, float2 *g, const float2 *g_prev,
                    const float2 *y_prev, float2 *dump_gd, float2 *dump_gwl, int stepping,
                    DevScalars *S, cudaStream_t st) {
    k_combine<<<blocks_for(d.n_obj, kThreads), kThreads, 0, st>>>(
        c.grid, d, field, gd_big, pin_grad, g, g_prev, y_prev, dump_gd, dump_gwl, stepping,
        c.part_comb, S);
}

void launch_update(const KernelCtx &c, const DeviceNetlist &d, float2 *pos, float2 *x,
                   const float2 *g, float2 *y_prev, float2 *g_prev, DevScalars *S,
                   cudaStream_t st) {
    k_update<<<blocks_for(d.n_obj, kThreads), kThreads, 0, st>>>(c.grid, d.n_obj, d.flags, d.size,
                                                                  pos, x, g, y_prev, g_prev, S);
}

void launch_stage_begin(const DeviceNetlist &d, const float2 *pos, float2 *x, DevScalars *S,
                        cudaStream_t st) {
    k_stage_begin<<<std::min(blocks_for(d.n_obj, kThreads), 148 * 4), kThreads, 0, st>>>(
        d.n_obj, d.flags, pos, x, S);
}

void launch_wrap_up(const KernelCtx &c, const DeviceNetlist &d, float2 *pos, const float2 *x,
                    cudaStream_t st) {
    k_wrap_up<<<blocks_for(d.n_obj, kThreads), kThreads, 0, st>>>(c.grid, d.n_obj, d.flags, d.size,
                                                                   pos, x);
}

void launch_hpwl(const KernelCtx &c, const DeviceNetlist &d, int mode, DevScalars *S,
                 cudaStream_t st) {
    launch_nets<false>(c, d, nullptr, c.part_hp, mode, S, st);
}

}  // namespace ep
