// common.cuh -- device-side helpers shared by the engine's kernels.
//
// Geometry follows the reference bit for bit where the density maps must be
// reproducible: products that feed a sum use explicit round-to-nearest
// intrinsics so nvcc cannot contract them into FMAs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ep {

constexpr double kEps = 1.0e-15;          // EPS, PlaceCommon/global.h:39
constexpr double kNegMaxExp = -300.0;     // NEGATIVE_MAX_EXP, global.h:46

enum ObjFlag : uint8_t {
    kMacro = 1,     // Module::isMacro
    kFiller = 2,    // Module::isFiller
    kInView = 4,    // member of the current stage view
    kBig = 8,       // spans more bins than a thread handles: block-per-object path
    kSmoothX = 16,  // narrower than a bin: widened to one bin (local smoothing)
    kSmoothY = 32,  // lower than a bin
};

// Device-resident scalars of one engine (EPlacer_2D + EplaceNesterovOpt state
// and the accumulators of the fused reductions).  Written only by the
// finalising block of each reduction; every kernel reads `done`.
struct DevScalars {
    // arrival counters of the grid-wide reductions (reset by their last block)
    unsigned int cnt_prep, cnt_wl, cnt_comb, cnt_upd, cnt_hp;
    double hpwl_query;                // result of the standalone HPWL pass
    // results
    double tau;
    double hpwl;
    double wirelength;
    double lambda;
    double last_hpwl;
    double inv_gamma_x, inv_gamma_y;
    double step;
    double a;          // Nesterov a_k
    double coef;       // (a_k - 1) / a_{k+1}
    double lip_step;   // 1/L of the last step (BB fallback)
    int iter;          // steps taken in this stage
    int done;          // stop condition reached: later kernels of the loop are no-ops
    int stop_pending;  // set by the combine finaliser, committed by the update
    int lambda_pending;// lambda update owed for the last step (uses the next HPWL)
    int lambda0_mode;  // the evaluation of initialization(): lambda = 0, then lambda_0
    int status;        // ep_status bits raised on the device
    int stage;
    int max_iter;
    float target_overflow;
    int step_rule;
    int mgp_iterations;
    int step_cap;      // > 0: also stop after this many steps (bounded runs)
    int bk_accept;     // backtracking: the last trial was accepted
    double bk_ratio;   // backtracking: a trial is accepted when 1/L >= bk_ratio * step
};

// ----- working precision ------------------------------------------------------
// The loop runs in one of two precisions (ep_params.precision): FP32 ("mixed":
// float positions, field and wirelength terms, FP64 reductions) or FP64
// throughout.  Kernels are templates on the real type R; Vec2<R> is its
// two-component vector (float2 / double2).
template <typename R>
struct Vec2;
template <>
struct Vec2<float> {
    using type = float2;
    static __host__ __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
};
template <>
struct Vec2<double> {
    using type = double2;
    static __host__ __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
};
template <typename R>
using vec2 = typename Vec2<R>::type;
template <typename R>
__host__ __device__ __forceinline__ vec2<R> mk2(R x, R y) {
    return Vec2<R>::make(x, y);
}

// Round-to-nearest arithmetic that nvcc does not contract into FMAs, in the
// working precision (the FP32 forms keep the reference's float rounding).
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float rcp_rn(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double rcp_rn(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float max_r(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double max_r(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float min_r(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double min_r(double a, double b) { return fmin(a, b); }

// ----- geometry (reference float semantics) -------------------------------
struct Grid {
    int nx, ny;
    float llx, lly, urx, ury;  // core region
    float sx, sy;              // bin step
    float td;                  // target density
    float isx, isy;            // 1 / bin step (gather only)
};

// getOverlap/getOverlapArea (PlaceCommon/global.h:477-518), FP64.
__device__ __forceinline__ double overlap_len(double a0, double a1, double b0, double b1) {
    double s = fmax(a0, b0);
    double e = fmin(a1, b1);
    return s >= e ? 0.0 : __dsub_rn(s, e);
}

__device__ __forceinline__ double overlap_area(double l1, double b1, double r1, double t1,
                                               double l2, double b2, double r2, double t2) {
    double h = overlap_len(l1, r1, l2, r2);
    if (h == 0.0) return 0.0;
    double v = overlap_len(b1, t1, b2, t2);
    if (v == 0.0) return 0.0;
    return __dmul_rn(h, v);
}

// float_less (global.h:350-353)
__device__ __forceinline__ bool f_less(float a, float b) {
    return (double)__fsub_rn(a, b) < -kEps;
}
__device__ __forceinline__ bool f_less(double a, double b) { return __dsub_rn(a, b) < -kEps; }

template <typename R>
struct RectT {
    R llx, lly, urx, ury, sx, sy;
};
using Rect = RectT<float>;

// Object rectangle with local smoothing, EPlace/eplace.cpp:1052-1072 (the
// reference's float steps for R = float; the same steps in double for the
// FP64 arm).
__device__ __forceinline__ Rect object_rect(const Grid &g, float cx, float cy, float w, float h) {
    Rect r;
    float cllx = __fsub_rn(cx, __fmul_rn(0.5f, w));
    float clly = __fsub_rn(cy, __fmul_rn(0.5f, h));
    r.llx = cllx;
    r.urx = __fadd_rn(cllx, w);
    r.lly = clly;
    r.ury = __fadd_rn(clly, h);
    r.sx = 1.0f;
    r.sy = 1.0f;
    if (f_less(w, g.sx)) {
        r.sx = __fdiv_rn(w, g.sx);
        double half = __dmul_rn(0.5, (double)g.sx);
        r.llx = (float)__dsub_rn((double)cx, half);
        r.urx = (float)__dadd_rn((double)cx, half);
    }
    if (f_less(h, g.sy)) {
        r.sy = __fdiv_rn(h, g.sy);
        double half = __dmul_rn(0.5, (double)g.sy);
        r.lly = (float)__dsub_rn((double)cy, half);
        r.ury = (float)__dadd_rn((double)cy, half);
    }
    return r;
}

__device__ __forceinline__ RectT<double> object_rect(const Grid &g, double cx, double cy, double w, double h) {
    RectT<double> r;
    const double gx = g.sx, gy = g.sy;
    r.llx = __dsub_rn(cx, __dmul_rn(0.5, w));
    r.urx = __dadd_rn(r.llx, w);
    r.lly = __dsub_rn(cy, __dmul_rn(0.5, h));
    r.ury = __dadd_rn(r.lly, h);
    r.sx = 1.0;
    r.sy = 1.0;
    if (f_less(w, gx)) {
        r.sx = __ddiv_rn(w, gx);
        r.llx = __dsub_rn(cx, __dmul_rn(0.5, gx));
        r.urx = __dadd_rn(cx, __dmul_rn(0.5, gx));
    }
    if (f_less(h, gy)) {
        r.sy = __ddiv_rn(h, gy);
        r.lly = __dsub_rn(cy, __dmul_rn(0.5, gy));
        r.ury = __dadd_rn(cy, __dmul_rn(0.5, gy));
    }
    return r;
}

// INT_DOWN bin range, end clamped (EPlace/eplace.cpp:1079-1104); the start is
// clamped at 0 (the reference asserts it; the core clamp keeps it there).
template <typename R>
__device__ __forceinline__ void bin_range(const Grid &g, const RectT<R> &r, int &i0, int &i1, int &j0,
                                          int &j1) {
    i0 = (int)div_rn(sub_rn(r.llx, (R)g.llx), (R)g.sx);
    i1 = (int)div_rn(sub_rn(r.urx, (R)g.llx), (R)g.sx);
    j0 = (int)div_rn(sub_rn(r.lly, (R)g.lly), (R)g.sy);
    j1 = (int)div_rn(sub_rn(r.ury, (R)g.lly), (R)g.sy);
    i0 = max(i0, 0);
    j0 = max(j0, 0);
    i1 = min(i1, g.nx - 1);
    j1 = min(j1, g.ny - 1);
}

// Bin corners as binInitialization stores them (EPlace/eplace.cpp:300-307).
template <typename R>
__device__ __forceinline__ void bin_box(const Grid &g, int i, int j, R &l, R &b, R &r, R &t) {
    l = add_rn(mul_rn((R)i, (R)g.sx), (R)g.llx);
    b = add_rn(mul_rn((R)j, (R)g.sy), (R)g.lly);
    r = add_rn(l, (R)g.sx);
    t = add_rn(b, (R)g.sy);
}

template <typename R>
__device__ __forceinline__ double rect_bin_overlap(const Grid &g, const RectT<R> &r, int i, int j) {
    R l, b, rr, t;
    bin_box<R>(g, i, j, l, b, rr, t);
    return overlap_area(l, b, rr, t, r.llx, r.lly, r.urx, r.ury);
}

// PlaceDB::setModuleCenter_2D clamp (PlaceDB/placedb.cpp:257-281), double
// compares and double sums stored in the working precision, as the reference
// evaluates them.
template <typename R>
__device__ __forceinline__ vec2<R> clamp_center(const Grid &g, vec2<R> c, float2 s) {
    double hw = 0.5 * (double)s.x, hh = 0.5 * (double)s.y;
    R x = c.x, y = c.y;
    if ((double)x - hw < (double)g.llx) x = (R)((double)g.llx + hw + kEps);
    if ((double)x + hw > (double)g.urx) x = (R)((double)g.urx - hw - kEps);
    if ((double)y - hh < (double)g.lly) y = (R)((double)g.lly + hh + kEps);
    if ((double)y + hh > (double)g.ury) y = (R)((double)g.ury - hh - kEps);
    return mk2<R>(x, y);
}

// fastExp, PlaceCommon/global.h:457-471 (ten squarings of 1 + a/1024).  a /
// 1024 is an exact power-of-two scaling, so the multiply rounds identically
// to the reference's division.
template <typename R>
__device__ __forceinline__ R fast_exp(R a) {
    a = add_rn((R)1, mul_rn(a, (R)0x1p-10));
#pragma unroll
    for (int i = 0; i < 10; i++) a = mul_rn(a, a);
    return a;
}

// ----- programmatic dependent launch ---------------------------------------------
// Every kernel of the loop starts with pdl_begin(): wait until the previous
// grid in the stream has completed and its writes are visible, then allow the
// next grid to be scheduled (its blocks wait in their own pdl_begin).
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ----- reductions ------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum of NV doubles; result valid in thread 0.  `sh` needs
// NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k * 32 + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = lane < nw ? sh[k * 32 + lane] : 0.0;
            v[k] = warp_sum(s);
        }
    }
    __syncthreads();
}

// "Last block done": returns true in thread 0 of the block that finishes
// last among `total` blocks (counted on *cnt, which it resets).
__device__ __forceinline__ unsigned int arrive_acq_rel(unsigned int *cnt);

__device__ __forceinline__ bool last_block(unsigned int *cnt, unsigned int total) {
    if (arrive_acq_rel(cnt) == total - 1) {
        *cnt = 0;
        return true;
    }
    return false;
}

// Deterministic grid-wide sum of NV doubles.  Every block writes its block
// total to partials[k * total + block_id]; the block that arrives last sums
// the partials in a fixed order (thread-strided, then a fixed tree), so the
// result does not depend on block scheduling.  The finalising block loads
// the NV partials of four blocks before it adds any of them (the additions
// keep the block order), so its L2 round trips overlap.  Must be called by all threads
// of every participating block.  Returns true in all threads of the last
// block; its thread 0 then holds the totals in v.
// Arrival count with acquire-release semantics at GPU scope: the partials this
// thread stored before are visible to whoever observes the increment, and the
// partials of every block counted before are visible to this thread after.
__device__ __forceinline__ unsigned int arrive_acq_rel(unsigned int *cnt) {
    unsigned int prev;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(cnt) : "memory");
    return prev;
}

template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *sh, double *partials,
                                         unsigned int *cnt, unsigned int total,
                                         unsigned int block_id) {
    __shared__ int is_last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[(size_t)k * total + block_id] = v[k];
        const unsigned int prev = arrive_acq_rel(cnt);
        is_last = (prev == total - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    // thread 0's acquire covers the block through the barrier above
    __threadfence_block();
    double s[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) s[k] = 0.0;
    constexpr int U = 4;
    unsigned int i = threadIdx.x;
    for (; i + (U - 1) * blockDim.x < total; i += U * blockDim.x) {
        double t[U][NV];
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int k = 0; k < NV; k++) t[u][k] = __ldcg(&partials[(size_t)k * total + i + u * blockDim.x]);
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int k = 0; k < NV; k++) s[k] += t[u][k];
    }
    for (; i < total; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; k++) s[k] += __ldcg(&partials[(size_t)k * total + i]);
    block_sum<NV>(s, sh);
    if (threadIdx.x == 0) {
        *cnt = 0;
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = s[k];
    }
    return true;
}

}  // namespace ep
