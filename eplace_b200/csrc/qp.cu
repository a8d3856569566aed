// qp.cu -- quadratic placement (QPPlacer::quadraticPlacement,
// QPlace/qplace.cpp:20-106) on the device: the initial placement ePlace
// starts from.
//
// Each outer round freezes the current centres, builds for X and for Y the
// system A x = b of the bound-pin model (QPPlacer::createSparseMatrix,
// qplace.cpp:125-272) and solves both with BiCGSTAB (identity
// preconditioner, warm start from the centres), then moves the nodes to the
// solution (clamped into the core) and recomputes the bound pins.
//
// The model, per net of p pins with bound pins found first-occurrence as
// Net::calcBoundPin does (PlaceCommon/objects.cpp:75-144): an unordered pin
// pair on different modules contributes w = (1/(p-1)) / max(d, 25) (d the
// pair's distance along the axis, MIN_DISTANCE 25, qplace.h) when, for X,
// either pin is the net's min- or max-x pin; for Y the reference tests
// "pin2 == Ymin || pin1 == Ymax || pin2 == Ymin || pin2 == Ymax" with pin1
// before pin2 in the net (qplace.cpp:206), which the engine reproduces: the
// Y system differs from the X one exactly as the reference's does.
// Movable-movable pairs add w to both diagonals, -w off the diagonal and
// -w (off_i - off_j) to b_i; a pair with a fixed pin adds w to the movable
// diagonal and w (abs_fixed - off_i) to its b.
//
// The matrices are built row by row (one thread per movable node, its pins in
// Module::modulePins order, each pin's partners in net order): a count pass,
// a prefix sum, a fill pass.  The row order of entries is fixed, and every
// dot product is an FP64 sum in a fixed tree, so the solve is bitwise
// repeatable.
#include <algorithm>

#include "engine.h"

namespace ep {

namespace {

constexpr int kQT = 256;
constexpr float kMinDistance = 25.0f;  // MIN_DISTANCE, QPlace/qplace.h

inline int qblocks(int n) { return (n + kQT - 1) / kQT; }
// Kernels that end in a grid reduction run on at most 8 blocks per SM and
// loop over their rows, so the finalising block adds few partials; the grid
// depends only on the sizes, so the sums are the same on every run.
constexpr int kQpMaxBlocks = 148 * 8;
inline int qgrid(int n) { return std::min(qblocks(n), kQpMaxBlocks); }

__device__ __forceinline__ float2 abs_pin(const float2 *__restrict__ pos, const float2 *__restrict__ off,
                                          int owner, int q) {
    const float2 c = pos[owner], o = off[q];
    return make_float2(__fadd_rn(c.x, o.x), __fadd_rn(c.y, o.y));
}

// Net::calcBoundPin: strict compares in double, the first pin at the
// extreme wins; bound = (x-min, x-max, y-min, y-max) as indices in the net.
__global__ void __launch_bounds__(kQT)
k_qp_bounds(int nnet, const int32_t *__restrict__ first, const int32_t *__restrict__ deg,
            const int32_t *__restrict__ owner, const float2 *__restrict__ off,
            const float2 *__restrict__ pos, int4 *__restrict__ bound, double *__restrict__ partials,
            unsigned *__restrict__ cnt, double *__restrict__ hpwl) {
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nnet; n += gridDim.x * blockDim.x) {
        const int f = first[n], d = deg[n];
        double mnx = 1.79769e308, mxx = -1.79769e308, mny = 1.79769e308, mxy = -1.79769e308;
        int4 b = make_int4(0, 0, 0, 0);
        for (int k = 0; k < d; k++) {
            const float2 a = abs_pin(pos, off, owner[f + k], f + k);
            if ((double)a.x < mnx) { mnx = a.x; b.x = k; }
            if ((double)a.x > mxx) { mxx = a.x; b.y = k; }
            if ((double)a.y < mny) { mny = a.y; b.z = k; }
            if ((double)a.y > mxy) { mxy = a.y; b.w = k; }
        }
        bound[n] = b;
        if (d > 0) acc[0] += (mxx - mnx) + (mxy - mny);
    }
    if (grid_sum<1>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) *hpwl = acc[0];
}

// Partners of pin a (index in its net of d pins) in the X model: every pin
// when a is a bound pin, else the two bound pins.
template <class F>
__device__ __forceinline__ void partners_x(int a, int d, int lo, int hi, F &&f) {
    if (a == lo || a == hi) {
        for (int b = 0; b < d; b++)
            if (b != a) f(b);
    } else {
        f(lo);
        if (hi != lo) f(hi);
    }
}

// Partners of pin a in the reference's Y model: the unordered pair (j < k)
// counts when k == y-min, j == y-max or k == y-max.
template <class F>
__device__ __forceinline__ void partners_y(int a, int d, int lo, int hi, F &&f) {
    if (a == hi) {
        for (int b = 0; b < d; b++)
            if (b != a) f(b);
    } else if (a == lo) {
        for (int b = 0; b < a; b++) f(b);
        if (hi > a) f(hi);
    } else {
        f(hi);
        if (lo > a && lo != hi) f(lo);
    }
}

// weightX / weightY of createSparseMatrix (qplace.cpp:172-183): float
// division, the distance held at MIN_DISTANCE from below (float_greaterorequal
// reduces to >= for float operands).
__device__ __forceinline__ float pair_weight(float c, float dist) {
    return dist >= kMinDistance ? __fdiv_rn(c, dist) : __fdiv_rn(c, kMinDistance);
}

// One movable node's row of both systems: counts (fill = 0) or entries,
// diagonal and right-hand side (fill = 1).
__global__ void __launch_bounds__(kQT)
k_qp_rows(int nn, int fill, const int32_t *__restrict__ obj_pin_start, const int32_t *__restrict__ obj_pin_dev,
          const int32_t *__restrict__ pin_net, const int32_t *__restrict__ first, const int32_t *__restrict__ deg,
          const int4 *__restrict__ bound, const int32_t *__restrict__ owner, const float2 *__restrict__ off,
          const float2 *__restrict__ pos, int32_t *__restrict__ count, const int32_t *__restrict__ row_x,
          const int32_t *__restrict__ row_y, int32_t *__restrict__ col_x, float *__restrict__ val_x,
          int32_t *__restrict__ col_y, float *__restrict__ val_y, float2 *__restrict__ diag,
          float2 *__restrict__ rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    int cx = 0, cy = 0;
    double dx = 0.0, dy = 0.0, bx = 0.0, by = 0.0;
    const int ox = fill ? row_x[i] : 0, oy = fill ? row_y[i] : 0;
    for (int k = obj_pin_start[i]; k < obj_pin_start[i + 1]; k++) {
        const int q = obj_pin_dev[k], n = pin_net[q], f = first[n], d = deg[n], a = q - f;
        const int4 bd = bound[n];
        const float c = (float)(1.0 / ((double)d - 1.0));
        const float2 pa = abs_pin(pos, off, i, q), oa = off[q];
        partners_x(a, d, bd.x, bd.y, [&](int b) {
            const int q2 = f + b, j = owner[q2];
            if (j == i) return;
            const float2 pb = abs_pin(pos, off, j, q2);
            const float w = pair_weight(c, fabsf(__fsub_rn(pa.x, pb.x)));
            dx += w;
            if (j < nn) {
                if (fill) {
                    col_x[ox + cx] = j;
                    val_x[ox + cx] = -w;
                }
                cx++;
                bx += -(double)w * (double)__fsub_rn(oa.x, off[q2].x);
            } else {
                bx += (double)w * (double)__fsub_rn(pb.x, oa.x);
            }
        });
        partners_y(a, d, bd.z, bd.w, [&](int b) {
            const int q2 = f + b, j = owner[q2];
            if (j == i) return;
            const float2 pb = abs_pin(pos, off, j, q2);
            const float w = pair_weight(c, fabsf(__fsub_rn(pa.y, pb.y)));
            dy += w;
            if (j < nn) {
                if (fill) {
                    col_y[oy + cy] = j;
                    val_y[oy + cy] = -w;
                }
                cy++;
                by += -(double)w * (double)__fsub_rn(oa.y, off[q2].y);
            } else {
                by += (double)w * (double)__fsub_rn(pb.y, oa.y);
            }
        });
    }
    if (!fill) {
        count[i] = cx;
        count[nn + i] = cy;
    } else {
        diag[i] = make_float2((float)dx, (float)dy);
        rhs[i] = make_float2((float)bx, (float)by);
    }
}

struct QpMat {
    const int32_t *row_x, *col_x, *row_y, *col_y;
    const float *val_x, *val_y;
    const float2 *diag;
};

// (A_x v.x, A_y v.y) for row i, computed by the 8 lanes of an aligned lane
// group (sub = lane index in the group): lane k sums entries k, k + 8, ...
// of the row in order, a fixed xor tree adds the 8 partial sums, and the
// diagonal term comes last, so the result is the same on every run.  Rows
// of bound pins of large nets hold hundreds of entries; eight lanes per row
// keep those from holding up a warp.  Every lane of the warp must call it
// (valid = false for lanes past the last row); all 8 lanes get the result.
constexpr int kRowLanes = 8, kRowsPerWarp = 32 / kRowLanes;
__device__ __forceinline__ float2 spmv_row8(const QpMat &m, const float2 *__restrict__ v, int i, int sub, bool valid) {
    float ax = 0.f, ay = 0.f;
    if (valid) {
        for (int e = m.row_x[i] + sub; e < m.row_x[i + 1]; e += kRowLanes) ax = fmaf(m.val_x[e], v[m.col_x[e]].x, ax);
        for (int e = m.row_y[i] + sub; e < m.row_y[i + 1]; e += kRowLanes) ay = fmaf(m.val_y[e], v[m.col_y[e]].y, ay);
    }
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (valid) {
        const float2 d = m.diag[i], vi = v[i];
        ax = fmaf(d.x, vi.x, ax);
        ay = fmaf(d.y, vi.y, ay);
    }
    return make_float2(ax, ay);
}

// Grid-stride loop over the rows of a matrix kernel, kRowsPerWarp rows per
// warp and pass; the loop bound is uniform over a warp (spmv_row8 shuffles),
// and row i, lane sub of its group, are declared for the body.
__device__ __forceinline__ int row_group_first() {
    return ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kRowsPerWarp;
}
__device__ __forceinline__ int row_group_stride() { return ((gridDim.x * blockDim.x) >> 5) * kRowsPerWarp; }
#define ROW_GROUPS(nn)                                                                                        \
    for (int base_ = row_group_first(), sub = threadIdx.x % kRowLanes, i = base_ + (threadIdx.x & 31) / kRowLanes; \
         base_ < (nn); base_ += row_group_stride(), i = base_ + (threadIdx.x & 31) / kRowLanes)

// ---- BiCGSTAB on the device -----------------------------------------------------
// Eigen's BiCGSTAB (van der Vorst's method, restart when r0.r vanishes,
// identity preconditioner) for both systems at once, every scalar of the
// recurrence kept in device memory (QpSolve) and updated by the finalising
// block of the grid reduction that produces its inputs; vector kernels read
// alpha, beta and omega from there.  Per axis c:
//   pre      rho_old = rho; rho = r0.r; restart when |rho| < eps^2 r0sq
//   restart  (only when flagged) r = b - A x, r0 = r; rho = r0sq = |r|^2,
//            the iteration count reset at the first restart
//   dir      p = r + beta (p - omega v), beta = (rho / rho_old)(alpha / omega)
//   av       v = A p; alpha = rho / (r0.v)
//   s        s = r - alpha v
//   at       t = A s; omega = t.s / t.t (0 when t.t = 0)
//   step     x += alpha p + omega s; r = s - omega t; |r|^2, r0.r; count;
//            the axis stays active while |r|^2 > (eps |b|)^2 and the count
//            is below the limit
// An inactive axis uses alpha = beta = omega = 0 (its x and r stay), and
// every kernel returns at once when neither axis is active, so iterations
// can be enqueued ahead of the convergence test.
__device__ __forceinline__ bool any_active(const QpSolve *S) { return S->active[0] || S->active[1]; }

// r = b - A x, r0 = r, p = v = 0; |r|^2 and |b|^2 per system, then the
// solver's initial state.
__global__ void __launch_bounds__(kQT)
k_qp_init(int nn, QpMat m, const float2 *__restrict__ rhs, const float2 *__restrict__ x, float2 *__restrict__ r,
          float2 *__restrict__ r0, float2 *__restrict__ p, float2 *__restrict__ v, double *__restrict__ partials,
          unsigned *__restrict__ cnt, int max_it, QpSolve *__restrict__ S) {
    __shared__ double sh[4 * 32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    ROW_GROUPS(nn) {
        const float2 ax = spmv_row8(m, x, i, sub, i < nn);
        if (i < nn && sub == 0) {
            const float2 bi = rhs[i];
            const float2 ri = make_float2(bi.x - ax.x, bi.y - ax.y);
            r[i] = ri;
            r0[i] = ri;
            p[i] = make_float2(0.f, 0.f);
            v[i] = make_float2(0.f, 0.f);
            acc[0] += (double)ri.x * ri.x;
            acc[1] += (double)ri.y * ri.y;
            acc[2] += (double)bi.x * bi.x;
            acc[3] += (double)bi.y * bi.y;
        }
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) {
        const double eps = 1.1920928955078125e-07, eps2 = eps * eps;
        S->zero_mask = 0;
        S->restart_mask = 0;
        S->iters = 0;
        for (int c = 0; c < 2; c++) {
            S->rr[c] = acc[c];
            S->bb[c] = acc[2 + c];
            S->r0sq[c] = acc[c];
            S->r0r[c] = acc[c];
            S->rho[c] = S->alpha[c] = S->w[c] = 1.0;
            S->it[c] = 0;
            S->restarts[c] = 0;
            S->tol2[c] = eps2 * S->bb[c];
            if (S->bb[c] == 0.0) {  // x = 0 (Eigen returns at once)
                S->zero_mask |= 1 << c;
                S->rr[c] = 0.0;
                S->active[c] = 0;
            } else {
                S->active[c] = S->rr[c] > S->tol2[c] && max_it > 0;
            }
        }
        S->max_it = max_it;
    }
}

// A zero right-hand side gives x = 0.
__global__ void k_qp_zero(int nn, const QpSolve *__restrict__ S, float2 *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn || !S->zero_mask) return;
    if (S->zero_mask & 1) x[i].x = 0.f;
    if (S->zero_mask & 2) x[i].y = 0.f;
}

__global__ void k_qp_pre(QpSolve *__restrict__ S) {
    if (threadIdx.x != 0 || !any_active(S)) return;
    const double eps = 1.1920928955078125e-07, eps2 = eps * eps;
    int restart = 0;
    for (int c = 0; c < 2; c++) {
        S->rho_old[c] = S->rho[c];
        if (!S->active[c]) continue;
        S->rho[c] = S->r0r[c];
        if (fabs(S->rho[c]) < eps2 * S->r0sq[c]) restart |= 1 << c;
    }
    S->restart_mask = restart;
}

// Restart of the flagged systems: r = b - A x, r0 = r; rho = r0sq = |r|^2.
__global__ void __launch_bounds__(kQT)
k_qp_restart(int nn, QpMat m, const float2 *__restrict__ rhs, const float2 *__restrict__ x, float2 *__restrict__ r,
             float2 *__restrict__ r0, double *__restrict__ partials, unsigned *__restrict__ cnt,
             QpSolve *__restrict__ S) {
    __shared__ double sh[2 * 32];
    const int mask = S->restart_mask;
    if (!mask || !any_active(S)) return;  // uniform over the grid
    double acc[2] = {0.0, 0.0};
    ROW_GROUPS(nn) {
        const float2 ax = spmv_row8(m, x, i, sub, i < nn);
        if (i < nn && sub == 0) {
            const float2 bi = rhs[i];
            float2 ri = r[i], zi = r0[i];
            if (mask & 1) ri.x = zi.x = bi.x - ax.x;
            if (mask & 2) ri.y = zi.y = bi.y - ax.y;
            r[i] = ri;
            r0[i] = zi;
            acc[0] += (double)ri.x * ri.x;
            acc[1] += (double)ri.y * ri.y;
        }
    }
    if (grid_sum<2>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) {
        for (int c = 0; c < 2; c++)
            if (mask & (1 << c)) {
                S->rho[c] = S->r0sq[c] = acc[c];
                if (S->restarts[c]++ == 0) S->it[c] = 0;
            }
        S->restart_mask = 0;
    }
}

// p = r + beta (p - omega v)
__global__ void __launch_bounds__(kQT)
k_qp_dir(int nn, const float2 *__restrict__ r, const float2 *__restrict__ v, float2 *__restrict__ p,
         const QpSolve *__restrict__ S) {
    if (!any_active(S)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    float b[2], w[2];
    for (int c = 0; c < 2; c++) {
        b[c] = S->active[c] ? (float)((S->rho[c] / S->rho_old[c]) * (S->alpha[c] / S->w[c])) : 0.f;
        w[c] = S->active[c] ? (float)S->w[c] : 0.f;
    }
    const float2 ri = r[i], vi = v[i], pi = p[i];
    p[i] = make_float2(ri.x + b[0] * (pi.x - w[0] * vi.x), ri.y + b[1] * (pi.y - w[1] * vi.y));
}

// v = A p; alpha = rho / (r0.v)
__global__ void __launch_bounds__(kQT)
k_qp_av(int nn, QpMat m, const float2 *__restrict__ p, const float2 *__restrict__ r0, float2 *__restrict__ v,
        double *__restrict__ partials, unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[2 * 32];
    if (!any_active(S)) return;
    double acc[2] = {0.0, 0.0};
    ROW_GROUPS(nn) {
        const float2 vi = spmv_row8(m, p, i, sub, i < nn);
        if (i < nn && sub == 0) {
            const float2 z = r0[i];
            v[i] = vi;
            acc[0] += (double)z.x * vi.x;
            acc[1] += (double)z.y * vi.y;
        }
    }
    if (grid_sum<2>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0)
        for (int c = 0; c < 2; c++) S->alpha[c] = S->active[c] ? S->rho[c] / acc[c] : 0.0;
}

// s = r - alpha v
__global__ void __launch_bounds__(kQT)
k_qp_s(int nn, const float2 *__restrict__ r, const float2 *__restrict__ v, float2 *__restrict__ s,
       const QpSolve *__restrict__ S) {
    if (!any_active(S)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const float ax = (float)S->alpha[0], ay = (float)S->alpha[1];
    const float2 ri = r[i], vi = v[i];
    s[i] = make_float2(ri.x - ax * vi.x, ri.y - ay * vi.y);
}

// t = A s; omega = t.s / t.t
__global__ void __launch_bounds__(kQT)
k_qp_at(int nn, QpMat m, const float2 *__restrict__ s, float2 *__restrict__ t, double *__restrict__ partials,
        unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[4 * 32];
    if (!any_active(S)) return;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    ROW_GROUPS(nn) {
        const float2 ti = spmv_row8(m, s, i, sub, i < nn);
        if (i < nn && sub == 0) {
            const float2 si = s[i];
            t[i] = ti;
            acc[0] += (double)ti.x * ti.x;
            acc[1] += (double)ti.y * ti.y;
            acc[2] += (double)ti.x * si.x;
            acc[3] += (double)ti.y * si.y;
        }
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0)
        for (int c = 0; c < 2; c++)
            if (S->active[c]) S->w[c] = acc[c] > 0.0 ? acc[2 + c] / acc[c] : 0.0;
}

// x += alpha p + omega s; r = s - omega t; |r|^2, r0.r; convergence per axis.
__global__ void __launch_bounds__(kQT)
k_qp_step(int nn, const float2 *__restrict__ p, const float2 *__restrict__ s, const float2 *__restrict__ t,
          const float2 *__restrict__ r0, float2 *__restrict__ x, float2 *__restrict__ r, double *__restrict__ partials,
          unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[4 * 32];
    if (!any_active(S)) return;
    float a[2], w[2];
    for (int c = 0; c < 2; c++) {
        a[c] = S->active[c] ? (float)S->alpha[c] : 0.f;
        w[c] = S->active[c] ? (float)S->w[c] : 0.f;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const float2 pi = p[i], si = s[i], ti = t[i], xi = x[i], z = r0[i];
        x[i] = make_float2(xi.x + a[0] * pi.x + w[0] * si.x, xi.y + a[1] * pi.y + w[1] * si.y);
        const float2 ri = make_float2(si.x - w[0] * ti.x, si.y - w[1] * ti.y);
        r[i] = ri;
        acc[0] += (double)ri.x * ri.x;
        acc[1] += (double)ri.y * ri.y;
        acc[2] += (double)z.x * ri.x;
        acc[3] += (double)z.y * ri.y;
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) {
        S->iters++;
        for (int c = 0; c < 2; c++) {
            if (!S->active[c]) continue;
            S->rr[c] = acc[c];
            S->r0r[c] = acc[2 + c];
            S->it[c]++;
            S->active[c] = S->rr[c] > S->tol2[c] && S->it[c] < S->max_it;
        }
    }
}

// Node centres <-> solution vector (setModuleCenter_2D clamp on the way back).
__global__ void k_qp_to_x(int nn, const float2 *__restrict__ pos, float2 *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nn) x[i] = pos[i];
}

__global__ void k_qp_from_x(Grid g, int nn, const float2 *__restrict__ x, const float2 *__restrict__ size,
                            float2 *__restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nn) pos[i] = clamp_center<float>(g, x[i], size[i]);
}

// PlaceDB::moveNodesCenterToCenter (PlaceDB/placedb.cpp:591-598).
__global__ void k_qp_center(Grid g, int nn, const float2 *__restrict__ size, float2 *__restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nn) {
        const float2 c = make_float2((float)(0.5 * ((double)g.urx + (double)g.llx)),
                                     (float)(0.5 * ((double)g.ury + (double)g.lly)));
        pos[i] = clamp_center<float>(g, c, size[i]);
    }
}

}  // namespace

void qp_bounds(const QpDev &q, const float2 *pos, double *hpwl, cudaStream_t st) {
    k_qp_bounds<<<qgrid(q.nnet), kQT, 0, st>>>(q.nnet, q.net_first, q.net_deg, q.owner, q.off, pos, q.bound,
                                                 q.partials, q.cnt, hpwl);
}

void qp_rows(const QpDev &q, int fill, const float2 *pos, cudaStream_t st) {
    k_qp_rows<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, fill, q.obj_pin_start, q.obj_pin_dev, q.pin_net, q.net_first,
                                             q.net_deg, q.bound, q.owner, q.off, pos, q.count, q.row_x, q.row_y,
                                             q.col_x, q.val_x, q.col_y, q.val_y, q.diag, q.rhs);
}

static QpMat mat(const QpDev &q) { return QpMat{q.row_x, q.col_x, q.row_y, q.col_y, q.val_x, q.val_y, q.diag}; }

void qp_init(const QpDev &q, int max_it, cudaStream_t st) {
    k_qp_init<<<qgrid(kRowLanes * q.nn), kQT, 0, st>>>(q.nn, mat(q), q.rhs, q.x, q.r, q.r0, q.p, q.v, q.partials,
                                                         q.cnt, max_it, q.solve);
    k_qp_zero<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, q.solve, q.x);
}

void qp_iterations(const QpDev &q, int count, cudaStream_t st) {
    const int b = qblocks(q.nn), bm = qgrid(kRowLanes * q.nn), br = qgrid(q.nn);
    for (int k = 0; k < count; k++) {
        k_qp_pre<<<1, 32, 0, st>>>(q.solve);
        k_qp_restart<<<bm, kQT, 0, st>>>(q.nn, mat(q), q.rhs, q.x, q.r, q.r0, q.partials, q.cnt, q.solve);
        k_qp_dir<<<b, kQT, 0, st>>>(q.nn, q.r, q.v, q.p, q.solve);
        k_qp_av<<<bm, kQT, 0, st>>>(q.nn, mat(q), q.p, q.r0, q.v, q.partials, q.cnt, q.solve);
        k_qp_s<<<b, kQT, 0, st>>>(q.nn, q.r, q.v, q.s, q.solve);
        k_qp_at<<<bm, kQT, 0, st>>>(q.nn, mat(q), q.s, q.t, q.partials, q.cnt, q.solve);
        k_qp_step<<<br, kQT, 0, st>>>(q.nn, q.p, q.s, q.t, q.r0, q.x, q.r, q.partials, q.cnt, q.solve);
    }
}

void qp_to_x(const QpDev &q, const float2 *pos, cudaStream_t st) {
    k_qp_to_x<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, pos, q.x);
}

void qp_from_x(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st) {
    k_qp_from_x<<<qblocks(q.nn), kQT, 0, st>>>(g, q.nn, q.x, size, pos);
}

void qp_center(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st) {
    k_qp_center<<<qblocks(q.nn), kQT, 0, st>>>(g, q.nn, size, pos);
}

int qp_partial_blocks(int nn, int nnet) { return std::max(qgrid(kRowLanes * nn), qgrid(nnet)); }

}  // namespace ep
