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
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (n < nnet) {
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
        if (d > 0) acc[0] = (mxx - mnx) + (mxy - mny);
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

// (A_x v.x, A_y v.y) for row i.
__device__ __forceinline__ float2 spmv_row(const QpMat &m, const float2 *__restrict__ v, int i) {
    const float2 d = m.diag[i], vi = v[i];
    float ax = d.x * vi.x, ay = d.y * vi.y;
    for (int e = m.row_x[i]; e < m.row_x[i + 1]; e++) ax = fmaf(m.val_x[e], v[m.col_x[e]].x, ax);
    for (int e = m.row_y[i]; e < m.row_y[i + 1]; e++) ay = fmaf(m.val_y[e], v[m.col_y[e]].y, ay);
    return make_float2(ax, ay);
}

__device__ __forceinline__ void qp_finish(double *acc, int nv, double *out) {
    for (int k = 0; k < nv; k++) out[k] = acc[k];
}

// r = b - A x, r0 = r, p = v = 0; sums (r.r per system, b.b per system).
__global__ void __launch_bounds__(kQT)
k_qp_init(int nn, QpMat m, const float2 *__restrict__ rhs, const float2 *__restrict__ x, float2 *__restrict__ r,
          float2 *__restrict__ r0, float2 *__restrict__ p, float2 *__restrict__ v, double *__restrict__ partials,
          unsigned *__restrict__ cnt, double *__restrict__ out) {
    __shared__ double sh[4 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < nn) {
        const float2 ax = spmv_row(m, x, i), bi = rhs[i];
        const float2 ri = make_float2(bi.x - ax.x, bi.y - ax.y);
        r[i] = ri;
        r0[i] = ri;
        p[i] = make_float2(0.f, 0.f);
        v[i] = make_float2(0.f, 0.f);
        acc[0] = (double)ri.x * ri.x;
        acc[1] = (double)ri.y * ri.y;
        acc[2] = (double)bi.x * bi.x;
        acc[3] = (double)bi.y * bi.y;
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) qp_finish(acc, 4, out);
}

// p = r + beta (p - w v)
__global__ void __launch_bounds__(kQT)
k_qp_dir(int nn, float2 beta, float2 w, const float2 *__restrict__ r, const float2 *__restrict__ v,
         float2 *__restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const float2 ri = r[i], vi = v[i], pi = p[i];
    p[i] = make_float2(ri.x + beta.x * (pi.x - w.x * vi.x), ri.y + beta.y * (pi.y - w.y * vi.y));
}

// v = A p; sums r0.v per system.
__global__ void __launch_bounds__(kQT)
k_qp_av(int nn, QpMat m, const float2 *__restrict__ p, const float2 *__restrict__ r0, float2 *__restrict__ v,
        double *__restrict__ partials, unsigned *__restrict__ cnt, double *__restrict__ out) {
    __shared__ double sh[2 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (i < nn) {
        const float2 vi = spmv_row(m, p, i), z = r0[i];
        v[i] = vi;
        acc[0] = (double)z.x * vi.x;
        acc[1] = (double)z.y * vi.y;
    }
    if (grid_sum<2>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) qp_finish(acc, 2, out);
}

// s = r - alpha v
__global__ void __launch_bounds__(kQT)
k_qp_s(int nn, float2 alpha, const float2 *__restrict__ r, const float2 *__restrict__ v, float2 *__restrict__ s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const float2 ri = r[i], vi = v[i];
    s[i] = make_float2(ri.x - alpha.x * vi.x, ri.y - alpha.y * vi.y);
}

// t = A s; sums t.t and t.s per system.
__global__ void __launch_bounds__(kQT)
k_qp_at(int nn, QpMat m, const float2 *__restrict__ s, float2 *__restrict__ t, double *__restrict__ partials,
        unsigned *__restrict__ cnt, double *__restrict__ out) {
    __shared__ double sh[4 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < nn) {
        const float2 ti = spmv_row(m, s, i), si = s[i];
        t[i] = ti;
        acc[0] = (double)ti.x * ti.x;
        acc[1] = (double)ti.y * ti.y;
        acc[2] = (double)ti.x * si.x;
        acc[3] = (double)ti.y * si.y;
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) qp_finish(acc, 4, out);
}

// x += alpha p + w s; r = s - w t; sums r.r and r0.r per system.
__global__ void __launch_bounds__(kQT)
k_qp_step(int nn, float2 alpha, float2 w, const float2 *__restrict__ p, const float2 *__restrict__ s,
          const float2 *__restrict__ t, const float2 *__restrict__ r0, float2 *__restrict__ x,
          float2 *__restrict__ r, double *__restrict__ partials, unsigned *__restrict__ cnt,
          double *__restrict__ out) {
    __shared__ double sh[4 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < nn) {
        const float2 pi = p[i], si = s[i], ti = t[i], xi = x[i], z = r0[i];
        x[i] = make_float2(xi.x + alpha.x * pi.x + w.x * si.x, xi.y + alpha.y * pi.y + w.y * si.y);
        const float2 ri = make_float2(si.x - w.x * ti.x, si.y - w.y * ti.y);
        r[i] = ri;
        acc[0] = (double)ri.x * ri.x;
        acc[1] = (double)ri.y * ri.y;
        acc[2] = (double)z.x * ri.x;
        acc[3] = (double)z.y * ri.y;
    }
    if (grid_sum<4>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) qp_finish(acc, 4, out);
}

// BiCGSTAB restart of the systems in `mask` (bit 0 X, bit 1 Y): r = b - A x,
// r0 = r; sums r.r per system.
__global__ void __launch_bounds__(kQT)
k_qp_restart(int nn, int mask, QpMat m, const float2 *__restrict__ rhs, const float2 *__restrict__ x,
             float2 *__restrict__ r, float2 *__restrict__ r0, double *__restrict__ partials,
             unsigned *__restrict__ cnt, double *__restrict__ out) {
    __shared__ double sh[2 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (i < nn) {
        const float2 ax = spmv_row(m, x, i), bi = rhs[i];
        float2 ri = r[i], zi = r0[i];
        if (mask & 1) ri.x = zi.x = bi.x - ax.x;
        if (mask & 2) ri.y = zi.y = bi.y - ax.y;
        r[i] = ri;
        r0[i] = zi;
        acc[0] = (double)ri.x * ri.x;
        acc[1] = (double)ri.y * ri.y;
    }
    if (grid_sum<2>(acc, sh, partials, cnt, gridDim.x, blockIdx.x) && threadIdx.x == 0) qp_finish(acc, 2, out);
}

// A zero right-hand side gives x = 0 (Eigen's BiCGSTAB returns at once).
__global__ void k_qp_zero_axis(int nn, int axis, float2 *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    if (axis == 0)
        x[i].x = 0.f;
    else
        x[i].y = 0.f;
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
    k_qp_bounds<<<qblocks(q.nnet), kQT, 0, st>>>(q.nnet, q.net_first, q.net_deg, q.owner, q.off, pos, q.bound,
                                                 q.partials, q.cnt, hpwl);
}

void qp_rows(const QpDev &q, int fill, const float2 *pos, cudaStream_t st) {
    k_qp_rows<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, fill, q.obj_pin_start, q.obj_pin_dev, q.pin_net, q.net_first,
                                             q.net_deg, q.bound, q.owner, q.off, pos, q.count, q.row_x, q.row_y,
                                             q.col_x, q.val_x, q.col_y, q.val_y, q.diag, q.rhs);
}

static QpMat mat(const QpDev &q) { return QpMat{q.row_x, q.col_x, q.row_y, q.col_y, q.val_x, q.val_y, q.diag}; }

void qp_init(const QpDev &q, cudaStream_t st) {
    k_qp_init<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, mat(q), q.rhs, q.x, q.r, q.r0, q.p, q.v, q.partials, q.cnt,
                                             q.out);
}

void qp_dir(const QpDev &q, float2 beta, float2 w, cudaStream_t st) {
    k_qp_dir<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, beta, w, q.r, q.v, q.p);
}

void qp_av(const QpDev &q, cudaStream_t st) {
    k_qp_av<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, mat(q), q.p, q.r0, q.v, q.partials, q.cnt, q.out);
}

void qp_s(const QpDev &q, float2 alpha, cudaStream_t st) {
    k_qp_s<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, alpha, q.r, q.v, q.s);
}

void qp_at(const QpDev &q, cudaStream_t st) {
    k_qp_at<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, mat(q), q.s, q.t, q.partials, q.cnt, q.out);
}

void qp_step(const QpDev &q, float2 alpha, float2 w, cudaStream_t st) {
    k_qp_step<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, alpha, w, q.p, q.s, q.t, q.r0, q.x, q.r, q.partials, q.cnt,
                                             q.out);
}

void qp_restart(const QpDev &q, int mask, cudaStream_t st) {
    k_qp_restart<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, mask, mat(q), q.rhs, q.x, q.r, q.r0, q.partials, q.cnt,
                                                q.out);
}

void qp_zero_axis(const QpDev &q, int axis, cudaStream_t st) {
    k_qp_zero_axis<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, axis, q.x);
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

int qp_partial_blocks(int nn, int nnet) { return std::max(qblocks(nn), qblocks(nnet)); }

}  // namespace ep
