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
// Nets in device order: the nets above kWarpPins pins (the head of that
// order) take a warp each -- lane l scans pins l, l + 32, ... and the lanes'
// (value, first index) pairs meet in a tree that keeps the extreme value and,
// among equal values, the lower index, which is the serial scan's answer --
// and the others a thread each.  A grid-stride loop over 32 n_big + (nnet -
// n_big) slots; the HPWL of the net (double) joins the grid sum.
struct Ext {
    double v;
    int k;
};
__device__ __forceinline__ void ext_min(Ext &a, double v, int k) {
    if (v < a.v || (v == a.v && k < a.k)) a = Ext{v, k};
}
__device__ __forceinline__ void ext_max(Ext &a, double v, int k) {
    if (v > a.v || (v == a.v && k < a.k)) a = Ext{v, k};
}

__global__ void __launch_bounds__(kQT)
k_qp_bounds(int nnet, int n_big, const int32_t *__restrict__ order, const int32_t *__restrict__ first,
            const int32_t *__restrict__ deg, const int32_t *__restrict__ owner, const float2 *__restrict__ off,
            const float2 *__restrict__ pos, int4 *__restrict__ bound, float2 *__restrict__ abspin,
            double *__restrict__ partials, unsigned *__restrict__ cnt, double *__restrict__ hpwl) {
    __shared__ double sh[32];
    double acc[1] = {0.0};
    const long long big = 32LL * n_big, slots = big + (nnet - n_big);
    const int lane = threadIdx.x & 31;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < slots;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < big) {  // whole warps (big is a multiple of 32, so is the stride)
            const int n = order[t >> 5], f = first[n], d = deg[n];
            Ext lx{1.79769e308, 0x7fffffff}, hx{-1.79769e308, 0x7fffffff};
            Ext ly{1.79769e308, 0x7fffffff}, hy{-1.79769e308, 0x7fffffff};
            for (int k = lane; k < d; k += 32) {
                const float2 a = abs_pin(pos, off, owner[f + k], f + k);
                abspin[f + k] = a;
                ext_min(lx, a.x, k);
                ext_max(hx, a.x, k);
                ext_min(ly, a.y, k);
                ext_max(hy, a.y, k);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ext_min(lx, __shfl_xor_sync(0xffffffffu, lx.v, o), __shfl_xor_sync(0xffffffffu, lx.k, o));
                ext_max(hx, __shfl_xor_sync(0xffffffffu, hx.v, o), __shfl_xor_sync(0xffffffffu, hx.k, o));
                ext_min(ly, __shfl_xor_sync(0xffffffffu, ly.v, o), __shfl_xor_sync(0xffffffffu, ly.k, o));
                ext_max(hy, __shfl_xor_sync(0xffffffffu, hy.v, o), __shfl_xor_sync(0xffffffffu, hy.k, o));
            }
            if (lane == 0) {
                bound[n] = make_int4(lx.k, hx.k, ly.k, hy.k);
                acc[0] += (hx.v - lx.v) + (hy.v - ly.v);
            }
            continue;
        }
        const int n = order[n_big + (int)(t - big)], f = first[n], d = deg[n];
        double mnx = 1.79769e308, mxx = -1.79769e308, mny = 1.79769e308, mxy = -1.79769e308;
        int4 b = make_int4(0, 0, 0, 0);
        for (int k = 0; k < d; k++) {
            const float2 a = abs_pin(pos, off, owner[f + k], f + k);
            abspin[f + k] = a;
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

// Pair (i, owner of pin q2) on one axis (pa, oa: pin a's coordinate and
// offset on that axis): adds the pair's weight to the diagonal sum and its
// term to the right-hand side; returns the partner node when it is movable
// (an off-diagonal entry of weight -w), -1 when it is i itself (no pair) or
// fixed (right-hand side only).
__device__ __forceinline__ int pair_terms(int i, int nn, int q2, int axis, const int32_t *__restrict__ owner,
                                          const float2 *__restrict__ abspin, const float2 *__restrict__ off, float c,
                                          float pa, float oa, float &w, double &dsum, double &bsum) {
    const int j = owner[q2];
    if (j == i) return -1;
    const float2 pb2 = abspin[q2];
    const float pb = axis ? pb2.y : pb2.x, ob = axis ? off[q2].y : off[q2].x;
    w = pair_weight(c, fabsf(__fsub_rn(pa, pb)));
    dsum += w;
    if (j < nn) {
        bsum += -(double)w * (double)__fsub_rn(oa, ob);
        return j;
    }
    bsum += (double)w * (double)__fsub_rn(pb, oa);
    return -1;
}

// The count pass's test of a pair: the partner node when it gives an
// off-diagonal entry (movable and not i itself), else -1 -- the entries
// pair_terms reports, without the weights.
__device__ __forceinline__ int pair_partner(int i, int nn, int q2, const int32_t *__restrict__ owner) {
    const int j = owner[q2];
    return j != i && j < nn ? j : -1;
}

// A pin's partner set as a range: pins [0, end) of its net but `skip`, then
// `extra` (-1: none) -- the bound pins' sets of partners_x / partners_y.
struct PartnerRange {
    int end, skip, extra;
};
__device__ __forceinline__ bool range_x(int a, int d, int lo, int hi, PartnerRange &r) {
    if (a != lo && a != hi) return false;
    r = PartnerRange{d, a, -1};
    return true;
}
__device__ __forceinline__ bool range_y(int a, int d, int lo, int hi, PartnerRange &r) {
    if (a == hi) {
        r = PartnerRange{d, a, -1};
        return true;
    }
    if (a != lo) return false;
    r = PartnerRange{a, -1, hi > a ? hi : -1};
    return true;
}
// partner sets above kLongPartners pins are taken by the whole warp (placed
// after the row's short sets; the threshold fixes the order of a row's
// entries, so the SpMV's sums)
constexpr int kLongPartners = 32;
__device__ __forceinline__ bool is_long(const PartnerRange &r) {
    return r.end - (r.skip >= 0) + (r.extra >= 0) > kLongPartners;
}

// ---- CSR row offsets on the device ------------------------------------------
// The counts of both systems lie in one array c[0 .. 2 nn) (X rows, then Y
// rows); with E the exclusive prefix sum of c over [0, 2 nn], row_x[i] =
// E[i] (i <= nn) and row_y[i] = E[nn + i] - E[nn].  Three passes over
// chunks of kScanChunk entries: chunk totals; one block scanning the totals
// (and finding E[nn], E[2 nn]); each chunk's prefix sums.  Integer sums:
// the same offsets the host loop gave.
constexpr int kScanItems = 4, kScanChunk = kQT * kScanItems;

__device__ __forceinline__ int block_excl_scan(int v, int &total) {
    __shared__ int warp_tot[kQT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    int before = 0;
    total = 0;
    for (int k = 0; k < kQT / 32; k++) {
        if (k < w) before += warp_tot[k];
        total += warp_tot[k];
    }
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kQT) k_qp_chunk_sums(const int32_t *__restrict__ c, int n2, int32_t *__restrict__ sums) {
    const int base = blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    int v = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; u++) v += base + u < n2 ? c[base + u] : 0;
    int total;
    block_excl_scan(v, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// one block: exclusive scan of the chunk totals in place, then E[nn] and
// E[2 nn] into sums[nb], sums[nb + 1], and the overflow flag
__global__ void __launch_bounds__(kQT) k_qp_chunk_scan(int32_t *__restrict__ sums, int nb, const int32_t *__restrict__ c,
                                                      int nn, int cap_x, int cap_y, QpSolve *__restrict__ S) {
    __shared__ int carry_s;
    int carry = 0;
    for (int t0 = 0; t0 < nb; t0 += kQT) {
        const int i = t0 + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        int total;
        const int ex = block_excl_scan(v, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
    // E[nn]: the scanned total of nn's chunk plus that chunk's entries before nn
    const int ch = nn / kScanChunk;
    int part = 0;
    for (int k = ch * kScanChunk + threadIdx.x; k < nn; k += kQT) part += c[k];
    int total;
    block_excl_scan(part, total);
    if (threadIdx.x == 0) carry_s = carry;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int enn = sums[ch] + total;
        sums[nb] = enn;
        sums[nb + 1] = carry_s;
        S->overflow = enn > cap_x || carry_s - enn > cap_y;
    }
}

__global__ void __launch_bounds__(kQT) k_qp_offsets(const int32_t *__restrict__ c, int nn, const int32_t *__restrict__ sums,
                                                   int nb, int32_t *__restrict__ row_x, int32_t *__restrict__ row_y) {
    const int n2 = 2 * nn, base = blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    int v[kScanItems], s = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; u++) {
        v[u] = base + u < n2 ? c[base + u] : 0;
        s += v[u];
    }
    int total;
    int e = sums[blockIdx.x] + block_excl_scan(s, total);
    const int enn = sums[nb];
#pragma unroll
    for (int u = 0; u < kScanItems; u++) {
        const int i = base + u;  // E[i] = e
        if (i <= n2) {
            if (i <= nn) row_x[i] = e;
            if (i >= nn) row_y[i - nn] = e - enn;
        }
        e += v[u];
    }
}

// One movable node's row of both systems: counts (FILL = false: the
// partners only, no weights) or entries, diagonal and right-hand side
// (FILL = true).  A thread per node takes its pins'
// short partner sets in pin order; then the warp takes the long ones (a bound
// pin of a large net pairs with every other pin of it), in pin order, 32
// partners at a time, entries placed by a ballot prefix so they keep the
// partner order, the sums of the pairs' terms through a fixed xor tree.
template <bool FILL>
__global__ void __launch_bounds__(kQT)
k_qp_rows(int nn, const int32_t *__restrict__ obj_pin_start, const int32_t *__restrict__ obj_pin_dev,
          const int32_t *__restrict__ pin_net, const int32_t *__restrict__ first, const int32_t *__restrict__ deg,
          const int4 *__restrict__ bound, const int32_t *__restrict__ owner, const float2 *__restrict__ off,
          const float2 *__restrict__ abspin, int32_t *__restrict__ count, const int32_t *__restrict__ row_x,
          const int32_t *__restrict__ row_y, int32_t *__restrict__ col_x, float *__restrict__ val_x,
          int32_t *__restrict__ col_y, float *__restrict__ val_y, float2 *__restrict__ diag,
          float2 *__restrict__ rhs, const QpSolve *__restrict__ S) {
    constexpr bool fill = FILL;
    if (fill && S->overflow) return;  // uniform: the offsets exceed the allocation, the solve reports it
    const int i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
    const bool valid = i < nn;  // every lane stays for the warp's long sets
    int cnt[2] = {0, 0};
    double dsum[2] = {0.0, 0.0}, bsum[2] = {0.0, 0.0};
    const int row0[2] = {fill && valid ? row_x[i] : 0, fill && valid ? row_y[i] : 0};
    int32_t *const col[2] = {col_x, col_y};
    float *const val[2] = {val_x, val_y};
    const int k0 = valid ? obj_pin_start[i] : 0, np_i = valid ? obj_pin_start[i + 1] - k0 : 0;
    auto entry = [&](int axis, int j, float w, int at) {
        if (fill) {
            col[axis][row0[axis] + at] = j;
            val[axis][row0[axis] + at] = -w;
        }
    };
    for (int k = k0; k < k0 + np_i; k++) {
        const int q = obj_pin_dev[k], n = pin_net[q], f = first[n], d = deg[n], a = q - f;
        const int4 bd = bound[n];
        const float c = (float)(1.0 / ((double)d - 1.0));
        const float2 pa = abspin[q], oa = off[q];
        PartnerRange rx, ry;
        const bool lx = range_x(a, d, bd.x, bd.y, rx) && is_long(rx);
        const bool ly = range_y(a, d, bd.z, bd.w, ry) && is_long(ry);
        if (!lx)
            partners_x(a, d, bd.x, bd.y, [&](int b) {
                if constexpr (FILL) {
                    float w;
                    const int j = pair_terms(i, nn, f + b, 0, owner, abspin, off, c, pa.x, oa.x, w, dsum[0], bsum[0]);
                    if (j >= 0) entry(0, j, w, cnt[0]++);
                } else if (pair_partner(i, nn, f + b, owner) >= 0) {
                    cnt[0]++;
                }
            });
        if (!ly)
            partners_y(a, d, bd.z, bd.w, [&](int b) {
                if constexpr (FILL) {
                    float w;
                    const int j = pair_terms(i, nn, f + b, 1, owner, abspin, off, c, pa.y, oa.y, w, dsum[1], bsum[1]);
                    if (j >= 0) entry(1, j, w, cnt[1]++);
                } else if (pair_partner(i, nn, f + b, owner) >= 0) {
                    cnt[1]++;
                }
            });
    }
    const int steps = __reduce_max_sync(0xffffffffu, np_i);
    for (int s = 0; s < steps; s++) {
        int q = 0, f = 0, d = 0;
        PartnerRange r[2] = {{0, -1, -1}, {0, -1, -1}};
        bool lg[2] = {false, false};
        if (s < np_i) {
            q = obj_pin_dev[k0 + s];
            const int n = pin_net[q];
            f = first[n];
            d = deg[n];
            const int4 bd = bound[n];
            lg[0] = range_x(q - f, d, bd.x, bd.y, r[0]) && is_long(r[0]);
            lg[1] = range_y(q - f, d, bd.z, bd.w, r[1]) && is_long(r[1]);
        }
        for (int axis = 0; axis < 2; axis++) {
            unsigned todo = __ballot_sync(0xffffffffu, lg[axis]);
            while (todo) {  // warp-uniform
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const int si = __shfl_sync(0xffffffffu, i, src), sq = __shfl_sync(0xffffffffu, q, src);
                const int sf = __shfl_sync(0xffffffffu, f, src), sd = __shfl_sync(0xffffffffu, d, src);
                const int end = __shfl_sync(0xffffffffu, r[axis].end, src);
                const int skip = __shfl_sync(0xffffffffu, r[axis].skip, src);
                const int extra = __shfl_sync(0xffffffffu, r[axis].extra, src);
                const int at0 = __shfl_sync(0xffffffffu, cnt[axis], src);
                const float c = (float)(1.0 / ((double)sd - 1.0));
                const float2 pa2 = abspin[sq], oa2 = off[sq];
                const float pa = axis ? pa2.y : pa2.x, oa = axis ? oa2.y : oa2.x;
                const int row = fill ? (axis ? row_y[si] : row_x[si]) : 0;
                double ds = 0.0, bs = 0.0;
                int added = 0;
                for (int base = 0; base < end; base += 32) {
                    const int b = base + lane;
                    float w = 0.f;
                    int j = -1;
                    if (b < end && b != skip)
                        j = FILL ? pair_terms(si, nn, sf + b, axis, owner, abspin, off, c, pa, oa, w, ds, bs)
                                 : pair_partner(si, nn, sf + b, owner);
                    const unsigned m = __ballot_sync(0xffffffffu, j >= 0);
                    if (fill && j >= 0) {
                        const int at = row + at0 + added + __popc(m & ((1u << lane) - 1));
                        col[axis][at] = j;
                        val[axis][at] = -w;
                    }
                    added += __popc(m);
                }
                if (extra >= 0) {
                    int j = -1;
                    float w = 0.f;
                    if (lane == 0)
                        j = FILL ? pair_terms(si, nn, sf + extra, axis, owner, abspin, off, c, pa, oa, w, ds, bs)
                                 : pair_partner(si, nn, sf + extra, owner);
                    if (fill && j >= 0) {
                        col[axis][row + at0 + added] = j;
                        val[axis][row + at0 + added] = -w;
                    }
                    added += __shfl_sync(0xffffffffu, j >= 0 ? 1 : 0, 0);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ds += __shfl_xor_sync(0xffffffffu, ds, o);
                    bs += __shfl_xor_sync(0xffffffffu, bs, o);
                }
                if (lane == src) {
                    cnt[axis] += added;
                    dsum[axis] += ds;
                    bsum[axis] += bs;
                }
            }
        }
    }
    if (!valid) return;
    if (!fill) {
        count[i] = cnt[0];
        count[nn + i] = cnt[1];
    } else {
        diag[i] = make_float2((float)dsum[0], (float)dsum[1]);
        rhs[i] = make_float2((float)bsum[0], (float)bsum[1]);
    }
}

struct QpMat {
    const int32_t *row_x, *col_x, *row_y, *col_y;
    const float *val_x, *val_y;
    const float2 *diag;
};

// (A_x v.x, A_y v.y) for row i.  A row takes the kRowLanes lanes of an
// aligned lane group (lane sub of the group sums entries sub, sub + 8, ...
// of both axes in order, a fixed xor tree adds the 8 partial sums); a row of
// more than kLongRow entries on either axis (the bound pins of large nets)
// takes the whole warp after the short rows are done (lane l sums entries
// l, l + 32, ..., a fixed xor tree over the warp).  The diagonal term comes
// last.  The split depends only on the row lengths, so the result is the
// same on every run.  Every lane of the warp must call it (valid = false
// for lanes past the last row); every lane of the row's group gets the
// result.
constexpr int kRowLanes = 8, kRowsPerWarp = 32 / kRowLanes, kLongRow = 4 * kRowLanes;

__device__ __forceinline__ void row_partial(const QpMat &m, const float2 *__restrict__ v, int bx, int lx, int by,
                                            int ly, int lane, int step, float &ax, float &ay) {
    const int len = max(lx, ly);
#pragma unroll 2
    for (int k = lane; k < len; k += step) {
        if (k < lx) ax = fmaf(m.val_x[bx + k], v[m.col_x[bx + k]].x, ax);
        if (k < ly) ay = fmaf(m.val_y[by + k], v[m.col_y[by + k]].y, ay);
    }
}

__device__ __forceinline__ float2 spmv_row8(const QpMat &m, const float2 *__restrict__ v, int i, int sub, bool valid) {
    const int lane = threadIdx.x & 31;
    int bx = 0, lx = 0, by = 0, ly = 0;
    if (valid) {
        bx = m.row_x[i];
        lx = m.row_x[i + 1] - bx;
        by = m.row_y[i];
        ly = m.row_y[i + 1] - by;
    }
    const bool is_long = max(lx, ly) > kLongRow;
    float ax = 0.f, ay = 0.f;
    if (!is_long) row_partial(m, v, bx, lx, by, ly, sub, kRowLanes, ax, ay);
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    unsigned longs = __ballot_sync(0xffffffffu, is_long && sub == 0);
    while (longs) {  // warp-uniform
        const int src = __ffs(longs) - 1;
        longs &= longs - 1;
        const int lbx = __shfl_sync(0xffffffffu, bx, src), llx = __shfl_sync(0xffffffffu, lx, src);
        const int lby = __shfl_sync(0xffffffffu, by, src), lly = __shfl_sync(0xffffffffu, ly, src);
        float sx = 0.f, sy = 0.f;
        row_partial(m, v, lbx, llx, lby, lly, lane, 32, sx, sy);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (lane / kRowLanes == src / kRowLanes) {
            ax = sx;
            ay = sy;
        }
    }
    if (valid) {
        const float2 d = m.diag[i], vi = v[i];
        ax = fmaf(d.x, vi.x, ax);
        ay = fmaf(d.y, vi.y, ay);
    }
    return make_float2(ax, ay);
}

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
//   head     rho_old = rho; rho = r0.r; restart when |rho| < eps^2 r0sq
//            (in the finaliser of the previous step, or of the set-up)
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

// The head of an iteration (rho_old = rho; rho = r0.r; the restart test),
// run by the finaliser that ends the previous iteration (or the set-up).
__device__ void qp_pre(QpSolve *S) {
    if (!any_active(S)) return;
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
        qp_pre(S);
    }
}

// A zero right-hand side gives x = 0.
__global__ void k_qp_zero(int nn, const QpSolve *__restrict__ S, float2 *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn || !S->zero_mask) return;
    if (S->zero_mask & 1) x[i].x = 0.f;
    if (S->zero_mask & 2) x[i].y = 0.f;
}



// Restart of the flagged systems: r = b - A x, r0 = r; rho = r0sq = |r|^2.
__global__ void __launch_bounds__(kQT)
k_qp_restart(int nn, QpMat m, const float2 *__restrict__ rhs, const float2 *__restrict__ x, float2 *__restrict__ r,
             float2 *__restrict__ r0, double *__restrict__ partials, unsigned *__restrict__ cnt,
             QpSolve *__restrict__ S) {
    __shared__ double sh[2 * 32];
    pdl_begin();
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

// p = r + beta (p - omega v); with a diagonal preconditioner (dinv, else
// null) also y = M^-1 p, the vector the SpMV then takes
__global__ void __launch_bounds__(kQT)
k_qp_dir(int nn, const float2 *__restrict__ r, const float2 *__restrict__ v, float2 *__restrict__ p,
         const float2 *__restrict__ dinv, float2 *__restrict__ y, const QpSolve *__restrict__ S) {
    pdl_begin();
    if (!any_active(S)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    float b[2], w[2];
    for (int c = 0; c < 2; c++) {
        b[c] = S->active[c] ? (float)((S->rho[c] / S->rho_old[c]) * (S->alpha[c] / S->w[c])) : 0.f;
        w[c] = S->active[c] ? (float)S->w[c] : 0.f;
    }
    const float2 ri = r[i], vi = v[i], pi = p[i];
    const float2 pn = make_float2(ri.x + b[0] * (pi.x - w[0] * vi.x), ri.y + b[1] * (pi.y - w[1] * vi.y));
    p[i] = pn;
    if (dinv) {
        const float2 d = dinv[i];
        y[i] = make_float2(pn.x * d.x, pn.y * d.y);
    }
}

// v = A p; alpha = rho / (r0.v)
__global__ void __launch_bounds__(kQT)
k_qp_av(int nn, QpMat m, const float2 *__restrict__ p, const float2 *__restrict__ r0, float2 *__restrict__ v,
        double *__restrict__ partials, unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[2 * 32];
    pdl_begin();
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

// s = r - alpha v; with the preconditioner also z = M^-1 s
__global__ void __launch_bounds__(kQT)
k_qp_s(int nn, const float2 *__restrict__ r, const float2 *__restrict__ v, float2 *__restrict__ s,
       const float2 *__restrict__ dinv, float2 *__restrict__ z, const QpSolve *__restrict__ S) {
    pdl_begin();
    if (!any_active(S)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const float ax = (float)S->alpha[0], ay = (float)S->alpha[1];
    const float2 ri = r[i], vi = v[i];
    const float2 si = make_float2(ri.x - ax * vi.x, ri.y - ay * vi.y);
    s[i] = si;
    if (dinv) {
        const float2 d = dinv[i];
        z[i] = make_float2(si.x * d.x, si.y * d.y);
    }
}

// t = A z (z = s, or M^-1 s); omega = t.s / t.t
__global__ void __launch_bounds__(kQT)
k_qp_at(int nn, QpMat m, const float2 *__restrict__ z, const float2 *__restrict__ s, float2 *__restrict__ t,
        double *__restrict__ partials, unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[4 * 32];
    pdl_begin();
    if (!any_active(S)) return;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    ROW_GROUPS(nn) {
        const float2 ti = spmv_row8(m, z, i, sub, i < nn);
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

// x += alpha y + omega z (y, z = p, s, or their preconditioned forms);
// r = s - omega t; |r|^2, r0.r; convergence per axis.
__global__ void __launch_bounds__(kQT)
k_qp_step(int nn, const float2 *__restrict__ p, const float2 *__restrict__ zs, const float2 *__restrict__ s,
          const float2 *__restrict__ t, const float2 *__restrict__ r0, float2 *__restrict__ x, float2 *__restrict__ r,
          double *__restrict__ partials, unsigned *__restrict__ cnt, QpSolve *__restrict__ S) {
    __shared__ double sh[4 * 32];
    pdl_begin();
    if (!any_active(S)) return;
    float a[2], w[2];
    for (int c = 0; c < 2; c++) {
        a[c] = S->active[c] ? (float)S->alpha[c] : 0.f;
        w[c] = S->active[c] ? (float)S->w[c] : 0.f;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const float2 pi = p[i], zi = zs[i], si = s[i], ti = t[i], xi = x[i], z = r0[i];
        x[i] = make_float2(xi.x + a[0] * pi.x + w[0] * zi.x, xi.y + a[1] * pi.y + w[1] * zi.y);
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
        qp_pre(S);
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
    k_qp_bounds<<<qgrid(31 * q.n_big + q.nnet), kQT, 0, st>>>(q.nnet, q.n_big, q.net_order, q.net_first, q.net_deg,
                                                               q.owner, q.off, pos, q.bound, q.abspin, q.partials,
                                                               q.cnt, hpwl);
}

void qp_rows(const QpDev &q, int fill, cudaStream_t st) {
    (fill ? k_qp_rows<true> : k_qp_rows<false>)<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, q.obj_pin_start, q.obj_pin_dev, q.pin_net, q.net_first,
                                             q.net_deg, q.bound, q.owner, q.off, q.abspin, q.count, q.row_x, q.row_y,
                                             q.col_x, q.val_x, q.col_y, q.val_y, q.diag, q.rhs, q.solve);
}

int qp_scan_blocks(int nn) { return (2 * nn + 1 + kScanChunk - 1) / kScanChunk; }

void qp_offsets(const QpDev &q, cudaStream_t st) {
    const int nb = qp_scan_blocks(q.nn);
    k_qp_chunk_sums<<<nb, kQT, 0, st>>>(q.count, 2 * q.nn, q.scan);
    k_qp_chunk_scan<<<1, kQT, 0, st>>>(q.scan, nb, q.count, q.nn, q.cap_x, q.cap_y, q.solve);
    k_qp_offsets<<<nb, kQT, 0, st>>>(q.count, q.nn, q.scan, nb, q.row_x, q.row_y);
}

static QpMat mat(const QpDev &q) { return QpMat{q.row_x, q.col_x, q.row_y, q.col_y, q.val_x, q.val_y, q.diag}; }

void qp_init(const QpDev &q, int max_it, cudaStream_t st) {
    k_qp_init<<<qgrid(kRowLanes * q.nn), kQT, 0, st>>>(q.nn, mat(q), q.rhs, q.x, q.r, q.r0, q.p, q.v, q.partials,
                                                         q.cnt, max_it, q.solve);
    k_qp_zero<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, q.solve, q.x);
}

// M^-1 of the Jacobi preconditioner: 1 / diagonal (1 where the diagonal is 0)
__global__ void k_qp_dinv(int nn, const float2 *__restrict__ diag, float2 *__restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const float2 d = diag[i];
    dinv[i] = make_float2(d.x != 0.f ? 1.f / d.x : 1.f, d.y != 0.f ? 1.f / d.y : 1.f);
}

void qp_iterations(const QpDev &q, int count, bool jacobi, cudaStream_t st) {
    const int b = qblocks(q.nn), bm = qgrid(kRowLanes * q.nn), br = qgrid(q.nn);
    for (int k = 0; k < count; k++) {
        // programmatic serialisation: each kernel's blocks are resident and
        // waiting (pdl_begin) while the previous one drains
        launch_k(k_qp_restart, bm, kQT, 0, st, q.nn, mat(q), q.rhs, q.x, q.r, q.r0, q.partials, q.cnt, q.solve);
        // Eigen's preconditioned form: y = M^-1 p and z = M^-1 s go into the
        // SpMVs and the update; without a preconditioner y = p and z = s
        const float2 *dinv = jacobi ? q.dinv : nullptr;
        const float2 *y = jacobi ? q.y : q.p, *z = jacobi ? q.z : q.s;
        launch_k(k_qp_dir, b, kQT, 0, st, q.nn, q.r, q.v, q.p, dinv, q.y, q.solve);
        launch_k(k_qp_av, bm, kQT, 0, st, q.nn, mat(q), y, q.r0, q.v, q.partials, q.cnt, q.solve);
        launch_k(k_qp_s, b, kQT, 0, st, q.nn, q.r, q.v, q.s, dinv, q.z, q.solve);
        launch_k(k_qp_at, bm, kQT, 0, st, q.nn, mat(q), z, q.s, q.t, q.partials, q.cnt, q.solve);
        launch_k(k_qp_step, br, kQT, 0, st, q.nn, y, z, q.s, q.t, q.r0, q.x, q.r, q.partials, q.cnt, q.solve);
    }
}

void qp_dinv(const QpDev &q, cudaStream_t st) { k_qp_dinv<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, q.diag, q.dinv); }

void qp_to_x(const QpDev &q, const float2 *pos, cudaStream_t st) {
    k_qp_to_x<<<qblocks(q.nn), kQT, 0, st>>>(q.nn, pos, q.x);
}

void qp_from_x(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st) {
    k_qp_from_x<<<qblocks(q.nn), kQT, 0, st>>>(g, q.nn, q.x, size, pos);
}

void qp_center(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st) {
    k_qp_center<<<qblocks(q.nn), kQT, 0, st>>>(g, q.nn, size, pos);
}

int qp_partial_blocks(int nn, int nnet) { return kQpMaxBlocks; }

}  // namespace ep
