// dct_fft.cu -- the electrostatic Poisson solve of FFT_2D::doFFT
// (FFT/fft.cpp:191-284) by fast transforms: the same sums as dct.cu,
//   a   = C_nx rho C_ny^T,   P = a .* K,
//   E_x = S_nx^T diag(wx) P C_ny,   E_y = C_nx^T P diag(wy) S_ny,   phi = C_nx^T P C_ny,
// evaluated as 1-D transforms along one axis at a time, each a length-n
// complex FFT in shared memory (n a power of two), O(n^2 log n) per map
// instead of the GEMMs' O(n^3).
//
// The 1-D transforms (C_n[k][j] = cos(pi k (j+1/2) / n)):
//   DCT-II  X = C_n x     by Makhoul's permutation v = (x0, x2, .., x3, x1),
//                         V = FFT(v), X[k] = Re(V[k] e^{-i pi k / 2n});
//   DCT-III y = C_n^T X   by the inverse of that: Z[k] = (X~[k] - i X[n-k])
//                         e^{i pi k / 2n} / 2 (X~[0] = 2 X[0], X[n] = 0),
//                         z = IFFT(Z) (unnormalised), y[2j] = z[j],
//                         y[2j+1] = z[n-1-j] (z is real: Z is Hermitian);
//   sine    y = S_n^T X   = (-1)^j C_n^T b with b[0] = 0, b[k] = X[n-k]
//                         (sin(pi (n-k)(j+1/2)/n) = (-1)^j cos(pi k (j+1/2)/n)).
// Two real sequences share one complex FFT (one in the real, one in the
// imaginary part) wherever the inputs or outputs are real.
//
// Three kernels, maps x-major [nx][ny] as everywhere in the engine:
//   k_fft_rows_fwd  T[x][v]  = DCT-II of rho[x][:] along y          (2 rows per FFT)
//   k_fft_cols      per column v of T: DCT-II along x, times K, then
//                   X1[:][v] = S^T diag(wx) P[:][v] and X2[:][v] = C^T P[:][v]
//                   (2 columns per block; X1 of two columns share one complex
//                   IFFT and X2 of two columns another: P is dominated by its
//                   low frequencies, so an FFT carrying P beside wx P would
//                   round the small E inputs relative to |P|)
//   k_fft_rows_inv  per row x: E_x = C^T X1[x][:], E_y = S^T diag(wy) X2[x][:]
//                   (one complex IFFT), phi = C^T X2[x][:] when asked
// Twiddles, the e^{i pi k / 2n} factors and the frequency weights come from
// tables computed in double on the host, staged in shared memory by every
// block before it waits on the previous grid.  The kernels are instantiated
// per log2 n so that every loop has a fixed trip count and a thread issues
// all its loads before it uses any, and per working precision R (float for
// the engine's mixed-precision form, double for the plain FP64 form; the
// tables are rounded to R).
#include <algorithm>
#include <array>
#include <cmath>
#include <new>
#include <utility>
#include <vector>

#include "engine.h"

namespace ep {

namespace {

constexpr int kThreads = 256;
// Columns per block of the column pass (128 threads per column).  Measured at
// 512^2 in FP32: 2 columns (256 blocks) 18.5 us for the three passes and
// 14.67 ms per solve, 4 columns (128 blocks, 512 threads) 19.0 us, 14.86 ms.
constexpr int kCols = 2;

struct FftPlan {
    int lognx = 0, logny = 0;
    int fp64 = 0;
    // twiddles, stage-major: stage s (half-size h = 2^s) holds e^{-i pi j / h},
    // j < h, at [h - 1 + j]; n - 1 entries per axis (vec2<R>)
    void *twx = nullptr, *twy = nullptr;
    // (cos, sin)(pi k / 2n), k <= n/2 (vec2<R>)
    void *qx = nullptr, *qy = nullptr;
    void *wx = nullptr, *wy = nullptr;  // frequency weights (R)
    double kscale = 0.0;                // 4 / (nx ny)
    void *T = nullptr;                  // [nx][ny] after the first pass (R)
    void *X = nullptr;                  // X1, X2: [2][nx][ny] (R)
    size_t smem_rows_fwd = 0, smem_cols = 0, smem_rows_inv = 0;
    int pairs_fwd = 1, rows_inv = 1;
};

__device__ __forceinline__ int makhoul(int j, int n) { return (j & 1) ? n - 1 - (j >> 1) : (j >> 1); }

__device__ __forceinline__ int brev(int i, int logn) { return (int)(__brev((unsigned)i) >> (32 - logn)); }

template <typename R>
__device__ __forceinline__ vec2<R> cmul(vec2<R> a, vec2<R> b) {
    return mk2<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// The dynamic shared memory of a kernel, as an array of R's complex type.
template <typename R>
__device__ __forceinline__ vec2<R> *smem_c() {
    extern __shared__ __align__(16) unsigned char fft_smem[];
    return reinterpret_cast<vec2<R> *>(fft_smem);
}

// In-place decimation-in-time FFT of nseq (<= NSEQ) length-2^LOGN sequences
// stored back to back in shared memory, input in bit-reversed order, output
// in natural order, by NT threads.  tw: the stage-major twiddles, in shared
// memory.  INV uses e^{+...} (unnormalised inverse).  The radix-2 stages run
// in pairs: a thread loads the four elements that stages s and s+1 combine,
// applies both stages in registers (the same operations as two radix-2
// passes) and stores them, one barrier per pair; an odd stage count starts
// with one radix-2 pass.  Ends with a block barrier.
template <bool INV, int LOGN, int NSEQ, int NT, typename R>
__device__ __forceinline__ void block_fft(vec2<R> *buf, int nseq, const vec2<R> *tw) {
    using C = vec2<R>;
    constexpr int half = 1 << (LOGN - 1), quarter = 1 << (LOGN - 2);
    constexpr int it2 = (NSEQ * half + NT - 1) / NT, it4 = (NSEQ * quarter + NT - 1) / NT;
    auto twiddle = [&](int i) {
        C w = tw[i];
        if (INV) w.y = -w.y;
        return w;
    };
    constexpr int first = LOGN & 1;  // stages done by the radix-2 pass
    if (first) {
        const int total = nseq * half;
#pragma unroll
        for (int it = 0; it < it2; it++) {
            const int j = threadIdx.x + it * NT;
            if (j >= total) break;
            const int i0 = 2 * j;  // stage 0: h = 1, twiddle 1
            const C a = buf[i0], c = buf[i0 + 1];
            buf[i0] = mk2<R>(a.x + c.x, a.y + c.y);
            buf[i0 + 1] = mk2<R>(a.x - c.x, a.y - c.y);
        }
        __syncthreads();
    }
    const int total = nseq * quarter;
#pragma unroll
    for (int s = first; s < LOGN; s += 2) {
        const int h = 1 << s;
#pragma unroll
        for (int it = 0; it < it4; it++) {
            const int j = threadIdx.x + it * NT;
            if (j >= total) break;
            const int q = j >> (LOGN - 2), b = j & (quarter - 1);
            const int pos = b & (h - 1);
            const int i0 = (q << LOGN) + ((b >> s) << (s + 2)) + pos;
            C a0 = buf[i0], a1 = buf[i0 + h], a2 = buf[i0 + 2 * h], a3 = buf[i0 + 3 * h];
            // stage s: pairs (i0, i0+h) and (i0+2h, i0+3h), one twiddle
            const C w1 = twiddle(h - 1 + pos);
            C t = cmul<R>(a1, w1);
            a1 = mk2<R>(a0.x - t.x, a0.y - t.y);
            a0 = mk2<R>(a0.x + t.x, a0.y + t.y);
            t = cmul<R>(a3, w1);
            a3 = mk2<R>(a2.x - t.x, a2.y - t.y);
            a2 = mk2<R>(a2.x + t.x, a2.y + t.y);
            // stage s+1: pairs (i0, i0+2h) at pos and (i0+h, i0+3h) at pos+h
            t = cmul<R>(a2, twiddle(2 * h - 1 + pos));
            buf[i0] = mk2<R>(a0.x + t.x, a0.y + t.y);
            buf[i0 + 2 * h] = mk2<R>(a0.x - t.x, a0.y - t.y);
            t = cmul<R>(a3, twiddle(2 * h - 1 + pos + h));
            buf[i0 + h] = mk2<R>(a1.x + t.x, a1.y + t.y);
            buf[i0 + 3 * h] = mk2<R>(a1.x - t.x, a1.y - t.y);
        }
        __syncthreads();
    }
}

// The twiddles (n - 1) and the (cos, sin)(pi k / 2n) factors (n/2 + 1) of
// one axis, and its frequency weights (n, when w is given), into shared
// memory, every load of a thread issued before its first store (one memory
// round trip).  These are constant tables, so blocks stage them before
// waiting on the previous grid; the caller's barrier publishes them.
template <int LOGN, int NT, typename R>
__device__ __forceinline__ void stage_tables(vec2<R> *tw_s, vec2<R> *q_s, R *w_s, const vec2<R> *__restrict__ tw,
                                             const vec2<R> *__restrict__ q, const R *__restrict__ w) {
    constexpr int n = 1 << LOGN;
    constexpr int it_t = (n - 1 + NT - 1) / NT, it_q = (n / 2 + 1 + NT - 1) / NT, it_w = (n + NT - 1) / NT;
    vec2<R> vt[it_t], vq[it_q];
    R vw[it_w];
#pragma unroll
    for (int it = 0; it < it_t; it++) {
        const int i = threadIdx.x + it * NT;
        if (i < n - 1) vt[it] = tw[i];
    }
#pragma unroll
    for (int it = 0; it < it_q; it++) {
        const int i = threadIdx.x + it * NT;
        if (i <= n / 2) vq[it] = q[i];
    }
#pragma unroll
    for (int it = 0; it < it_w; it++) {
        const int i = threadIdx.x + it * NT;
        if (w && i < n) vw[it] = w[i];
    }
#pragma unroll
    for (int it = 0; it < it_t; it++) {
        const int i = threadIdx.x + it * NT;
        if (i < n - 1) tw_s[i] = vt[it];
    }
#pragma unroll
    for (int it = 0; it < it_q; it++) {
        const int i = threadIdx.x + it * NT;
        if (i <= n / 2) q_s[i] = vq[it];
    }
#pragma unroll
    for (int it = 0; it < it_w; it++) {
        const int i = threadIdx.x + it * NT;
        if (w && i < n) w_s[i] = vw[it];
    }
}

// Spectrum entry k (1 <= k <= n/2) of the DCT-III input X (entry n-k is its
// conjugate): (X[k] c + X[n-k] s, X[k] s - X[n-k] c) / 2.
template <typename R>
__device__ __forceinline__ vec2<R> dct3_spec(R xk, R xm, vec2<R> cs) {
    return mk2<R>((R)0.5 * (xk * cs.x + xm * cs.y), (R)0.5 * (xk * cs.y - xm * cs.x));
}

// Entries k and n-k (bit-reversed positions) of the complex spectrum that
// carries DCT-III input a in its real part and b in its imaginary part.
template <typename R>
__device__ __forceinline__ void pack_spec(vec2<R> *o, int k, int m, int logn, vec2<R> sa, vec2<R> sb, bool self) {
    o[brev(k, logn)] = mk2<R>(sa.x - sb.y, sa.y + sb.x);
    if (!self) o[brev(m, logn)] = mk2<R>(sa.x + sb.y, sb.x - sa.y);
}

// Shared-memory bytes of the per-axis tables (twiddles, factors, weights).
template <typename R>
__host__ __device__ constexpr size_t table_bytes(int n) {
    return sizeof(vec2<R>) * ((size_t)n - 1 + n / 2 + 1) + sizeof(R) * n;
}

// Row pairs (pass 1) and rows (pass 3) per block: enough sequences that a
// butterfly stage has a thread each.
template <int LOGN>
__host__ __device__ constexpr int seqs_per_block() {
    return (2 * kThreads) >> LOGN > 1 ? (2 * kThreads) >> LOGN : 1;
}

// ---- pass 1: rows along y --------------------------------------------------
template <int LOGN, typename R>
__global__ void __launch_bounds__(kThreads)
k_fft_rows_fwd(const R *__restrict__ rho, R *__restrict__ T, int pairs, const vec2<R> *__restrict__ tw,
               const vec2<R> *__restrict__ q, const DevScalars *__restrict__ S) {
    using C = vec2<R>;
    constexpr int n = 1 << LOGN, NS = seqs_per_block<LOGN>();
    C *sm = smem_c<R>();
    C *tw_s = sm + NS * n, *q_s = tw_s + n - 1;
    stage_tables<LOGN, kThreads, R>(tw_s, q_s, nullptr, tw, q, nullptr);
    pdl_begin();
    if (S && S->done) return;
    const int x0 = blockIdx.x * pairs * 2;
    constexpr int li = (NS * n + kThreads - 1) / kThreads;
    C v[li];
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e < (pairs << LOGN)) {
            const int p = e >> LOGN, y = e & (n - 1);
            const size_t ra = (size_t)(x0 + 2 * p) * n;
            v[it] = mk2<R>(rho[ra + y], rho[ra + n + y]);
        }
    }
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e < (pairs << LOGN)) sm[(e & ~(n - 1)) + brev(makhoul(e & (n - 1), n), LOGN)] = v[it];
    }
    __syncthreads();
    block_fft<false, LOGN, NS, kThreads, R>(sm, pairs, tw_s);
    constexpr int hk = n / 2 + 1;
    constexpr int pi_ = (NS * hk + kThreads - 1) / kThreads;
#pragma unroll
    for (int it = 0; it < pi_; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e >= pairs * hk) break;
        const int p = e / hk, k = e - p * hk;
        const C *z = sm + (p << LOGN);
        const C Z = z[k], M = z[(n - k) & (n - 1)];
        // V_a = (Z + conj M) / 2, V_b = (Z - conj M) / 2i
        const R ar = (R)0.5 * (Z.x + M.x), ai = (R)0.5 * (Z.y - M.y);
        const R br = (R)0.5 * (Z.y + M.y), bi = (R)-0.5 * (Z.x - M.x);
        const C cs = q_s[k];
        R *ta = T + (size_t)(x0 + 2 * p) * n, *tb = ta + n;
        ta[k] = ar * cs.x + ai * cs.y;
        tb[k] = br * cs.x + bi * cs.y;
        if (k != 0 && k != n / 2) {
            ta[n - k] = ar * cs.y - ai * cs.x;
            tb[n - k] = br * cs.y - bi * cs.x;
        }
    }
}

// ---- pass 2: columns along x -----------------------------------------------
// COLS (2 or 4) columns per block, 128 * COLS threads; column pairs
// (v0 + 2p, v0 + 2p + 1) share the forward FFT, the E-branch IFFT and the
// cosine-branch IFFT.  The spectral scale K[u][v] = kscale h_u h_v /
// (wx_u^2 + wy_v^2) (h_0 = 1/2, K[0][0] = 0) is formed here from the weight
// tables.  ColVec: COLS consecutive R values of a row, loaded as one vector.
template <typename R, int COLS>
struct ColVec;
template <>
struct ColVec<float, 2> {
    using T = float2;
};
template <>
struct ColVec<float, 4> {
    using T = float4;
};
template <>
struct ColVec<double, 2> {
    using T = double2;
};

template <int LOGN, int COLS, typename R>
__global__ void __launch_bounds__(128 * COLS)
k_fft_cols(const R *__restrict__ T, const R *__restrict__ wx, const R *__restrict__ wy, R kscale, R *__restrict__ X1,
           R *__restrict__ X2, int ny, const vec2<R> *__restrict__ tw, const vec2<R> *__restrict__ q,
           const DevScalars *__restrict__ S) {
    using C = vec2<R>;
    constexpr int n = 1 << LOGN;
    constexpr int kThreads = 128 * COLS, NP = COLS / 2;
    using V = typename ColVec<R, COLS>::T;
    C *sm = smem_c<R>();
    C *fw = sm;  // NP packed forward sequences (columns v0 + 2p, v0 + 2p + 1)
    C *iv = sm;  // then COLS inverse sequences: E branch of each pair, then cosine branch of each pair
    C *tw_s = sm + COLS * n, *q_s = tw_s + n - 1;
    R *wx_s = (R *)(q_s + n / 2 + 1);
    stage_tables<LOGN, kThreads, R>(tw_s, q_s, wx_s, tw, q, wx);
    const int v0 = blockIdx.x * COLS;
    const V wvv = *reinterpret_cast<const V *>(wy + v0);
    const R *wvc = reinterpret_cast<const R *>(&wvv);
    pdl_begin();
    if (S && S->done) return;
    constexpr int li = (n + kThreads - 1) / kThreads;
    V t[li];
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int x = threadIdx.x + it * kThreads;
        if (x < n) t[it] = *reinterpret_cast<const V *>(T + (size_t)x * ny + v0);
    }
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int x = threadIdx.x + it * kThreads;
        if (x < n) {
            const int pos = brev(makhoul(x, n), LOGN);
            const R *tv = reinterpret_cast<const R *>(&t[it]);
#pragma unroll
            for (int p = 0; p < NP; p++) fw[p * n + pos] = mk2<R>(tv[2 * p], tv[2 * p + 1]);
        }
    }
    __syncthreads();
    block_fft<false, LOGN, NP, kThreads, R>(fw, NP, tw_s);
    constexpr int hk = n / 2 + 1;
    constexpr int pi_ = (NP * hk + kThreads - 1) / kThreads;
    // the forward spectra into registers: the inverse sequences overwrite them
    C zk[pi_], zm[pi_];
#pragma unroll
    for (int it = 0; it < pi_; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e < NP * hk) {
            const int p = e / hk, k = e - p * hk;
            zk[it] = fw[p * n + k];
            zm[it] = fw[p * n + ((n - k) & (n - 1))];
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < pi_; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e >= NP * hk) break;
        const int p = e / hk, k = e - p * hk;
        const int m = (n - k) & (n - 1);
        const bool self = (k == n / 2);
        const C Z = zk[it], M = zm[it];
        const C cs = q_s[k];
        const R re[2] = {(R)0.5 * (Z.x + M.x), (R)0.5 * (Z.y + M.y)};
        const R im[2] = {(R)0.5 * (Z.y - M.y), (R)-0.5 * (Z.x - M.x)};
        const R wk = wx_s[k], wm = wx_s[m];
        R pk[2], pm[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int v = v0 + 2 * p + h;
            const R wv = wvc[2 * p + h];
            const R cv = (v == 0 ? (R)0.5 : (R)1) * kscale;
            // DCT-II outputs k and n-k, times K
            const R kk = (k == 0) ? (v == 0 ? (R)0 : (R)0.5 * cv / (wv * wv)) : cv / fma_r(wk, wk, wv * wv);
            pk[h] = (re[h] * cs.x + im[h] * cs.y) * kk;
            pm[h] = (self || k == 0) ? pk[h] : (re[h] * cs.y - im[h] * cs.x) * (cv / fma_r(wm, wm, wv * wv));
        }
        C *oe = iv + p * n, *oc = iv + (NP + p) * n;
        if (k == 0) {
            oe[0] = mk2<R>((R)0, (R)0);  // sine branch: b[0] = 0
            oc[0] = mk2<R>(pk[0], pk[1]);
            continue;
        }
        // sine branch: b[k] = wx[n-k] P[n-k], b[n-k] = wx[k] P[k]
        pack_spec<R>(oe, k, m, LOGN, dct3_spec<R>(wm * pm[0], wk * pk[0], cs), dct3_spec<R>(wm * pm[1], wk * pk[1], cs),
                     self);
        pack_spec<R>(oc, k, m, LOGN, dct3_spec<R>(pk[0], pm[0], cs), dct3_spec<R>(pk[1], pm[1], cs), self);
    }
    __syncthreads();
    block_fft<true, LOGN, COLS, kThreads, R>(iv, COLS, tw_s);
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int x = threadIdx.x + it * kThreads;
        if (x >= n) break;
        const int m = makhoul(x, n);
        const R sg = (x & 1) ? (R)-1 : (R)1;
        V o1, o2;
        R *f1 = reinterpret_cast<R *>(&o1), *f2 = reinterpret_cast<R *>(&o2);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            const C e = iv[p * n + m], c = iv[(NP + p) * n + m];
            f1[2 * p] = sg * e.x;
            f1[2 * p + 1] = sg * e.y;
            f2[2 * p] = c.x;
            f2[2 * p + 1] = c.y;
        }
        *reinterpret_cast<V *>(X1 + (size_t)x * ny + v0) = o1;
        *reinterpret_cast<V *>(X2 + (size_t)x * ny + v0) = o2;
    }
}

// ---- pass 3: rows along y, to the field -------------------------------------
template <typename R>
struct Quad;
template <>
struct Quad<float> {
    using T = float4;
    static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};
template <>
struct Quad<double> {
    struct T {
        double x, y, z, w;
    };
    static __device__ __forceinline__ T make(double a, double b, double c, double d) { return T{a, b, c, d}; }
};

template <int LOGN, bool PHI, typename R>
__global__ void __launch_bounds__(kThreads)
k_fft_rows_inv(const R *__restrict__ X1, const R *__restrict__ X2, const R *__restrict__ wy, vec2<R> *__restrict__ field,
               R *__restrict__ phi, int rows, const vec2<R> *__restrict__ tw, const vec2<R> *__restrict__ q,
               const DevScalars *__restrict__ S) {
    using C = vec2<R>;
    constexpr int n = 1 << LOGN, NS = seqs_per_block<LOGN>();
    constexpr int nseq = PHI ? 2 : 1;  // per row: (E_x, E_y) packed, then phi
    C *sm = smem_c<R>();
    C *tw_s = sm + NS * nseq * n, *q_s = tw_s + n - 1;
    R *wy_s = (R *)(q_s + n / 2 + 1);
    stage_tables<LOGN, kThreads, R>(tw_s, q_s, wy_s, tw, q, wy);
    pdl_begin();
    if (S && S->done) return;
    const int x0 = blockIdx.x * rows;
    constexpr int hk = n / 2 + 1;
    constexpr int li = (NS * hk + kThreads - 1) / kThreads;
    typename Quad<R>::T v[li];  // X1[k], X1[n-k], X2[k], X2[n-k]
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e < rows * hk) {
            const int r = e / hk, k = e - r * hk;
            const int m = (n - k) & (n - 1);
            const size_t base = (size_t)(x0 + r) * n;
            v[it] = Quad<R>::make(X1[base + k], X1[base + m], X2[base + k], X2[base + m]);
        }
    }
    __syncthreads();  // the tables
#pragma unroll
    for (int it = 0; it < li; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e >= rows * hk) break;
        const int r = e / hk, k = e - r * hk;
        const int m = (n - k) & (n - 1);
        C *o = sm + ((r * nseq) << LOGN);
        const R a_k = v[it].x, a_m = v[it].y, b_k = v[it].z, b_m = v[it].w;
        if (k == 0) {
            o[0] = mk2<R>(a_k, (R)0);
            if (PHI) o[n] = mk2<R>(b_k, (R)0);
            continue;
        }
        const C cs = q_s[k];
        const bool self = (k == n / 2);
        // sine branch of wy X2: b[k] = wy[n-k] X2[n-k], b[n-k] = wy[k] X2[k]
        pack_spec<R>(o, k, m, LOGN, dct3_spec<R>(a_k, a_m, cs), dct3_spec<R>(wy_s[m] * b_m, wy_s[k] * b_k, cs), self);
        if (PHI) pack_spec<R>(o + n, k, m, LOGN, dct3_spec<R>(b_k, b_m, cs), mk2<R>((R)0, (R)0), self);
    }
    __syncthreads();
    block_fft<true, LOGN, NS * nseq, kThreads, R>(sm, rows * nseq, tw_s);
    constexpr int oi = (NS * n + kThreads - 1) / kThreads;
#pragma unroll
    for (int it = 0; it < oi; it++) {
        const int e = threadIdx.x + it * kThreads;
        if (e >= (rows << LOGN)) break;
        const int r = e >> LOGN, y = e & (n - 1);
        const int m = makhoul(y, n);
        const C *z = sm + ((r * nseq) << LOGN);
        const size_t at = (size_t)(x0 + r) * n + y;
        field[at] = mk2<R>(z[m].x, (y & 1) ? -z[m].y : z[m].y);
        if (PHI) phi[at] = z[n + m].x;
    }
}

// Kernel instances for log2 n = kMinLog .. kMaxLog, per precision.
constexpr int kMinLog = 3, kMaxLog = 11;
constexpr int kLogs = kMaxLog - kMinLog + 1;
template <typename R>
struct FftFns {
    using RowsFwdFn = void (*)(const R *, R *, int, const vec2<R> *, const vec2<R> *, const DevScalars *);
    using ColsFn = void (*)(const R *, const R *, const R *, R, R *, R *, int, const vec2<R> *, const vec2<R> *,
                            const DevScalars *);
    using RowsInvFn = void (*)(const R *, const R *, const R *, vec2<R> *, R *, int, const vec2<R> *,
                               const vec2<R> *, const DevScalars *);
    template <int... L>
    static constexpr std::array<RowsFwdFn, sizeof...(L)> rows_fwd(std::integer_sequence<int, L...>) {
        return {k_fft_rows_fwd<L + kMinLog, R>...};
    }
    template <int... L>
    static constexpr std::array<ColsFn, sizeof...(L)> cols(std::integer_sequence<int, L...>) {
        return {k_fft_cols<L + kMinLog, kCols, R>...};
    }
    template <bool PHI, int... L>
    static constexpr std::array<RowsInvFn, sizeof...(L)> rows_inv(std::integer_sequence<int, L...>) {
        return {k_fft_rows_inv<L + kMinLog, PHI, R>...};
    }
    using LogSeq = std::make_integer_sequence<int, kLogs>;
    static const std::array<RowsFwdFn, kLogs> kRowsFwd;
    static const std::array<ColsFn, kLogs> kCols_;
    static const std::array<RowsInvFn, kLogs> kRowsInv, kRowsInvPhi;
};
template <typename R>
const std::array<typename FftFns<R>::RowsFwdFn, kLogs> FftFns<R>::kRowsFwd = FftFns<R>::rows_fwd(LogSeq{});
template <typename R>
const std::array<typename FftFns<R>::ColsFn, kLogs> FftFns<R>::kCols_ = FftFns<R>::cols(LogSeq{});
template <typename R>
const std::array<typename FftFns<R>::RowsInvFn, kLogs> FftFns<R>::kRowsInv = FftFns<R>::template rows_inv<false>(LogSeq{});
template <typename R>
const std::array<typename FftFns<R>::RowsInvFn, kLogs> FftFns<R>::kRowsInvPhi =
    FftFns<R>::template rows_inv<true>(LogSeq{});
template struct FftFns<float>;
template struct FftFns<double>;

int seqs_per_block_rt(int logn) { return std::max(1, (2 * kThreads) >> logn); }

int ilog2_exact(int n) {
    int l = 0;
    while ((1 << l) < n) l++;
    return (1 << l) == n ? l : -1;
}

template <typename T>
int upload_vec(void *&dst, const std::vector<T> &src, std::string &err) {
    if (cudaMalloc(&dst, src.size() * sizeof(T)) != cudaSuccess) {
        err = "cudaMalloc failed for FFT tables";
        return EP_ERR_NOMEM;
    }
    if (cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
        err = "copy of FFT tables failed";
        return EP_ERR_CUDA;
    }
    return EP_OK;
}

template <typename R>
void tables(int n, std::vector<vec2<R>> &tw, std::vector<vec2<R>> &q) {
    const double pi = 3.14159265358979323846;
    tw.assign(n - 1, mk2<R>((R)0, (R)0));
    for (int h = 1; h < n; h <<= 1)
        for (int j = 0; j < h; j++) tw[h - 1 + j] = mk2<R>((R)cos(pi * j / h), (R)-sin(pi * j / h));
    q.assign(n / 2 + 1, mk2<R>((R)0, (R)0));
    for (int k = 0; k <= n / 2; k++) q[k] = mk2<R>((R)cos(pi * k / (2.0 * n)), (R)sin(pi * k / (2.0 * n)));
}

template <typename R>
int fft_init_t(FftPlan *f, int nx, int ny, const std::vector<double> &wx, const std::vector<double> &wy,
               std::string &err) {
    const int lx = f->lognx, ly = f->logny;
    std::vector<vec2<R>> tw, q;
    int rc;
    tables<R>(nx, tw, q);
    if ((rc = upload_vec(f->twx, tw, err)) || (rc = upload_vec(f->qx, q, err))) return rc;
    tables<R>(ny, tw, q);
    if ((rc = upload_vec(f->twy, tw, err)) || (rc = upload_vec(f->qy, q, err))) return rc;
    std::vector<R> wxr(nx), wyr(ny);
    for (int u = 0; u < nx; u++) wxr[u] = (R)wx[u];
    for (int v = 0; v < ny; v++) wyr[v] = (R)wy[v];
    if ((rc = upload_vec(f->wx, wxr, err)) || (rc = upload_vec(f->wy, wyr, err))) return rc;
    f->kscale = (double)(R)(4.0 / nx / ny);
    if (cudaMalloc(&f->T, sizeof(R) * nx * ny) != cudaSuccess ||
        cudaMalloc(&f->X, sizeof(R) * 2 * nx * ny) != cudaSuccess) {
        err = "cudaMalloc failed for FFT intermediates";
        return EP_ERR_NOMEM;
    }
    const int nsf = seqs_per_block_rt(ly);
    f->pairs_fwd = std::min(nsf, nx / 2);
    f->rows_inv = std::min(nsf, nx);
    f->smem_rows_fwd = sizeof(vec2<R>) * (size_t)nsf * ny + table_bytes<R>(ny);
    f->smem_cols = sizeof(vec2<R>) * (size_t)kCols * nx + table_bytes<R>(nx);
    f->smem_rows_inv = sizeof(vec2<R>) * (size_t)nsf * 2 * ny + table_bytes<R>(ny);
    using F = FftFns<R>;
    const std::pair<const void *, size_t> attr[4] = {
        {(const void *)F::kRowsFwd[ly - kMinLog], f->smem_rows_fwd},
        {(const void *)F::kCols_[lx - kMinLog], f->smem_cols},
        {(const void *)F::kRowsInv[ly - kMinLog], f->smem_rows_inv - sizeof(vec2<R>) * (size_t)nsf * ny},
        {(const void *)F::kRowsInvPhi[ly - kMinLog], f->smem_rows_inv}};
    for (auto &a : attr) {
        if (a.second > 48 * 1024 &&
            cudaFuncSetAttribute(a.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.second) != cudaSuccess) {
            err = "shared memory of the FFT Poisson kernels refused";
            return EP_ERR_UNSUPPORTED;
        }
        // the loop's split, unless this block needs more (1 KB per block is
        // reserved by the hardware)
        cudaFuncSetAttribute(a.first, cudaFuncAttributePreferredSharedMemoryCarveout,
                             carveout_percent(std::max(kLoopSmemBytes, a.second + 1024)));
    }
    return EP_OK;
}

template <typename R>
void fft_run_t(const FftPlan *f, int nx, int ny, const R *rho, vec2<R> *field, R *phi, const DevScalars *S,
               cudaStream_t st) {
    using F = FftFns<R>;
    R *X1 = (R *)f->X, *X2 = X1 + (size_t)nx * ny;
    const int pr = launch_priority(true);
    const int lx = f->lognx - kMinLog, ly = f->logny - kMinLog;
    launch_kp(F::kRowsFwd[ly], nx / (2 * f->pairs_fwd), kThreads, f->smem_rows_fwd, st, pr, rho, (R *)f->T,
              f->pairs_fwd, (const vec2<R> *)f->twy, (const vec2<R> *)f->qy, S);
    launch_kp(F::kCols_[lx], ny / kCols, 128 * kCols, f->smem_cols, st, pr, (const R *)f->T, (const R *)f->wx,
              (const R *)f->wy, (R)f->kscale, X1, X2, ny, (const vec2<R> *)f->twx, (const vec2<R> *)f->qx, S);
    const size_t phi_seqs = sizeof(vec2<R>) * (size_t)seqs_per_block_rt(f->logny) * ny;
    launch_kp(phi ? F::kRowsInvPhi[ly] : F::kRowsInv[ly], nx / f->rows_inv, kThreads,
              phi ? f->smem_rows_inv : f->smem_rows_inv - phi_seqs, st, pr, (const R *)X1, (const R *)X2,
              (const R *)f->wy, field, phi, f->rows_inv, (const vec2<R> *)f->twy, (const vec2<R> *)f->qy, S);
}

}  // namespace

int dct_fft_init(DctPlan &p, const std::vector<double> &wx, const std::vector<double> &wy, int fp64,
                 std::string &err) {
    const int nx = p.nx, ny = p.ny;
    const int lx = ilog2_exact(nx), ly = ilog2_exact(ny);
    if (lx < kMinLog || ly < kMinLog || lx > kMaxLog || ly > kMaxLog) {
        err = "the FFT Poisson path needs power-of-two bin counts in [8, 2048]";
        return EP_ERR_UNSUPPORTED;
    }
    FftPlan *f = new (std::nothrow) FftPlan;
    if (!f) {
        err = "out of host memory for the FFT plan";
        return EP_ERR_NOMEM;
    }
    p.fft = f;
    f->lognx = lx;
    f->logny = ly;
    f->fp64 = fp64;
    return fp64 ? fft_init_t<double>(f, nx, ny, wx, wy, err) : fft_init_t<float>(f, nx, ny, wx, wy, err);
}

void dct_fft_free(DctPlan &p) {
    FftPlan *f = (FftPlan *)p.fft;
    if (!f) return;
    for (void *d : {f->twx, f->twy, f->qx, f->qy, f->wx, f->wy, f->T, f->X})
        if (d) cudaFree(d);
    delete f;
    p.fft = nullptr;
}

int dct_fft_run(DctPlan &p, const void *rho, void *field, void *phi, const DevScalars *S, cudaStream_t st) {
    const FftPlan *f = (const FftPlan *)p.fft;
    if (f->fp64)
        fft_run_t<double>(f, p.nx, p.ny, (const double *)rho, (double2 *)field, (double *)phi, S, st);
    else
        fft_run_t<float>(f, p.nx, p.ny, (const float *)rho, (float2 *)field, (float *)phi, S, st);
    return EP_OK;
}

}  // namespace ep
