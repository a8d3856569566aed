// dct.cu -- the electrostatic Poisson solve of FFT_2D::doFFT
// (FFT/fft.cpp:191-284) restated as dense GEMMs.
//
// With C_n[u][x] = cos(pi u (x+1/2) / n) and S_n[u][x] = sin(pi u (x+1/2) / n),
// the reference's Ooura calls compute (rho is [nx][ny], x-major):
//   a      = C_nx rho C_ny^T                       (ddct2d, isgn = -1)
//   P      = a .* K,  K[u][v] = 4/(nx ny) h_u h_v / (wx_u^2 + wy_v^2),
//            h_0 = 1/2, K[0][0] = 0,  wx_u = pi u / nx,
//            wy_v = pi v / ny * (step_y / step_x)      (fft.cpp:129-147,200-266)
//   phi    = C_nx^T P C_ny                         (ddct2d,  isgn = +1)
//   E_x    = S_nx^T diag(wx) P C_ny                (ddsct2d, isgn = +1)
//   E_y    = C_nx^T P diag(wy) S_ny                (ddcst2d, isgn = +1)
// Four GEMM launches, every operand K-major ("NT": C[m][n] = sum_k A[m][k] B[n][k]):
//   G1  Tt[v][x] = sum_y rho[x][y] Cy[v][y]            (transposed store)
//   G2  P[u][v]  = K[u][v] sum_x Cx[u][x] Tt[v][x]      (spectral epilogue)
//   G3  T3[n][u] = sum_v P[u][v] B3[n][v],  B3 = [C_ny^T ; (diag(wy) S_ny)^T]
//       so T3 = [Ut ; Vt] with U = P C_ny, V = P diag(wy) S_ny (transposed store)
//   G4  E_x[x][y] = sum_u A4x[x][u] Ut[y][u],  A4x[x][u] = wx_u S_nx[u][x]
//       E_y[x][y] = sum_u A4y[x][u] Vt[y][u],  A4y[x][u] = C_nx[u][x]
//       (phi, when asked: A4y against Ut)          (interleaved float2 field)
// This file holds the tables and the FP32 CUDA-core GEMM; dct_tc.cu runs the
// same four GEMMs on the tcgen05 tensor cores, dct_fft.cu evaluates the same
// sums by fast transforms.
#include <cmath>
#include <vector>

#include "engine.h"

namespace ep {

int dct_tc_init(DctPlan &p, std::string &err);
void dct_tc_free(DctPlan &p);
int dct_tc_run(DctPlan &p, float2 *field, float *phi, const DevScalars *S, cudaStream_t st);
int dct_fft_init(DctPlan &p, const std::vector<double> &wx, const std::vector<double> &wy, int fp64, std::string &err);
void dct_fft_free(DctPlan &p);
int dct_fft_run(DctPlan &p, const void *rho, void *field, void *phi, const DevScalars *S, cudaStream_t st);

namespace {

enum Epi { kEpiT = 0, kEpiSpectral = 1, kEpiField = 2 };

struct GemmArgs {
    const float *A[3];
    const float *B[3];
    float *C;          // kEpiT / kEpiSpectral output
    int ldc;
    const float *K;    // spectral scale [M][N]
    float2 *field;     // kEpiField output [M][N]
    float *phi;        // kEpiField batch 2 output
};

constexpr int BM = 64, BN = 64, BK = 16;

// C[m][n] = sum_k A[m][k] B[n][k]; 256 threads, 4x4 outputs each.
template <int EPI>
__global__ void __launch_bounds__(256)
k_sgemm_nt(int M, int N, int K, GemmArgs a, const DevScalars *__restrict__ S) {
    pdl_begin();
    if (S && S->done) return;
    const int bz = blockIdx.z;
    const float *__restrict__ A = a.A[bz];
    const float *__restrict__ B = a.B[bz];
    __shared__ float As[BK][BM + 4];
    __shared__ float Bs[BK][BN + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
        for (int e = threadIdx.x; e < BM * BK; e += 256) {
            int r = e / BK, c = e % BK;
            int m = m0 + r, k = k0 + c;
            As[c][r] = (m < M && k < K) ? A[(size_t)m * K + k] : 0.f;
            int n = n0 + r;
            Bs[c][r] = (n < N && k < K) ? B[(size_t)n * K + k] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m >= M || n >= N) continue;
            float v = acc[i][j];
            if (EPI == kEpiT) {
                a.C[(size_t)n * a.ldc + m] = v;
            } else if (EPI == kEpiSpectral) {
                a.C[(size_t)m * a.ldc + n] = v * a.K[(size_t)m * N + n];
            } else {
                if (bz == 0)
                    a.field[(size_t)m * N + n].x = v;
                else if (bz == 1)
                    a.field[(size_t)m * N + n].y = v;
                else
                    a.phi[(size_t)m * N + n] = v;
            }
        }
}

template <int EPI>
void sgemm(int M, int N, int K, int batch, const GemmArgs &a, const DevScalars *S, cudaStream_t st) {
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, batch);
    launch_k(k_sgemm_nt<EPI>, grid, 256, 0, st, M, N, K, a, S);
}

}  // namespace

void set_sgemm_carveout(int carveout) {
    for (const void *f : {(const void *)k_sgemm_nt<kEpiT>, (const void *)k_sgemm_nt<kEpiSpectral>,
                          (const void *)k_sgemm_nt<kEpiField>})
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
}

namespace {

template <typename T>
int upload(T *&dst, const std::vector<T> &src, std::string &err) {
    if (cudaMalloc(&dst, src.size() * sizeof(T)) != cudaSuccess) {
        err = "cudaMalloc failed for DCT tables";
        return EP_ERR_NOMEM;
    }
    cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    return EP_OK;
}

}  // namespace

int dct_plan_init(DctPlan &p, int nx, int ny, float step_x, float step_y, int mode, int fp64,
                  std::string &err) {
    p.nx = nx;
    p.ny = ny;
    p.mode = mode;
    p.fp64 = fp64;
    if (fp64 && mode != EP_DCT_FFT) {
        err = "the FP64 Poisson solve uses the fast transforms only (power-of-two bin counts in [8, 2048])";
        return EP_ERR_UNSUPPORTED;
    }
    const double pi = 3.14159265358979323846;
    std::vector<double> wx(nx), wy(ny);
    for (int u = 0; u < nx; u++) wx[u] = pi * u / nx;
    for (int v = 0; v < ny; v++) wy[v] = pi * v / ny * ((double)step_y / (double)step_x);
    if (mode == EP_DCT_FFT) return dct_fft_init(p, wx, wy, fp64, err);
    std::vector<float> Cy((size_t)ny * ny), Cx((size_t)nx * nx), K((size_t)nx * ny),
        B3((size_t)2 * ny * ny), A4((size_t)2 * nx * nx);
    for (int v = 0; v < ny; v++)
        for (int y = 0; y < ny; y++) {
            double ang = pi * v * (y + 0.5) / ny;
            Cy[(size_t)v * ny + y] = (float)cos(ang);
            B3[(size_t)y * ny + v] = (float)cos(ang);                    // C_ny^T
            B3[(size_t)(ny + y) * ny + v] = (float)(wy[v] * sin(ang));   // (diag(wy) S_ny)^T
        }
    for (int u = 0; u < nx; u++)
        for (int x = 0; x < nx; x++) {
            double ang = pi * u * (x + 0.5) / nx;
            Cx[(size_t)u * nx + x] = (float)cos(ang);
            A4[(size_t)x * nx + u] = (float)(wx[u] * sin(ang));               // A4x
            A4[(size_t)nx * nx + (size_t)x * nx + u] = (float)cos(ang);       // A4y
        }
    for (int u = 0; u < nx; u++)
        for (int v = 0; v < ny; v++) {
            double h = (u == 0 ? 0.5 : 1.0) * (v == 0 ? 0.5 : 1.0);
            double den = wx[u] * wx[u] + wy[v] * wy[v];
            K[(size_t)u * ny + v] = (u == 0 && v == 0) ? 0.0f : (float)(4.0 / nx / ny * h / den);
        }
    int rc;
    if ((rc = upload(p.Cy, Cy, err)) || (rc = upload(p.Cx, Cx, err)) || (rc = upload(p.K, K, err)) ||
        (rc = upload(p.B3, B3, err)) || (rc = upload(p.A4, A4, err)))
        return rc;
    if (cudaMalloc(&p.Tt, sizeof(float) * nx * ny) != cudaSuccess ||
        cudaMalloc(&p.P, sizeof(float) * nx * ny) != cudaSuccess ||
        cudaMalloc(&p.T3, sizeof(float) * 2 * nx * ny) != cudaSuccess) {
        err = "cudaMalloc failed for DCT intermediates";
        return EP_ERR_NOMEM;
    }
    if (mode == EP_DCT_BF16X3) return dct_tc_init(p, err);
    return EP_OK;
}

void dct_plan_free(DctPlan &p) {
    if (p.tc) dct_tc_free(p);
    if (p.fft) dct_fft_free(p);
    for (float *q : {p.Cy, p.Cx, p.K, p.B3, p.A4, p.Tt, p.P, p.T3})
        if (q) cudaFree(q);
    p = DctPlan();
}

int dct_run(DctPlan &p, const void *rho_v, void *field_v, void *phi_v, const DevScalars *S, cudaStream_t st) {
    if (p.mode == EP_DCT_FFT) return dct_fft_run(p, rho_v, field_v, phi_v, S, st);
    // the dense paths are FP32 only (dct_plan_init refuses them for FP64)
    const float *rho = (const float *)rho_v;
    float2 *field = (float2 *)field_v;
    float *phi = (float *)phi_v;
    if (p.mode == EP_DCT_BF16X3) return dct_tc_run(p, field, phi, S, st);
    const int nx = p.nx, ny = p.ny;
    GemmArgs a{};
    // G1: Tt = (rho Cy^T)^T
    a.A[0] = rho;
    a.B[0] = p.Cy;
    a.C = p.Tt;
    a.ldc = nx;
    sgemm<kEpiT>(nx, ny, ny, 1, a, S, st);
    // G2: P = (Cx T) .* K
    a.A[0] = p.Cx;
    a.B[0] = p.Tt;
    a.C = p.P;
    a.ldc = ny;
    a.K = p.K;
    sgemm<kEpiSpectral>(nx, ny, nx, 1, a, S, st);
    // G3: T3 = [Ut; Vt]
    a.A[0] = p.P;
    a.B[0] = p.B3;
    a.C = p.T3;
    a.ldc = nx;
    sgemm<kEpiT>(nx, 2 * ny, ny, 1, a, S, st);
    // G4: field (and phi)
    a.A[0] = p.A4;
    a.B[0] = p.T3;
    a.A[1] = p.A4 + (size_t)nx * nx;
    a.B[1] = p.T3 + (size_t)ny * nx;
    a.A[2] = p.A4 + (size_t)nx * nx;
    a.B[2] = p.T3;
    a.field = field;
    a.phi = phi;
    sgemm<kEpiField>(nx, ny, nx, phi ? 3 : 2, a, S, st);
    return EP_OK;
}

}  // namespace ep
