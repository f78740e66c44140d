// life_simulation_b200/csrc/lenia_fft.cu -- the multi-kernel FFT convolution
// step, B200 form of the reference's FFT path (Modules/FieldModules/
// Lenia.cpp:576-643 driving Shaders/Common/FFT.metal and leniaGrowthMulti,
// Shaders/Field/Lenia.metal:161-232).
//
// The reference spends 1 + (log2 W + log2 H) + 1 + K*(1 + log2 W + log2 H + 1)
// + 1 full-field passes per substep (85 at 1024x512, K=3), each a radix-2
// stage through memory, and needs power-of-two sizes. Here a substep is
// three sweeps, any W (even) and H whose factors are 2, 3 and 5:
//
//   row pass     A -> S          length-M complex FFT of each row packed as
//                                z[n] = A[2n] + i*A[2n+1] (M = W/2), then the
//                                real-FFT split to X[0..M]; X[0] and X[M] are
//                                real and share column 0 as (re, im).
//   column pass  S -> U_k        per column: forward length-H FFT, then for
//                                every kernel k the product with its real,
//                                even spectrum and the inverse FFT.
//   row pass     U_k -> A'       per row and kernel: C2R (inverse of the
//                                split above, then a length-M inverse FFT),
//                                growth accumulated over k in the
//                                reference's order, Euler step, noise,
//                                injection, clip, store A'; and, fused, the
//                                row FFT of A' -- the next substep's first
//                                sweep -- so steady state is two launches.
//
// Spectra are stored column-major ([kx][ky], H contiguous per column) so the
// column pass streams whole columns and the row passes move rows_per_cta
// consecutive rows per column (32 B segments at 4 rows). The 1/(W*H)
// normalisation is folded into the kernel spectra (FP64 on the host).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "fft_core.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

using fft::cadd;
using fft::cconj;
using fft::cmul;
using fft::cscale;
using fft::csub;

namespace {

__device__ __forceinline__ void load_table(float2* dst, const float2* __restrict__ src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Real-FFT split of one row spectrum z (length M) into the packed half
// spectrum, stored to S column-major. For k >= 1:
//   E = (Z[k] + conj Z[M-k]) / 2,  O = (Z[k] - conj Z[M-k]) / (2i),
//   X[k] = E + exp(-2 pi i k / W) * O;
// for k = 0: X[0] = Re Z0 + Im Z0 and X[M] = Re Z0 - Im Z0 (both real).
__device__ __forceinline__ void r2c_store(const float2* z, const float2* twr, float2* S,
                                          int y0, int rows, int M, int H) {
    const int total = M * rows;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int k = q / rows;
        const int r = q - k * rows;
        const float2* zr = z + r * M;
        const float2 Z = zr[k];
        float2 X;
        if (k == 0) {
            X = make_float2(Z.x + Z.y, Z.x - Z.y);
        } else {
            const float2 Zc = cconj(zr[M - k]);
            const float2 E = cscale(cadd(Z, Zc), 0.5f);
            const float2 D = csub(Z, Zc);
            const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);  // D / (2i)
            X = cadd(E, cmul(twr[k], O));
        }
        S[size_t(k) * H + y0 + r] = X;
    }
}

__global__ void row_r2c_kernel(FftGeometry g, const float* __restrict__ A, float2* __restrict__ S) {
    extern __shared__ __align__(16) float2 sm[];
    const int M = g.M, H = g.H, W = g.W, RB = g.rows_per_cta;
    float2* tw = sm;
    float2* twr = tw + M;
    float2* ba = twr + (M + 1);
    float2* bb = ba + RB * M;
    load_table(tw, g.tw_row, M);
    load_table(twr, g.tw_r2c, M + 1);
    for (int y0 = blockIdx.x * RB; y0 < H; y0 += gridDim.x * RB) {
        const int rows = min(RB, H - y0);
        for (int q = threadIdx.x; q < rows * M; q += blockDim.x) {
            const int r = q / M, n = q - r * M;
            ba[q] = __ldg(reinterpret_cast<const float2*>(A + size_t(y0 + r) * W) + n);
        }
        __syncthreads();
        float2* z = fft::run<false>(ba, bb, g.row, rows, tw);
        r2c_store(z, twr, S, y0, rows, M, H);
        __syncthreads();
    }
}

__global__ void col_conv_kernel(FftGeometry g, const float2* __restrict__ S, float2* __restrict__ U) {
    extern __shared__ __align__(16) float2 sm[];
    const int M = g.M, H = g.H, CB = g.cols_per_cta, Hh = H / 2 + 1;
    float2* tw = sm;
    float2* b0 = tw + H;
    float2* b1 = b0 + CB * H;
    float2* b2 = b1 + CB * H;
    load_table(tw, g.tw_col, H);
    for (int k0 = blockIdx.x * CB; k0 < M; k0 += gridDim.x * CB) {
        const int cols = min(CB, M - k0);
        const float2* src = S + size_t(k0) * H;  // cols*H contiguous
        for (int q = threadIdx.x; q < cols * H; q += blockDim.x) b0[q] = __ldg(src + q);
        __syncthreads();
        float2* C = fft::run<false>(b0, b1, g.col, cols, tw);
        float2* X = (C == b0) ? b1 : b0;  // two free buffers for the inverses
        float2* Y = b2;
        for (int kk = 0; kk < g.nk; ++kk) {
            const float* kh = g.khat + size_t(kk) * (M + 1) * Hh;
            for (int q = threadIdx.x; q < cols * H; q += blockDim.x) {
                const int c = q / H, ky = q - c * H;
                const int kx = k0 + c;
                const int kyr = min(ky, H - ky);
                const float2 Cv = C[q];
                float2 D;
                if (kx == 0) {
                    // Packed DC/Nyquist column: C = FFT(a + i b) with a, b real;
                    // want FFT^-1 of (A^ P + i B^ Q) with P, Q the two real spectra.
                    const float P = __ldg(kh + kyr), Q = __ldg(kh + size_t(M) * Hh + kyr);
                    const float2 Cm = cconj(C[c * H + (ky == 0 ? 0 : H - ky)]);
                    D = cadd(cscale(Cv, 0.5f * (P + Q)), cscale(Cm, 0.5f * (P - Q)));
                } else {
                    D = cscale(Cv, __ldg(kh + size_t(kx) * Hh + kyr));
                }
                X[q] = D;
            }
            __syncthreads();
            float2* res = fft::run<true>(X, Y, g.col, cols, tw);
            float2* dst = U + size_t(kk) * M * H + size_t(k0) * H;
            for (int q = threadIdx.x; q < cols * H; q += blockDim.x) dst[q] = res[q];
            __syncthreads();
        }
    }
}

__global__ void row_c2r_growth_kernel(FftGeometry g, const float2* __restrict__ U,
                                      const float* __restrict__ A, float* __restrict__ A_out,
                                      float2* __restrict__ S_next, StepParams p) {
    extern __shared__ __align__(16) float2 sm[];
    const int M = g.M, H = g.H, W = g.W, RB = g.rows_per_cta;
    float2* tw = sm;
    float2* twr = tw + M;
    float2* ba = twr + (M + 1);
    float2* bb = ba + RB * M;
    float* acc = reinterpret_cast<float*>(bb + RB * M);  // [RB][W]
    load_table(tw, g.tw_row, M);
    load_table(twr, g.tw_r2c, M + 1);
    const bool asym = p.growth_mode == 1u;
    for (int y0 = blockIdx.x * RB; y0 < H; y0 += gridDim.x * RB) {
        const int rows = min(RB, H - y0);
        for (int kk = 0; kk < g.nk; ++kk) {
            const float2* Uk = U + size_t(kk) * M * H;
            for (int q = threadIdx.x; q < M * rows; q += blockDim.x) {
                const int k = q / rows, r = q - k * rows;
                ba[r * M + k] = __ldg(Uk + size_t(k) * H + y0 + r);
            }
            __syncthreads();
            // Inverse of the real-FFT split: Z'[k] = (X[k] + conj X[M-k])
            //   + i * exp(+2 pi i k / W) * (X[k] - conj X[M-k]);
            // the unnormalised length-M inverse of Z' is W * (u[2n] + i u[2n+1]).
            for (int q = threadIdx.x; q < M * rows; q += blockDim.x) {
                const int r = q / M, k = q - r * M;
                const float2* xr = ba + r * M;
                float2 Z;
                if (k == 0) {
                    const float2 x0 = xr[0];
                    Z = make_float2(x0.x + x0.y, x0.x - x0.y);
                } else {
                    const float2 Xk = xr[k];
                    const float2 Xm = cconj(xr[M - k]);
                    const float2 D = cmul(cconj(twr[k]), csub(Xk, Xm));
                    Z = cadd(cadd(Xk, Xm), make_float2(-D.y, D.x));
                }
                bb[q] = Z;
            }
            __syncthreads();
            const float2* z = fft::run<true>(bb, ba, g.row, rows, tw);
            const float mu = p.mu[kk], sigma = p.sigma[kk], h = p.weight[kk];
            for (int q = threadIdx.x; q < M * rows; q += blockDim.x) {
                const int r = q / M, n = q - r * M;
                const float2 u = z[q];
                const uint32_t gy = uint32_t(y0 + r);
                float* ar = acc + r * W + 2 * n;
                const float m0 = mu + mu_jitter_shift(p, uint32_t(2 * n), gy);
                const float m1 = mu + mu_jitter_shift(p, uint32_t(2 * n + 1), gy);
                const float bl0 = bell(u.x, m0, sigma), bl1 = bell(u.y, m1, sigma);
                const float c0 = asym ? h * bl0 : h * (2.0f * bl0 - 1.0f);
                const float c1 = asym ? h * bl1 : h * (2.0f * bl1 - 1.0f);
                if (kk == 0) {
                    ar[0] = c0;
                    ar[1] = c1;
                } else {
                    ar[0] += c0;
                    ar[1] += c1;
                }
            }
            __syncthreads();
        }
        float* af = reinterpret_cast<float*>(ba);  // A' staged as row pairs
        for (int q = threadIdx.x; q < rows * W; q += blockDim.x) {
            const int r = q / W, x = q - r * W;
            const size_t gi = size_t(y0 + r) * W + x;
            GrowthAcc ga;
            ga.weighted = acc[q];
            ga.std_sum = acc[q];
            const float a2 = growth_finish(p, __ldg(A + gi), ga, uint32_t(x), uint32_t(y0 + r));
            A_out[gi] = a2;
            af[q] = a2;
        }
        __syncthreads();
        if (S_next) {
            float2* z2 = fft::run<false>(ba, bb, g.row, rows, tw);
            r2c_store(z2, twr, S_next, y0, rows, M, H);
            __syncthreads();
        }
    }
}

int g_num_sms = 0;

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

template <typename K>
int persistent_grid(K kernel, int threads, size_t smem, int work_items) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (per_sm < 1) per_sm = 1;
    return std::max(1, std::min(work_items, per_sm * num_sms()));
}

constexpr int kThreads = 256;

}  // namespace

size_t fft_row_smem_bytes(const FftGeometry& g) {
    // twiddles (M + M+1), two work buffers, growth accumulators.
    return sizeof(float2) * (size_t(2 * g.M + 1) + 2 * size_t(g.rows_per_cta) * g.M) +
           sizeof(float) * size_t(g.rows_per_cta) * g.W;
}

size_t fft_col_smem_bytes(const FftGeometry& g) {
    return sizeof(float2) * (size_t(g.H) + 3 * size_t(g.cols_per_cta) * g.H);
}

cudaError_t launch_row_r2c(const FftGeometry& g, const float* A, float2* S, cudaStream_t s) {
    const size_t smem = sizeof(float2) * (size_t(2 * g.M + 1) + 2 * size_t(g.rows_per_cta) * g.M);
    cudaError_t e = cudaFuncSetAttribute(row_r2c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return e;
    const int items = (g.H + g.rows_per_cta - 1) / g.rows_per_cta;
    const int grid = persistent_grid(row_r2c_kernel, kThreads, smem, items);
    row_r2c_kernel<<<grid, kThreads, smem, s>>>(g, A, S);
    return cudaGetLastError();
}

cudaError_t launch_col_conv(const FftGeometry& g, const float2* S, float2* U, cudaStream_t s) {
    const size_t smem = fft_col_smem_bytes(g);
    cudaError_t e = cudaFuncSetAttribute(col_conv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return e;
    const int items = (g.M + g.cols_per_cta - 1) / g.cols_per_cta;
    const int grid = persistent_grid(col_conv_kernel, kThreads, smem, items);
    col_conv_kernel<<<grid, kThreads, smem, s>>>(g, S, U);
    return cudaGetLastError();
}

cudaError_t launch_row_c2r_growth(const FftGeometry& g, const float2* U, const float* A,
                                  float* A_out, float2* S_next, const StepParams& p,
                                  cudaStream_t s) {
    const size_t smem = fft_row_smem_bytes(g);
    cudaError_t e = cudaFuncSetAttribute(row_c2r_growth_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    const int items = (g.H + g.rows_per_cta - 1) / g.rows_per_cta;
    const int grid = persistent_grid(row_c2r_growth_kernel, kThreads, smem, items);
    row_c2r_growth_kernel<<<grid, kThreads, smem, s>>>(g, U, A, A_out, S_next, p);
    return cudaGetLastError();
}

}  // namespace lenia
