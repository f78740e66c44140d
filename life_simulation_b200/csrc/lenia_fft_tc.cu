// life_simulation_b200/csrc/lenia_fft_tc.cu -- the spectral path's column
// pass with its DFT stages on the tensor cores (split-precision BF16 or FP16
// hi/lo operands, FP32 accumulation; fft_tc.cuh), for column lengths whose
// compile-time plan is all radix 16 (256 = 16^2, 4096 = 16^3).
//
// Same contract and blocked layout as col_fast_kernel (lenia_fft_fast.cu):
// S (row spectrum, packed column 0) -> per kernel k the inverse column FFT of
// FFT_H(S) * khat_k into U_k. The forward column spectrum stays in shared
// memory (the tensor-core passes distribute their outputs by MMA fragment,
// not by thread item, so it cannot stay in registers as in the CUDA-core
// kernel): three buffers of B columns -- the spectrum and two work buffers.
// Every stage scales by 1/16 (folded into the DFT matrix); the product with
// the kernel spectrum restores the scale (x H^2, exact), so U_k has exactly
// the CUDA-core kernel's scale and the row pass is shared.
#include <cuda_runtime.h>

#include <algorithm>

#include "fft_fast_common.cuh"
#include "fft_tc.cuh"
#include "lenia_kernels.h"

namespace lenia {
namespace {

using fft::cadd;
using fft::cconj;
using fft::cscale;
using namespace fftct;
using namespace fastfft;

template <class PF, int B>
struct ColTcK {
    static constexpr int H = PF::n;
    static constexpr int Hh = H / 2 + 1;
    static constexpr int T = 256;
    static constexpr int PITCH = row_pitch(H);
    static constexpr size_t smem() { return sizeof(float2) * 3 * size_t(B) * PITCH; }
};

template <class PF, int B, int PREC>
__global__ void __launch_bounds__(256)
    col_tc_kernel(SpectralWorld w0, const SpectralWorld* __restrict__ worlds, const float2* __restrict__ twf,
                  const float2* __restrict__ twi) {
    using K = ColTcK<PF, B>;
    constexpr int H = K::H, Hh = K::Hh, T = K::T, PITCH = K::PITCH, NP = PF::np;
    static_assert(NP == 2 || NP == 3, "plans of two or three radix-16 passes");
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SpectralWorld sw;
    if (threadIdx.x == 0) sw = worlds ? worlds[blockIdx.y] : w0;
    float2* Cb = sm;             // forward column spectrum / 16^NP
    float2* X = Cb + B * PITCH;  // work buffers
    float2* Y = X + B * PITCH;
    tcfft::Dft16<PREC, false> Ff;
    tcfft::Dft16<PREC, true> Fi;
    Ff.init();
    Fi.init();
    __syncthreads();
    const float2* __restrict__ S = sw.S;
    float2* __restrict__ U = sw.U;
    const float* __restrict__ khat = sw.khat;
    const int M = sw.M, nk = sw.nk;
    const float kscale = float(H) * float(H);  // 16^(2 NP)
    const auto at = [](float2* buf) { return [buf](int b, int i, float2 v) { buf[b * PITCH + i] = v; }; };
    const auto from = [](const float2* buf) { return [buf](int b, int i) { return buf[b * PITCH + i]; }; };
    // Product elements per thread; up to 16, their kernel spectrum values are
    // fetched one kernel ahead into registers (kernel 0's during the forward
    // transform, kernel k+1's during kernel k's inverse).
    constexpr int PER = (B * H + T - 1) / T;
    constexpr bool kAhead = PER <= 16;
    for (int k0 = blockIdx.x * B; k0 < M; k0 += gridDim.x * B) {
        const int cols = min(B, M - k0);
        const size_t gbase = size_t(k0 / KB) * H * KB + (k0 % KB);
        float kv[kAhead ? PER : 1];
        const auto fetch_k = [&](int kk) {
            if constexpr (kAhead) {
                const float* kh = khat + size_t(kk) * (M + 1) * Hh;
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const int idx = int(threadIdx.x) + j * T;
                    const int b = idx % B, ky = idx / B;
                    const int kyr = min(ky, H - ky);
                    kv[j] = (idx < B * H && b < cols) ? __ldg(kh + size_t(k0 + b) * Hh + kyr) : 0.0f;
                }
            }
        };
        if (nk > 0) fetch_k(0);
        // Forward column FFT: global -> X (-> Y) -> Cb.
        tcfft::pass16<PF, 0, false, PREC, B, T>(
            [&](int b, int i) { return __ldg(S + gbase + size_t(i) * KB + b); }, at(X), twf, Ff, cols);
        __syncthreads();
        if constexpr (NP == 2) {
            tcfft::pass16<PF, 1, false, PREC, B, T>(from(X), at(Cb), twf, Ff, cols);
        } else {
            tcfft::pass16<PF, 1, false, PREC, B, T>(from(X), at(Y), twf, Ff, cols);
            __syncthreads();
            tcfft::pass16<PF, 2, false, PREC, B, T>(from(Y), at(Cb), twf, Ff, cols);
        }
        __syncthreads();
        for (int kk = 0; kk < nk; ++kk) {
            const float* kh = khat + size_t(kk) * (M + 1) * Hh;
            // Spectrum product (packed column 0 split with C[k] and conj C[-k]).
            const auto product = [&](int idx, float kval) {
                const int b = idx % B, ky = idx / B;
                const int kx = k0 + b;
                const int kyr = min(ky, H - ky);
                const float2 c = Cb[b * PITCH + ky];
                float2 d;
                if (kx == 0) {
                    const float P = kval, Q = __ldg(kh + size_t(M) * Hh + kyr);
                    const float2 cm = cconj(Cb[ky == 0 ? 0 : H - ky]);
                    d = cadd(cscale(c, 0.5f * (P + Q)), cscale(cm, 0.5f * (P - Q)));
                } else {
                    d = cscale(c, kval);
                }
                X[b * PITCH + ky] = cscale(d, kscale);
            };
            if constexpr (kAhead) {
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const int idx = int(threadIdx.x) + j * T;
                    if (idx < B * H && idx % B < cols) product(idx, kv[j]);
                }
            } else {
                for (int idx = threadIdx.x; idx < B * H; idx += T) {
                    const int b = idx % B, ky = idx / B;
                    if (b >= cols) continue;
                    product(idx, __ldg(kh + size_t(k0 + b) * Hh + min(ky, H - ky)));
                }
            }
            if (kk + 1 < nk) fetch_k(kk + 1);
            __syncthreads();
            // Inverse column FFT: X -> Y (-> X) -> U_k (global).
            float2* dst = U + size_t(kk) * M * H + gbase;
            const auto out = [dst](int b, int i, float2 v) { dst[size_t(i) * KB + b] = v; };
            tcfft::pass16<PF, 0, true, PREC, B, T>(from(X), at(Y), twi, Fi, cols);
            __syncthreads();
            if constexpr (NP == 2) {
                tcfft::pass16<PF, 1, true, PREC, B, T>(from(Y), out, twi, Fi, cols);
            } else {
                tcfft::pass16<PF, 1, true, PREC, B, T>(from(Y), at(X), twi, Fi, cols);
                __syncthreads();
                tcfft::pass16<PF, 2, true, PREC, B, T>(from(X), out, twi, Fi, cols);
            }
            __syncthreads();
        }
    }
}

template <class PF, int B, int PREC>
cudaError_t launch_t(const SpectralWorld& w0, const SpectralWorld* worlds, int n, int M, const FastTables& t,
                     cudaStream_t s) {
    using K = ColTcK<PF, B>;
    auto fn = col_tc_kernel<PF, B, PREC>;
    const size_t smem = K::smem();
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
    fn<<<world_grid(per, (M + B - 1) / B, n), K::T, smem, s>>>(w0, worlds, t.col_twf, t.col_twi);
    return cudaGetLastError();
}

template <class PF, int B>
cudaError_t launch_prec(int precision, const SpectralWorld& w0, const SpectralWorld* worlds, int n, int M,
                        const FastTables& t, cudaStream_t s) {
    if (precision == tcfft::kBF16x3) return launch_t<PF, B, tcfft::kBF16x3>(w0, worlds, n, M, t, s);
    if (precision == tcfft::kFP16x3) return launch_t<PF, B, tcfft::kFP16x3>(w0, worlds, n, M, t, s);
    return cudaErrorInvalidValue;
}

cudaError_t dispatch(int H, int M, int precision, int batch, const SpectralWorld& w0, const SpectralWorld* worlds,
                     int n, const FastTables& t, cudaStream_t s) {
    switch (H) {
        case 256:
            if (batch >= 8) return launch_prec<Plan<16, 16>, 8>(precision, w0, worlds, n, M, t, s);
            if (batch >= 4) return launch_prec<Plan<16, 16>, 4>(precision, w0, worlds, n, M, t, s);
            return launch_prec<Plan<16, 16>, 2>(precision, w0, worlds, n, M, t, s);
        case 4096:
            if (batch >= 2) return launch_prec<Plan<16, 16, 16>, 2>(precision, w0, worlds, n, M, t, s);
            return launch_prec<Plan<16, 16, 16>, 1>(precision, w0, worlds, n, M, t, s);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace

bool tc_col_plan(int H) { return H == 256 || H == 4096; }

cudaError_t launch_col_tc(const FftGeometry& g, const FastTables& t, int precision, int batch, const float2* S,
                          float2* U, cudaStream_t s) {
    SpectralWorld w{};
    w.S = S;
    w.U = U;
    w.khat = g.khat;
    w.M = g.M;
    w.nk = g.nk;
    return dispatch(g.H, g.M, precision, batch, w, nullptr, 1, t, s);
}

}  // namespace lenia
