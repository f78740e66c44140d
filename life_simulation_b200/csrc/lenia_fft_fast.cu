// life_simulation_b200/csrc/lenia_fft_fast.cu -- the spectral path's column
// and row passes for field sizes with a compile-time FFT plan (the sizes of
// the benchmark configs and common sim resolutions; others use the
// runtime-plan kernels of lenia_fft.cu, which produce the same layout).
//
// What compile-time plans buy over the runtime-plan kernels:
//   * every division/modulo of the Stockham index algebra is by a constant;
//   * composite radices (9, 15, ...) run in registers, so 1080 = 15*9*8 and
//     960 = 8*15*8 take three passes instead of five;
//   * the forward transform's last pass and the inverse's first pass use the
//     same radix (the inverse plan is the forward plan reversed), so item j
//     of the last pass holds exactly the elements item j of the next first
//     pass reads: the column spectrum stays in registers through the
//     per-kernel products, and in the row pass the potentials, the growth
//     accumulators and A' stay in registers from the inverse row FFT,
//     through the growth, into the forward row FFT of A'.
// Both kernels are persistent and software-pipelined: while a CTA transforms
// one work item (a column group; a row group x kernel), cp.async streams the
// next item's inputs into the other half of a double-buffered stage.
// Each pass loads all of a thread's items before computing any (ILP), and
// per-pass twiddle tables are laid out [t][m] so lanes with consecutive m
// read consecutive words.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "fft_ct.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

using fft::cadd;
using fft::cconj;
using fft::cmul;
using fft::cscale;
using fft::csub;
using namespace fftct;

namespace {

constexpr int roundup32(int x) { return (x + 31) / 32 * 32; }

// Smallest pitch >= n with 2*pitch = 8 (mod 32): rows of a batch then start
// 8 banks apart, so lanes that differ only in the row index do not collide.
constexpr int row_pitch(int n) {
    int p = n;
    while ((2 * p) % 32 != 8) ++p;
    return p;
}

// One Stockham pass over a batch: all of a thread's items are loaded first,
// then twiddled, transformed and stored. src(b, i) / dst(b, i, v) address
// element i of transform b.
template <class P, int PASS, bool INV, int B, int T, class Src, class Dst>
__device__ __forceinline__ void pass_gen(Src&& src, Dst&& dst, const float2* __restrict__ tw, int cols) {
    using I = PassIdx<P, PASS>;
    constexpr int TOT = B * I::NR;
    constexpr int ITEMS = (TOT + T - 1) / T;
    float2 v[ITEMS][I::R];
    int jj[ITEMS], bi[ITEMS];
    bool ok[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const int q = int(threadIdx.x) + it * T;
        bi[it] = q / I::NR;
        jj[it] = q - bi[it] * I::NR;
        ok[it] = (TOT % T == 0 || q < TOT) && bi[it] < cols;
        if (ok[it]) {
#pragma unroll
            for (int t = 0; t < I::R; ++t) v[it][t] = src(bi[it], I::in(jj[it], t));
        }
    }
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        if (ok[it]) {
            I::template twiddle<INV>(v[it], jj[it], tw);
            Dft<I::R, INV>::run(v[it]);
            const int ob = I::out_base(jj[it]);
#pragma unroll
            for (int t = 0; t < I::R; ++t) dst(bi[it], ob + t * I::NS, v[it][t]);
        }
    }
}

// Passes PASS..LAST-1 between two shared buffers (barrier after each);
// returns the buffer that holds the data afterwards.
template <class P, int PASS, int LAST, bool INV, int B, int T, int PITCH>
__device__ __forceinline__ float2* mid_passes(float2* a, float2* b, const float2* __restrict__ tw, int cols) {
    if constexpr (PASS < LAST) {
        pass_gen<P, PASS, INV, B, T>([&](int bb, int i) { return a[bb * PITCH + i]; },
                                     [&](int bb, int i, float2 v) { b[bb * PITCH + i] = v; }, tw, cols);
        __syncthreads();
        return mid_passes<P, PASS + 1, LAST, INV, B, T, PITCH>(b, a, tw, cols);
    } else {
        return a;
    }
}

__device__ __forceinline__ void copy_table(float2* dst, const float2* __restrict__ src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Asynchronous global -> shared copies (cp.async): the next work item's
// inputs stream into a second staging buffer while the current one is
// transformed. Completion is awaited per thread with cp.async.wait_group
// (a hardware wait, no spin loop) followed by a block barrier.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until at most one committed group of this thread is still pending.
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// ------------------------------------------------------------- columns

template <class PF, int B>
struct ColK {
    using PI = typename Reverse<PF>::type;
    static constexpr int H = PF::n;
    static constexpr int Hh = H / 2 + 1;
    static constexpr int RL = PF::last();
    static constexpr int NRL = H / RL;
    static constexpr int T = roundup32(B * NRL);
    static constexpr int ITL = (B * NRL + T - 1) / T;
    static constexpr int PITCH = H;
    static constexpr int KHP = (Hh + 3) / 4 * 4;  // staged kernel-spectrum column pitch (floats)
    // Stage of one column group: B columns of S, then nk x B kernel columns
    // (a multiple of 4 floats so both halves start 16-byte aligned).
    static constexpr size_t stage_floats(int nk) {
        return (size_t(2 * B * H) + size_t(nk) * B * KHP + 3) / 4 * 4;
    }
    // Float offset of the stage from the start of shared memory, rounded up
    // to 16 bytes.
    static constexpr size_t stage_offset() {
        return (2 * (size_t(PF::tw_size()) + PI::tw_size() + 2 * size_t(B) * PITCH + H) + 3) / 4 * 4;
    }
    static size_t smem(int nk) { return sizeof(float) * (stage_offset() + 2 * stage_floats(nk)); }
};

template <class PF, int B>
__global__ void __launch_bounds__(ColK<PF, B>::T)
    col_fast_kernel(const float2* __restrict__ S, float2* __restrict__ U, const float* __restrict__ khat,
                    const float2* __restrict__ twf_g, const float2* __restrict__ twi_g, int M, int nk) {
    using K = ColK<PF, B>;
    using PI = typename K::PI;
    using IL = PassIdx<PF, PF::np - 1>;
    constexpr int H = K::H, T = K::T, PITCH = K::PITCH, RL = K::RL, NRL = K::NRL, Hh = K::Hh, KHP = K::KHP;
    extern __shared__ __align__(16) float2 sm[];
    float2* twf = sm;
    float2* twi = twf + PF::tw_size();
    float2* ba = twi + PI::tw_size();
    float2* bb = ba + B * PITCH;
    float2* c0 = bb + B * PITCH;
    float* stage = reinterpret_cast<float*>(sm) + K::stage_offset();  // [2][stage_floats]
    const size_t sfl = K::stage_floats(nk);
    copy_table(twf, twf_g, PF::tw_size());
    copy_table(twi, twi_g, PI::tw_size());

    // Queues the copies of column group k0 (k0 > 0) into stage half `h`:
    // its columns of S (contiguous) and its kernel-spectrum columns. The
    // group holding the packed column kx = 0 reads global memory directly.
    auto issue = [&](int k0, int h) {
        float* st = stage + h * sfl;
        const int cols = min(B, M - k0);
        const float* src = reinterpret_cast<const float*>(S + size_t(k0) * H);
        const int nf = cols * H * 2;  // floats of S
        if ((size_t(k0) * H) % 2 == 0) {  // 16-byte aligned source
            for (int i = threadIdx.x; i < nf / 4; i += T) cp_async16(st + 4 * i, src + 4 * i);
            if (nf % 4 && threadIdx.x == 0) cp_async8(st + nf - 2, src + nf - 2);
        } else {
            for (int i = threadIdx.x; i < nf / 2; i += T) cp_async8(st + 2 * i, src + 2 * i);
        }
        float* ks = st + 2 * B * H;
        for (int kk = 0; kk < nk; ++kk)
            for (int b = 0; b < cols; ++b) {
                const float* kh = khat + size_t(kk) * (M + 1) * Hh + size_t(k0 + b) * Hh;
                float* dst = ks + (kk * B + b) * KHP;
                for (int i = threadIdx.x; i < Hh; i += T) cp_async4(dst + i, kh + i);
            }
    };
    int h = 0;
    int k0 = blockIdx.x * B;
    if (k0 < M) {
        if (k0 != 0) issue(k0, 0);
        cp_async_commit();
    }
    __syncthreads();
    for (; k0 < M; k0 += gridDim.x * B) {
        const int cols = min(B, M - k0);
        const int kn = k0 + gridDim.x * B;
        if (kn < M && kn != 0) issue(kn, h ^ 1);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        const bool staged = k0 != 0;  // the kx = 0 group reads global memory directly
        const float2* st = reinterpret_cast<const float2*>(stage + h * sfl);
        const float* ks = stage + h * sfl + 2 * B * H;
        const float2* gsrc = S + size_t(k0) * H;
        pass_gen<PF, 0, false, B, T>(
            [&](int b, int i) { return staged ? st[b * H + i] : __ldg(gsrc + b * H + i); },
            [&](int b, int i, float2 v) { ba[b * PITCH + i] = v; }, twf, cols);
        __syncthreads();
        float2* X = mid_passes<PF, 1, PF::np - 1, false, B, T, PITCH>(ba, bb, twf, cols);
        float2* Y = (X == ba) ? bb : ba;
        // Last forward pass: the column spectrum C stays in registers.
        float2 C[K::ITL][RL];
        int jj[K::ITL], bi[K::ITL];
        bool ok[K::ITL];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            bi[it] = q / NRL;
            jj[it] = q - bi[it] * NRL;
            ok[it] = q < B * NRL && bi[it] < cols;
            if (ok[it]) {
#pragma unroll
                for (int t = 0; t < RL; ++t) C[it][t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
                IL::template twiddle<false>(C[it], jj[it], twf);
                Dft<RL, false>::run(C[it]);
                if (k0 == 0 && bi[it] == 0) {
#pragma unroll
                    for (int t = 0; t < RL; ++t) c0[jj[it] + t * NRL] = C[it][t];
                }
            }
        }
        if (k0 == 0) __syncthreads();  // c0 (packed DC/Nyquist column) visible
        for (int kk = 0; kk < nk; ++kk) {
            const float* khg = khat + size_t(kk) * (M + 1) * Hh;
            // Spectrum product, then the inverse's first pass (radix RL, no
            // twiddles) from registers into Y.
#pragma unroll
            for (int it = 0; it < K::ITL; ++it) {
                if (!ok[it]) continue;
                const int kx = k0 + bi[it];
                const float* kcol = ks + (kk * B + bi[it]) * KHP;
                float2 D[RL];
#pragma unroll
                for (int t = 0; t < RL; ++t) {
                    const int ky = jj[it] + t * NRL;
                    const int kyr = min(ky, H - ky);
                    if (kx == 0) {
                        const float P = __ldg(khg + kyr), Q = __ldg(khg + size_t(M) * Hh + kyr);
                        const float2 Cm = cconj(c0[ky == 0 ? 0 : H - ky]);
                        D[t] = cadd(cscale(C[it][t], 0.5f * (P + Q)), cscale(Cm, 0.5f * (P - Q)));
                    } else {
                        D[t] = cscale(C[it][t], staged ? kcol[kyr] : __ldg(khg + size_t(kx) * Hh + kyr));
                    }
                }
                Dft<RL, true>::run(D);
#pragma unroll
                for (int t = 0; t < RL; ++t) Y[bi[it] * PITCH + jj[it] * RL + t] = D[t];
            }
            __syncthreads();
            float2* Z = mid_passes<PI, 1, PI::np - 1, true, B, T, PITCH>(Y, X, twi, cols);
            float2* dst = U + size_t(kk) * M * H + size_t(k0) * H;
            pass_gen<PI, PI::np - 1, true, B, T>([&](int b, int i) { return Z[b * PITCH + i]; },
                                                  [&](int b, int i, float2 v) { dst[b * H + i] = v; }, twi, cols);
            __syncthreads();
        }
        h ^= 1;
    }
}

// ---------------------------------------------------------------- rows

template <class PI, int RB>
struct RowK {
    using PF = typename Reverse<PI>::type;
    static constexpr int M = PI::n;
    static constexpr int RC = PI::last();
    static constexpr int NRC = M / RC;
    static constexpr int T = roundup32(RB * NRC);
    static constexpr int ITL = (RB * NRC + T - 1) / T;
    static constexpr int PITCH = row_pitch(M);
    static constexpr size_t smem() {
        return sizeof(float2) * (size_t(M + 1) + PI::tw_size() + PF::tw_size() + 4 * size_t(RB) * PITCH);
    }
};

template <class PI, int RB>
__global__ void __launch_bounds__(RowK<PI, RB>::T)
    row_fast_kernel(const float2* __restrict__ U, const float* __restrict__ A, float* __restrict__ A_out,
                    float2* __restrict__ S_next, const float2* __restrict__ twr_g,
                    const float2* __restrict__ twi_g, const float2* __restrict__ twf_g, int H, int nk,
                    StepParams p) {
    using K = RowK<PI, RB>;
    using PF = typename K::PF;
    using IL = PassIdx<PI, PI::np - 1>;
    constexpr int M = K::M, W = 2 * M, T = K::T, PITCH = K::PITCH, RC = K::RC, NRC = K::NRC;
    extern __shared__ __align__(16) float2 sm[];
    float2* twr = sm;
    float2* twi = twr + (M + 1);
    float2* twf = twi + PI::tw_size();
    float2* stg = twf + PF::tw_size();  // [2][RB * PITCH]
    float2* ba = stg + 2 * RB * PITCH;
    float2* bb = ba + RB * PITCH;
    copy_table(twr, twr_g, M + 1);
    copy_table(twi, twi_g, PI::tw_size());
    copy_table(twf, twf_g, PF::tw_size());
    const bool asym = p.growth_mode == 1u;
    const int ystride = gridDim.x * RB;

    // Queues kernel kk's spectrum rows y0..y0+RB (column-major in U) into
    // stage half h, transposed to row-major with pitch PITCH.
    auto issue = [&](int y0, int kk, int h) {
        const int rows = min(RB, H - y0);
        const float2* Uk = U + size_t(kk) * M * H + y0;
        float2* st = stg + h * RB * PITCH;
        for (int q = threadIdx.x; q < M * RB; q += T) {
            const int k = q / RB, b = q - k * RB;
            if (b < rows) cp_async8(st + b * PITCH + k, Uk + size_t(k) * H + b);
        }
    };
    int h = 0;
    if (int(blockIdx.x) * RB < H) issue(blockIdx.x * RB, 0, 0);
    cp_async_commit();
    __syncthreads();
    for (int y0 = blockIdx.x * RB; y0 < H; y0 += ystride) {
        const int rows = min(RB, H - y0);
        int jj[K::ITL], bi[K::ITL];
        bool ok[K::ITL];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            bi[it] = q / NRC;
            jj[it] = q - bi[it] * NRC;
            ok[it] = q < RB * NRC && bi[it] < rows;
        }
        float acc[K::ITL][RC][2];
        for (int kk = 0; kk < nk; ++kk) {
            // Prefetch the next work item: the next kernel of these rows, or
            // the first kernel of the next row group.
            if (kk + 1 < nk) issue(y0, kk + 1, h ^ 1);
            else if (y0 + ystride < H) issue(y0 + ystride, 0, h ^ 1);
            cp_async_commit();
            cp_async_wait_prev();
            __syncthreads();
            const float2* st = stg + h * RB * PITCH;
            // Inverse of the real-FFT split folded into the first pass's loads:
            // Z'[k] = (X[k] + conj X[M-k]) + i exp(+2 pi i k/W) (X[k] - conj X[M-k]).
            pass_gen<PI, 0, true, RB, T>(
                [&](int b, int i) {
                    const float2* xr = st + b * PITCH;
                    if (i == 0) {
                        const float2 x0 = xr[0];
                        return make_float2(x0.x + x0.y, x0.x - x0.y);
                    }
                    const float2 Xk = xr[i];
                    const float2 Xm = cconj(xr[M - i]);
                    const float2 D = cmul(cconj(twr[i]), csub(Xk, Xm));
                    return cadd(cadd(Xk, Xm), make_float2(-D.y, D.x));
                },
                [&](int b, int i, float2 v) { ba[b * PITCH + i] = v; }, twi, rows);
            __syncthreads();
            float2* X = mid_passes<PI, 1, PI::np - 1, true, RB, T, PITCH>(ba, bb, twi, rows);
            // Last inverse pass into registers: u[2n], u[2n+1] for n = j + t*NRC.
            // Selects instead of a dynamic index into the parameter block (which
            // would spill it to local memory).
            const auto pick = [&](const float(&a)[kMaxKernels]) {
                return kk == 0 ? a[0] : kk == 1 ? a[1] : kk == 2 ? a[2] : a[3];
            };
            const float mu = pick(p.mu), inv_sigma = 1.0f / pick(p.sigma), hw = pick(p.weight);
            const bool jitter = p.mu_jitter > 0.0f;
#pragma unroll
            for (int it = 0; it < K::ITL; ++it) {
                if (!ok[it]) continue;
                float2 z[RC];
#pragma unroll
                for (int t = 0; t < RC; ++t) z[t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
                IL::template twiddle<true>(z, jj[it], twi);
                Dft<RC, true>::run(z);
                const uint32_t gy = uint32_t(y0 + bi[it]);
#pragma unroll
                for (int t = 0; t < RC; ++t) {
                    const uint32_t x0 = uint32_t(2 * (jj[it] + t * NRC));
                    const float m0 = jitter ? mu + mu_jitter_shift(p, x0, gy) : mu;
                    const float m1 = jitter ? mu + mu_jitter_shift(p, x0 + 1u, gy) : mu;
                    const float b0 = bell_fast(z[t].x, m0, inv_sigma);
                    const float b1 = bell_fast(z[t].y, m1, inv_sigma);
                    const float c0 = asym ? hw * b0 : hw * (2.0f * b0 - 1.0f);
                    const float c1 = asym ? hw * b1 : hw * (2.0f * b1 - 1.0f);
                    acc[it][t][0] = kk == 0 ? c0 : acc[it][t][0] + c0;
                    acc[it][t][1] = kk == 0 ? c1 : acc[it][t][1] + c1;
                }
            }
            __syncthreads();
            h ^= 1;
        }
        // Euler step, noise, injection, clip; A' stored and kept for the
        // next substep's row transform (forward first pass, radix RC).
        float2 za[K::ITL][RC];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            if (!ok[it]) continue;
            const int gy = y0 + bi[it];
#pragma unroll
            for (int t = 0; t < RC; ++t) {
                const int n = jj[it] + t * NRC;
                const size_t gi = size_t(gy) * W + 2 * n;
                const float2 a = __ldg(reinterpret_cast<const float2*>(A + gi));
                GrowthAcc g0, g1;
                g0.weighted = g0.std_sum = acc[it][t][0];
                g1.weighted = g1.std_sum = acc[it][t][1];
                const float2 r = make_float2(growth_finish(p, a.x, g0, uint32_t(2 * n), uint32_t(gy)),
                                             growth_finish(p, a.y, g1, uint32_t(2 * n + 1), uint32_t(gy)));
                *reinterpret_cast<float2*>(A_out + gi) = r;
                za[it][t] = r;
            }
        }
        if (S_next == nullptr) continue;
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            if (!ok[it]) continue;
            Dft<RC, false>::run(za[it]);
#pragma unroll
            for (int t = 0; t < RC; ++t) ba[bi[it] * PITCH + jj[it] * RC + t] = za[it][t];
        }
        __syncthreads();
        float2* Y = mid_passes<PF, 1, PF::np - 1, false, RB, T, PITCH>(ba, bb, twf, rows);
        float2* Zo = (Y == ba) ? bb : ba;
        pass_gen<PF, PF::np - 1, false, RB, T>([&](int b, int i) { return Y[b * PITCH + i]; },
                                                [&](int b, int i, float2 v) { Zo[b * PITCH + i] = v; }, twf, rows);
        __syncthreads();
        // Real-FFT split and the column-major store (rows fastest).
        for (int q = threadIdx.x; q < M * RB; q += T) {
            const int k = q / RB, b = q - k * RB;
            if (b >= rows) continue;
            const float2* zr = Zo + b * PITCH;
            const float2 Zk = zr[k];
            float2 Xv;
            if (k == 0) {
                Xv = make_float2(Zk.x + Zk.y, Zk.x - Zk.y);
            } else {
                const float2 Zc = cconj(zr[M - k]);
                const float2 E = cscale(cadd(Zk, Zc), 0.5f);
                const float2 D = csub(Zk, Zc);
                const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
                Xv = cadd(E, cmul(twr[k], O));
            }
            S_next[size_t(k) * H + y0 + b] = Xv;
        }
        __syncthreads();
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ------------------------------------------------------------- catalog

template <class P>
void plan_radices(FastPlan& out) {
    out.n = P::n;
    out.np = P::np;
    for (int i = 0; i < P::np; ++i) out.radix[i] = P::radix(i);
}

int g_sms = 0;
int sms() {
    if (!g_sms) {
        int d = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
        if (g_sms <= 0) g_sms = 148;
    }
    return g_sms;
}

template <typename F>
cudaError_t prepare(F fn, size_t smem) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

template <class PF, int B>
cudaError_t launch_col_t(const FftGeometry& g, const FastTables& t, const float2* S, float2* U,
                         cudaStream_t s) {
    using K = ColK<PF, B>;
    auto fn = col_fast_kernel<PF, B>;
    const size_t smem = K::smem(g.nk);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
    const int groups = (g.M + B - 1) / B;
    const int grid = std::max(1, std::min(groups, std::max(1, per) * sms()));
    fn<<<grid, K::T, smem, s>>>(S, U, g.khat, t.col_twf, t.col_twi, g.M, g.nk);
    return cudaGetLastError();
}

template <class PI, int RB>
cudaError_t launch_row_t(const FftGeometry& g, const FastTables& t, const float2* U, const float* A,
                         float* A_out, float2* S_next, const StepParams& p, cudaStream_t s) {
    using K = RowK<PI, RB>;
    auto fn = row_fast_kernel<PI, RB>;
    const size_t smem = K::smem();
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
    const int groups = (g.H + RB - 1) / RB;
    const int grid = std::max(1, std::min(groups, std::max(1, per) * sms()));
    fn<<<grid, K::T, smem, s>>>(U, A, A_out, S_next, g.tw_r2c, t.row_twi, t.row_twf, g.H, g.nk, p);
    return cudaGetLastError();
}

// Column plans (forward order) by transform length. The last radix is
// kept small: the column spectrum of the last pass lives in registers.
#define LENIA_COL_PLANS(X)     \
    X(1080, Plan<15, 9, 8>)    \
    X(512, Plan<8, 8, 8>)      \
    X(1024, Plan<16, 8, 8>)    \
    X(4096, Plan<16, 16, 16>)  \
    X(2048, Plan<16, 16, 8>)   \
    X(256, Plan<16, 16>)       \
    X(128, Plan<16, 8>)        \
    X(216, Plan<6, 6, 6>)      \
    X(64, Plan<8, 8>)
// Row plans (inverse order) by M = W/2.
#define LENIA_ROW_PLANS(X)     \
    X(960, Plan<8, 15, 8>)     \
    X(512, Plan<8, 8, 8>)      \
    X(2048, Plan<16, 8, 16>)   \
    X(256, Plan<16, 16>)       \
    X(192, Plan<8, 3, 8>)      \
    X(128, Plan<16, 8>)        \
    X(64, Plan<8, 8>)

}  // namespace

bool fast_col_plan(int H, FastPlan& fwd) {
    switch (H) {
#define X(n, ...) \
    case n: plan_radices<__VA_ARGS__>(fwd); return true;
        LENIA_COL_PLANS(X)
#undef X
    default: return false;
    }
}

bool fast_row_plan(int M, FastPlan& inv) {
    switch (M) {
#define X(n, ...) \
    case n: plan_radices<__VA_ARGS__>(inv); return true;
        LENIA_ROW_PLANS(X)
#undef X
    default: return false;
    }
}

// Per-pass twiddles of a plan in the device layout: for pass p >= 1 with
// span Ns and radix R, entry [(t-1)*Ns + m] = exp(-2 pi i m t / (Ns R)).
void fast_plan_twiddles(const FastPlan& plan, std::vector<float2>& out) {
    out.clear();
    int ns = plan.radix[0];
    for (int p = 1; p < plan.np; ++p) {
        const int r = plan.radix[p];
        for (int t = 1; t < r; ++t)
            for (int m = 0; m < ns; ++m) {
                const double a = 2.0 * M_PI * double(m) * double(t) / double(ns * r);
                out.push_back(make_float2(float(std::cos(a)), float(-std::sin(a))));
            }
        ns *= r;
    }
}

cudaError_t launch_col_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* S,
                            float2* U, cudaStream_t s) {
    switch (g.H) {
#define X(n, ...)                                                             \
    case n:                                                                   \
        if (batch == 2) return launch_col_t<__VA_ARGS__, 2>(g, t, S, U, s);   \
        if (batch == 4) return launch_col_t<__VA_ARGS__, 4>(g, t, S, U, s);   \
        return launch_col_t<__VA_ARGS__, 1>(g, t, S, U, s);
        LENIA_COL_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

cudaError_t launch_row_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* U,
                            const float* A, float* A_out, float2* S_next, const StepParams& p,
                            cudaStream_t s) {
    switch (g.M) {
#define X(n, ...)                                                                           \
    case n:                                                                                 \
        if (batch == 2) return launch_row_t<__VA_ARGS__, 2>(g, t, U, A, A_out, S_next, p, s); \
        if (batch == 4) return launch_row_t<__VA_ARGS__, 4>(g, t, U, A, A_out, S_next, p, s); \
        return launch_row_t<__VA_ARGS__, 1>(g, t, U, A, A_out, S_next, p, s);
        LENIA_ROW_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

}  // namespace lenia
