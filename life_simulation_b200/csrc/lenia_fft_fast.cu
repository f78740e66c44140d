// life_simulation_b200/csrc/lenia_fft_fast.cu -- the spectral path's column
// and row passes for field sizes with a compile-time FFT plan (the sizes of
// the benchmark configs and common sim resolutions; other sizes use the
// runtime-plan kernels of lenia_fft.cu).
//
// Spectral layout of this path ("blocked"): spectra S and U_k are stored in
// blocks of 8 columns, element (kx, ky) at ((kx/8)*H + ky)*8 + kx%8, so a row
// of a block is 64 contiguous bytes. The column pass reads/writes 4- or
// 8-column slices of a block (32/64 B per row), the row pass reads/writes
// RB rows x 8 columns (RB*64 contiguous bytes per block): both coalesced.
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
// Items are mapped with the batch index fastest (lane -> (b, j)), which makes
// the global loads/stores of the first/last passes contiguous, and shared
// buffers use a row pitch of 8 banks (mod 32) so lanes of different b do not
// collide. Complex arithmetic uses the packed FP32x2 instructions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "fft_ct.cuh"
#include "colormap.cuh"
#include "fft_fast_common.cuh"
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

using namespace fastfft;

// ------------------------------------------------------------- columns

// Shared-memory staging of the next column group's row spectrum (B columns
// x H rows, row-major, 16-byte asynchronous copies): used when B is even and
// the extra buffer fits the 227 KB a CTA may have.
template <class PF, int B, int S = 1>
struct ColStage {
    using K = ColK<PF, B, S>;
    static constexpr int OFF = (K::BUF0 + 2 * B * K::PITCH + K::H + 1) / 2 * 2;  // 16-byte aligned
    static constexpr size_t with_stage = sizeof(float2) * (size_t(OFF) + size_t(B) * K::H);
    // Not with S = 2, whose CTAs are meant to fit two per SM.
    static constexpr bool on = S == 1 && B % 2 == 0 && with_stage <= 227 * 1024;
    static constexpr size_t smem() { return on ? with_stage : K::smem(); }
};

template <class PF, int B, int SPLIT>
__global__ void __launch_bounds__(ColK<PF, B, SPLIT>::T)
    col_fast_kernel(SpectralWorld w0, const SpectralWorld* __restrict__ worlds,
                    const float2* __restrict__ twf_g, const float2* __restrict__ twi_g) {
    using K = ColK<PF, B, SPLIT>;
    using PI = typename K::PI;
    using IL = PassIdx<PF, PF::np - 1>;
    constexpr int H = K::H, T = K::T, PITCH = K::PITCH, RL = K::RL, NRL = K::NRL, Hh = K::Hh;
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SpectralWorld sw;  // this CTA's world
    float2* twf = sm;
    float2* twi = twf + PF::tw_size();
    float2* ba = sm + K::BUF0;
    float2* bb = ba + B * PITCH;
    float2* c0 = bb + B * PITCH;
    copy_table(twf, twf_g, PF::tw_size());
    copy_table(twi, twi_g, PI::tw_size());
    grid_dependency_wait();
    if (threadIdx.x == 0) sw = worlds ? worlds[blockIdx.y] : w0;
    __syncthreads();
    const float2* __restrict__ S = sw.S;
    float2* __restrict__ U = sw.U;
    const float* __restrict__ khat = sw.khat;
    const int M = sw.M, nk = sw.nk;
    using CS = ColStage<PF, B, SPLIT>;
    float2* bs = sm + CS::OFF;
    // Rows of columns g0..g0+B-1 of S into bs as bs[i * B + b].
    const auto stage_group = [&](int g0) {
        const float2* src = S + size_t(g0 / KB) * H * KB + (g0 % KB);
        for (int q = threadIdx.x; q < H * (B / 2); q += T) {
            const int i = q / (B / 2), c2 = q - i * (B / 2);
            cp_async16(bs + i * B + 2 * c2, src + size_t(i) * KB + 2 * c2);
        }
        cp_async_commit();
    };
    if constexpr (CS::on) {
        if (int(blockIdx.x) * B < M) stage_group(int(blockIdx.x) * B);
    }
    if (int(blockIdx.x) * B >= M) allow_dependents();
    for (int k0 = blockIdx.x * B; k0 < M; k0 += gridDim.x * B) {
        if (k0 + int(gridDim.x) * B >= M) allow_dependents();  // this CTA's last group
        const int cols = min(B, M - k0);
        // Element (b, ky) of this group in the blocked layout.
        const size_t gbase = size_t(k0 / KB) * H * KB + (k0 % KB);
        int jj[K::ITL], bi[K::ITL];
        bool ok[K::ITL];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            jj[it] = q / B;
            bi[it] = q - jj[it] * B;
            ok[it] = q < B * NRL && bi[it] < cols;
        }
        // Kernel spectrum values of this thread's last-pass elements, one
        // kernel ahead: kernel 0's are in flight during the forward
        // transform, kernel k+1's during kernel k's inverse. Only for last
        // passes of radix <= 8: with 16 values per item the extra registers
        // cost more occupancy than the hidden latency gains.
        constexpr bool kAhead = RL <= 8;
        float kv[K::ITL][kAhead ? RL : 1], kv2[K::ITL][kAhead ? RL : 1];  // kv2: Nyquist column (packed column 0)
        const auto fetch_k = [&](int kk) {
            if constexpr (kAhead) {
                const float* kh = khat + size_t(kk) * (M + 1) * Hh;
#pragma unroll
                for (int it = 0; it < K::ITL; ++it) {
                    const int kx = k0 + bi[it];
#pragma unroll
                    for (int t = 0; t < RL; ++t) {
                        const int ky = jj[it] + t * NRL;
                        const int kyr = min(ky, H - ky);
                        kv[it][t] = ok[it] ? __ldg(kh + size_t(kx) * Hh + kyr) : 0.0f;
                        kv2[it][t] = (ok[it] && kx == 0) ? __ldg(kh + size_t(M) * Hh + kyr) : 0.0f;
                    }
                }
            }
        };
        if (nk > 0) fetch_k(0);
        if constexpr (CS::on) {
            cp_async_wait_all();
            __syncthreads();  // this group's rows staged
            pass0_buf<PF, false, B, T, PITCH>([&](int b, int i) { return bs[i * B + b]; }, ba, cols);
            __syncthreads();  // bs read: the next group's rows may land
            const int next = k0 + int(gridDim.x) * B;
            if (next < M) stage_group(next);
        } else {
            pass0_buf<PF, false, B, T, PITCH>([&](int b, int i) { return __ldg(S + gbase + size_t(i) * KB + b); }, ba,
                                              cols);
            __syncthreads();
        }
        float2* X = mid_passes<PF, 1, PF::np - 1, false, B, T, PITCH>(ba, bb, twf, cols);
        // The other buffer, chosen by the (compile-time) pass count rather than
        // by comparing pointers, so every access through it stays a
        // shared-memory access (a runtime select between buffers compiles to
        // generic loads and stores).
        float2* Y = (PF::np - 2) % 2 ? ba : bb;
        // Last forward pass: the column spectrum C stays in registers.
        float2 C[K::ITL][RL];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
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
        // Spectrum product of kernel kk, then the inverse's first pass (radix
        // RL, no twiddles) from registers into Y; kernel kk+1's spectrum values
        // are fetched while kk's remaining passes run.
        const auto first_inverse = [&](int kk) {
#pragma unroll
            for (int it = 0; it < K::ITL; ++it) {
                if (!ok[it]) continue;
                const int kx = k0 + bi[it];
                float2 D[RL];
                const float* kh = khat + size_t(kk) * (M + 1) * Hh;
#pragma unroll
                for (int t = 0; t < RL; ++t) {
                    const int ky = jj[it] + t * NRL;
                    const int kyr = min(ky, H - ky);
                    float kval, knyq;
                    if constexpr (kAhead) {
                        kval = kv[it][t];
                        knyq = kv2[it][t];
                    } else {
                        kval = __ldg(kh + size_t(kx) * Hh + kyr);
                        knyq = kx == 0 ? __ldg(kh + size_t(M) * Hh + kyr) : 0.0f;
                    }
                    if (kx == 0) {
                        const float P = kval, Q = knyq;
                        const float2 Cm = cconj(c0[ky == 0 ? 0 : H - ky]);
                        D[t] = cadd(cscale(C[it][t], 0.5f * (P + Q)), cscale(Cm, 0.5f * (P - Q)));
                    } else {
                        D[t] = cscale(C[it][t], kval);
                    }
                }
                Dft<RL, true>::run(D);
                store_run<RL>(Y + bi[it] * PITCH, jj[it] * RL, D);
            }
            if (kk + 1 < nk) fetch_k(kk + 1);
        };
        // The inverse's last pass of kernel kk from Z into U_kk.
        const auto last_inverse = [&](int kk, const float2* Z) {
            float2* dst = U + size_t(kk) * M * H + gbase;
            pass_gen<PI, PI::np - 1, true, B, T>(
                [&](int b, int i) { return Z[b * PITCH + i]; },
                [&](int b, int i, float2 v) { dst[size_t(i) * KB + b] = v; }, twi, cols);
        };
        // With an odd number of middle passes the last pass reads X while the
        // next kernel's first pass writes Y, so the two share one barrier
        // interval: the last pass's threads (radix 15 at 1080: 288 of 544)
        // are joined by the whole CTA's next first pass instead of idling at
        // a barrier. Same operations, same bits.
        constexpr bool kMerge = (PI::np - 2) % 2 == 1;
        if (nk > 0) first_inverse(0);
        for (int kk = 0; kk < nk; ++kk) {
            __syncthreads();  // Y holds kernel kk's first pass
            float2* Z = mid_passes<PI, 1, PI::np - 1, true, B, T, PITCH>(Y, X, twi, cols);
            last_inverse(kk, Z);
            if (kk + 1 < nk) {
                if constexpr (!kMerge) __syncthreads();  // Z is Y: read before it is rewritten
                first_inverse(kk + 1);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- rows

// The colour layer of two adjacent pixels of A' (the module's output pass,
// fused into the last substep): both RGBA16F texels in one 16-byte store.
// Out of line: the rare path costs the row pass no registers.
static __device__ __noinline__ void palette_pair(const ColorMapParams& cm, float2 v, uint2* dst) {
    __half t0[4], t1[4];
    palette_rgba16f(cm, channel_of(v.x, cm.channel), t0);
    palette_rgba16f(cm, channel_of(v.y, cm.channel), t1);
    uint4 q;
    q.x = uint32_t(__half_as_ushort(t0[0])) | (uint32_t(__half_as_ushort(t0[1])) << 16);
    q.y = uint32_t(__half_as_ushort(t0[2])) | (uint32_t(__half_as_ushort(t0[3])) << 16);
    q.z = uint32_t(__half_as_ushort(t1[0])) | (uint32_t(__half_as_ushort(t1[1])) << 16);
    q.w = uint32_t(__half_as_ushort(t1[2])) | (uint32_t(__half_as_ushort(t1[3])) << 16);
    *reinterpret_cast<uint4*>(dst) = q;
}

// nk > 0: inverse row transforms of U_k, growth, A' (+ the next step's row
// spectrum when S_next != null). nk == 0: only the forward row transform of
// A into S_next (the first step after an upload or init).
//
// PIPE: software pipeline over two staging buffers and one work buffer.
// While the rows of U_k go through their inverse transform, the rows of
// U_{k+1} (after the last kernel: the rows of A) are already in flight by
// cp.async, and while A' goes through the forward transform, the next row
// group's U_0 is: a CTA always has one staged load in flight. Without PIPE
// (one staging buffer, which doubles as the second work buffer) each item is
// staged and waited for in turn: less shared memory per CTA, which wins
// where shared memory limits the resident CTAs (long rows).
template <class PI, int RB, bool PIPE, bool CM, int SPLIT>
__global__ void __launch_bounds__(RowK<PI, RB, SPLIT>::T,
                                  (512 / RowK<PI, RB, SPLIT>::T > 1 ? 512 / RowK<PI, RB, SPLIT>::T : 1))
    row_fast_kernel(SpectralWorld w0, const SpectralWorld* __restrict__ worlds,
                    const float2* __restrict__ twr_g, const float2* __restrict__ twi_g,
                    const float2* __restrict__ twf_g) {
    using K = RowK<PI, RB, SPLIT>;
    using PF = typename K::PF;
    using IL = PassIdx<PI, PI::np - 1>;
    constexpr int M = K::M, W = 2 * M, T = K::T, PITCH = K::PITCH, RC = K::RC, NRC = K::NRC;
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SpectralWorld sw;  // this CTA's world
    float2* twr = sm;
    float2* twi = twr + (M + 1);
    float2* twf = twi + PI::tw_size();
    // Staging (16-byte aligned) and work buffers.
    // Staging buffer i & 1 by address arithmetic on the shared array (a
    // runtime-indexed pointer table would make every access through it a
    // generic load).
    const auto stg = [&](int i) { return sm + K::BUF0 + (PIPE ? (i & 1) * (RB * PITCH) : 0); };
    float2* bw = sm + K::BUF0 + (PIPE ? 2 : 1) * RB * PITCH;
    copy_table(twr, twr_g, M + 1);
    copy_table(twi, twi_g, PI::tw_size());
    copy_table(twf, twf_g, PF::tw_size());
    grid_dependency_wait();
    if (threadIdx.x == 0) sw = worlds ? worlds[blockIdx.y] : w0;
    __syncthreads();
    const float2* __restrict__ U = sw.U;
    const float* __restrict__ A = sw.A;
    float* __restrict__ A_out = sw.A_out;
    float2* __restrict__ S_next = sw.S_next;
    float* __restrict__ U_px = sw.U_px;
    const int H = int(sw.p.height), nk = sw.nk;
    const StepParams& p = sw.p;
    const bool asym = p.growth_mode == 1u;
    const bool jitter = p.mu_jitter > 0.0f;
    // The Euler step's parameters in registers (the rare noise / injection
    // path reads them from the shared block out of line).
    const bool extras = p.noise_amount > 0.0f || p.inject_amount > 0.0f;
    const float dt = p.dt, sum_w = p.sum_weights;
    const bool sw_ok = sum_w > 1e-6f;
    // Item idx of a row group: the rows of U_idx for idx < nk, else of A.
    const auto stage = [&](float2* dst, int y, int idx) {
        if (y >= H) return;
        const int n = min(RB, H - y);
        if (idx < nk)
            stage_rows<M, RB, T, PITCH>(dst, U + size_t(idx) * M * H, H, y, n);
        else
            stage_field_rows<M, RB, T, PITCH>(dst, A, y, n);
    };
    int base = 0;  // staging buffer of the group's first item
    if constexpr (PIPE) {
        stage(stg(0), int(blockIdx.x) * RB, 0);
        cp_async_commit();
    }
    if (int(blockIdx.x) * RB >= H) allow_dependents();
    for (int y0 = blockIdx.x * RB; y0 < H; y0 += gridDim.x * RB) {
        if (y0 + int(gridDim.x) * RB >= H) allow_dependents();  // this CTA's last row group
        const int rows = min(RB, H - y0);
        int jj[K::ITL], bi[K::ITL];
        bool ok[K::ITL];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            jj[it] = q / RB;
            bi[it] = q - jj[it] * RB;
            ok[it] = q < RB * NRC && bi[it] < rows;
        }
        float2 acc[K::ITL][RC];  // growth sums of the pixel pair (2n, 2n + 1)
        for (int kk = 0; kk < nk; ++kk) {
            float2* cur = stg(base + kk);
            if constexpr (PIPE) {
                // One barrier makes item kk's rows visible and frees the
                // other staging buffer (item kk-1's, whose last pass every
                // thread has finished); item kk+1 then lands there while kk
                // is transformed.
                cp_async_wait_all();
                __syncthreads();
                stage(stg(base + kk + 1), y0, kk + 1);
                cp_async_commit();
            } else {
                stage(cur, y0, kk);
                cp_async_wait_all();
                __syncthreads();
            }
            // Inverse of the real-FFT split folded into the first pass's loads.
            pass0_buf<PI, true, RB, T, PITCH>([&](int b, int i) { return c2r_split<M>(cur + b * PITCH, twr, i); }, bw,
                                              rows);
            __syncthreads();
            float2* X = mid_passes<PI, 1, PI::np - 1, true, RB, T, PITCH>(bw, cur, twi, rows);
            // Selects instead of a dynamic index into the parameter block (which
            // would spill it to local memory).
            const auto pick = [&](const float(&a)[kMaxKernels]) {
                return kk == 0 ? a[0] : kk == 1 ? a[1] : kk == 2 ? a[2] : a[3];
            };
            const GrowthPair gp(pick(p.mu), 1.0f / pick(p.sigma), pick(p.weight), asym);
            // Last inverse pass into registers: u[2n], u[2n+1] for n = j + t*NRC.
#pragma unroll
            for (int it = 0; it < K::ITL; ++it) {
                if (!ok[it]) continue;
                float2 z[RC];
#pragma unroll
                for (int t = 0; t < RC; ++t) z[t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
                IL::template twiddle<true>(z, jj[it], twi);
                Dft<RC, true>::run(z);
                const uint32_t gy = uint32_t(y0 + bi[it]);
                if (U_px) {  // keep the potentials (the adjoint's recomputation)
                    float* up = U_px + (size_t(kk) * H + gy) * W;
#pragma unroll
                    for (int t = 0; t < RC; ++t) *reinterpret_cast<float2*>(up + 2 * (jj[it] + t * NRC)) = z[t];
                }
#pragma unroll
                for (int t = 0; t < RC; ++t) {
                    const float2 c = gp.term(z[t], p, jitter, uint32_t(2 * (jj[it] + t * NRC)), gy);
                    acc[it][t] = kk == 0 ? c : __fadd2_rn(acc[it][t], c);
                }
            }
            if constexpr (!PIPE) __syncthreads();  // cur (the one staging buffer) read
        }
        // The rows of A are in sA; the other staging buffer takes the next
        // row group's first item.
        float2* sA = stg(base + nk);
        if constexpr (PIPE) {
            cp_async_wait_all();
            __syncthreads();  // A's rows visible; the last kernel's buffer free
            stage(stg(base + nk + 1), y0 + int(gridDim.x) * RB, 0);
            cp_async_commit();
        } else {
            stage(sA, y0, nk);
            cp_async_wait_all();
            __syncthreads();
        }
        // Euler step, noise, injection, clip (or, with nk == 0, the field as
        // is); the result is kept for the forward row transform (first
        // pass radix RC, the same elements per thread).
        float2 za[K::ITL][RC];
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            if (!ok[it]) continue;
            const int gy = y0 + bi[it];
#pragma unroll
            for (int t = 0; t < RC; ++t) {
                const int n = jj[it] + t * NRC;
                const float2 a = sA[bi[it] * PITCH + n];
                if (nk == 0) {
                    za[it][t] = a;
                    continue;
                }
                // growth_finish_lean with the parameters in registers.
                const auto finish = [&](float A, float s, uint32_t gx) {
                    if (extras) return growth_finish_call(p, A, s, s, gx, uint32_t(gy));
                    const float A2 = asym ? A + dt * ((sw_ok ? s / sum_w : A) - A) : A + dt * s;
                    return fminf(fmaxf(A2, 0.0f), 1.0f);
                };
                const float2 r = make_float2(finish(a.x, acc[it][t].x, uint32_t(2 * n)),
                                             finish(a.y, acc[it][t].y, uint32_t(2 * n + 1)));
                *reinterpret_cast<float2*>(A_out + size_t(gy) * W + 2 * n) = r;
                if constexpr (CM) palette_pair(sw.cm, r, sw.rgba + size_t(gy) * W + 2 * n);
                za[it][t] = r;
            }
        }
        if constexpr (PIPE) base = (base + nk + 1) & 1;
        if (S_next == nullptr) {
            __syncthreads();  // sA read before it is staged into again
            continue;
        }
#pragma unroll
        for (int it = 0; it < K::ITL; ++it) {
            if (!ok[it]) continue;
            Dft<RC, false>::run(za[it]);
            store_run<RC>(bw + bi[it] * PITCH, jj[it] * RC, za[it]);
        }
        __syncthreads();
        float2* Y = mid_passes<PF, 1, PF::np - 1, false, RB, T, PITCH>(bw, sA, twf, rows);
        float2* Zo = (PF::np - 2) % 2 ? bw : sA;  // the other buffer (see the column pass)
        pass_gen<PF, PF::np - 1, false, RB, T>([&](int b, int i) { return Y[b * PITCH + i]; },
                                                [&](int b, int i, float2 v) { Zo[b * PITCH + i] = v; }, twf, rows);
        __syncthreads();
        r2c_store_rows<M, RB, T, PITCH>(Zo, twr, S_next, H, y0, rows);
        __syncthreads();
    }
    cp_async_wait_all();
}

// ------------------------------------------------------------- catalog

template <class P>
void plan_radices(FastPlan& out) {
    out.n = P::n;
    out.np = P::np;
    for (int i = 0; i < P::np; ++i) out.radix[i] = P::radix(i);
}

template <class PF, int B, int S = 1>
cudaError_t launch_col_t(const SpectralWorld& w0, const SpectralWorld* worlds, int n, int M,
                         const FastTables& t, cudaStream_t s) {
    using K = ColK<PF, B, S>;
    auto fn = col_fast_kernel<PF, B, S>;
    const size_t smem = ColStage<PF, B, S>::smem();
    if (smem > 227 * 1024 || K::T > 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
    return launch_chained(fn, world_grid(per, (M + B - 1) / B, n), K::T, smem, s, w0, worlds, t.col_twf, t.col_twi);
}

template <class PI, int RB, bool PIPE, bool CM, int S = 1>
cudaError_t launch_row_t(const SpectralWorld& w0, const SpectralWorld* worlds, int n, int H,
                         const float2* tw_r2c, const FastTables& t, cudaStream_t s) {
    using K = RowK<PI, RB, S>;
    auto fn = row_fast_kernel<PI, RB, PIPE, CM, S>;
    const size_t smem = K::smem(PIPE ? 3 : 2);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
    return launch_chained(fn, world_grid(per, (H + RB - 1) / RB, n), K::T, smem, s, w0, worlds, tw_r2c, t.row_twi,
                          t.row_twf);
}

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

bool fast_twiddle_tables(int H, int M, std::vector<float2> (&out)[4]) {
    FastPlan cf, ri;
    if (!fast_col_plan(H, cf) || !fast_row_plan(M, ri)) return false;
    FastPlan rcf = cf, rri = ri;
    for (int i = 0; i < cf.np; ++i) rcf.radix[i] = cf.radix[cf.np - 1 - i];
    for (int i = 0; i < ri.np; ++i) rri.radix[i] = ri.radix[ri.np - 1 - i];
    const FastPlan* plans[4] = {&cf, &rcf, &ri, &rri};
    for (int q = 0; q < 4; ++q) {
        fast_plan_twiddles(*plans[q], out[q]);
        if (out[q].empty()) out[q].push_back(make_float2(1.0f, 0.0f));
    }
    return true;
}

namespace {

cudaError_t col_dispatch(int H, int M, int batch, const SpectralWorld& w0, const SpectralWorld* worlds, int n,
                         const FastTables& t, cudaStream_t s) {
    switch (H) {
#define X(h, ...)                                                                                  \
    case h:                                                                                        \
        if (batch == (4 | kHalfThreads)) return launch_col_t<__VA_ARGS__, 4, 2>(w0, worlds, n, M, t, s); \
        if (batch == 8) return launch_col_t<__VA_ARGS__, 8>(w0, worlds, n, M, t, s);               \
        if (batch == 4) return launch_col_t<__VA_ARGS__, 4>(w0, worlds, n, M, t, s);               \
        return launch_col_t<__VA_ARGS__, 2>(w0, worlds, n, M, t, s);
        LENIA_COL_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

// CM: the variant that also writes the colour layer (w0.rgba); the other
// launches use the one compiled without that store, which would otherwise
// cost every row pass a few per cent.
template <bool CM>
cudaError_t row_dispatch_t(int H, int M, int batch, const SpectralWorld& w0, const SpectralWorld* worlds, int n,
                           const float2* tw_r2c, const FastTables& t, cudaStream_t s) {
    const int rb = batch & 7;
    const bool pipe = (batch & kRowPipelined) != 0;
    if (batch & kHalfThreads) return cudaErrorInvalidConfiguration;  // columns only
    switch (M) {
#define X(m, ...)                                                                                      \
    case m:                                                                                            \
        if (pipe) {                                                                                    \
            if (rb == 4) return launch_row_t<__VA_ARGS__, 4, true, CM>(w0, worlds, n, H, tw_r2c, t, s); \
            if (rb == 2) return launch_row_t<__VA_ARGS__, 2, true, CM>(w0, worlds, n, H, tw_r2c, t, s); \
            return launch_row_t<__VA_ARGS__, 1, true, CM>(w0, worlds, n, H, tw_r2c, t, s);              \
        }                                                                                              \
        if (rb == 4) return launch_row_t<__VA_ARGS__, 4, false, CM>(w0, worlds, n, H, tw_r2c, t, s);    \
        if (rb == 2) return launch_row_t<__VA_ARGS__, 2, false, CM>(w0, worlds, n, H, tw_r2c, t, s);    \
        return launch_row_t<__VA_ARGS__, 1, false, CM>(w0, worlds, n, H, tw_r2c, t, s);
        LENIA_ROW_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

cudaError_t row_dispatch(int H, int M, int batch, const SpectralWorld& w0, const SpectralWorld* worlds, int n,
                         const float2* tw_r2c, const FastTables& t, cudaStream_t s) {
    if (w0.rgba && !worlds) return row_dispatch_t<true>(H, M, batch, w0, worlds, n, tw_r2c, t, s);
    return row_dispatch_t<false>(H, M, batch, w0, worlds, n, tw_r2c, t, s);
}

template <class PF, int B, int S = 1>
bool col_shape_ok() {
    using K = ColK<PF, B, S>;
    return K::T <= 1024 && ColStage<PF, B, S>::smem() <= 227 * 1024;
}

template <class PI, int RB, bool PIPE, int S = 1>
bool row_shape_ok() {
    using K = RowK<PI, RB, S>;
    return K::T <= 1024 && K::smem(PIPE ? 3 : 2) <= 227 * 1024;
}

}  // namespace

bool fast_shapes_supported(int H, int M, int col_batch, int row_batch) {
    bool col = false, row = false;
    switch (H) {
#define X(h, ...)                                                        \
    case h:                                                              \
        col = col_batch == 8                    ? col_shape_ok<__VA_ARGS__, 8>()    \
              : col_batch == 4                  ? col_shape_ok<__VA_ARGS__, 4>()    \
              : col_batch == (4 | kHalfThreads) ? col_shape_ok<__VA_ARGS__, 4, 2>() \
              : col_batch == 2                  ? col_shape_ok<__VA_ARGS__, 2>() : false; \
        break;
        LENIA_COL_PLANS(X)
#undef X
    default: break;
    }
    const int rb = row_batch & 7;
    const bool pipe = (row_batch & kRowPipelined) != 0;
    if ((row_batch & ~(kRowPipelined | 7)) != 0) return false;
    switch (M) {
#define X(m, ...)                                                                                      \
    case m:                                                                                            \
        row = pipe ? (rb == 4   ? row_shape_ok<__VA_ARGS__, 4, true>()                                 \
                      : rb == 2 ? row_shape_ok<__VA_ARGS__, 2, true>()                                 \
                      : rb == 1 ? row_shape_ok<__VA_ARGS__, 1, true>() : false)                        \
                   : (rb == 4   ? row_shape_ok<__VA_ARGS__, 4, false>()                                \
                      : rb == 2 ? row_shape_ok<__VA_ARGS__, 2, false>()                                \
                      : rb == 1 ? row_shape_ok<__VA_ARGS__, 1, false>() : false);                      \
        break;
        LENIA_ROW_PLANS(X)
#undef X
    default: break;
    }
    return col && row;
}

cudaError_t launch_col_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* S,
                            float2* U, cudaStream_t s) {
    SpectralWorld w{};
    w.S = S;
    w.U = U;
    w.khat = g.khat;
    w.M = g.M;
    w.nk = g.nk;
    return col_dispatch(g.H, g.M, batch, w, nullptr, 1, t, s);
}

cudaError_t launch_row_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* U,
                            const float* A, float* A_out, float2* S_next, const StepParams& p,
                            int nk, cudaStream_t s, void* rgba16f, const ColorMapParams* cm) {
    SpectralWorld w{};
    if (rgba16f && cm && nk > 0) {
        w.rgba = static_cast<uint2*>(rgba16f);
        w.cm = *cm;
    }
    w.U = const_cast<float2*>(U);  // read only by the row pass
    w.A = A;
    w.A_out = A_out;
    w.S_next = S_next;
    w.M = g.M;
    w.nk = nk;
    w.p = p;
    w.p.height = uint32_t(g.H);
    return row_dispatch(g.H, g.M, batch, w, nullptr, 1, g.tw_r2c, t, s);
}

cudaError_t launch_col_fast_worlds(int H, int M, const FastTables& t, int batch, const SpectralWorld* worlds,
                                   int n, cudaStream_t s) {
    return col_dispatch(H, M, batch, SpectralWorld{}, worlds, n, t, s);
}

cudaError_t launch_row_fast_worlds(int H, int M, const FastTables& t, const float2* tw_r2c, int batch,
                                   const SpectralWorld* worlds, int n, cudaStream_t s) {
    return row_dispatch(H, M, batch, SpectralWorld{}, worlds, n, tw_r2c, t, s);
}

}  // namespace lenia
