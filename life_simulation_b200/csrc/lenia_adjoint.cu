// life_simulation_b200/csrc/lenia_adjoint.cu -- gradient of a Lenia rollout
// through the spectral path (lenia_adjoint_* in include/lenia_b200.h). The
// reference only steps forward; this is the step's exact derivative, run
// backwards over T steps with checkpoints.
//
// One forward step (Lenia.metal:188-231, no noise/jitter/injection):
//   U_k = K_k (*) A_t,  pre = A_t + dt * sum_k h_k (2 bell_k(U_k) - 1)
//   (mode 1: A_t + dt (sum_k h_k bell_k / sum h - A_t)),  A_{t+1} = clamp(pre).
// Its adjoint, given dL/dA_{t+1}:
//   g    = dL/dpre   = dL/dA_{t+1} where 0 < A_{t+1} < 1, else 0
//   q_k  = g dpre/dU_k,  dpre/dU_k = dt h_k 2 bell_k (mu_k - U_k) / sigma_k^2
//   dL/dA_t = ca g + sum_k K_k (*) q_k         (K_k even: adjoint = same conv)
//   dL/dmu_k += -sum q_k,  dL/dsigma_k += sum q_k (mu_k - U_k) / sigma_k,
//   dL/dh_k += sum g dt (2 bell_k - 1),  dL/ddt += sum g sum_k h_k (2 bell_k - 1)
//   dL/dbeta_i += sum_x q_k (E_i - c_i U_k) = sum_w d_i(w) Re(conj Q_k(w) A(w))
// with E_i the potential of ring i alone (normalised by the kernel's total),
// c_i its share of the normalisation, and d_i = (E^_i - c_i K^_k) / (W H) a
// real even table: the ring sums come from the spectra the passes already
// hold (Parseval), with no extra convolutions.
//
// Per backward step, two launches mirror the forward's two:
//   row pass: inverse row FFT of the previous column pass's output -> dL/dA_{t+1};
//     clip mask -> g; the potentials U_k of step t (kept as planes by the
//     forward row pass) -> q_k and the parameter sums; forward row FFTs of q_k.
//   column pass: column FFTs of q_k, sum_k K^_k Q_k (and the beta sums against
//     the column FFT of A_t's row spectrum), one inverse column FFT.
// The forward keeps the potentials, row spectra and fields of the current
// segment of `checkpoint_every` steps and A at every checkpoint; the
// backward recomputes each earlier segment from its checkpoint with the
// forward kernels (bit-identical), then runs the segment's adjoint steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lenia_b200.h"
#include "abi_guard.h"
#include "fft_fast_common.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"
#include "lenia_module.h"

namespace lenia {

constexpr int kPerKernel = LENIA_ADJOINT_PARAMS_PER_KERNEL;
constexpr int kSlotDt = kMaxKernels * kPerKernel;  // 44
constexpr int kSlotMode1 = kSlotDt + 1;            // mode 1: sum g dt G / sum h
constexpr int kAcc = kSlotMode1 + 1;
constexpr int kMaxTables = kMaxKernels * kMaxBetas;
static_assert(kSlotDt == LENIA_ADJOINT_NUM_PARAMS - 1, "gradient layout");

// One world of an adjoint row launch (blockIdx.y = world).
struct AdjRowWorld {
    const float2* SG;     // convolution part of dL/dA_{t+1} (row spectra), or null
    const float* g_in;    // with SG: dL/dpre_{t+1}; without: dL/dA_{t+1}
    const float* A_next;  // A_{t+1}: clip mask of step t
    const float* A_cur;   // A_t (growth mode 1's dt term)
    const float* U;       // nk potential planes (H x W) of step t; null: only write dL/dA_{t+1}
    float* g_out;         // dL/dpre_t
    float2* SQ;           // nk row spectra of q_k
    float* gA_out;        // dL/dA_{t+1} when U is null
};
struct AdjRowArgs {
    StepParams p;
    double* acc;  // kAcc accumulators
    float ca;     // dpre/dA_t
    int nk;
};
// One world of an adjoint column launch.
struct AdjColWorld {
    const float2* SQ;  // nk row spectra of q_k
    float2* SG;        // out: sum_k K^_k Q_k after the inverse column FFT
    const float2* S;   // row spectrum of A_t (beta sums), or null
};
struct AdjColArgs {
    const float* khat;  // nk x (M+1) x (H/2+1), / (W H)
    const float* dtab;  // ntab x (M+1) x (H/2+1) ring tables d_i
    double* acc;
    int nk, ntab, M;
    int tab_kernel[kMaxTables];  // kernel of table i
    int tab_slot[kMaxTables];    // accumulator slot of table i
};

namespace {

using fft::cadd;
using fft::cconj;
using fft::cscale;
using fft::csub;
using namespace fftct;
using namespace fastfft;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Adds every thread's v into a shared FP64 accumulator, one atomic per warp.
// All threads of the block call it. The per-thread partial sums are FP64 as
// well: which pixels a thread sums depends on the tuned rows or columns per
// CTA, so only FP64 keeps the parameter gradients independent of the tuning
// (up to the order of FP64 additions).
__device__ __forceinline__ void block_add(double* red, double v) {
    v = warp_sum(v);
    if ((threadIdx.x & 31u) == 0u) atomicAdd(red, double(v));
}

// ------------------------------------------------------------------- rows

template <class PI, int RB>
__global__ void __launch_bounds__(RowK<PI, RB>::T, (512 / RowK<PI, RB>::T > 1 ? 512 / RowK<PI, RB>::T : 1))
    row_adj_kernel(const AdjRowWorld* __restrict__ worlds, AdjRowArgs a, const float2* __restrict__ twr_g,
                   const float2* __restrict__ twi_g, const float2* __restrict__ twf_g) {
    using K = RowK<PI, RB>;
    using PF = typename K::PF;
    using IL = PassIdx<PI, PI::np - 1>;
    constexpr int M = K::M, W = 2 * M, T = K::T, PITCH = K::PITCH, RC = K::RC, NRC = K::NRC, ITL = K::ITL;
    extern __shared__ __align__(16) float2 sm[];
    __shared__ AdjRowWorld sw;
    __shared__ double red[kAcc];
    if (threadIdx.x == 0) sw = worlds[blockIdx.y];
    for (int i = threadIdx.x; i < kAcc; i += T) red[i] = 0.0;
    float2* twr = sm;
    float2* twi = twr + (M + 1);
    float2* twf = twi + PI::tw_size();
    float2* ba = sm + K::BUF0;
    float2* bb = ba + RB * PITCH;
    copy_table(twr, twr_g, M + 1);
    copy_table(twi, twi_g, PI::tw_size());
    copy_table(twf, twf_g, PF::tw_size());
    __syncthreads();
    const StepParams& p = a.p;
    const int H = int(p.height), nk = a.nk;
    const bool asym = p.growth_mode == 1u;
    const bool sw_ok = p.sum_weights > 1e-6f;
    const float inv_sw = sw_ok ? 1.0f / p.sum_weights : 0.0f;
    const float dt = p.dt, ca = a.ca;
    const bool has_q = sw.U != nullptr;
    double pdt = 0.0, pcommon = 0.0;
    for (int y0 = blockIdx.x * RB; y0 < H; y0 += gridDim.x * RB) {
        const int rows = min(RB, H - y0);
        int jj[ITL], bi[ITL];
        bool ok[ITL];
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            jj[it] = q / RB;
            bi[it] = q - jj[it] * RB;
            ok[it] = q < RB * NRC && bi[it] < rows;
        }
        const auto gidx = [&](int it, int t) { return size_t(y0 + bi[it]) * W + 2 * (jj[it] + t * NRC); };
        // The potentials of step t (kept by the recomputation's row pass) at
        // this thread's pixel pairs, one kernel ahead: kernel 0's are in
        // flight during the inverse row transform below, kernel k+1's during
        // kernel k's forward transform.
        float2 zn[ITL][RC];
        const auto fetch_u = [&](int kk) {
            const float* Uk = sw.U + size_t(kk) * H * W;
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
#pragma unroll
                for (int t = 0; t < RC; ++t) zn[it][t] = __ldg(reinterpret_cast<const float2*>(Uk + gidx(it, t)));
            }
        };
        if (has_q && nk > 0) fetch_u(0);
        // dL/dA_{t+1} at this thread's pixel pairs (2n, 2n+1), n = j + t*NRC.
        float2 gv[ITL][RC];
        if (sw.SG) {
            stage_rows<M, RB, T, PITCH>(ba, sw.SG, H, y0, rows);
            cp_async_wait_all();
            __syncthreads();
            pass_gen<PI, 0, true, RB, T>([&](int b, int i) { return c2r_split<M>(ba + b * PITCH, twr, i); },
                                         [&](int b, int i, float2 v) { bb[b * PITCH + i] = v; }, twi, rows);
            __syncthreads();
            float2* X = mid_passes<PI, 1, PI::np - 1, true, RB, T, PITCH>(bb, ba, twi, rows);
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
                float2 z[RC];
#pragma unroll
                for (int t = 0; t < RC; ++t) z[t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
                IL::template twiddle<true>(z, jj[it], twi);
                Dft<RC, true>::run(z);
#pragma unroll
                for (int t = 0; t < RC; ++t) {
                    const float2 gi = __ldg(reinterpret_cast<const float2*>(sw.g_in + gidx(it, t)));
                    gv[it][t] = make_float2(fmaf(ca, gi.x, z[t].x), fmaf(ca, gi.y, z[t].y));
                }
            }
            __syncthreads();  // X read; the buffers are free again
        } else {
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
#pragma unroll
                for (int t = 0; t < RC; ++t)
                    gv[it][t] = __ldg(reinterpret_cast<const float2*>(sw.g_in + gidx(it, t)));
            }
        }
        if (!has_q) {
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
#pragma unroll
                for (int t = 0; t < RC; ++t) *reinterpret_cast<float2*>(sw.gA_out + gidx(it, t)) = gv[it][t];
            }
            continue;
        }
        // Clip mask of step t: A_{t+1} strictly inside (0, 1) <=> pre was.
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            if (!ok[it]) continue;
#pragma unroll
            for (int t = 0; t < RC; ++t) {
                const float2 an = __ldg(reinterpret_cast<const float2*>(sw.A_next + gidx(it, t)));
                gv[it][t].x = (an.x > 0.0f && an.x < 1.0f) ? gv[it][t].x : 0.0f;
                gv[it][t].y = (an.y > 0.0f && an.y < 1.0f) ? gv[it][t].y : 0.0f;
                *reinterpret_cast<float2*>(sw.g_out + gidx(it, t)) = gv[it][t];
            }
        }
        // The dt and mode-1 terms are linear in the kernels' contributions,
        // so they are summed kernel by kernel (no per-pixel accumulator).
        for (int kk = 0; kk < nk; ++kk) {
            const auto pick = [&](const float(&v)[kMaxKernels]) {
                return kk == 0 ? v[0] : kk == 1 ? v[1] : kk == 2 ? v[2] : v[3];
            };
            const float mu = pick(p.mu), inv_sigma = 1.0f / pick(p.sigma), hw = pick(p.weight);
            const float coef = asym ? (sw_ok ? dt * hw * inv_sw : 0.0f) : 2.0f * dt * hw;
            double pmu = 0.0, psig = 0.0, ph = 0.0;
            float2 zq[ITL][RC];
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
                float2 z[RC];
#pragma unroll
                for (int t = 0; t < RC; ++t) z[t] = zn[it][t];
#pragma unroll
                for (int t = 0; t < RC; ++t) {
                    float qv[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const float u = e ? z[t].y : z[t].x;
                        const float g = e ? gv[it][t].y : gv[it][t].x;
                        const float b = bell_fast(u, mu, inv_sigma);
                        const float dmu = (mu - u) * inv_sigma;
                        const float q = g * coef * b * dmu * inv_sigma;
                        pmu -= q;
                        psig += q * dmu;
                        if (asym) {
                            // dpre/dh_k = dt (b_k - G) / sum h; dpre/ddt = G - A_t.
                            const float gb = sw_ok ? g * hw * b * inv_sw : 0.0f;
                            ph += sw_ok ? g * dt * b * inv_sw : 0.0f;
                            pdt += gb;
                            pcommon += dt * inv_sw * gb;
                        } else {
                            ph += g * dt * (2.0f * b - 1.0f);
                            pdt += g * hw * (2.0f * b - 1.0f);
                        }
                        qv[e] = q;
                    }
                    zq[it][t] = make_float2(qv[0], qv[1]);
                }
            }
            if (kk + 1 < nk) fetch_u(kk + 1);
            block_add(&red[kk * kPerKernel + 0], pmu);
            block_add(&red[kk * kPerKernel + 1], psig);
            block_add(&red[kk * kPerKernel + 2], ph);
            // (The shared buffers are free: the last reader of them was
            // followed by a barrier.) Forward row transform of q_k: first pass (radix RC) from registers.
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
                Dft<RC, false>::run(zq[it]);
#pragma unroll
                for (int t = 0; t < RC; ++t) ba[bi[it] * PITCH + jj[it] * RC + t] = zq[it][t];
            }
            __syncthreads();
            float2* Y = mid_passes<PF, 1, PF::np - 1, false, RB, T, PITCH>(ba, bb, twf, rows);
            float2* Zo = (PF::np - 2) % 2 ? ba : bb;  // the other buffer, chosen at compile time (shared accesses)
            pass_gen<PF, PF::np - 1, false, RB, T>([&](int b, int i) { return Y[b * PITCH + i]; },
                                                    [&](int b, int i, float2 v) { Zo[b * PITCH + i] = v; }, twf,
                                                    rows);
            __syncthreads();
            r2c_store_rows<M, RB, T, PITCH>(Zo, twr, sw.SQ + size_t(kk) * M * H, H, y0, rows);
            __syncthreads();
        }
        // Mode 1's dt term: the -A_t part.
        if (asym && sw_ok) {
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
#pragma unroll
                for (int t = 0; t < RC; ++t) {
                    const float2 ac = __ldg(reinterpret_cast<const float2*>(sw.A_cur + gidx(it, t)));
                    pdt -= gv[it][t].x * ac.x + gv[it][t].y * ac.y;
                }
            }
        }
    }
    block_add(&red[kSlotDt], pdt);
    block_add(&red[kSlotMode1], pcommon);
    __syncthreads();
    for (int i = threadIdx.x; i < kAcc; i += T)
        if (red[i] != 0.0) atomicAdd(a.acc + i, red[i]);
}

// ---------------------------------------------------------------- columns

// Forward column FFT of B columns of a blocked-layout plane (group base
// gbase) up to the last pass, which the caller runs into registers; returns
// the buffer holding the last pass's input.
template <class PF, int B, int T, int PITCH>
__device__ __forceinline__ float2* col_forward(const float2* __restrict__ src, float2* ba, float2* bb,
                                               const float2* twf, int cols) {
    pass_gen<PF, 0, false, B, T>([&](int b, int i) { return __ldg(src + size_t(i) * KB + b); },
                                  [&](int b, int i, float2 v) { ba[b * PITCH + i] = v; }, twf, cols);
    __syncthreads();
    return mid_passes<PF, 1, PF::np - 1, false, B, T, PITCH>(ba, bb, twf, cols);
}

template <class PF, int B>
struct ColAdjK {
    using K = ColK<PF, B>;
    // ColK's buffers (twiddles, two work buffers, one packed column) plus a
    // second packed column (A's), then (when B is even and it fits) a staging
    // buffer of B columns x H rows for the next first-pass input.
    static constexpr int OFF =
        (PF::tw_size() + K::PI::tw_size() + 2 * B * K::PITCH + 2 * K::H + 1) / 2 * 2;  // 16-byte aligned
    static constexpr size_t with_stage = sizeof(float2) * (size_t(OFF) + size_t(B) * K::H);
    static constexpr bool stage = B % 2 == 0 && with_stage <= 227 * 1024;
    static constexpr size_t smem() {
        return stage ? with_stage : K::smem() + sizeof(float2) * size_t(K::H);
    }
};

template <class PF, int B>
__global__ void __launch_bounds__(ColK<PF, B>::T)
    col_adj_kernel(const AdjColWorld* __restrict__ worlds, AdjColArgs a, const float2* __restrict__ twf_g,
                   const float2* __restrict__ twi_g) {
    using K = ColK<PF, B>;
    using PI = typename K::PI;
    using IL = PassIdx<PF, PF::np - 1>;
    constexpr int H = K::H, T = K::T, PITCH = K::PITCH, RL = K::RL, NRL = K::NRL, Hh = K::Hh, ITL = K::ITL;
    extern __shared__ __align__(16) float2 sm[];
    __shared__ AdjColWorld sw;
    __shared__ double red[kMaxTables];
    if (threadIdx.x == 0) sw = worlds[blockIdx.y];
    for (int i = threadIdx.x; i < kMaxTables; i += T) red[i] = 0.0;
    float2* twf = sm;
    float2* twi = twf + PF::tw_size();
    float2* ba = twi + PI::tw_size();
    float2* bb = ba + B * PITCH;
    float2* c0q = bb + B * PITCH;  // packed column 0 of Q_k (DC + i Nyquist)
    float2* c0a = c0q + H;         // packed column 0 of A^
    copy_table(twf, twf_g, PF::tw_size());
    copy_table(twi, twi_g, PI::tw_size());
    __syncthreads();
    const int M = a.M, nk = a.nk;
    const bool beta = a.ntab > 0 && sw.S != nullptr;
    // First-pass inputs of a column group, in order: A_t's row spectrum
    // (with beta), then SQ_0 .. SQ_{nk-1}. With staging, input j + 1 (or the
    // next group's first) is copied into bs by cp.async while input j is
    // transformed.
    using CAK = ColAdjK<PF, B>;
    float2* bs = sm + CAK::OFF;
    const int nin = nk + (beta ? 1 : 0);
    const auto input_plane = [&](int j) -> const float2* {
        return beta ? (j == 0 ? sw.S : sw.SQ + size_t(j - 1) * M * H) : sw.SQ + size_t(j) * M * H;
    };
    const auto stage_input = [&](int g0, int j) {
        const float2* src = input_plane(j) + size_t(g0 / KB) * H * KB + (g0 % KB);
        for (int q = threadIdx.x; q < H * (B / 2); q += T) {
            const int i = q / (B / 2), c2 = q - i * (B / 2);
            cp_async16(bs + i * B + 2 * c2, src + size_t(i) * KB + 2 * c2);
        }
        cp_async_commit();
    };
    // Forward column FFT of the group's input j up to its last pass (which
    // the caller runs into registers); returns the buffer holding the last
    // pass's input.
    const auto forward_input = [&](int k0, int j, int cols) -> float2* {
        if constexpr (CAK::stage) {
            cp_async_wait_all();
            __syncthreads();  // input j staged
            pass_gen<PF, 0, false, B, T>([&](int b, int i) { return bs[i * B + b]; },
                                          [&](int b, int i, float2 v) { ba[b * PITCH + i] = v; }, twf, cols);
            __syncthreads();  // bs read
            if (j + 1 < nin)
                stage_input(k0, j + 1);
            else if (k0 + int(gridDim.x) * B < M)
                stage_input(k0 + int(gridDim.x) * B, 0);
            return mid_passes<PF, 1, PF::np - 1, false, B, T, PITCH>(ba, bb, twf, cols);
        } else {
            return col_forward<PF, B, T, PITCH>(input_plane(j) + size_t(k0 / KB) * H * KB + (k0 % KB), ba, bb, twf,
                                                cols);
        }
    };
    if constexpr (CAK::stage) {
        if (int(blockIdx.x) * B < M && nin > 0) stage_input(int(blockIdx.x) * B, 0);
    }
    for (int k0 = blockIdx.x * B; k0 < M; k0 += gridDim.x * B) {
        const int cols = min(B, M - k0);
        const size_t gbase = size_t(k0 / KB) * H * KB + (k0 % KB);
        int jj[ITL], bi[ITL];
        bool ok[ITL];
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            const int q = int(threadIdx.x) + it * T;
            jj[it] = q / B;
            bi[it] = q - jj[it] * B;
            ok[it] = q < B * NRL && bi[it] < cols;
        }
        // Kernel spectrum values of this thread's elements, one kernel
        // ahead (last passes of radix <= 8 only, as in the forward pass).
        constexpr bool kAhead = RL <= 8;
        float kv[ITL][kAhead ? RL : 1], kv2[ITL][kAhead ? RL : 1];  // kv2: Nyquist column (packed column 0)
        const auto fetch_k = [&](int kk) {
            if constexpr (kAhead) {
                const float* kh = a.khat + size_t(kk) * (M + 1) * Hh;
#pragma unroll
                for (int it = 0; it < ITL; ++it) {
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
        // Last forward pass of a column FFT into registers (+ packed column).
        const auto last_pass = [&](const float2* X, float2 (&C)[ITL][RL], float2* c0) {
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
#pragma unroll
                for (int t = 0; t < RL; ++t) C[it][t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
                IL::template twiddle<false>(C[it], jj[it], twf);
                Dft<RL, false>::run(C[it]);
                if (k0 == 0 && bi[it] == 0) {
#pragma unroll
                    for (int t = 0; t < RL; ++t) c0[jj[it] + t * NRL] = C[it][t];
                }
            }
        };
        float2 Ah[ITL][RL];
        if (beta) {
            float2* X = forward_input(k0, 0, cols);
            last_pass(X, Ah, c0a);
            __syncthreads();  // X read
        }
        float2 G[ITL][RL];
        for (int kk = 0; kk < nk; ++kk) {
            float2 Q[ITL][RL];
            float2* X = forward_input(k0, kk + (beta ? 1 : 0), cols);
            last_pass(X, Q, c0q);
            __syncthreads();  // X read; packed columns visible
#pragma unroll
            for (int it = 0; it < ITL; ++it) {
                if (!ok[it]) continue;
                const int kx = k0 + bi[it];
                const float* kh = a.khat + size_t(kk) * (M + 1) * Hh;
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
                    float2 D;
                    if (kx == 0) {
                        const float P = kval, Qn = knyq;
                        const float2 Cm = cconj(c0q[ky == 0 ? 0 : H - ky]);
                        D = cadd(cscale(Q[it][t], 0.5f * (P + Qn)), cscale(Cm, 0.5f * (P - Qn)));
                    } else {
                        D = cscale(Q[it][t], kval);
                    }
                    G[it][t] = kk == 0 ? D : cadd(G[it][t], D);
                }
            }
            if (kk + 1 < nk) fetch_k(kk + 1);
            if (beta) {
                for (int tb = 0; tb < a.ntab; ++tb) {
                    if (a.tab_kernel[tb] != kk) continue;
                    const float* dtb = a.dtab + size_t(tb) * (M + 1) * Hh;
                    double part = 0.0;
#pragma unroll
                    for (int it = 0; it < ITL; ++it) {
                        if (!ok[it]) continue;
                        const int kx = k0 + bi[it];
#pragma unroll
                        for (int t = 0; t < RL; ++t) {
                            const int ky = jj[it] + t * NRL;
                            const int kyr = min(ky, H - ky);
                            const float2 q = Q[it][t], ah = Ah[it][t];
                            if (kx != 0) {
                                part += 2.0f * __ldg(dtb + size_t(kx) * Hh + kyr) * (q.x * ah.x + q.y * ah.y);
                            } else {
                                // Unpack DC (x) and Nyquist (y) columns:
                                // X0 = (C + conj C-)/2, XN = (C - conj C-)/2i.
                                const int km = ky == 0 ? 0 : H - ky;
                                const float2 qm = cconj(c0q[km]), am = cconj(c0a[km]);
                                const float2 sq = cadd(q, qm), sa = cadd(ah, am);
                                const float2 dq = csub(q, qm), da = csub(ah, am);
                                part += 0.25f * (__ldg(dtb + kyr) * (sq.x * sa.x + sq.y * sa.y) +
                                                 __ldg(dtb + size_t(M) * Hh + kyr) * (dq.x * da.x + dq.y * da.y));
                            }
                        }
                    }
                    block_add(&red[tb], part);
                }
            }
            __syncthreads();  // packed column read before the next kernel's
        }
        // Inverse column FFT of G: first pass (radix RL) from registers.
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            if (!ok[it]) continue;
            Dft<RL, true>::run(G[it]);
#pragma unroll
            for (int t = 0; t < RL; ++t) ba[bi[it] * PITCH + jj[it] * RL + t] = G[it][t];
        }
        __syncthreads();
        float2* Z = mid_passes<PI, 1, PI::np - 1, true, B, T, PITCH>(ba, bb, twi, cols);
        float2* dst = sw.SG + gbase;
        pass_gen<PI, PI::np - 1, true, B, T>([&](int b, int i) { return Z[b * PITCH + i]; },
                                              [&](int b, int i, float2 v) { dst[size_t(i) * KB + b] = v; }, twi,
                                              cols);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < a.ntab; i += T)
        if (red[i] != 0.0) atomicAdd(a.acc + a.tab_slot[i], red[i]);
}

// Final parameter gradients: mode 1's weight gradients lose the common term.
__global__ void finalize_kernel(const double* __restrict__ acc, double* __restrict__ out, int nk, int mode1) {
    const int i = threadIdx.x;
    if (i >= LENIA_ADJOINT_NUM_PARAMS) return;
    double v = acc[i];
    if (mode1 && i < nk * kPerKernel && i % kPerKernel == 2) v -= acc[kSlotMode1];
    out[i] = v;
}

// ---------------------------------------------------------------- dispatch

template <class PF, int B>
cudaError_t launch_col_adj_t(const AdjColWorld* worlds, int n, const AdjColArgs& args, const FastTables& t,
                             cudaStream_t s) {
    using K = ColK<PF, B>;
    if constexpr (K::T > 1024) {
        return cudaErrorInvalidConfiguration;
    } else {
        auto fn = col_adj_kernel<PF, B>;
        const size_t smem = ColAdjK<PF, B>::smem();
        if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
        cudaError_t e = prepare(fn, smem);
        if (e != cudaSuccess) return e;
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
        fn<<<world_grid(per, (args.M + B - 1) / B, n), K::T, smem, s>>>(worlds, args, t.col_twf, t.col_twi);
        return cudaGetLastError();
    }
}

template <class PI, int RB>
cudaError_t launch_row_adj_t(const AdjRowWorld* worlds, int n, const AdjRowArgs& args, const float2* tw_r2c,
                             const FastTables& t, cudaStream_t s) {
    using K = RowK<PI, RB>;
    if constexpr (K::T > 1024) {
        return cudaErrorInvalidConfiguration;
    } else {
        auto fn = row_adj_kernel<PI, RB>;
        const size_t smem = K::smem();
        if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
        cudaError_t e = prepare(fn, smem);
        if (e != cudaSuccess) return e;
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, K::T, smem);
        const int H = int(args.p.height);
        fn<<<world_grid(per, (H + RB - 1) / RB, n), K::T, smem, s>>>(worlds, args, tw_r2c, t.row_twi, t.row_twf);
        return cudaGetLastError();
    }
}

// batch: columns per CTA iteration (2, 4, 8); rows per CTA iteration (1, 2,
// 4, 8). Candidates that do not fit a CTA return cudaErrorInvalidConfiguration.
cudaError_t launch_col_adj(int H, int batch, const AdjColWorld* worlds, int n, const AdjColArgs& args,
                           const FastTables& t, cudaStream_t s) {
    switch (H) {
#define X(h, ...)                                                                         \
    case h:                                                                               \
        if (batch == 8) return launch_col_adj_t<__VA_ARGS__, 8>(worlds, n, args, t, s);   \
        if (batch == 4) return launch_col_adj_t<__VA_ARGS__, 4>(worlds, n, args, t, s);   \
        return launch_col_adj_t<__VA_ARGS__, 2>(worlds, n, args, t, s);
        LENIA_COL_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

cudaError_t launch_row_adj(int M, int batch, const AdjRowWorld* worlds, int n, const AdjRowArgs& args,
                           const float2* tw_r2c, const FastTables& t, cudaStream_t s) {
    switch (M) {
#define X(m, ...)                                                                                 \
    case m:                                                                                       \
        if (batch == 8) return launch_row_adj_t<__VA_ARGS__, 8>(worlds, n, args, tw_r2c, t, s);   \
        if (batch == 4) return launch_row_adj_t<__VA_ARGS__, 4>(worlds, n, args, tw_r2c, t, s);   \
        if (batch == 2) return launch_row_adj_t<__VA_ARGS__, 2>(worlds, n, args, tw_r2c, t, s);   \
        return launch_row_adj_t<__VA_ARGS__, 1>(worlds, n, args, tw_r2c, t, s);
        LENIA_ROW_PLANS(X)
#undef X
    default: return cudaErrorNotSupported;
    }
}

}  // namespace
}  // namespace lenia

// ================================================================== context

struct lenia_adjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string message;
    lenia_adjoint_config cfg{};
    int W = 0, H = 0, M = 0, Hh = 0, nb = 0, nk = 0, T = 0, C = 0, nck = 0;
    size_t P = 0, SPX = 0;
    uint64_t bytes = 0, launches = 0;
    std::vector<void*> allocs;
    // Buffers (all worlds of a slot contiguous).
    float* ckpt = nullptr;   // nck x nb x P: A_{jC} (last slot: A_T)
    float* seg = nullptr;    // C x nb x P: A_{s+i} inside a segment (i >= 1)
    float2* Sring = nullptr; // (C+1) x nb x SPX: row spectra of A_t
    float2* Uspec = nullptr; // nb x nk x SPX: potential spectra (column -> row pass scratch)
    float* Upx = nullptr;    // C x nb x nk x P: potentials of step t (kept by the row pass)
    float2* SQ = nullptr;    // nb x nk x SPX
    float2* SG = nullptr;    // nb x SPX
    float* g[2] = {nullptr, nullptr};  // nb x P: dL/dpre
    float* gio = nullptr;    // nb x P: dL/dA_T in, dL/dA_0 out
    double* acc = nullptr;
    float* khat = nullptr;
    float* dtab = nullptr;
    float2* tw_r2c = nullptr;
    float2* tw[4] = {nullptr, nullptr, nullptr, nullptr};
    lenia::FastTables ft{};
    // Launch tables.
    lenia::SpectralWorld* d_r2c = nullptr;   // (nck-1) x nb
    lenia::SpectralWorld* d_fcol = nullptr;  // T x nb
    lenia::SpectralWorld* d_frow = nullptr;  // T x nb, recomputation (keeps every step's potentials)
    lenia::SpectralWorld* d_ffwd = nullptr;  // T x nb, forward (keeps the last segment's potentials)
    lenia::AdjRowWorld* d_arow = nullptr;    // (T+1) x nb
    lenia::AdjColWorld* d_acol = nullptr;    // T x nb
    lenia::AdjRowArgs rargs{};
    lenia::AdjColArgs cargs{};
    lenia::StepParams params{};
    int col_batch = 4, row_batch = 2;          // forward passes (autotuned)
    int adj_col_batch = 4, adj_row_batch = 2;  // adjoint passes (autotuned)
    bool forward_done = false, last_segment_fresh = false;

    template <typename Tp>
    cudaError_t alloc(Tp** p, size_t count) {
        const size_t nbytes = std::max<size_t>(count, 1) * sizeof(Tp);
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), nbytes);
        if (e == cudaSuccess) {
            allocs.push_back(*p);
            bytes += nbytes;
        }
        return e;
    }
    ~lenia_adjoint() {
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    int fail(int code, std::string m) {
        message = std::move(m);
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        message = std::string(what) + ": " + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    float* slot(int t, int b) const {
        if (t == T) return ckpt + (size_t(nck - 1) * nb + b) * P;
        if (t % C == 0) return ckpt + (size_t(t / C) * nb + b) * P;
        return seg + (size_t(t % C) * nb + b) * P;
    }
    float2* S_of(int t, int b) const { return Sring + (size_t(t % (C + 1)) * nb + b) * SPX; }
    float2* Uspec_of(int b) const { return Uspec + size_t(b) * nk * SPX; }
    float* U_of(int t, int b) const { return Upx + (size_t(t % C) * nb + b) * nk * P; }

    int set_kernels(const lenia_kernel_def* kd, uint32_t n, float dt_new);
    int build_tables();
};

namespace {

int check_kernels(const lenia_kernel_def* kd, uint32_t n, std::string& why) {
    if (n < 1 || n > uint32_t(lenia::kMaxKernels)) {
        why = "num_kernels must be 1..4";
        return LENIA_ERR_INVALID_ARG;
    }
    for (uint32_t k = 0; k < n; ++k) {
        const lenia_kernel_def& d = kd[k];
        if (d.num_betas < 1 || d.num_betas > uint32_t(lenia::kMaxBetas)) {
            why = "num_betas must be 1..8";
            return LENIA_ERR_INVALID_ARG;
        }
        if (!(d.sigma > 0.0f) || !(d.radius_scale > 0.0f) || !std::isfinite(d.mu) || !std::isfinite(d.weight)) {
            why = "kernel sigma and radius_scale must be positive, mu and weight finite";
            return LENIA_ERR_INVALID_ARG;
        }
        double z = 0.0;
        for (uint32_t i = 0; i < d.num_betas; ++i) z += d.betas[i];
        if (!(z > 0.0)) {
            why = "the betas of a kernel must have a positive sum";
            return LENIA_ERR_INVALID_ARG;
        }
    }
    return LENIA_OK;
}

}  // namespace

// Kernel spectra and ring tables (FP64, rounded once), and the step
// parameters, for new kernel values.
int lenia_adjoint::set_kernels(const lenia_kernel_def* kd, uint32_t n, float dt_new) {
    using namespace lenia;
    const size_t tab = size_t(M + 1) * Hh;
    const double inv_n = 1.0 / (double(W) * double(H));
    std::vector<float> kh(tab * nk, 0.0f), dt_tabs;
    AdjColArgs ca{};
    ca.nk = nk;
    ca.M = M;
    for (int k = 0; k < nk; ++k) {
        const lenia_kernel_def& d = kd[k];
        std::vector<std::vector<double>> rings;
        ring_shells_f64(uint32_t(W), uint32_t(H), double(cfg.radius) * double(d.radius_scale), double(cfg.shell_sigma),
                        d.num_betas, cfg.kernel_core, rings);
        std::vector<double> sums(d.num_betas, 0.0);
        double z = 0.0;
        for (uint32_t i = 0; i < d.num_betas; ++i) {
            for (double v : rings[i]) sums[i] += v;
            z += double(d.betas[i]) * sums[i];
        }
        if (!(z > 0.0)) return fail(LENIA_ERR_INVALID_ARG, "kernel " + std::to_string(k) + " has no taps");
        std::vector<std::vector<double>> ehat(d.num_betas);
        std::vector<double> khat_k(tab, 0.0);
        for (uint32_t i = 0; i < d.num_betas; ++i) {
            even_spectrum_f64(rings[i], uint32_t(W), uint32_t(H), ehat[i]);
            for (size_t j = 0; j < tab; ++j) {
                ehat[i][j] /= z;
                khat_k[j] += double(d.betas[i]) * ehat[i][j];
            }
        }
        for (size_t j = 0; j < tab; ++j) kh[size_t(k) * tab + j] = float(khat_k[j] * inv_n);
        if (d.num_betas > 1) {
            for (uint32_t i = 0; i < d.num_betas; ++i) {
                const double c = sums[i] / z;
                const size_t base = dt_tabs.size();
                dt_tabs.resize(base + tab);
                for (size_t j = 0; j < tab; ++j) dt_tabs[base + j] = float((ehat[i][j] - c * khat_k[j]) * inv_n);
                ca.tab_kernel[ca.ntab] = k;
                ca.tab_slot[ca.ntab] = k * kPerKernel + 3 + int(i);
                ++ca.ntab;
            }
        }
    }
    cudaError_t e;
    if ((e = cudaMemcpy(khat, kh.data(), kh.size() * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "copy kernel spectra");
    if (ca.ntab > 0 &&
        (e = cudaMemcpy(dtab, dt_tabs.data(), dt_tabs.size() * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "copy ring tables");
    ca.khat = khat;
    ca.dtab = dtab;
    ca.acc = acc;
    cargs = ca;

    StepParams p{};
    p.dt = dt_new;
    float sw = 0.0f;
    for (int k = 0; k < nk; ++k) {
        p.mu[k] = kd[k].mu;
        p.sigma[k] = kd[k].sigma;
        p.weight[k] = kd[k].weight;
        sw += kd[k].weight;
    }
    for (int k = nk; k < kMaxKernels; ++k) p.sigma[k] = 1.0f;
    p.sum_weights = sw;
    p.num_kernels = uint32_t(nk);
    p.growth_mode = cfg.growth_mode;
    p.radius = cfg.radius;
    p.width = uint32_t(W);
    p.height = uint32_t(H);
    params = p;
    rargs.p = p;
    rargs.acc = acc;
    rargs.nk = nk;
    rargs.ca = (cfg.growth_mode == 1u && sw > 1e-6f) ? 1.0f - dt_new : 1.0f;
    for (int k = 0; k < nk; ++k) cfg.kernels[k] = kd[k];
    cfg.dt = dt_new;
    forward_done = false;
    last_segment_fresh = false;
    return build_tables();
}

// Every launch's world table (pointers per step and world).
int lenia_adjoint::build_tables() {
    using namespace lenia;
    std::vector<SpectralWorld> r2c(size_t(nck - 1) * nb), fcol(size_t(T) * nb), frow(size_t(T) * nb),
        ffwd(size_t(T) * nb);
    const int last_segment = (nck - 2) * C;
    std::vector<AdjRowWorld> arow(size_t(T + 1) * nb);
    std::vector<AdjColWorld> acol(size_t(T) * nb);
    for (int b = 0; b < nb; ++b) {
        for (int j = 0; j + 1 < nck; ++j) {
            SpectralWorld& w = r2c[size_t(j) * nb + b];
            w = SpectralWorld{};
            w.A = slot(j * C, b);
            w.S_next = S_of(j * C, b);
            w.M = M;
            w.nk = 0;
            w.p = params;
        }
        for (int t = 0; t < T; ++t) {
            SpectralWorld& c = fcol[size_t(t) * nb + b];
            c = SpectralWorld{};
            c.S = S_of(t, b);
            c.U = Uspec_of(b);
            c.khat = khat;
            c.M = M;
            c.nk = nk;
            c.p = params;
            SpectralWorld& r = frow[size_t(t) * nb + b];
            r = SpectralWorld{};
            r.U = Uspec_of(b);
            r.U_px = U_of(t, b);
            r.A = slot(t, b);
            r.A_out = slot(t + 1, b);
            r.S_next = (t + 1 < T) ? S_of(t + 1, b) : nullptr;
            r.M = M;
            r.nk = nk;
            r.p = params;
            ffwd[size_t(t) * nb + b] = r;
            if (t < last_segment) ffwd[size_t(t) * nb + b].U_px = nullptr;
            AdjRowWorld& ar = arow[size_t(t) * nb + b];
            ar = AdjRowWorld{};
            ar.SG = (t == T - 1) ? nullptr : SG + size_t(b) * SPX;
            ar.g_in = (t == T - 1) ? gio + size_t(b) * P : g[(t + 1) % 2] + size_t(b) * P;
            ar.A_next = slot(t + 1, b);
            ar.A_cur = slot(t, b);
            ar.U = U_of(t, b);
            ar.g_out = g[t % 2] + size_t(b) * P;
            ar.SQ = SQ + size_t(b) * nk * SPX;
            AdjColWorld& ac = acol[size_t(t) * nb + b];
            ac.SQ = SQ + size_t(b) * nk * SPX;
            ac.SG = SG + size_t(b) * SPX;
            ac.S = cargs.ntab > 0 ? S_of(t, b) : nullptr;
        }
        AdjRowWorld& fin = arow[size_t(T) * nb + b];
        fin = AdjRowWorld{};
        fin.SG = SG + size_t(b) * SPX;
        fin.g_in = g[0] + size_t(b) * P;
        fin.gA_out = gio + size_t(b) * P;
    }
    cudaError_t e = cudaSuccess;
    const auto up = [&](void* dst, const void* src, size_t n) {
        if (e == cudaSuccess && n) e = cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
    };
    up(d_r2c, r2c.data(), r2c.size() * sizeof(SpectralWorld));
    up(d_fcol, fcol.data(), fcol.size() * sizeof(SpectralWorld));
    up(d_frow, frow.data(), frow.size() * sizeof(SpectralWorld));
    up(d_ffwd, ffwd.data(), ffwd.size() * sizeof(SpectralWorld));
    up(d_arow, arow.data(), arow.size() * sizeof(AdjRowWorld));
    up(d_acol, acol.data(), acol.size() * sizeof(AdjColWorld));
    if (e != cudaSuccess) return cuda_fail(e, "copy launch tables");
    return LENIA_OK;
}

namespace {

thread_local std::string g_adjoint_create_error;

cudaStream_t pick_stream(lenia_adjoint* a, void* s) { return s ? static_cast<cudaStream_t>(s) : a->stream; }

// The forward kernels over one step's world table.
// The forward kernels over one step's world tables (`recompute`: the tables
// that keep the step's potentials).
cudaError_t forward_step(lenia_adjoint* a, int t, bool recompute, cudaStream_t s) {
    using namespace lenia;
    cudaError_t e = launch_col_fast_worlds(a->H, a->M, a->ft, a->col_batch, a->d_fcol + size_t(t) * a->nb, a->nb, s);
    const SpectralWorld* rt = (recompute ? a->d_frow : a->d_ffwd) + size_t(t) * a->nb;
    if (e == cudaSuccess) e = launch_row_fast_worlds(a->H, a->M, a->ft, a->tw_r2c, a->row_batch, rt, a->nb, s);
    a->launches += 2;
    return e;
}

cudaError_t row_spectrum(lenia_adjoint* a, int j, cudaStream_t s) {
    a->launches += 1;
    return lenia::launch_row_fast_worlds(a->H, a->M, a->ft, a->tw_r2c, a->row_batch, a->d_r2c + size_t(j) * a->nb,
                                         a->nb, s);
}

// Columns per CTA iteration of the forward column pass and rows of the row
// pass: each candidate timed (CUDA events, after one warm-up launch) on step
// 0's tables over zeroed buffers; the fastest is kept.
cudaError_t autotune(lenia_adjoint* a) {
    const cudaStream_t s = a->stream;
    cudaError_t e = cudaMemsetAsync(a->ckpt, 0, sizeof(float) * a->nb * a->P, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a->Sring, 0, sizeof(float2) * a->nb * a->SPX, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a->SG, 0, sizeof(float2) * a->nb * a->SPX, s);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMemsetAsync(a->g[i], 0, sizeof(float) * a->nb * a->P, s);
    if (e != cudaSuccess) return e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const auto timed = [&](auto launch, float* ms) -> cudaError_t {
        cudaError_t r = launch();
        if (r != cudaSuccess) return r;
        cudaEventRecord(t0, s);
        for (int i = 0; i < 3 && r == cudaSuccess; ++i) r = launch();
        cudaEventRecord(t1, s);
        if (r == cudaSuccess) r = cudaEventSynchronize(t1);
        if (r == cudaSuccess) r = cudaEventElapsedTime(ms, t0, t1);
        return r;
    };
    float best = 1e30f;
    for (int cb : lenia::kColCandidates) {
        float ms = 0.0f;
        const cudaError_t r = timed([&] {
            return lenia::launch_col_fast_worlds(a->H, a->M, a->ft, cb, a->d_fcol, a->nb, s);
        }, &ms);
        if (r == cudaErrorInvalidConfiguration) continue;  // candidate too large for this size
        if (r != cudaSuccess) {
            e = r;
            break;
        }
        if (ms < best) {
            best = ms;
            a->col_batch = cb;
        }
    }
    best = 1e30f;
    for (int rb : lenia::kRowCandidates) {
        if (e != cudaSuccess) break;
        float ms = 0.0f;
        const cudaError_t r = timed([&] {
            return lenia::launch_row_fast_worlds(a->H, a->M, a->ft, a->tw_r2c, rb, a->d_frow, a->nb, s);
        }, &ms);
        if (r == cudaErrorInvalidConfiguration) continue;
        if (r != cudaSuccess) {
            e = r;
            break;
        }
        if (ms < best) {
            best = ms;
            a->row_batch = rb;
        }
    }
    // The adjoint passes, on step 0's tables (the row pass with the
    // previous column pass's input, as in the steady state).
    const int ta = a->T > 1 ? a->T - 2 : 0;
    best = 1e30f;
    for (int rb : {8, 4, 2, 1}) {
        if (e != cudaSuccess) break;
        float ms = 0.0f;
        const cudaError_t r = timed([&] {
            return lenia::launch_row_adj(a->M, rb, a->d_arow + size_t(ta) * a->nb, a->nb, a->rargs, a->tw_r2c, a->ft,
                                         s);
        }, &ms);
        if (r == cudaErrorInvalidConfiguration) continue;
        if (r != cudaSuccess) {
            e = r;
            break;
        }
        if (ms < best) {
            best = ms;
            a->adj_row_batch = rb;
        }
    }
    best = 1e30f;
    for (int cb : {8, 4, 2}) {
        if (e != cudaSuccess) break;
        float ms = 0.0f;
        const cudaError_t r = timed([&] {
            return lenia::launch_col_adj(a->H, cb, a->d_acol, a->nb, a->cargs, a->ft, s);
        }, &ms);
        if (r == cudaErrorInvalidConfiguration) continue;
        if (r != cudaSuccess) {
            e = r;
            break;
        }
        if (ms < best) {
            best = ms;
            a->adj_col_batch = cb;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaGetLastError();
    return e;
}

}  // namespace

extern "C" {

int lenia_adjoint_create(const lenia_adjoint_config* cfg, lenia_adjoint** out) {
    return lenia::abi_guard(&g_adjoint_create_error, [&]() -> int {
        using namespace lenia;
        if (!cfg || !out) return LENIA_ERR_INVALID_ARG;
        *out = nullptr;
        std::unique_ptr<lenia_adjoint> holder(new lenia_adjoint());
        lenia_adjoint* a = holder.get();
        const auto bail = [&](int code) {
            g_adjoint_create_error = a->message;
            return code;  // the holder frees the half-built engine
        };
        a->cfg = *cfg;
        std::string why;
        if (check_kernels(cfg->kernels, cfg->num_kernels, why) != LENIA_OK) return bail(a->fail(LENIA_ERR_INVALID_ARG, why));
        if (cfg->batch < 1 || cfg->steps < 1 || cfg->checkpoint_every < 1 || cfg->checkpoint_every > cfg->steps)
            return bail(a->fail(LENIA_ERR_INVALID_ARG, "need batch >= 1, steps >= 1, 1 <= checkpoint_every <= steps"));
        if (cfg->radius < 1 || cfg->growth_mode > 1u || cfg->kernel_core > 1u || !std::isfinite(cfg->dt))
            return bail(a->fail(LENIA_ERR_INVALID_ARG, "radius >= 1, growth_mode 0/1, kernel_core 0/1, finite dt"));
        if (cfg->kernel_core == LENIA_CORE_GAUSS_SHELL && !(cfg->shell_sigma > 0.0f))
            return bail(a->fail(LENIA_ERR_INVALID_ARG, "shell_sigma must be positive"));
        FastPlan cf, ri;
        if (cfg->width % 2 || cfg->width / 2 % kSpectralBlock || !fast_col_plan(int(cfg->height), cf) ||
            !fast_row_plan(int(cfg->width / 2), ri))
            return bail(a->fail(LENIA_ERR_UNSUPPORTED, "field size " + std::to_string(cfg->width) + "x" +
                                                           std::to_string(cfg->height) +
                                                           " has no compile-time FFT plan"));
        a->W = int(cfg->width);
        a->H = int(cfg->height);
        a->M = a->W / 2;
        a->Hh = a->H / 2 + 1;
        a->nb = int(cfg->batch);
        a->nk = int(cfg->num_kernels);
        a->T = int(cfg->steps);
        a->C = int(cfg->checkpoint_every);
        a->nck = (a->T + a->C - 1) / a->C + 1;
        a->P = size_t(a->W) * a->H;
        a->SPX = size_t(a->M) * a->H;
        cudaGetDevice(&a->device);
        cudaError_t e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bail(a->cuda_fail(e, "cudaStreamCreate"));
        const size_t nb = size_t(a->nb), nk = size_t(a->nk);
        int ntab = 0;
        for (int k = 0; k < a->nk; ++k)
            if (cfg->kernels[k].num_betas > 1) ntab += int(cfg->kernels[k].num_betas);
        const size_t tab = size_t(a->M + 1) * a->Hh;
        if ((e = a->alloc(&a->ckpt, size_t(a->nck) * nb * a->P)) != cudaSuccess ||
            (e = a->alloc(&a->seg, size_t(a->C) * nb * a->P)) != cudaSuccess ||
            (e = a->alloc(&a->Sring, size_t(a->C + 1) * nb * a->SPX)) != cudaSuccess ||
            (e = a->alloc(&a->Uspec, nb * nk * a->SPX)) != cudaSuccess ||
            (e = a->alloc(&a->Upx, size_t(a->C) * nb * nk * a->P)) != cudaSuccess ||
            (e = a->alloc(&a->SQ, nb * nk * a->SPX)) != cudaSuccess || (e = a->alloc(&a->SG, nb * a->SPX)) != cudaSuccess ||
            (e = a->alloc(&a->g[0], nb * a->P)) != cudaSuccess || (e = a->alloc(&a->g[1], nb * a->P)) != cudaSuccess ||
            (e = a->alloc(&a->gio, nb * a->P)) != cudaSuccess || (e = a->alloc(&a->acc, size_t(kAcc))) != cudaSuccess ||
            (e = a->alloc(&a->khat, nk * tab)) != cudaSuccess ||
            (e = a->alloc(&a->dtab, std::max<size_t>(1, size_t(ntab)) * tab)) != cudaSuccess ||
            (e = a->alloc(&a->d_r2c, size_t(a->nck - 1) * nb)) != cudaSuccess ||
            (e = a->alloc(&a->d_fcol, size_t(a->T) * nb)) != cudaSuccess ||
            (e = a->alloc(&a->d_frow, size_t(a->T) * nb)) != cudaSuccess ||
            (e = a->alloc(&a->d_ffwd, size_t(a->T) * nb)) != cudaSuccess ||
            (e = a->alloc(&a->d_arow, size_t(a->T + 1) * nb)) != cudaSuccess ||
            (e = a->alloc(&a->d_acol, size_t(a->T) * nb)) != cudaSuccess)
            return bail(a->cuda_fail(e, "cudaMalloc"));
        std::vector<float2> t2;
        fill_twiddles(a->W, t2);
        t2.resize(size_t(a->M) + 1);
        std::vector<float2> tws[4];
        fast_twiddle_tables(a->H, a->M, tws);
        if ((e = a->alloc(&a->tw_r2c, t2.size())) != cudaSuccess) return bail(a->cuda_fail(e, "cudaMalloc"));
        cudaMemcpy(a->tw_r2c, t2.data(), t2.size() * sizeof(float2), cudaMemcpyHostToDevice);
        for (int q = 0; q < 4; ++q) {
            if ((e = a->alloc(&a->tw[q], tws[q].size())) != cudaSuccess) return bail(a->cuda_fail(e, "cudaMalloc"));
            cudaMemcpy(a->tw[q], tws[q].data(), tws[q].size() * sizeof(float2), cudaMemcpyHostToDevice);
        }
        a->ft.col_twf = a->tw[0];
        a->ft.col_twi = a->tw[1];
        a->ft.row_twi = a->tw[2];
        a->ft.row_twf = a->tw[3];
        int rc = a->set_kernels(cfg->kernels, cfg->num_kernels, cfg->dt);
        if (rc != LENIA_OK) return bail(rc);
        if ((e = autotune(a)) != cudaSuccess) return bail(a->cuda_fail(e, "autotune"));
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(a->cuda_fail(e, "setup"));
        *out = holder.release();
        return LENIA_OK;
    });
}

int lenia_adjoint_destroy(lenia_adjoint* a) {
    return lenia::abi_guard(a ? &a->message : nullptr, [&]() -> int {
        if (!a) return LENIA_ERR_INVALID_ARG;
        delete a;
        return LENIA_OK;
    });
}

int lenia_adjoint_set_params(lenia_adjoint* a, const lenia_kernel_def* kernels, uint32_t num_kernels, float dt) {
    return lenia::abi_guard(a ? &a->message : nullptr, [&]() -> int {
        if (!a || !kernels) return LENIA_ERR_INVALID_ARG;
        std::string why;
        if (check_kernels(kernels, num_kernels, why) != LENIA_OK) return a->fail(LENIA_ERR_INVALID_ARG, why);
        if (int(num_kernels) != a->nk) return a->fail(LENIA_ERR_INVALID_ARG, "num_kernels differs from creation");
        for (int k = 0; k < a->nk; ++k) {
            if (kernels[k].num_betas != a->cfg.kernels[k].num_betas)
                return a->fail(LENIA_ERR_INVALID_ARG, "num_betas of a kernel differs from creation");
            if (kernels[k].radius_scale != a->cfg.kernels[k].radius_scale)
                return a->fail(LENIA_ERR_INVALID_ARG, "radius_scale of a kernel differs from creation");
        }
        if (!std::isfinite(dt)) return a->fail(LENIA_ERR_INVALID_ARG, "dt must be finite");
        // The tables are read by queued launches (on any stream): wait first.
        cudaDeviceSynchronize();
        return a->set_kernels(kernels, num_kernels, dt);
    });
}

int lenia_adjoint_forward(lenia_adjoint* a, const float* a0, float* a_final, void* stream) {
    return lenia::abi_guard(a ? &a->message : nullptr, [&]() -> int {
        if (!a || !a0 || !a_final) return LENIA_ERR_INVALID_ARG;
        const cudaStream_t s = pick_stream(a, stream);
        const size_t n = size_t(a->nb) * a->P * sizeof(float);
        cudaError_t e = cudaMemcpyAsync(a->ckpt, a0, n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = row_spectrum(a, 0, s);
        for (int t = 0; t < a->T && e == cudaSuccess; ++t) e = forward_step(a, t, false, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(a_final, a->slot(a->T, 0), n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return a->cuda_fail(e, "forward");
        a->forward_done = true;
        a->last_segment_fresh = true;
        return LENIA_OK;
    });
}

int lenia_adjoint_backward(lenia_adjoint* a, const float* g_final, float* g_initial, double* grad_params,
                           void* stream) {
    return lenia::abi_guard(a ? &a->message : nullptr, [&]() -> int {
        using namespace lenia;
        if (!a || !g_final || !g_initial) return LENIA_ERR_INVALID_ARG;
        if (!a->forward_done) return a->fail(LENIA_ERR_STATE, "backward needs a forward with the current parameters");
        const cudaStream_t s = pick_stream(a, stream);
        const size_t n = size_t(a->nb) * a->P * sizeof(float);
        cudaError_t e = cudaMemsetAsync(a->acc, 0, sizeof(double) * kAcc, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(a->gio, g_final, n, cudaMemcpyDeviceToDevice, s);
        for (int j = a->nck - 2; j >= 0 && e == cudaSuccess; --j) {
            const int s0 = j * a->C, e0 = std::min(s0 + a->C, a->T);
            if (!(j == a->nck - 2 && a->last_segment_fresh)) {
                e = row_spectrum(a, j, s);
                for (int t = s0; t < e0 && e == cudaSuccess; ++t) e = forward_step(a, t, true, s);
            }
            for (int t = e0 - 1; t >= s0 && e == cudaSuccess; --t) {
                e = launch_row_adj(a->M, a->adj_row_batch, a->d_arow + size_t(t) * a->nb, a->nb, a->rargs, a->tw_r2c,
                                   a->ft, s);
                if (e == cudaSuccess)
                    e = launch_col_adj(a->H, a->adj_col_batch, a->d_acol + size_t(t) * a->nb, a->nb, a->cargs, a->ft, s);
                a->launches += 2;
            }
        }
        if (e == cudaSuccess) {
            e = launch_row_adj(a->M, a->adj_row_batch, a->d_arow + size_t(a->T) * a->nb, a->nb, a->rargs, a->tw_r2c,
                               a->ft, s);
            a->launches += 1;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(g_initial, a->gio, n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && grad_params) {
            finalize_kernel<<<1, 64, 0, s>>>(a->acc, grad_params, a->nk, a->cfg.growth_mode == 1u ? 1 : 0);
            e = cudaGetLastError();
            a->launches += 1;
        }
        a->last_segment_fresh = false;
        if (e != cudaSuccess) return a->cuda_fail(e, "backward");
        return LENIA_OK;
    });
}

int lenia_adjoint_stats(lenia_adjoint* a, uint64_t* device_bytes, uint64_t* launches) {
    return lenia::abi_guard(a ? &a->message : nullptr, [&]() -> int {
        if (!a) return LENIA_ERR_INVALID_ARG;
        if (device_bytes) *device_bytes = a->bytes;
        if (launches) *launches = a->launches;
        return LENIA_OK;
    });
}

// NULL: the calling thread's last failed lenia_adjoint_create.
const char* lenia_adjoint_last_message(lenia_adjoint* a) {
    return a ? a->message.c_str() : g_adjoint_create_error.c_str();
}

}  // extern "C"
