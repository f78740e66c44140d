// life_simulation_b200/csrc/fft_fast_common.cuh -- shared pieces of the
// compile-time-plan spectral kernels (forward step, adjoint step): the
// Stockham pass runner over a batch of transforms, the shared-memory pitch,
// table copies and 16-byte asynchronous copies.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "fft_ct.cuh"
#include "lenia_kernels.h"

namespace lenia {
namespace fastfft {

using namespace fftct;

constexpr int KB = kSpectralBlock;  // columns per block of the blocked layout

constexpr int roundup32(int x) { return (x + 31) / 32 * 32; }

// Smallest pitch >= n with 2*pitch = 8 (mod 32) (in float2): transforms of a
// batch start 8 banks apart.
constexpr int row_pitch(int n) {
    int p = n;
    while ((2 * p) % 32 != 8) ++p;
    return p;
}

// One Stockham pass over a batch of B transforms: item q -> (b = q % B,
// j = q / B). All of a thread's items are loaded first, then twiddled,
// transformed and stored. src(b, i) / dst(b, i, v) address element i of
// transform b.
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
        jj[it] = q / B;
        bi[it] = q - jj[it] * B;
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

// The R outputs of one item of a first pass (span 1) are R consecutive
// elements of a row: written two at a time (16-byte stores, half the store
// instructions and shared-memory wavefronts) when R is even.
// `row + base` must be 16-byte aligned when R is even (shared buffers at
// even float2 offsets, even pitches, base a multiple of R).
template <int R>
__device__ __forceinline__ void store_run(float2* row, int base, const float2* v) {
    if constexpr (R % 2 == 0) {
        float4* d = reinterpret_cast<float4*>(row + base);
#pragma unroll
        for (int t = 0; t < R / 2; ++t) d[t] = make_float4(v[2 * t].x, v[2 * t].y, v[2 * t + 1].x, v[2 * t + 1].y);
    } else {
#pragma unroll
        for (int t = 0; t < R; ++t) row[base + t] = v[t];
    }
}

// Pass 0 (span 1) of plan P over a batch of B transforms into the shared
// buffer `buf` (row pitch PITCH, even): pass_gen with store_run's stores.
template <class P, bool INV, int B, int T, int PITCH, class Src>
__device__ __forceinline__ void pass0_buf(Src&& src, float2* buf, int cols) {
    using I = PassIdx<P, 0>;
    static_assert(I::NS == 1, "the first pass has span 1");
    constexpr int TOT = B * I::NR;
    constexpr int ITEMS = (TOT + T - 1) / T;
    float2 v[ITEMS][I::R];
    int jj[ITEMS], bi[ITEMS];
    bool ok[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const int q = int(threadIdx.x) + it * T;
        jj[it] = q / B;
        bi[it] = q - jj[it] * B;
        ok[it] = (TOT % T == 0 || q < TOT) && bi[it] < cols;
        if (ok[it]) {
#pragma unroll
            for (int t = 0; t < I::R; ++t) v[it][t] = src(bi[it], I::in(jj[it], t));
        }
    }
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        if (ok[it]) {
            Dft<I::R, INV>::run(v[it]);
            store_run<I::R>(buf + bi[it] * PITCH, jj[it] * I::R, v[it]);
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

// Asynchronous 16-byte global -> shared copy (completion: cp.async.wait_all,
// a hardware wait, then a block barrier).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Launch geometry of a column pass over B columns per CTA iteration (forward
// plan PF; the inverse is PF reversed): T threads, ITL last-pass items per
// thread, shared buffers of pitch PITCH. S = 2 halves the thread count (each
// thread takes two last-pass items): fewer warps per CTA, twice the
// independent work per thread, and CTAs small enough for two per SM.
template <class PF, int B, int S = 1>
struct ColK {
    static_assert(KB % B == 0, "a column group lies inside one block");
    using PI = typename Reverse<PF>::type;
    static constexpr int H = PF::n;
    static constexpr int Hh = H / 2 + 1;
    static constexpr int RL = PF::last();
    static constexpr int NRL = H / RL;
    static constexpr int T = roundup32((B * NRL + S - 1) / S);
    static constexpr int ITL = (B * NRL + T - 1) / T;
    static constexpr int PITCH = row_pitch(H);
    // The work buffers start after the twiddle tables at an even float2
    // offset (16-byte aligned, for store_run's paired stores).
    static constexpr int BUF0 = (PF::tw_size() + PI::tw_size() + 1) / 2 * 2;
    static_assert(PITCH % 2 == 0, "column pitch must keep 16-byte alignment");
    static constexpr size_t smem() { return sizeof(float2) * (size_t(BUF0) + 2 * size_t(B) * PITCH + H); }
};

// Launch geometry of a row pass over RB rows per CTA iteration (inverse plan
// PI; the forward is PI reversed); S as for ColK.
template <class PI, int RB, int S = 1>
struct RowK {
    using PF = typename Reverse<PI>::type;
    static constexpr int M = PI::n;
    static_assert(M % KB == 0, "row length must be a whole number of blocks");
    static constexpr int RC = PI::last();
    static constexpr int NRC = M / RC;
    static constexpr int T = roundup32((RB * NRC + S - 1) / S);
    static constexpr int ITL = (RB * NRC + T - 1) / T;
    static constexpr int PITCH = row_pitch(M);  // even: rows start 16-byte aligned
    // Twiddle tables, then the buffers from an even float2 offset so the
    // 16-byte cp.async destinations are 16-byte aligned.
    static constexpr int TABLES = (M + 1) + PI::tw_size() + PF::tw_size();
    static constexpr int BUF0 = (TABLES + 1) / 2 * 2;
    static_assert(PITCH % 2 == 0, "row pitch must keep 16-byte alignment");
    // Tables plus `nbuf` buffers of RB rows.
    static constexpr size_t smem(int nbuf = 2) { return sizeof(float2) * (size_t(BUF0) + nbuf * size_t(RB) * PITCH); }
};

// Real rows of W = 2M values are transformed as M complex values
// z[n] = x[2n] + i x[2n+1]; the half spectrum X[0..M] is stored as M entries
// with X[0] + i X[M] in column 0 (both are real). twr[k] = exp(-2 pi i k / W).

// Stages rows y0..y0+rows-1 of a blocked-layout plane (H rows, M columns)
// into shared rows of pitch PITCH: per block, rows x 8 columns are
// contiguous (16-byte asynchronous copies, two columns each). The caller
// waits (cp_async_wait_all + barrier).
template <int M, int RB, int T, int PITCH>
__device__ __forceinline__ void stage_rows(float2* dst, const float2* __restrict__ plane, int H, int y0, int rows) {
    for (int q = threadIdx.x; q < (M / KB) * RB * (KB / 2); q += T) {
        const int c2 = q % (KB / 2);
        const int b = (q / (KB / 2)) % RB;
        const int kb = q / ((KB / 2) * RB);
        if (b < rows) cp_async16(dst + b * PITCH + kb * KB + 2 * c2, plane + (size_t(kb) * H + y0 + b) * KB + 2 * c2);
    }
}

// Stages rows y0..y0+rows-1 of a row-major real field (W = 2M floats per
// row) into shared rows of pitch PITCH, as M float2 pairs (x[2n], x[2n+1]):
// 16-byte asynchronous copies. The caller waits.
template <int M, int RB, int T, int PITCH>
__device__ __forceinline__ void stage_field_rows(float2* dst, const float* __restrict__ field, int y0, int rows) {
    for (int q = threadIdx.x; q < RB * (M / 2); q += T) {
        const int c = q % (M / 2), b = q / (M / 2);
        if (b < rows) cp_async16(dst + b * PITCH + 2 * c, field + (size_t(y0 + b) * M + 2 * c) * 2);
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until at most one committed group of this thread is still in flight.
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Inverse of the real-FFT split for element i of a staged half-spectrum row:
// Z'[k] = (X[k] + conj X[M-k]) + i exp(+2 pi i k/W) (X[k] - conj X[M-k]);
// the length-M inverse transform of Z' gives 2 z[n].
template <int M>
__device__ __forceinline__ float2 c2r_split(const float2* xr, const float2* twr, int i) {
    if (i == 0) {
        const float2 x0 = xr[0];
        return make_float2(x0.x + x0.y, x0.x - x0.y);
    }
    const float2 Xk = xr[i];
    const float2 Xm = fft::cconj(xr[M - i]);
    const float2 D = fft::cmul(fft::cconj(twr[i]), fft::csub(Xk, Xm));
    return fft::cadd(fft::cadd(Xk, Xm), make_float2(-D.y, D.x));
}

// Real-FFT split of the length-M forward transforms Z of `rows` packed real
// rows (shared, pitch PITCH) into half spectra, stored to rows y0.. of a
// blocked-layout plane two columns at a time.
template <int M, int RB, int T, int PITCH>
__device__ __forceinline__ void r2c_store_rows(const float2* Z, const float2* twr, float2* __restrict__ plane, int H,
                                               int y0, int rows) {
    for (int q = threadIdx.x; q < (M / KB) * RB * (KB / 2); q += T) {
        const int c2 = q % (KB / 2);
        const int b = (q / (KB / 2)) % RB;
        const int kb = q / ((KB / 2) * RB);
        if (b >= rows) continue;
        const float2* zr = Z + b * PITCH;
        float2 xv[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int k = kb * KB + 2 * c2 + e;
            const float2 Zk = zr[k];
            if (k == 0) {
                xv[e] = make_float2(Zk.x + Zk.y, Zk.x - Zk.y);
            } else {
                const float2 Zc = fft::cconj(zr[M - k]);
                const float2 E = fft::cscale(fft::cadd(Zk, Zc), 0.5f);
                const float2 D = fft::csub(Zk, Zc);
                const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
                xv[e] = fft::cadd(E, fft::cmul(twr[k], O));
            }
        }
        *reinterpret_cast<float4*>(plane + (size_t(kb) * H + y0 + b) * KB + 2 * c2) =
            make_float4(xv[0].x, xv[0].y, xv[1].x, xv[1].y);
    }
}

// ------------------------------------------------------- launch helpers

inline int sms() {
    static int n = 0;
    if (!n) {
        int d = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
        if (n <= 0) n = 148;
    }
    return n;
}

// Opt a kernel into `smem` bytes of dynamic shared memory and the largest
// shared-memory carveout.
template <typename F>
cudaError_t prepare(F fn, size_t smem) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

// Programmatic dependent launch. A kernel launched by `launch_chained` may
// start while the kernel before it in the stream is still running: it does
// its data-independent prologue (twiddle tables into shared memory), then
// `grid_dependency_wait` blocks until that kernel has completed and its
// writes are visible. `allow_dependents`, called when a CTA starts its last
// work item, lets the next chained kernel launch once every CTA of this one
// has called it (or exited): the next kernel's CTAs then do their prologue
// while this kernel's last items finish. Every CTA of a chained kernel
// waits before it touches data, so kernel completion stays transitive along
// the stream. Both instructions are no-ops in a kernel launched without the
// attribute.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// LENIA_CHAINED_LAUNCH=0 in the environment turns the attribute off (plain
// stream order), e.g. for tools that serialise launches anyway.
inline bool chained_launch_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("LENIA_CHAINED_LAUNCH");
        return !(v && v[0] == '0' && v[1] == '\0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*fn)(KArgs...), dim3 grid, int threads, size_t smem, cudaStream_t s,
                           Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(unsigned(threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = chained_launch_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, fn, args...);
}

// Persistent grid over n worlds: grid.y = world, grid.x = CTAs per world
// (the resident CTAs of the device shared out, at most one per group).
// Rounded down: every CTA loops over its share of the pass, so a CTA beyond
// the resident slots would wait for a whole persistent CTA to finish -- a
// second wave as long as the first (e.g. 19 x 32 = 608 CTAs for 592 slots).
inline dim3 world_grid(int per_sm, int groups, int n) {
    const int resident = std::max(1, per_sm) * sms();
    const int x = std::max(1, std::min(groups, resident / std::max(1, n)));
    return dim3(unsigned(x), unsigned(n));
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
// Row plans (inverse order) by M = W/2 (a multiple of 8).
#define LENIA_ROW_PLANS(X)     \
    X(960, Plan<8, 15, 8>)     \
    X(512, Plan<8, 8, 8>)      \
    X(2048, Plan<16, 16, 8>)   \
    X(256, Plan<8, 4, 8>)      \
    X(192, Plan<8, 3, 8>)      \
    X(128, Plan<16, 8>)        \
    X(64, Plan<8, 8>)

}  // namespace fastfft
}  // namespace lenia
