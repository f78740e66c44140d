// life_simulation_b200/csrc/lenia_fft_tc05.cu -- the column pass of a
// 4096-row field with its DFT stages as GEMMs on the fifth-generation tensor
// cores (tcgen05.mma: operands in shared memory, accumulators in tensor
// memory), split-precision FP16 or BF16 hi/lo operands, FP32 accumulation.
//
// Same contract and blocked layout as col_fast_kernel (lenia_fft_fast.cu):
// S (row spectrum, packed column 0) -> for every kernel k, U_k = the inverse
// column FFT of FFT_H(S) * khat_k.
//
// 4096 = 64 x 64: two radix-64 Stockham passes per transform. One pass over
// B = 2 columns is one GEMM: 128 items (64 per column, the two columns'
// items interleaved: GEMM item 2j + b is item j of column b) of 64 complex inputs,
// i.e. in real arithmetic a 128 x 128 operand X (K = 128: re/im of the 64
// inputs interleaved) against the 128 x 128 real DFT matrix
//     F[2u + c][2t + c'] = ([[cos, sin], [-sin, cos]] of 2 pi u t / 64) / 64
// (row 2u + c: re/im of output u; the 1/64 keeps every pass's magnitudes in
// FP16's range). Every product is taken in split precision: a = a_hi + a_lo
// (the 16-bit rounding of a, then the rounding of the remainder) and
//     F X ~ F_hi X_hi + F_hi X_lo + F_lo X_hi,
// 24 MMAs of K = 16 accumulated in FP32 in tensor memory.
//
// Orientation. A transform's first pass computes D = F X (D rows = outputs,
// one tensor-memory lane each; columns = items): a lane then holds, for one
// output u, the values of consecutive items j -- the consecutive K inputs
// that item u of the second pass reads (the Stockham transpose), so the
// second pass's operand rows are written from registers after a twiddle.
// The second pass computes D = X F^T (rows = items, columns = outputs): each
// lane then holds the consecutive outputs of one item -- for the forward
// transform exactly the inputs of one item of the inverse's first pass (the
// spectrum product needs no exchange), for the inverse the elements of one
// output column. The inverse transform is the forward one conjugated,
// IDFT(x) = conj(DFT(conj(x))), and with conjugated data the inverse
// twiddles become the forward ones: one DFT matrix and one twiddle rule
// serve both directions.
//
// Sixteen warps: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 and
// columns kCW (w / 4) .. + kCW - 1 of every result.
//
// Tensor memory: 256 columns per CTA, [0, 128) the current pass's result,
// [128, 256) the forward column spectrum, kept for all kernels' products
// (pipelined form: 512, two result regions and the spectrum).
// Waits on the MMA completion barrier are bounded; a wait that runs out
// counts into `err` and the CTA stops issuing work, frees its tensor memory
// and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "fft_fast_common.cuh"
#include "fft_tc.cuh"
#include "lenia_kernels.h"

namespace lenia {
namespace {

using namespace fastfft;

constexpr int kH = 4096;                     // column length
constexpr int kHh = kH / 2 + 1;              // kernel spectrum rows
constexpr int kB = 2;                        // columns per group
constexpr int kT = 512;                      // 16 warps: four per tensor-memory lane quadrant
constexpr int kCW = 128 / (kT / 128);        // tensor-memory columns per warp (32)
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t kOp = 128u * 128u * 2u;   // one 128 x 128 16-bit operand (32 KB)
// Dynamic shared memory: F hi/lo, operand slot 0 hi/lo, (pipelined: slot 1
// hi/lo,) the second pass's 4096 twiddles.
constexpr uint32_t kSmFhi = 0, kSmFlo = kOp, kSmXhi = 2 * kOp, kSmXlo = 3 * kOp, kSmRoot = 4 * kOp;
constexpr size_t kSmem = 4 * size_t(kOp) + size_t(kH) * sizeof(float2);  // 160 KB (224 KB pipelined)
constexpr float kProductScale = 16777216.0f;  // 2^24 = 4096^2: the two 1/64 of each transform's passes
constexpr uint32_t kPolls = 1u << 22;         // polls of the MMA barrier before a CTA gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row r, k) of a 128 x 128 operand in the canonical
// K-major layout without swizzle: 8 x 8 core matrices of 16-byte rows (8
// consecutive k), core (r / 8, k / 8) at ((k / 8) * 16 + r / 8) * 128. Core
// matrices adjacent in k are 2048 bytes apart (the descriptor's leading
// byte offset), adjacent in r 128 bytes (its stride byte offset).
__device__ __forceinline__ uint32_t kmaj(int r, int k) {
    return (uint32_t(((k >> 3) << 4) + (r >> 3)) << 7) + (uint32_t(r & 7) << 4) + (uint32_t(k & 7) << 1);
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// byte offset 2048, stride byte offset 128 (all >> 4), descriptor version 1,
// no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t(2048u >> 4) << 16) | (uint64_t(128u >> 4) << 32) |
           (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, A and B FP16 (0)
// or BF16 (1), both K-major, N = 128 (>> 3), M = 128 (>> 4).
template <int PREC>
constexpr uint32_t idesc() {
    constexpr uint32_t f = PREC == tcfft::kBF16x3 ? 1u : 0u;
    return (1u << 4) | (f << 7) | (f << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kPolls; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// One pass: D = A B^T over K = 128 (both operands 128 x 128, K-major), as
// A_hi B_hi + A_hi B_lo + A_lo B_hi; the barrier's phase completes when
// every MMA has. Issued by one thread.
template <int PREC>
__device__ __forceinline__ void issue_pass(uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo,
                                           uint64_t* bar) {
    constexpr uint32_t id = idesc<PREC>();
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        const uint32_t o = uint32_t(kc) * 4096u;  // K = 16 kc .. 16 kc + 15: core columns 2 kc, 2 kc + 1
        mma(d, smem_desc(a_hi + o), smem_desc(b_hi + o), id, kc > 0 ? 1u : 0u);
        mma(d, smem_desc(a_hi + o), smem_desc(b_lo + o), id, 1u);
        mma(d, smem_desc(a_lo + o), smem_desc(b_hi + o), id, 1u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive tensor-memory columns of this warp's lane quadrant: one
// load, one wait (a wait per 16 columns left the warps idle on its latency).
__device__ __forceinline__ void tmem_ld(uint32_t addr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
// Four complex values (eight consecutive K elements of one operand row),
// split into hi and lo 16-bit parts: one 16-byte store each.
template <int PREC>
__device__ __forceinline__ void put4(unsigned char* xhi, unsigned char* xlo, uint32_t off, const float2* z) {
    uint4 h, l;
    tcfft::split2<PREC>(z[0].x, z[0].y, h.x, l.x);
    tcfft::split2<PREC>(z[1].x, z[1].y, h.y, l.y);
    tcfft::split2<PREC>(z[2].x, z[2].y, h.z, l.z);
    tcfft::split2<PREC>(z[3].x, z[3].y, h.w, l.w);
    *reinterpret_cast<uint4*>(xhi + off) = h;
    *reinterpret_cast<uint4*>(xlo + off) = l;
}

// From a first-pass result D = F X in tensor memory (rows 2u + c, columns
// n = 2j + b: item j of column b): the second pass's operand
// X'[2u + b][2j + c] = D(u; j, b) * exp(-2 pi i u j / 4096). Warp (quadrant
// q4, part hh) takes outputs u = 16 q4 .. 16 q4 + 15 and D columns kCW hh ..
// kCW hh + kCW - 1 (items of both columns). A lane pair (re row, im row)
// trades halves so the even lane holds the complex values of column b = 0's
// items and the odd lane column b = 1's: the pair reads one twiddle
// (tw[j * 64 + u] = exp(-2 pi i u j / 4096), a broadcast) and writes rows
// 2u and 2u + 1 of one operand chunk (distinct shared-memory bank quads).
template <int PREC>
__device__ __forceinline__ void second_pass_operand(uint32_t dtm, const float2* tw, unsigned char* xhi,
                                                    unsigned char* xlo, int q4, int hh, int lane) {
    const int u = 16 * q4 + (lane >> 1);
    const int odd = lane & 1;
    float v[kCW];
    tmem_ld(dtm + uint32_t(kCW * hh), v);
#pragma unroll
    for (int c16 = 0; c16 < kCW / 16; ++c16) {
        float2 z[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            // Column 16 c16 + 2i (b = 0) and + 2i + 1 (b = 1) of this row.
            const float send = odd ? v[16 * c16 + 2 * i] : v[16 * c16 + 2 * i + 1];
            const float got = __shfl_xor_sync(0xffffffffu, send, 1);
            z[i] = odd ? make_float2(got, v[16 * c16 + 2 * i + 1]) : make_float2(v[16 * c16 + 2 * i], got);
        }
        const int j0 = (kCW * hh + 16 * c16) >> 1;  // items j0 .. j0 + 7
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 w = tw[(j0 + i) * 64 + u];
            z[i] = make_float2(__fmaf_rn(z[i].x, w.x, -z[i].y * w.y), __fmaf_rn(z[i].x, w.y, z[i].y * w.x));
        }
        put4<PREC>(xhi, xlo, kmaj(2 * u + odd, 2 * j0), z);
        put4<PREC>(xhi, xlo, kmaj(2 * u + odd, 2 * j0 + 8), z + 4);
    }
}

// PIPE: two operand slots (shared-memory operand, tensor-memory result and
// completion barrier each), so the MMAs of one kernel's inverse transform
// run while the CUDA cores build the next kernel's operands: kernel k uses
// slot k % 2, its first pass is issued as soon as the slot is free, and the
// CUDA-core work of kernel k (second-pass operand, output) is interleaved
// with kernel k + 1's. Without PIPE every pass waits for its own MMAs.
template <int PREC, bool PIPE>
__global__ void __launch_bounds__(kT, 1)
    col_tc05_kernel(const float2* __restrict__ S, float2* __restrict__ U, const float* __restrict__ khat, int M, int nk,
                    int* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int stop;  // a wait for an MMA ran out (read after block barriers)
    if (nk <= 0) return;
    constexpr uint32_t kCols = PIPE ? 2 * kTmemCols : kTmemCols;
    const int tid = int(threadIdx.x), warp = tid >> 5, lane = tid & 31;
    const int q4 = warp & 3, hh = warp >> 2;
    unsigned char* fhi = sm + kSmFhi;
    unsigned char* flo = sm + kSmFlo;
    // Operand slot s: hi at (2 + 2s) * kOp, lo at (3 + 2s) * kOp.
    const auto xhi = [&](int sl) { return sm + kSmXhi + uint32_t(sl) * 2u * kOp; };
    const auto xlo = [&](int sl) { return sm + kSmXlo + uint32_t(sl) * 2u * kOp; };
    float2* tw = reinterpret_cast<float2*>(sm + (PIPE ? kSmRoot + 2 * kOp : kSmRoot));
    const uint32_t a_fhi = smem_u32(fhi), a_flo = smem_u32(flo);

    // Second-pass twiddles tw[j * 64 + u] = exp(-2 pi i u j / 4096).
    for (int a = tid; a < kH; a += kT) {
        float sn, cs;
        sincospif(float((a >> 6) * (a & 63)) * (1.0f / 2048.0f), &sn, &cs);
        tw[a] = make_float2(cs, -sn);
    }
    // F: row 2u (re of output u) holds (cos, sin) of 2 pi u t / 64 against
    // (re, im) of input t, row 2u + 1 (im) holds (-sin, cos); over 64.
    for (int e = tid; e < 128 * 64; e += kT) {
        const int r = e >> 6, t = e & 63, u = r >> 1;
        float sn, cs;
        sincospif(float((u * t) & 63) * (1.0f / 32.0f), &sn, &cs);
        const float2 w = make_float2(cs, -sn);  // exp(-2 pi i u t / 64)
        const float a0 = ((r & 1) ? w.y : w.x) * (1.0f / 64.0f);
        const float a1 = ((r & 1) ? w.x : -w.y) * (1.0f / 64.0f);
        uint32_t h, l;
        tcfft::split2<PREC>(a0, a1, h, l);
        *reinterpret_cast<uint32_t*>(fhi + kmaj(r, 2 * t)) = h;
        *reinterpret_cast<uint32_t*>(flo + kmaj(r, 2 * t)) = l;
    }
    if (tid == 0) {
        stop = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t quad = uint32_t(32 * q4) << 16;  // this warp's lane quadrant
    // Slot s's pass results at columns [128 s, 128 s + 128); the spectrum after them.
    const auto wcol = [&](int sl) { return tmem + uint32_t(sl) * 128u; };
    const uint32_t spec = tmem + (PIPE ? 256u : 128u);
    uint32_t phases = 0, pending = 0;  // per slot: barrier phase to wait for; MMAs issued, not yet waited
    bool ok = true;

    // One pass on slot sl: operand writes made visible to the tensor cores,
    // D = A B^T issued by one thread (not waited for). False for every
    // thread, and nothing issued, once a wait has run out anywhere.
    const auto issue = [&](int sl, uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (*reinterpret_cast<volatile int*>(&stop)) return false;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_pass<PREC>(d, a_hi, a_lo, b_hi, b_lo, &bars[sl]);
        }
        pending |= 1u << sl;
        return true;
    };
    // Waits (bounded) for slot sl's pass. A wait that runs out raises `stop`
    // and the thread carries on (its values are not used: the next `issue`,
    // or the end of the kernel, stops every thread after a block barrier).
    const auto wait = [&](int sl) {
        if (mbar_wait(&bars[sl], (phases >> sl) & 1u)) {
            phases ^= 1u << sl;
            pending &= ~(1u << sl);
        } else {
            *reinterpret_cast<volatile int*>(&stop) = 1;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    };
    const auto sx = [&](int sl) { return smem_u32(xhi(sl)); };
    const auto sxl = [&](int sl) { return smem_u32(xlo(sl)); };

    // Column 0 of U_{nk-1}: scratch for the packed DC/Nyquist column's
    // spectrum (element ky at c0[ky * 8]) between the forward transform and
    // the last kernel's output, which overwrites it. Only the CTA holding
    // column 0 touches it.
    float2* c0 = U + size_t(nk - 1) * size_t(M) * kH;

    for (int k0 = int(blockIdx.x) * kB; k0 < M && ok; k0 += int(gridDim.x) * kB) {
        const size_t gbase = size_t(k0 / KB) * kH * KB + size_t(k0 % KB);
        // Forward first pass operand: X[2j + b][2t + c] = S[j + 64 t][b] (the
        // two columns' items interleaved);
        // this thread's rows (j = tid % 64, t = 4q .. 4q + 3 for q =
        // tid / 64 + (kT / 64) it) all requested before any is used.
        {
            constexpr int kIt = 1024 / kT;
            const int j = tid & 63;
            float4 sv[4 * kIt];
#pragma unroll
            for (int it = 0; it < kIt; ++it)
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int t = 4 * ((tid >> 6) + (kT / 64) * it) + i;
                    sv[4 * it + i] = __ldg(reinterpret_cast<const float4*>(S + gbase + size_t(j + 64 * t) * KB));
                }
#pragma unroll
            for (int it = 0; it < kIt; ++it) {
                const int q = (tid >> 6) + (kT / 64) * it;
                // Rows 2j (column 0) and 2j + 1 (column 1); lanes with j % 8 >= 4
                // write the odd row first, so each store's eight-lane phase
                // covers eight distinct bank quads.
                const int sw = (j >> 2) & 1;
                float2 z0[4], z1[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float4 a = sv[4 * it + i];
                    z0[i] = sw ? make_float2(a.z, a.w) : make_float2(a.x, a.y);
                    z1[i] = sw ? make_float2(a.x, a.y) : make_float2(a.z, a.w);
                }
                put4<PREC>(xhi(0), xlo(0), kmaj(2 * j + sw, 8 * q), z0);
                put4<PREC>(xhi(0), xlo(0), kmaj(2 * j + 1 - sw, 8 * q), z1);
            }
        }
        // The next group's rows into L2 while this group's passes run (a
        // 128-byte line holds two 64-byte block rows).
        {
            const int nxt = k0 + int(gridDim.x) * kB;
            if (nxt < M) {
                const float2* ns = S + size_t(nxt / KB) * kH * KB + size_t(nxt % KB);
                for (int r = 2 * tid; r < kH; r += 2 * kT)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(ns + size_t(r) * KB));
                // and its two columns of every kernel spectrum (2049 floats each)
                constexpr int kLines = (kHh + 31) / 32;
                for (int q = tid; q < nk * 2 * kLines; q += kT) {
                    const int kk = q / (2 * kLines), c = (q / kLines) & 1, l = q % kLines;
                    const float* kp = khat + (size_t(kk) * size_t(M + 1) + size_t(nxt + c)) * kHh + size_t(32 * l);
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(kp));
                }
            }
        }
        if (!(ok = issue(0, wcol(0), a_fhi, a_flo, sx(0), sxl(0)))) break;
        wait(0);
        second_pass_operand<PREC>(wcol(0) + quad, tw, xhi(0), xlo(0), q4, hh, lane);
        // Column spectrum C = X F^T: row 2j' + b (item j' of column b),
        // columns 2u' + c: C at ky = j' + 64 u' (over 4096).
        if (!(ok = issue(0, spec, sx(0), sxl(0), a_fhi, a_flo))) break;
        wait(0);

        // This lane's item of the spectrum: row m = 32 q4 + lane (item j of
        // column b; the lane pair (b = 0, 1) holds the same item of both).
        const int b = lane & 1, j = 16 * q4 + (lane >> 1), m = 32 * q4 + lane;
        const int kx = k0 + b;
        if (k0 == 0) {
            // Every lane loads (the tensor-memory load is warp-wide); the
            // lanes of column 0 store.
            float v[kCW];
            tmem_ld(spec + quad + uint32_t(kCW * hh), v);
            if (b == 0) {
#pragma unroll
                for (int i = 0; i < kCW / 2; ++i)
                    c0[size_t(j + 64 * ((kCW / 2) * hh + i)) * KB] = make_float2(v[2 * i], v[2 * i + 1]);
            }
            __syncthreads();  // column 0's spectrum visible to the block
        }
        // Inverse first pass operand of kernel kk (conjugated) into slot sl:
        // X[m][2u' + c] = conj(C * khat) * 2^24, u' = (kCW / 2) hh + e for
        // e < kCW / 2; the kernel values are requested first.
        const auto product = [&](int kk, int sl) {
            const float* kh = khat + size_t(kk) * size_t(M + 1) * kHh;
            float kv[kCW / 2];
#pragma unroll
            for (int i = 0; i < kCW / 2; ++i) {
                const int ky = j + 64 * ((kCW / 2) * hh + i);
                kv[i] = __ldg(kh + size_t(kx) * kHh + min(ky, kH - ky));
            }
            float v[kCW];
            tmem_ld(spec + quad + uint32_t(kCW * hh), v);
#pragma unroll
            for (int c8 = 0; c8 < kCW / 16; ++c8) {
                float2 z[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int e = 8 * c8 + i;  // u' = (kCW / 2) hh + e
                    const float P = kv[e] * kProductScale;
                    if (kx == 0) {
                        // Packed column 0: X[0] and X[M] (both real) as re/im;
                        // the product splits them with C[ky] and conj C[-ky].
                        const int ky = j + 64 * ((kCW / 2) * hh + e);
                        const float Q = __ldg(kh + size_t(M) * kHh + min(ky, kH - ky)) * kProductScale;
                        const float2 cm = c0[size_t(ky == 0 ? 0 : kH - ky) * KB];
                        const float ev = 0.5f * (P + Q), od = 0.5f * (P - Q);
                        z[i] = make_float2(ev * v[2 * e] + od * cm.x, -ev * v[2 * e + 1] + od * cm.y);
                    } else {
                        z[i] = make_float2(v[2 * e] * P, -v[2 * e + 1] * P);
                    }
                }
                const int kc = kCW * hh + 16 * c8;
                put4<PREC>(xhi(sl), xlo(sl), kmaj(m, kc), z);
                put4<PREC>(xhi(sl), xlo(sl), kmaj(m, kc + 8), z + 4);
            }
        };
        // U_kk = conj(D) from slot sl: row m = item j of column b, columns
        // 2u' + c at ky = j + 64 u'. The lane pair swaps halves so each lane
        // writes both columns of a row (16 bytes, the group's whole share of
        // a block row): lane b = 0 the first half of its outputs u', lane
        // b = 1 the second.
        const auto output = [&](int kk, int sl) {
            float2* dst = U + size_t(kk) * size_t(M) * kH + gbase;
            float v[kCW];
            tmem_ld(wcol(sl) + quad + uint32_t(kCW * hh), v);
            constexpr int kH4 = kCW / 4;  // outputs per lane after the swap
#pragma unroll
            for (int i = 0; i < kH4; ++i) {
                const float sr = b ? v[2 * i] : v[2 * (kH4 + i)], si = b ? v[2 * i + 1] : v[2 * (kH4 + i) + 1];
                const float gr = __shfl_xor_sync(0xffffffffu, sr, 1), gi = __shfl_xor_sync(0xffffffffu, si, 1);
                const int e = b ? kH4 + i : i;  // u' = (kCW / 2) hh + e
                const float4 q = b ? make_float4(gr, -gi, v[2 * e], -v[2 * e + 1])
                                   : make_float4(v[2 * e], -v[2 * e + 1], gr, -gi);
                *reinterpret_cast<float4*>(dst + size_t(j + 64 * ((kCW / 2) * hh + e)) * KB) = q;
            }
        };
        // Inverse transforms of kernel kk on slot sl: first pass issued by
        // `first`, the second pass's operand built and issued by `second`.
        const auto first = [&](int kk, int sl) {
            product(kk, sl);
            return issue(sl, wcol(sl), a_fhi, a_flo, sx(sl), sxl(sl));
        };
        const auto second = [&](int sl) {
            second_pass_operand<PREC>(wcol(sl) + quad, tw, xhi(sl), xlo(sl), q4, hh, lane);
            return issue(sl, wcol(sl), sx(sl), sxl(sl), a_fhi, a_flo);
        };
        if constexpr (!PIPE) {
            for (int kk = 0; kk < nk; ++kk) {
                if (!(ok = first(kk, 0))) break;
                wait(0);
                if (!(ok = second(0))) break;
                wait(0);
                output(kk, 0);
            }
        } else {
            if (!(ok = first(0, 0))) break;
            if (nk > 1 && !(ok = first(1, 1))) break;
            for (int k = 0; k < nk; ++k) {
                const int sl = k & 1;
                wait(sl);  // kernel k's first pass
                if (!(ok = second(sl))) break;
                if (k >= 1) {
                    wait(sl ^ 1);  // kernel k - 1's second pass
                    output(k - 1, sl ^ 1);
                    if (k + 1 < nk && !(ok = first(k + 1, sl ^ 1))) break;
                }
            }
            if (ok) {
                wait((nk - 1) & 1);
                output(nk - 1, (nk - 1) & 1);
            }
        }
    }
    __syncthreads();
    if (*reinterpret_cast<volatile int*>(&stop)) ok = false;
    if (!ok) {
        // A wait ran out: count it once per CTA and give the MMAs still in
        // flight one more bounded wait before the tensor memory is freed.
        if (tid == 0 && err) atomicAdd(err, 1);
        for (int sl = 0; sl < 2; ++sl)
            if ((pending >> sl) & 1u) mbar_wait(&bars[sl], (phases >> sl) & 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
}

template <int PREC, bool PIPE>
cudaError_t launch_t(const FftGeometry& g, const float2* S, float2* U, int* err, cudaStream_t s) {
    auto fn = col_tc05_kernel<PREC, PIPE>;
    constexpr size_t smem = PIPE ? kSmem + 2 * size_t(kOp) : kSmem;
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    const int groups = g.M / kB;
    const int grid = std::max(1, std::min(groups, sms()));
    fn<<<grid, kT, smem, s>>>(S, U, g.khat, g.M, g.nk, err);
    return cudaGetLastError();
}

}  // namespace

bool tc05_col_plan(int H) { return H == kH; }

cudaError_t launch_col_tc05(const FftGeometry& g, int precision, bool pipelined, const float2* S, float2* U, int* err,
                            cudaStream_t s) {
    if (g.H != kH || g.M % KB != 0 || g.M <= 0) return cudaErrorNotSupported;
    if (precision == tcfft::kBF16x3)
        return pipelined ? launch_t<tcfft::kBF16x3, true>(g, S, U, err, s) : launch_t<tcfft::kBF16x3, false>(g, S, U, err, s);
    if (precision == tcfft::kFP16x3)
        return pipelined ? launch_t<tcfft::kFP16x3, true>(g, S, U, err, s) : launch_t<tcfft::kFP16x3, false>(g, S, U, err, s);
    return cudaErrorInvalidValue;
}

}  // namespace lenia
