// life_simulation_b200/csrc/fft_tc.cuh -- radix-16 FFT passes on the tensor
// cores with split precision (BF16 or FP16 hi/lo operands, FP32 accumulation).
//
// One radix-16 Stockham pass computes, per item, y = F16 (w .* x) for 16
// complex inputs x (twiddles w, then the 16-point DFT). Eight items of a warp
// form the B operand of mma.m16n8k16 (K = 16 inputs, N = 8 items); the DFT
// matrix F = C + iS is the constant A operand, kept in registers for the
// whole kernel. In real arithmetic
//     y_re = C x_re - S x_im,   y_im = S x_re + C x_im,
// and every product is taken in split precision: a = a_hi + a_lo with a_hi
// the 16-bit rounding of a and a_lo the rounding of the remainder, and
//     A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi      (FP32 accumulators)
// which keeps ~16 (BF16) or ~22 (FP16) significant bits of every product;
// 12 MMAs per 8 items. Twiddles are applied in FP32 on the CUDA cores before
// the split. F is scaled by 1/16 (exact in both formats) so that every stage
// of a transform keeps the magnitudes of its input (FP16's range).
//
// Fragment layouts (PTX ISA, mma.m16n8k16 .bf16/.f16): with g = lane / 4 and
// q = lane % 4, A register r holds (row, col) = (g + 8 (r & 1), 2q + 8 (r >> 1))
// and the next column; B register r holds (k, n) = (2q + 8r, g) and (2q + 8r
// + 1, g); accumulator r holds (g + 8 (r >> 1), 2q + (r & 1)). The lower 16
// bits of a register hold the element with the smaller index.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fft_ct.cuh"

namespace lenia {
namespace tcfft {

using namespace fftct;

enum Precision { kBF16x3 = 1, kFP16x3 = 2 };

// (cos, -sin)(2 pi t / 16), t < 16, from the constexpr trig of fft_ct.cuh.
#define LENIA_TW16(t) {float(cs2pi(t, 16).c), float(-cs2pi(t, 16).s)}
static __constant__ float2 kTw16[16] = {
    LENIA_TW16(0),  LENIA_TW16(1),  LENIA_TW16(2),  LENIA_TW16(3),  LENIA_TW16(4),  LENIA_TW16(5),
    LENIA_TW16(6),  LENIA_TW16(7),  LENIA_TW16(8),  LENIA_TW16(9),  LENIA_TW16(10), LENIA_TW16(11),
    LENIA_TW16(12), LENIA_TW16(13), LENIA_TW16(14), LENIA_TW16(15)};
#undef LENIA_TW16

// Split a pair (a, b) into packed hi and lo 16-bit pairs (a in the low half).
template <int PREC>
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    if constexpr (PREC == kBF16x3) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    } else {
        const __half2 h = __floats2half2_rn(a, b);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    }
}

// d += A B for one m16n8k16 tile (FP32 accumulators).
template <int PREC>
__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    if constexpr (PREC == kBF16x3) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    } else {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
}

// This lane's A fragments of (C, S, -S) / 16 for the 16-point DFT, hi and lo.
template <int PREC, bool INV>
struct Dft16 {
    uint32_t c_hi[4], c_lo[4], s_hi[4], s_lo[4], n_hi[4], n_lo[4];
    __device__ __forceinline__ void init() {
        const int lane = int(threadIdx.x & 31u), g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int row = g + 8 * (r & 1), col = 2 * q + 8 * (r >> 1);
            float c[2], s[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float2 w = kTw16[(row * (col + e)) & 15];
                c[e] = w.x * 0.0625f;
                s[e] = (INV ? -w.y : w.y) * 0.0625f;
            }
            split2<PREC>(c[0], c[1], c_hi[r], c_lo[r]);
            split2<PREC>(s[0], s[1], s_hi[r], s_lo[r]);
            split2<PREC>(-s[0], -s[1], n_hi[r], n_lo[r]);
        }
    }
};

// One radix-16 pass (pass PASS of plan P, all of whose radices are 16) over
// a batch of B transforms, items q -> (b = q % B, j = q / B) as in the
// CUDA-core passes; src(b, i) / dst(b, i, v) address element i of transform
// b. tw: the plan's per-pass twiddle table (global memory). Every thread of
// the block calls it; warps take chunks of 8 items.
template <class P, int PASS, bool INV, int PREC, int B, int T, class Src, class Dst>
__device__ __forceinline__ void pass16(Src&& src, Dst&& dst, const float2* __restrict__ tw,
                                       const Dft16<PREC, INV>& F, int cols) {
    using I = PassIdx<P, PASS>;
    static_assert(I::R == 16, "tensor-core passes are radix 16");
    constexpr int ITEMS = B * I::NR;
    static_assert(ITEMS % 8 == 0, "whole chunks of 8 items");
    constexpr int CHUNKS = ITEMS / 8;
    const int lane = int(threadIdx.x & 31u), warp = int(threadIdx.x >> 5), g = lane >> 2, q = lane & 3;
    for (int c = warp; c < CHUNKS; c += T / 32) {
        const int n = 8 * c + g;
        const int bi = n % B, j = n / B;
        const int ks[4] = {2 * q, 2 * q + 1, 2 * q + 8, 2 * q + 9};
        float2 x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) x[e] = bi < cols ? src(bi, I::in(j, ks[e])) : make_float2(0.0f, 0.0f);
        if constexpr (I::NS > 1) {
            const int m = j % I::NS;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if (ks[e] == 0) continue;
                float2 w = __ldg(tw + I::TWO + (ks[e] - 1) * I::NS + m);
                if (INV) w.y = -w.y;
                x[e] = make_float2(x[e].x * w.x - x[e].y * w.y, x[e].x * w.y + x[e].y * w.x);
            }
        }
        uint32_t rh[2], rl[2], ih[2], il[2];
        split2<PREC>(x[0].x, x[1].x, rh[0], rl[0]);
        split2<PREC>(x[2].x, x[3].x, rh[1], rl[1]);
        split2<PREC>(x[0].y, x[1].y, ih[0], il[0]);
        split2<PREC>(x[2].y, x[3].y, ih[1], il[1]);
        float dr[4] = {0.0f, 0.0f, 0.0f, 0.0f}, di[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        mma<PREC>(dr, F.c_hi, rh[0], rh[1]);
        mma<PREC>(dr, F.c_hi, rl[0], rl[1]);
        mma<PREC>(dr, F.c_lo, rh[0], rh[1]);
        mma<PREC>(dr, F.n_hi, ih[0], ih[1]);
        mma<PREC>(dr, F.n_hi, il[0], il[1]);
        mma<PREC>(dr, F.n_lo, ih[0], ih[1]);
        mma<PREC>(di, F.s_hi, rh[0], rh[1]);
        mma<PREC>(di, F.s_hi, rl[0], rl[1]);
        mma<PREC>(di, F.s_lo, rh[0], rh[1]);
        mma<PREC>(di, F.c_hi, ih[0], ih[1]);
        mma<PREC>(di, F.c_hi, il[0], il[1]);
        mma<PREC>(di, F.c_lo, ih[0], ih[1]);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int n2 = 8 * c + 2 * q + e;
            const int b2 = n2 % B, j2 = n2 / B;
            if (b2 >= cols) continue;
            const int ob = I::out_base(j2);
            dst(b2, ob + g * I::NS, make_float2(dr[e], di[e]));
            dst(b2, ob + (g + 8) * I::NS, make_float2(dr[2 + e], di[2 + e]));
        }
    }
}

}  // namespace tcfft
}  // namespace lenia
