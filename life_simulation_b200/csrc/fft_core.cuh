// life_simulation_b200/csrc/fft_core.cuh -- block-level mixed-radix FFT in
// shared memory.
//
// A transform of length N = r_0 * r_1 * ... runs as one Stockham autosort
// pass per factor (the radix-r generalisation of the radix-2 stage in
// Shaders/Common/FFT.metal:13-27): for j < N/r, m = j mod Ns,
//   v_t = x[j + t*N/r] * w_{Ns*r}^{m*t}   (t = 0..r-1)
//   V   = DFT_r(v)
//   y[(j - m)*r + m + t*Ns] = V_t,        Ns *= r
// so no digit-reversal pass is needed. Each pass reads one shared buffer and
// writes the other (ping-pong); a batch of independent transforms is spread
// over the whole block. The radix-r DFTs are straight-line register code
// whose constants are exact values of cos/sin at multiples of 2*pi/r
// (r = 2, 3, 4, 5, 8, 16). Twiddles come from an N-entry table of
// exp(-2*pi*i*t/N) evaluated in FP64 on the host and rounded once.
#pragma once
#include <cuda_runtime.h>

#include "lenia_kernels.h"

namespace lenia {
namespace fft {

// Complex arithmetic on float2 with the packed FP32x2 instructions of sm_100
// (one add/mul/fma per complex lane pair instead of two); each lane is an
// IEEE round-to-nearest operation, the same result as the scalar form.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(__fmaf_rn(-a.y, b.y, __fmul_rn(a.x, b.x)), __fmaf_rn(a.y, b.x, __fmul_rn(a.x, b.y)));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(__fmul_rn(a.x, s), __fmul_rn(a.y, s)); }
// -i*a (forward quarter turn) and +i*a.
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }
// Multiply by -i (forward) or +i (inverse).
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a) { return INV ? mul_pi(a) : mul_mi(a); }

// cos and sin of pi/4, pi/8, 3*pi/8; cos(2pi/3); sin(2pi/3); cos/sin(2pi/5),
// cos/sin(4pi/5).
constexpr float kS2 = 0.70710678118654752440f;
constexpr float kC8 = 0.92387953251128675613f;
constexpr float kS8 = 0.38268343236508977173f;
constexpr float kC3 = -0.5f;
constexpr float kS3 = 0.86602540378443864676f;
constexpr float kC51 = 0.30901699437494742410f;
constexpr float kC52 = -0.80901699437494742410f;
constexpr float kS51 = 0.95105651629515357212f;
constexpr float kS52 = 0.58778525229247312917f;

template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
    float2 t = cadd(v[1], v[2]);
    float2 d = csub(v[1], v[2]);
    float2 m = make_float2(__fmaf_rn(t.x, kC3, v[0].x), __fmaf_rn(t.y, kC3, v[0].y));
    v[0] = cadd(v[0], t);
    float2 r = rot90<INV>(cscale(d, kS3));  // -i*s*d forward
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* v) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2* v) {
    float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    float2 x0 = v[0];
    v[0] = cadd(x0, cadd(a1, a2));
    const auto fma2 = [](float2 a, float k, float2 c) { return make_float2(__fmaf_rn(a.x, k, c.x), __fmaf_rn(a.y, k, c.y)); };
    float2 c1 = fma2(a2, kC52, fma2(a1, kC51, x0));
    float2 c2 = fma2(a2, kC51, fma2(a1, kC52, x0));
    float2 s1 = rot90<INV>(fma2(b2, kS52, cscale(b1, kS51)));
    float2 s2 = rot90<INV>(fma2(b2, -kS51, cscale(b1, kS52)));
    v[1] = cadd(c1, s1);
    v[4] = csub(c1, s1);
    v[2] = cadd(c2, s2);
    v[3] = csub(c2, s2);
}

// w_8^k for k = 1, 2, 3 applied to b (forward w = exp(-i*pi/4)).
template <bool INV>
__device__ __forceinline__ float2 w8_1(float2 b) {
    // forward: sqrt(1/2) * (b.x + b.y, b.y - b.x); inverse: sqrt(1/2) * (b.x - b.y, b.x + b.y)
    const float2 s = INV ? make_float2(__fsub_rn(b.x, b.y), __fadd_rn(b.x, b.y))
                         : make_float2(__fadd_rn(b.x, b.y), __fsub_rn(b.y, b.x));
    return make_float2(__fmul_rn(s.x, kS2), __fmul_rn(s.y, kS2));
}
template <bool INV>
__device__ __forceinline__ float2 w8_3(float2 b) {
    // forward: sqrt(1/2) * (b.y - b.x, -(b.x + b.y)); inverse: sqrt(1/2) * (-(b.x + b.y), b.x - b.y)
    const float2 s = INV ? make_float2(-__fadd_rn(b.x, b.y), __fsub_rn(b.x, b.y))
                         : make_float2(__fsub_rn(b.y, b.x), -__fadd_rn(b.x, b.y));
    return make_float2(__fmul_rn(s.x, kS2), __fmul_rn(s.y, kS2));
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<INV>(e);
    dft4<INV>(o);
    o[1] = w8_1<INV>(o[1]);
    o[2] = rot90<INV>(o[2]);
    o[3] = w8_3<INV>(o[3]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = cadd(e[k], o[k]);
        v[k + 4] = csub(e[k], o[k]);
    }
}

template <bool INV>
__device__ __forceinline__ void dft16(float2* v) {
    float2 e[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        e[k] = v[2 * k];
        o[k] = v[2 * k + 1];
    }
    dft8<INV>(e);
    dft8<INV>(o);
    // w_16^k, k = 0..7 (forward exp(-i*pi*k/8)).
    const float c[8] = {1.0f, kC8, kS2, kS8, 0.0f, -kS8, -kS2, -kC8};
    const float s[8] = {0.0f, kS8, kS2, kC8, 1.0f, kC8, kS2, kS8};
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        float2 w = make_float2(c[k], INV ? s[k] : -s[k]);
        o[k] = cmul(o[k], w);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[k] = cadd(e[k], o[k]);
        v[k + 8] = csub(e[k], o[k]);
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v[0], v[1]);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
}

// One Stockham pass of radix R over `batch` transforms of length N laid out
// back to back (transform b at in + b*N). tw: N-entry forward table.
template <int R, bool INV>
__device__ __forceinline__ void pass(const float2* __restrict__ in, float2* __restrict__ out,
                                     int N, int Ns, int batch, const float2* __restrict__ tw) {
    const int NR = N / R;
    const int tstep = N / (Ns * R);
    const int total = batch * NR;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int b = q / NR;
        const int j = q - b * NR;
        const int m = j % Ns;
        const float2* ib = in + b * N;
        float2 v[R];
#pragma unroll
        for (int t = 0; t < R; ++t) v[t] = ib[j + t * NR];
        if (Ns > 1) {
#pragma unroll
            for (int t = 1; t < R; ++t) {
                float2 w = tw[m * t * tstep];
                if (INV) w.y = -w.y;
                v[t] = cmul(v[t], w);
            }
        }
        dft<R, INV>(v);
        float2* ob = out + b * N + (j - m) * R + m;
#pragma unroll
        for (int t = 0; t < R; ++t) ob[t * Ns] = v[t];
    }
}

// All passes of `plan` over `batch` transforms held in buffer a (b is the
// ping-pong partner). Returns the buffer holding the result. Every pass is
// followed by a block barrier; the caller must have synchronised before.
template <bool INV>
__device__ float2* run(float2* a, float2* b, const FftPlan& plan, int batch,
                       const float2* __restrict__ tw) {
    int Ns = 1;
    for (int p = 0; p < plan.npass; ++p) {
        const int R = plan.radix[p];
        switch (R) {
        case 2: pass<2, INV>(a, b, plan.n, Ns, batch, tw); break;
        case 3: pass<3, INV>(a, b, plan.n, Ns, batch, tw); break;
        case 4: pass<4, INV>(a, b, plan.n, Ns, batch, tw); break;
        case 5: pass<5, INV>(a, b, plan.n, Ns, batch, tw); break;
        case 8: pass<8, INV>(a, b, plan.n, Ns, batch, tw); break;
        case 16: pass<16, INV>(a, b, plan.n, Ns, batch, tw); break;
        default: break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace fft
}  // namespace lenia
