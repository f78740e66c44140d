// life_simulation_b200/csrc/fft_ct.cuh -- compile-time FFT building blocks:
// radix-r DFT codelets in registers and the index algebra of a Stockham
// pass whose length, radix and span are template constants.
//
// Codelets exist for r = 2, 3, 4, 5, 6, 8, 9, 10, 12, 15, 16. Composite
// radices are built as a two-level Cooley-Tukey split in registers,
// r = A*B:  Y[n2][k1] = DFT_A(v[B*n1 + n2]) * w_r^(n2*k1),
//           X[k1 + A*k2] = DFT_B(Y[.][k1]),
// whose internal twiddles are compile-time constants: cos/sin of 2*pi*p/q
// evaluated in double by a constexpr series (exact octant reduction, then a
// Taylor series on [0, pi/4)) and rounded once to float.
#pragma once
#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace lenia {
namespace fftct {

using fft::cadd;
using fft::cmul;
using fft::cscale;
using fft::csub;

// ----------------------------------------------------- constexpr trig

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kSqrtHalf = 0.70710678118654752440084436210484904;

constexpr double taylor_sin(double x) {
    double x2 = x * x, term = x, sum = x;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / double((2 * n) * (2 * n + 1));
        sum += term;
    }
    return sum;
}
constexpr double taylor_cos(double x) {
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / double((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sum;
}

// cos and sin of 2*pi*p/q for integers p, q > 0.
struct CS {
    double c, s;
};
constexpr CS cs2pi(long p, long q) {
    p %= q;
    if (p < 0) p += q;
    const long o = (8 * p) / q;      // octant 0..7
    const long rem = 8 * p - o * q;  // angle = o*pi/4 + 2*pi*rem/(8q)
    const double th = 2.0 * kPi * double(rem) / double(8 * q);
    const double c = taylor_cos(th), s = taylor_sin(th);
    // cos/sin(o*pi/4 + th) from the octant's exact cos/sin.
    const double oc[8] = {1.0, kSqrtHalf, 0.0, -kSqrtHalf, -1.0, -kSqrtHalf, 0.0, kSqrtHalf};
    const double os[8] = {0.0, kSqrtHalf, 1.0, kSqrtHalf, 0.0, -kSqrtHalf, -1.0, -kSqrtHalf};
    return CS{oc[o] * c - os[o] * s, os[o] * c + oc[o] * s};
}

// w_q^(p) of the transform direction: exp(-2 pi i p / q) forward,
// exp(+2 pi i p / q) inverse.
template <long P, long Q, bool INV>
struct Tw {
    static constexpr CS v = cs2pi(P, Q);
    static constexpr float re = float(v.c);
    static constexpr float im = INV ? float(v.s) : float(-v.s);
};

template <long P, long Q, bool INV>
__device__ __forceinline__ float2 twmul(float2 a) {
    constexpr long p = ((P % Q) + Q) % Q;
    if constexpr (p == 0) {
        return a;
    } else if constexpr (4 * p == Q) {  // quarter turn
        return INV ? fft::mul_pi(a) : fft::mul_mi(a);
    } else if constexpr (2 * p == Q) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * p == 3 * Q) {
        return INV ? fft::mul_mi(a) : fft::mul_pi(a);
    } else {
        constexpr float wr = Tw<p, Q, INV>::re, wi = Tw<p, Q, INV>::im;
        return make_float2(__fmaf_rn(a.y, -wi, __fmul_rn(a.x, wr)), __fmaf_rn(a.y, wr, __fmul_rn(a.x, wi)));
    }
}

// ------------------------------------------------------------ codelets

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<1, INV> {
    __device__ __forceinline__ static void run(float2*) {}
};
template <bool INV>
struct Dft<2, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft2<INV>(v[0], v[1]); }
};
template <bool INV>
struct Dft<3, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft3<INV>(v); }
};
template <bool INV>
struct Dft<4, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft4<INV>(v); }
};
template <bool INV>
struct Dft<5, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft5<INV>(v); }
};
template <bool INV>
struct Dft<8, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft8<INV>(v); }
};
template <bool INV>
struct Dft<16, INV> {
    __device__ __forceinline__ static void run(float2* v) { fft::dft16<INV>(v); }
};

// Two-level split R = A*B (n = B*n1 + n2, k = k1 + A*k2).
template <int A, int B, bool INV>
struct DftSplit {
    static constexpr int R = A * B;
    template <int N2>
    __device__ __forceinline__ static void inner(float2* v, float2 (&y)[B][A]) {
        if constexpr (N2 < B) {
            float2 t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + N2];
            Dft<A, INV>::run(t);
            tw_row<N2, 0>(t, y);
            inner<N2 + 1>(v, y);
        }
    }
    template <int N2, int K1>
    __device__ __forceinline__ static void tw_row(const float2* t, float2 (&y)[B][A]) {
        if constexpr (K1 < A) {
            y[N2][K1] = twmul<long(N2) * K1, R, INV>(t[K1]);
            tw_row<N2, K1 + 1>(t, y);
        }
    }
    __device__ __forceinline__ static void run(float2* v) {
        float2 y[B][A];
        inner<0>(v, y);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 t[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2][k1];
            Dft<B, INV>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
        }
    }
};

template <bool INV>
struct Dft<6, INV> : DftSplit<2, 3, INV> {};
template <bool INV>
struct Dft<9, INV> : DftSplit<3, 3, INV> {};
template <bool INV>
struct Dft<10, INV> : DftSplit<2, 5, INV> {};
template <bool INV>
struct Dft<12, INV> : DftSplit<4, 3, INV> {};
template <bool INV>
struct Dft<15, INV> : DftSplit<3, 5, INV> {};

// ------------------------------------------------------------- plans

// A transform of length N = product of Rs, one Stockham pass per radix.
template <int... Rs>
struct Plan {
    static_assert(sizeof...(Rs) > 0, "a plan needs at least one pass");
    static constexpr int np = int(sizeof...(Rs));
    static constexpr int r[np] = {Rs...};
    static constexpr int n = (1 * ... * Rs);
    static constexpr int radix(int p) { return r[p]; }
    static constexpr int span(int p) {
        int s = 1;
        for (int i = 0; i < p; ++i) s *= r[i];
        return s;
    }
    // Offset of pass p's twiddle block in the per-plan table (passes >= 1;
    // block p holds w_{span*r}^(m*t) at [(t-1)*span + m]).
    static constexpr int tw_offset(int p) {
        int o = 0;
        for (int i = 1; i < p; ++i) o += span(i) * (r[i] - 1);
        return o;
    }
    static constexpr int tw_size() { return tw_offset(np); }
    static constexpr int last() { return r[np - 1]; }
    static constexpr int first() { return r[0]; }
};

template <int... Xs>
struct Seq {};

template <class Acc, int... Xs>
struct RevImpl;
template <int... Acc>
struct RevImpl<Seq<Acc...>> {
    using type = Plan<Acc...>;
};
template <int... Acc, int X, int... Xs>
struct RevImpl<Seq<Acc...>, X, Xs...> {
    using type = typename RevImpl<Seq<X, Acc...>, Xs...>::type;
};

// The plan with its passes in the opposite order: the inverse of a
// transform whose last pass leaves item j's outputs at j + t*N/R then reads
// exactly those elements in its first pass (same radix R).
template <class P>
struct Reverse;
template <int... Rs>
struct Reverse<Plan<Rs...>> {
    using type = typename RevImpl<Seq<>, Rs...>::type;
};

// Index algebra of pass p of plan P: item j of a transform reads
// x[j + t*N/R] and writes y[(j - m)*R + m + t*Ns] (m = j mod Ns).
template <class P, int PASS>
struct PassIdx {
    static constexpr int N = P::n;
    static constexpr int R = P::radix(PASS);
    static constexpr int NS = P::span(PASS);
    static constexpr int NR = N / R;
    static constexpr int TWO = P::tw_offset(PASS);
    __device__ __forceinline__ static int in(int j, int t) { return j + t * NR; }
    __device__ __forceinline__ static int out_base(int j) {
        const int m = j % NS;
        return (j - m) * R + m;
    }
    // Twiddles of the pass applied to v (no-op for the first pass).
    template <bool INV>
    __device__ __forceinline__ static void twiddle(float2* v, int j, const float2* __restrict__ tw) {
        if constexpr (NS > 1) {
            const int m = j % NS;
#pragma unroll
            for (int t = 1; t < R; ++t) {
                float2 w = tw[TWO + (t - 1) * NS + m];
                if (INV) w.y = -w.y;
                v[t] = cmul(v[t], w);
            }
        }
    }
};

}  // namespace fftct
}  // namespace lenia
