// life_simulation_b200/csrc/lenia_batch_persistent.cu -- the batched form's
// substep as ONE persistent launch over a device work list (the reference
// steps its sweep variants one SceneRunner at a time,
// Apps/LifePresetLab/main.cpp:718-795).
//
// Work items (PersistItem): a column group of one spectral world (forward
// column FFT, spectrum product, inverse), a row group of one spectral world
// (inverse row FFT, growth, Euler step, clip, forward row FFT of A'), or a
// 64x32 output tile of one direct world. Every CTA (256 threads) claims
// items in list order from a device counter and runs the body compiled for
// the item's field size; the list holds every column item first, then the
// direct tiles, then the row items, so a row item only ever waits for
// column items that running CTAs have already claimed (no deadlock, however
// many CTAs are resident). A row item waits -- one thread polling an
// acquire load, bounded, with a device error flag when the bound runs out --
// until its world's column items are all done; worlds never wait on each
// other, so column work of one world overlaps row work of another and the
// size classes share one grid.
//
// Bodies are the compile-time-plan passes of lenia_fft_fast.cu re-shaped for
// a fixed CTA of 256 threads: columns (rows) per item chosen per size so an
// item's last pass has about one element group per thread. They compute the
// same operations in the same order as those passes (same plans, same
// twiddle tables). A CTA stages the twiddle tables of an item's shape in
// shared memory and keeps them while the next items have the same shape (the
// list keeps a size class's items together). An item covers a few
// consecutive groups of one world, so its set-up (descriptor, world entry,
// dependency check) is shared by them. Each spectral body is a
// separate (non-inlined) function: inlined into one kernel, the bodies'
// register demands add up (the row bodies alone reach 230 registers), while
// called they are allocated one at a time within the kernel's 128.
//
// Per launch: counter set `par` (two sets alternate with the table parity;
// block 0 clears the other set for the next launch), and the last CTA to
// finish advances every world's frame index and substep seed, so a captured
// graph of k substeps is k kernel nodes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "direct_tile.cuh"
#include "fft_ct.cuh"
#include "fft_fast_common.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

using fft::cadd;
using fft::cconj;
using fft::cscale;
using namespace fftct;

namespace {

using namespace fastfft;

constexpr int kPT = kPersistThreads;  // threads per CTA
// Polls of a row item's dependency counter before it gives up (about a
// second with the back-off; a healthy device needs a few microseconds).
constexpr uint32_t kPersistPolls = 1u << 22;

// Column bodies (length, columns per item, forward plan = the catalogue's)
// and row bodies (length, rows per item, inverse plan).
#define LENIA_PERSIST_COLS(X)  \
    X(64, 32, Plan<8, 8>)      \
    X(128, 16, Plan<16, 8>)    \
    X(216, 7, Plan<6, 6, 6>)   \
    X(256, 16, Plan<16, 16>)   \
    X(512, 4, Plan<8, 8, 8>)   \
    X(1024, 2, Plan<16, 8, 8>)
#define LENIA_PERSIST_ROWS(X)  \
    X(64, 32, Plan<8, 8>)      \
    X(128, 16, Plan<16, 8>)    \
    X(192, 10, Plan<8, 3, 8>)  \
    X(256, 8, Plan<8, 4, 8>)   \
    X(512, 4, Plan<8, 8, 8>)

// Twiddle tables of a body, staged in shared memory while consecutive items
// have the same shape (the work list keeps a size class's items together).
template <class PF>
constexpr int col_tables() {
    return PF::tw_size() + Reverse<PF>::type::tw_size();
}
template <class PI>
constexpr int row_tables() {
    return PI::n + 1 + PI::tw_size() + Reverse<PI>::type::tw_size();
}
constexpr int tables_max() {
    int m = 0;
#define X(h, B, ...) m = m > col_tables<__VA_ARGS__>() ? m : col_tables<__VA_ARGS__>();
    LENIA_PERSIST_COLS(X)
#undef X
#define X(mm, RB, ...) m = m > row_tables<__VA_ARGS__>() ? m : row_tables<__VA_ARGS__>();
    LENIA_PERSIST_ROWS(X)
#undef X
    return (m + 15) / 16 * 16;  // the body buffers after it stay 128-byte aligned
}
constexpr int kTables = tables_max();

template <class PF, int B>
struct PCol {
    using PI = typename Reverse<PF>::type;
    static constexpr int H = PF::n, RL = PF::last(), NRL = H / RL, Hh = H / 2 + 1;
    static constexpr int PITCH = row_pitch(H);
    static constexpr int ITL = (B * NRL + kPT - 1) / kPT;
    static constexpr size_t smem = sizeof(float2) * (2 * size_t(B) * PITCH + H);
};
template <class PI, int RB>
struct PRow {
    using PF = typename Reverse<PI>::type;
    static constexpr int M = PI::n, RC = PI::last(), NRC = M / RC;
    static constexpr int PITCH = row_pitch(M);
    static constexpr int ITL = (RB * NRC + kPT - 1) / kPT;
    static constexpr size_t smem = sizeof(float2) * 3 * size_t(RB) * PITCH;
};

// Column group [k0, k0 + B) of one world: forward FFT of the columns of S,
// per kernel the product with its real spectrum and the inverse FFT into
// U_k. The same steps as col_fast_kernel's loop body (its non-staged form).
template <class PF, int B>
__device__ __noinline__ void col_item(const SpectralWorld& sw, int k0, const float2* __restrict__ twf,
                                         const float2* __restrict__ twi, float2* sm) {
    using K = PCol<PF, B>;
    using PI = typename K::PI;
    using IL = PassIdx<PF, PF::np - 1>;
    constexpr int H = K::H, RL = K::RL, NRL = K::NRL, Hh = K::Hh, PITCH = K::PITCH, ITL = K::ITL;
    float2* ba = sm;
    float2* bb = ba + B * PITCH;
    float2* c0 = bb + B * PITCH;
    const float2* __restrict__ S = sw.S;
    float2* __restrict__ U = sw.U;
    const float* __restrict__ khat = sw.khat;
    const int M = sw.M, nk = sw.nk;
    const int cols = min(B, M - k0);
    // Element (column k0 + b, row i) of a blocked plane (a group may span
    // several blocks of KB columns).
    const auto at = [&](int b, int i) {
        const int c = k0 + b;
        return size_t(c / KB) * H * KB + size_t(i) * KB + size_t(c % KB);
    };
    int jj[ITL], bi[ITL];
    bool ok[ITL];
#pragma unroll
    for (int it = 0; it < ITL; ++it) {
        const int q = int(threadIdx.x) + it * kPT;
        jj[it] = q / B;
        bi[it] = q - jj[it] * B;
        ok[it] = q < B * NRL && bi[it] < cols;
    }
    // S was written by the previous launch's row items; loads at L2.
    pass_gen<PF, 0, false, B, kPT>([&](int b, int i) { return __ldcg(S + at(b, i)); },
                                   [&](int b, int i, float2 v) { ba[b * PITCH + i] = v; }, twf, cols);
    __syncthreads();
    float2* X = mid_passes<PF, 1, PF::np - 1, false, B, kPT, PITCH>(ba, bb, twf, cols);
    float2* Y = (PF::np - 2) % 2 ? ba : bb;
    float2 C[ITL][RL];
#pragma unroll
    for (int it = 0; it < ITL; ++it) {
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
    const auto first_inverse = [&](int kk) {
        const float* kh = khat + size_t(kk) * (M + 1) * Hh;
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            if (!ok[it]) continue;
            const int kx = k0 + bi[it];
            float2 D[RL];
#pragma unroll
            for (int t = 0; t < RL; ++t) {
                const int ky = jj[it] + t * NRL;
                const int kyr = min(ky, H - ky);
                const float kval = __ldg(kh + size_t(kx) * Hh + kyr);
                if (kx == 0) {
                    const float P = kval, Q = __ldg(kh + size_t(M) * Hh + kyr);
                    const float2 Cm = cconj(c0[ky == 0 ? 0 : H - ky]);
                    D[t] = cadd(cscale(C[it][t], 0.5f * (P + Q)), cscale(Cm, 0.5f * (P - Q)));
                } else {
                    D[t] = cscale(C[it][t], kval);
                }
            }
            Dft<RL, true>::run(D);
#pragma unroll
            for (int t = 0; t < RL; ++t) Y[bi[it] * PITCH + jj[it] * RL + t] = D[t];
        }
    };
    const auto last_inverse = [&](int kk, const float2* Z) {
        float2* dst = U + size_t(kk) * M * H;
        pass_gen<PI, PI::np - 1, true, B, kPT>([&](int b, int i) { return Z[b * PITCH + i]; },
                                               [&](int b, int i, float2 v) { dst[at(b, i)] = v; }, twi, cols);
    };
    constexpr bool kMerge = (PI::np - 2) % 2 == 1;
    if (nk > 0) first_inverse(0);
    for (int kk = 0; kk < nk; ++kk) {
        __syncthreads();  // Y holds kernel kk's first pass
        float2* Z = mid_passes<PI, 1, PI::np - 1, true, B, kPT, PITCH>(Y, X, twi, cols);
        last_inverse(kk, Z);
        if (kk + 1 < nk) {
            if constexpr (!kMerge) __syncthreads();
            first_inverse(kk + 1);
        }
    }
    __syncthreads();
}

// Row group [y0, y0 + RB) of one world: per kernel the inverse row FFT of
// U_k and the growth sums, then the Euler step, clip and store of A', and
// the forward row FFT of A' into S_next. The same steps as row_fast_kernel's
// loop body; the rows of A are staged while U_0's rows are transformed.
template <class PI, int RB>
__device__ __noinline__ void row_item(const SpectralWorld& sw, int y0, const float2* __restrict__ twr,
                                         const float2* __restrict__ twi, const float2* __restrict__ twf,
                                         float2* sm) {
    using K = PRow<PI, RB>;
    using PF = typename K::PF;
    using IL = PassIdx<PI, PI::np - 1>;
    constexpr int M = K::M, W = 2 * M, RC = K::RC, NRC = K::NRC, PITCH = K::PITCH, ITL = K::ITL;
    float2* sU = sm;
    float2* sA = sU + RB * PITCH;
    float2* bw = sA + RB * PITCH;
    const float2* __restrict__ U = sw.U;
    float* __restrict__ A_out = sw.A_out;
    float2* __restrict__ S_next = sw.S_next;
    const StepParams& p = sw.p;
    const int H = int(p.height), nk = sw.nk;
    const int rows = min(RB, H - y0);
    const bool asym = p.growth_mode == 1u;
    const bool jitter = p.mu_jitter > 0.0f;
    const bool extras = p.noise_amount > 0.0f || p.inject_amount > 0.0f;
    const float dt = p.dt, sum_w = p.sum_weights;
    const bool sw_ok = sum_w > 1e-6f;
    if (nk > 0) stage_rows<M, RB, kPT, PITCH>(sU, U, H, y0, rows);
    cp_async_commit();
    stage_field_rows<M, RB, kPT, PITCH>(sA, sw.A, y0, rows);
    cp_async_commit();
    int jj[ITL], bi[ITL];
    bool ok[ITL];
#pragma unroll
    for (int it = 0; it < ITL; ++it) {
        const int q = int(threadIdx.x) + it * kPT;
        jj[it] = q / RB;
        bi[it] = q - jj[it] * RB;
        ok[it] = q < RB * NRC && bi[it] < rows;
    }
    float2 acc[ITL][RC];  // growth sums of the pixel pair (2n, 2n + 1)
    for (int kk = 0; kk < nk; ++kk) {
        if (kk == 0) {
            cp_async_wait_prev();  // U_0's rows (A's may still be in flight)
        } else {
            stage_rows<M, RB, kPT, PITCH>(sU, U + size_t(kk) * M * H, H, y0, rows);
            cp_async_commit();
            cp_async_wait_all();
        }
        __syncthreads();
        pass_gen<PI, 0, true, RB, kPT>([&](int b, int i) { return c2r_split<M>(sU + b * PITCH, twr, i); },
                                       [&](int b, int i, float2 v) { bw[b * PITCH + i] = v; }, twi, rows);
        __syncthreads();
        float2* X = mid_passes<PI, 1, PI::np - 1, true, RB, kPT, PITCH>(bw, sU, twi, rows);
        const auto pick = [&](const float(&a)[kMaxKernels]) {
            return kk == 0 ? a[0] : kk == 1 ? a[1] : kk == 2 ? a[2] : a[3];
        };
        const GrowthPair gp(pick(p.mu), 1.0f / pick(p.sigma), pick(p.weight), asym);
#pragma unroll
        for (int it = 0; it < ITL; ++it) {
            if (!ok[it]) continue;
            float2 z[RC];
#pragma unroll
            for (int t = 0; t < RC; ++t) z[t] = X[bi[it] * PITCH + IL::in(jj[it], t)];
            IL::template twiddle<true>(z, jj[it], twi);
            Dft<RC, true>::run(z);
            const uint32_t gy = uint32_t(y0 + bi[it]);
#pragma unroll
            for (int t = 0; t < RC; ++t) {
                const float2 c = gp.term(z[t], p, jitter, uint32_t(2 * (jj[it] + t * NRC)), gy);
                acc[it][t] = kk == 0 ? c : __fadd2_rn(acc[it][t], c);
            }
        }
        __syncthreads();  // sU and X read before sU is staged again
    }
    cp_async_wait_all();
    __syncthreads();  // A's rows visible
    float2 za[ITL][RC];
#pragma unroll
    for (int it = 0; it < ITL; ++it) {
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
            const auto finish = [&](float A, float s, uint32_t gx) {
                if (extras) return growth_finish_call(p, A, s, s, gx, uint32_t(gy));
                const float A2 = asym ? A + dt * ((sw_ok ? s / sum_w : A) - A) : A + dt * s;
                return fminf(fmaxf(A2, 0.0f), 1.0f);
            };
            const float2 r = make_float2(finish(a.x, acc[it][t].x, uint32_t(2 * n)),
                                         finish(a.y, acc[it][t].y, uint32_t(2 * n + 1)));
            *reinterpret_cast<float2*>(A_out + size_t(gy) * W + 2 * n) = r;
            za[it][t] = r;
        }
    }
    if (S_next == nullptr) {
        __syncthreads();
        return;
    }
#pragma unroll
    for (int it = 0; it < ITL; ++it) {
        if (!ok[it]) continue;
        Dft<RC, false>::run(za[it]);
#pragma unroll
        for (int t = 0; t < RC; ++t) bw[bi[it] * PITCH + jj[it] * RC + t] = za[it][t];
    }
    __syncthreads();
    float2* Y = mid_passes<PF, 1, PF::np - 1, false, RB, kPT, PITCH>(bw, sA, twf, rows);
    float2* Zo = (PF::np - 2) % 2 ? bw : sA;
    pass_gen<PF, PF::np - 1, false, RB, kPT>([&](int b, int i) { return Y[b * PITCH + i]; },
                                              [&](int b, int i, float2 v) { Zo[b * PITCH + i] = v; }, twf, rows);
    __syncthreads();
    r2c_store_rows<M, RB, kPT, PITCH>(Zo, twr, S_next, H, y0, rows);
    __syncthreads();
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(uint32_t* p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// ctl layout per counter set: [0] next item, [1] CTAs finished, [2..] unused,
// [kPersistCtlHead + w] column items of world w done.
__global__ void __launch_bounds__(kPT, 2)
    persist_kernel(const PersistItem* __restrict__ items, int nitems, uint32_t* ctl, int nworlds, int par,
                   StepParams* const* loc, const uint32_t* __restrict__ base_seed, uint32_t* frame, int advance,
                   int* err) {
    extern __shared__ __align__(128) float2 psm[];
    __shared__ PersistItem s_it;
    __shared__ SpectralWorld s_sw;
    __shared__ DirectWorld s_dw;
    __shared__ int s_next, s_skip;
    float2* tab = psm;              // the current shape's twiddle tables
    float2* body = psm + kTables;   // the body's buffers
    int tab_kind = -1, tab_shape = -1;
    const int stride = kPersistCtlHead + nworlds;
    uint32_t* cs = ctl + size_t(par) * stride;
    if (blockIdx.x == 0) {
        // The other set is idle during this launch (the launches before and
        // after this one, which use it, are ordered by the stream).
        uint32_t* other = ctl + size_t(par ^ 1) * stride;
        for (int i = threadIdx.x; i < stride; i += kPT) other[i] = 0u;
    }
    if (threadIdx.x == 0) s_next = int(atomicAdd(cs, 1u));
    __syncthreads();
    int cur = s_next;
    while (cur < nitems) {
        if (threadIdx.x == 0) {
            s_it = items[cur];
            s_next = int(atomicAdd(cs, 1u));  // used after this item: its latency is hidden
            s_skip = 0;
        }
        __syncthreads();
        const int kind = s_it.kind;
        // The item's world entry (parameters and buffers) into shared memory.
        if (kind == kPersistDirect) {
            const uint32_t* src = static_cast<const uint32_t*>(s_it.world);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&s_dw);
            for (int i = threadIdx.x; i < int(sizeof(DirectWorld) / 4); i += kPT) dst[i] = src[i];
        } else {
            const uint32_t* src = static_cast<const uint32_t*>(s_it.world);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&s_sw);
            for (int i = threadIdx.x; i < int(sizeof(SpectralWorld) / 4); i += kPT) dst[i] = src[i];
        }
        if (kind == kPersistRow && threadIdx.x == 0) {
            const uint32_t* d = cs + kPersistCtlHead + s_it.world_id;
            uint32_t polls = 0;
            while (ld_acquire(d) < uint32_t(s_it.need)) {
                if (++polls > kPersistPolls) {
                    atomicExch(err, 1);
                    s_skip = 1;
                    break;
                }
                __nanosleep(200);
            }
        }
        __syncthreads();
        if (kind == kPersistCol) {
            switch (s_it.shape) {
#define X(h, B, ...)                                                               \
    case h: {                                                                    \
        using PF = __VA_ARGS__;                                                  \
        if (tab_kind != kind || tab_shape != h) {                                \
            copy_table(tab, s_it.tw0, PF::tw_size());                            \
            copy_table(tab + PF::tw_size(), s_it.tw1, Reverse<PF>::type::tw_size()); \
            tab_kind = kind;                                                     \
            tab_shape = h;                                                       \
            __syncthreads();                                                     \
        }                                                                        \
        for (int g = 0, k0 = s_it.group; g < s_it.count && k0 < s_sw.M; ++g, k0 += B) \
            col_item<PF, B>(s_sw, k0, tab, tab + PF::tw_size(), body);           \
        break;                                                                   \
    }
                LENIA_PERSIST_COLS(X)
#undef X
            default: break;
            }
            if (threadIdx.x == 0) {
                __threadfence();
                red_release_add(cs + kPersistCtlHead + s_it.world_id, 1u);
            }
        } else if (kind == kPersistRow) {
            if (!s_skip) {
                switch (s_it.shape) {
#define X(m, RB, ...)                                                                   \
    case m: {                                                                         \
        using PI = __VA_ARGS__;                                                       \
        constexpr int NI = PI::tw_size();                                             \
        if (tab_kind != kind || tab_shape != m) {                                     \
            copy_table(tab, s_it.tw2, m + 1);                                         \
            copy_table(tab + m + 1, s_it.tw0, NI);                                    \
            copy_table(tab + m + 1 + NI, s_it.tw1, Reverse<PI>::type::tw_size());     \
            tab_kind = kind;                                                          \
            tab_shape = m;                                                            \
            __syncthreads();                                                          \
        }                                                                             \
        for (int g = 0, y0 = s_it.group; g < s_it.count && y0 < int(s_sw.p.height); ++g, y0 += RB) \
            row_item<PI, RB>(s_sw, y0, tab, tab + m + 1, tab + m + 1 + NI, body);     \
        break;                                                                        \
    }
                    LENIA_PERSIST_ROWS(X)
#undef X
                default: break;
                }
            }
        } else {
            const int g = s_it.group;
            direct_tile<64, 32, 1, 1, 8, 1>(s_dw.src, s_dw.dst, s_dw.weights, s_dw.spans, s_dw.g, s_dw.p,
                                            (g & 0xFFFF) * 64, (g >> 16) * 32, nullptr, nullptr);
            tab_kind = -1;  // the tile overwrote the tables
        }
        cur = s_next;
        __syncthreads();  // s_it, s_sw, s_dw and the shared buffers free for the next item
    }
    // The last CTA to finish advances every world's frame index and substep
    // seed (pcgHash(seed ^ (frame * 197)), Modules/FieldModules/Lenia.cpp:564)
    // in both parity tables: every item of this launch has read them.
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(cs + 1, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && advance) {
        __threadfence();
        for (int i = threadIdx.x; i < nworlds; i += kPT) {
            const uint32_t f = frame[i] + 1u;
            frame[i] = f;
            const uint32_t seed = pcg_hash(base_seed[i] ^ (f * 197u));
            for (int k = 0; k < 2; ++k) {
                StepParams* q = loc[2 * i + k];
                q->frame_index = f;
                q->audio_frame = f;
                q->seed = seed;
            }
        }
    }
}

size_t direct_item_smem(int max_r) {
    if (max_r <= 0) return 0;
    DirectGeometry g{max_r, 2 * max_r + 1, (max_r + 3) / 4 * 4, 0};
    g.wp = 2 * g.xp + 8;
    return direct_smem_bytes(kDirectTile64x32, 1, g);
}

}  // namespace

int persist_col_group(int H) {
    switch (H) {
#define X(h, B, ...) \
    case h: return B;
        LENIA_PERSIST_COLS(X)
#undef X
    default: return 0;
    }
}

int persist_row_group(int M) {
    switch (M) {
#define X(m, RB, ...) \
    case m: return RB;
        LENIA_PERSIST_ROWS(X)
#undef X
    default: return 0;
    }
}

size_t persist_smem_bytes(const std::vector<int>& col_h, const std::vector<int>& row_m, int direct_max_r) {
    size_t s = direct_item_smem(direct_max_r), f = 0;
    for (int h : col_h) {
        switch (h) {
#define X(hh, B, ...) \
    case hh: f = std::max(f, PCol<__VA_ARGS__, B>::smem); break;
            LENIA_PERSIST_COLS(X)
#undef X
        default: break;
        }
    }
    for (int m : row_m) {
        switch (m) {
#define X(mm, RB, ...) \
    case mm: f = std::max(f, PRow<__VA_ARGS__, RB>::smem); break;
            LENIA_PERSIST_ROWS(X)
#undef X
        default: break;
        }
    }
    // Spectral bodies sit after the twiddle tables; a direct tile uses the whole
    // area from the start (and invalidates the tables).
    if (f > 0) s = std::max(s, sizeof(float2) * size_t(kTables) + f);
    return s;
}

int persist_grid(size_t smem) {
    if (cudaFuncSetAttribute(persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return 0;
    cudaFuncSetAttribute(persist_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, persist_kernel, kPT, smem) != cudaSuccess) return 0;
    return per * fastfft::sms();
}

cudaError_t launch_persistent(const PersistItem* items, int nitems, uint32_t* ctl, int nworlds, int par,
                              StepParams* const* loc, const uint32_t* base_seed, uint32_t* frame, bool advance,
                              int* err, size_t smem, int grid, cudaStream_t s) {
    if (grid <= 0) return cudaErrorInvalidConfiguration;
    persist_kernel<<<grid, kPT, smem, s>>>(items, nitems, ctl, nworlds, par, loc, base_seed, frame,
                                           advance ? 1 : 0, err);
    return cudaGetLastError();
}

}  // namespace lenia
