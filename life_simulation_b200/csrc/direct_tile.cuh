// life_simulation_b200/csrc/direct_tile.cuh -- the direct path's tile body
// (halo tile in shared memory, 8-tap chunks, growth epilogue), shared by
// the single-world and batched direct kernels (lenia_direct.cu) and the
// batch's persistent launch (lenia_batch_persistent.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {
namespace {


constexpr int PX = 8;  // taps per chunk along x (and the default outputs per thread)

// OX outputs per thread along x: 8, or 16 on large tiles (half the input
// loads per multiply-add); OY output rows per thread: 1, or 2 on large tiles
// (each staged input row chunk then feeds two kernel rows: half the input
// loads again). Each output's sum runs in the same order in every variant,
// so they all give the same bits.
template <int TW, int TH, int OX = PX, int OY = 1>
struct DirectTile {
    static constexpr int kThreads = (TW / OX) * (TH / OY);
};

// Shared memory serves a warp's 16-byte loads eight lanes at a time; a
// phase of eight lanes is conflict-free when its lanes hit eight different
// 16-byte bank quads. A thread reads its inputs OX floats to the right of its
// x-neighbour's and one tile row (TP floats) below its y-neighbour's. So the
// halo tile's row pitch is 4 modulo 8 floats (consecutive rows start on
// bank quads of opposite parity), and each phase holds 32 / OX threads along
// x (distinct quads within a row) times 8 OX / 32 rows.
__host__ __device__ constexpr int tile_pitch(int tw, int xp) { return tw + 2 * xp + 12; }

// Thread lt of a tile group (TW / OX threads per output row): its thread
// column tx and output row within the tile, lanes ordered so every phase of
// eight lanes is two or four threads along x by four or two rows. The
// mapping only changes which thread computes which outputs.
template <int TW, int OX>
__device__ __forceinline__ void tile_thread(int lt, int& tx, int& row) {
    constexpr int NX = TW / OX;           // threads along x
    constexpr int XP = 32 / OX;           // threads along x in one phase (2 or 4)
    constexpr int RP = 8 / XP;            // rows in one phase
    constexpr int XH = NX / XP;           // phases along x in one warp
    constexpr int RW = 32 / NX;           // rows per warp
    static_assert(NX % XP == 0 && 32 % NX == 0, "tile width and outputs per thread");
    const int lane = lt & 31, phase = lane >> 3;
    tx = lane % XP + XP * (phase % XH);
    row = (lt >> 5) * RW + (lane / XP) % RP + RP * (phase / XH);
}

// Per-kernel-row chunk plan, filled on the host: for row dy (0..2R), the first
// 8-tap chunk starts at dx = start (relative to -XP... see host) and `count`
// chunks follow. Packed as (start + 128) | (count << 16).
__device__ __forceinline__ void unpack_span(uint32_t v, int& start, int& count) {
    start = int(v & 0xFFFFu) - 128;
    count = int(v >> 16);
}

// --- TMA halo load (sm_90+ PTX: mbarrier + cp.async.bulk.tensor) ---------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// Makes the initialised barrier visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Box (x, y) of a 2D tensor map into shared memory; x (the innermost
// coordinate) is a multiple of 4 floats, as a TMA copy requires.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
// Polls of the halo-load barrier before a CTA gives up (the load of a few
// tens of KB lands within microseconds; this bound is reached only if the
// device stops delivering it).
constexpr uint32_t kTmaPolls = 1u << 22;

// One output tile at (x0, y0) of one world. `tmap` (or null): the state's
// halo-tile tensor map; `err` counts halo loads whose wait ran out. S > 1
// splits the kernel rows over S thread groups (group s takes rows dy = s,
// s + S, ...) for fields too small to fill the GPU one thread per 8 outputs:
// the groups' partial sums meet in shared memory and are added in group
// order before the epilogue.
template <int TW, int TH, int NK, int S = 1, int OX = PX, int OY = 1>
__device__ __forceinline__ void direct_tile(const float* __restrict__ src, float* __restrict__ dst,
                                            const float* __restrict__ weights,  // [NK][2R+1][WP], zero padded
                                            const uint32_t* __restrict__ spans, // [NK][2R+1]
                                            const DirectGeometry& g, const StepParams& p, int x0, int y0,
                                            const CUtensorMap* tmap, int* err) {
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t tma_bar;
    const int TP = tile_pitch(TW, g.xp);       // tile pitch (floats), 4 modulo 8
    const int TR = TH + 2 * g.r;               // tile rows
    float* tile = smem;                        // [TR][TP]
    float* wts = tile + TR * TP;               // [NK][2R+1][WP]
    uint32_t* sp = reinterpret_cast<uint32_t*>(wts + NK * g.ksize * g.wp);

    const int W = int(p.width), H = int(p.height);
    const int tid = threadIdx.x;
    static_assert(OY == 1 || S == 1, "two output rows per thread only without the kernel-row split");
    constexpr int NT0 = DirectTile<TW, TH, OX, OY>::kThreads;  // threads per row group
    constexpr int NT = NT0 * S;
    const int grp = S > 1 ? tid / NT0 : 0;
    const int lt = tid - grp * NT0;

    // Stage the halo tile: tile[r][c] = A[(y0 - R + r) mod H][(x0 - XP + c) mod W].
    // A box inside the field is one TMA load (its TR x TP layout is the
    // tile's); a box that wraps around the torus is loaded element by element.
    const int bx = x0 - g.xp, by = y0 - g.r;
    const bool tma = tmap != nullptr && bx >= 0 && bx + TP <= W && by >= 0 && by + TR <= H &&
                     (smem_addr(tile) & 127u) == 0u;
    if (tma) {
        if (tid == 0) {
            mbar_init(&tma_bar, 1);
            mbar_init_fence();
        }
        __syncthreads();
        if (tid == 0) {
            mbar_arrive_expect_tx(&tma_bar, uint32_t(TR * TP) * uint32_t(sizeof(float)));
            tma_load_2d(tile, tmap, bx, by, &tma_bar);
        }
    } else {
        for (int i = tid; i < TR * TP; i += NT) {
            int r = i / TP, c = i - r * TP;
            int gy = y0 - g.r + r;
            int gx = x0 - g.xp + c;
            gy %= H;
            if (gy < 0) gy += H;
            gx %= W;
            if (gx < 0) gx += W;
            tile[i] = __ldg(src + size_t(gy) * W + gx);
        }
    }
    const int nw = NK * g.ksize * g.wp;
    for (int i = tid; i < nw; i += NT) wts[i] = __ldg(weights + i);
    for (int i = tid; i < NK * g.ksize; i += NT) sp[i] = __ldg(spans + i);
    if (tma) {
        bool done = false;
        for (uint32_t i = 0; i < kTmaPolls && !done; ++i) done = mbar_try_wait(&tma_bar, 0);
        if (!__syncthreads_and(done)) {
            // The load did not arrive: count it, give the copy in flight one
            // more bounded wait, and leave this tile unwritten.
            if (tid == 0 && err) atomicAdd(err, 1);
            for (uint32_t i = 0; i < kTmaPolls && !mbar_try_wait(&tma_bar, 0); ++i) {
            }
            return;
        }
    }
    __syncthreads();

    int tx, ty;  // thread column; first output row within the tile
    tile_thread<TW, OX>(lt, tx, ty);
    ty *= OY;
    const int ox = tx * OX;  // first output column within the tile
    float acc[OY][NK][OX];
#pragma unroll
    for (int o = 0; o < OY; ++o)
#pragma unroll
        for (int k = 0; k < NK; ++k)
#pragma unroll
            for (int j = 0; j < OX; ++j) acc[o][k][j] = 0.0f;

    if constexpr (OY > 1) {
        // Walk the input rows ty + r; row r meets kernel row dy = r - o of
        // output row ty + o. A chunk of the row is loaded once for every
        // kernel row it meets: the union of those rows' chunk spans (spans
        // lie on one 8-tap grid, and taps outside a row's own span weigh
        // zero, adding an exact +0 to its sums). Each output still sums its
        // kernel rows in ascending dy and taps in ascending dx.
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            for (int r = 0; r < g.ksize + OY - 1; ++r) {
                int lo = 1 << 20, hi = -(1 << 20);
#pragma unroll
                for (int o = 0; o < OY; ++o) {
                    const int dyi = r - o;
                    if (dyi < 0 || dyi >= g.ksize) continue;
                    int start, count;
                    unpack_span(sp[k * g.ksize + dyi], start, count);
                    if (count > 0) {
                        lo = min(lo, start);
                        hi = max(hi, start + count * PX);
                    }
                }
                const float* in_row = tile + (ty + r) * TP + ox + g.xp;
                for (int d0 = lo; d0 < hi; d0 += PX) {
                    const float4* ip = reinterpret_cast<const float4*>(in_row + d0);
                    float in[OX + PX];
#pragma unroll
                    for (int q = 0; q < (OX + PX) / 4; ++q) {
                        const float4 a = ip[q];
                        in[4 * q] = a.x;
                        in[4 * q + 1] = a.y;
                        in[4 * q + 2] = a.z;
                        in[4 * q + 3] = a.w;
                    }
#pragma unroll
                    for (int o = 0; o < OY; ++o) {
                        const int dyi = r - o;
                        if (dyi < 0 || dyi >= g.ksize) continue;
                        const float4* wp =
                            reinterpret_cast<const float4*>(wts + (k * g.ksize + dyi) * g.wp + g.xp + d0);
                        const float4 w0 = wp[0], w1 = wp[1];
                        const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                        for (int i = 0; i < PX; ++i)
#pragma unroll
                            for (int j = 0; j < OX; ++j) acc[o][k][j] = fmaf(wv[i], in[i + j], acc[o][k][j]);
                    }
                }
            }
        }
    } else {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        for (int dyi = grp; dyi < g.ksize; dyi += S) {
            int start, count;
            unpack_span(sp[k * g.ksize + dyi], start, count);
            // Input row for kernel row dy = dyi - R of output row ty.
            const float* in_row = tile + (ty + dyi) * TP + ox + g.xp;
            const float* w_row = wts + (k * g.ksize + dyi) * g.wp + g.xp;
            for (int c = 0; c < count; ++c) {
                const int d0 = start + c * PX;  // multiple of 4
                const float4* ip = reinterpret_cast<const float4*>(in_row + d0);
                const float4* wp = reinterpret_cast<const float4*>(w_row + d0);
                float in[OX + PX];
#pragma unroll
                for (int q = 0; q < (OX + PX) / 4; ++q) {
                    const float4 a = ip[q];
                    in[4 * q] = a.x;
                    in[4 * q + 1] = a.y;
                    in[4 * q + 2] = a.z;
                    in[4 * q + 3] = a.w;
                }
                const float4 w0 = wp[0], w1 = wp[1];
                const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                for (int i = 0; i < PX; ++i)
#pragma unroll
                    for (int j = 0; j < OX; ++j) acc[0][k][j] = fmaf(wv[i], in[i + j], acc[0][k][j]);
            }
        }
    }
    }

    if constexpr (S > 1) {
        float* part = reinterpret_cast<float*>(sp + NK * g.ksize);  // [S-1][NK][NT0][OX]
        if (grp > 0) {
#pragma unroll
            for (int k = 0; k < NK; ++k)
#pragma unroll
                for (int j = 0; j < OX; ++j) part[(((grp - 1) * NK + k) * NT0 + lt) * OX + j] = acc[0][k][j];
        }
        __syncthreads();
        if (grp > 0) return;
        for (int q = 1; q < S; ++q)
#pragma unroll
            for (int k = 0; k < NK; ++k)
#pragma unroll
                for (int j = 0; j < OX; ++j) acc[0][k][j] += part[(((q - 1) * NK + k) * NT0 + lt) * OX + j];
    }
#pragma unroll
    for (int o = 0; o < OY; ++o) {
        const int gy = y0 + ty + o;
        if (gy >= H) return;
        const float* arow = tile + (ty + o + g.r) * TP + ox + g.xp;
#pragma unroll
        for (int j = 0; j < OX; ++j) {
            const int gx = x0 + ox + j;
            if (gx >= W) break;
            const float A = arow[j];
            const float muJ = mu_jitter_shift(p, uint32_t(gx), uint32_t(gy));
            GrowthAcc ga;
#pragma unroll
            for (int k = 0; k < NK; ++k) ga.add(p.weight[k], bell(acc[o][k][j], p.mu[k] + muJ, p.sigma[k]));
            dst[size_t(gy) * W + gx] = growth_finish(p, A, ga, uint32_t(gx), uint32_t(gy));
        }
    }
}

}  // namespace
}  // namespace lenia
