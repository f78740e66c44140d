// life_simulation_b200/csrc/lenia_direct.cu -- direct toroidal convolution +
// growth + clip, fused in one pass (the work of leniaStep,
// Shaders/Field/Lenia.metal:63-128, generalised to up to 4 kernel LUTs with
// the leniaGrowthMulti epilogue, Lenia.metal:161-232).
//
// Design (FP32 CUDA cores; the op is 2*nnz FLOP per pixel against 8 bytes
// of state, so it is compute-bound):
//   * a CTA owns a TW x TH output tile; the (TH+2R) x (TW+2R) halo tile is
//     staged once in shared memory: by one TMA box load (cp.async.bulk.tensor,
//     completion on an mbarrier) when the box lies inside the field, else by
//     element loads with the toroidal wrap folded into the index;
//   * every thread owns 8 consecutive outputs of one row and walks the
//     kernel row by row; along x it consumes 8 taps at a time: 4 LDS.128 of
//     inputs and 2 LDS.128 of (warp-uniform, broadcast) weights feed 64 FFMA,
//     so shared-memory issue stays below a tenth of the FMA issue;
//   * per kernel row only the chunks covering its nonzero span are visited
//     (the disc's zero corners are skipped, like the reference's `w == 0`
//     test), taps within a row are summed in ascending dx, rows in
//     ascending dy (the reference's order);
//   * the growth map, Euler step, noise, blob injection and clip run on the
//     accumulators before the single store of A'.
#include <cuda.h>  // CUtensorMap and its encoding enums (the driver entry point is fetched at run time)
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

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

template <int TW, int TH, int NK, int S, int OX, int OY>
__global__ void __launch_bounds__(DirectTile<TW, TH, OX, OY>::kThreads * S)
    direct_step_kernel(const float* __restrict__ src, float* __restrict__ dst,
                       const float* __restrict__ weights, const uint32_t* __restrict__ spans,
                       DirectGeometry g, StepParams p, const __grid_constant__ CUtensorMap tmap, int use_tma,
                       int* err) {
    direct_tile<TW, TH, NK, S, OX, OY>(src, dst, weights, spans, g, p, blockIdx.x * TW, blockIdx.y * TH,
                                       use_tma ? &tmap : nullptr, err);
}

// Many worlds in one launch: CTA i computes tile tiles[i] = (world, tile x,
// tile y) of that world; each world brings its own state buffers, LUT,
// geometry and growth parameters.
template <int TW, int TH>
__global__ void __launch_bounds__(DirectTile<TW, TH>::kThreads)
    direct_worlds_kernel(const DirectWorld* __restrict__ worlds, const int3* __restrict__ tiles) {
    __shared__ DirectWorld w;
    const int3 t = tiles[blockIdx.x];
    if (threadIdx.x == 0) w = worlds[t.x];
    __syncthreads();
    direct_tile<TW, TH, 1>(w.src, w.dst, w.weights, w.spans, w.g, w.p, t.y * TW, t.z * TH, nullptr, nullptr);
}

template <int TW, int TH, int NK, int S, int OX, int OY>
cudaError_t launch_t(const float* src, float* dst, const float* weights, const uint32_t* spans,
                     const DirectGeometry& g, const StepParams& p, cudaStream_t stream, const DirectTma* tma,
                     int buffer) {
    const int TP = tile_pitch(TW, g.xp);
    const size_t smem = sizeof(float) * (size_t(TH + 2 * g.r) * TP + size_t(NK) * g.ksize * g.wp) +
                        sizeof(uint32_t) * NK * g.ksize +
                        sizeof(float) * size_t(S - 1) * NK * DirectTile<TW, TH, OX, OY>::kThreads * OX;
    auto fn = direct_step_kernel<TW, TH, NK, S, OX, OY>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    CUtensorMap map;
    std::memset(&map, 0, sizeof map);
    const bool on = tma && tma->on && (buffer == 0 || buffer == 1);
    if (on) std::memcpy(&map, tma->map[buffer], sizeof map);
    dim3 grid((p.width + TW - 1) / TW, (p.height + TH - 1) / TH);
    fn<<<grid, DirectTile<TW, TH, OX, OY>::kThreads * S, smem, stream>>>(src, dst, weights, spans, g, p, map,
                                                                     on ? 1 : 0, on ? tma->err : nullptr);
    return cudaGetLastError();
}

template <int TW, int TH, int S, int OX = PX, int OY = 1>
cudaError_t launch_nk(int nk, const float* src, float* dst, const float* weights,
                      const uint32_t* spans, const DirectGeometry& g, const StepParams& p,
                      cudaStream_t s, const DirectTma* tma, int buffer) {
    switch (nk) {
    case 1: return launch_t<TW, TH, 1, S, OX, OY>(src, dst, weights, spans, g, p, s, tma, buffer);
    case 2: return launch_t<TW, TH, 2, S, OX, OY>(src, dst, weights, spans, g, p, s, tma, buffer);
    case 3: return launch_t<TW, TH, 3, S, OX, OY>(src, dst, weights, spans, g, p, s, tma, buffer);
    case 4: return launch_t<TW, TH, 4, S, OX, OY>(src, dst, weights, spans, g, p, s, tma, buffer);
    default: return cudaErrorInvalidValue;
    }
}

void tile_shape(int tile_cfg, int& TW, int& TH) {
    TW = 64;
    TH = 16;
    if (tile_cfg == kDirectTile32x16) { TW = 32; TH = 16; }
    if (tile_cfg == kDirectTile64x32) { TW = 64; TH = 32; }
}

}  // namespace

size_t direct_smem_bytes(int tile_cfg, int nk, const DirectGeometry& g) {
    int TW, TH;
    tile_shape(tile_cfg, TW, TH);
    const int TP = tile_pitch(TW, g.xp);
    return sizeof(float) * (size_t(TH + 2 * g.r) * TP + size_t(nk) * g.ksize * g.wp) +
           sizeof(uint32_t) * nk * g.ksize;
}

cudaError_t launch_direct_step(int tile_cfg, int nk, const float* src, float* dst,
                               const float* weights, const uint32_t* spans,
                               const DirectGeometry& g, const StepParams& p,
                               cudaStream_t stream, const DirectTma* tma, int buffer, int split, int ox,
                               int oy) {
    if (oy != 1 && oy != 2) return cudaErrorInvalidValue;
    if (oy == 2 && split != 1) return cudaErrorInvalidValue;
    if (ox == 16) {
        if (tile_cfg != kDirectTile64x32 || split != 1) return cudaErrorInvalidValue;
        if (oy == 2) return launch_nk<64, 32, 1, 16, 2>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        return launch_nk<64, 32, 1, 16>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
    }
    if (ox != PX) return cudaErrorInvalidValue;
    if (oy == 2) {
        if (tile_cfg == kDirectTile64x32)
            return launch_nk<64, 32, 1, PX, 2>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        if (tile_cfg == kDirectTile64x16)
            return launch_nk<64, 16, 1, PX, 2>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        return cudaErrorInvalidValue;
    }
    if (tile_cfg == kDirectTile32x16) {
        switch (split) {
        case 1: return launch_nk<32, 16, 1>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        case 2: return launch_nk<32, 16, 2>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        case 4: return launch_nk<32, 16, 4>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        case 8: return launch_nk<32, 16, 8>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
        default: return cudaErrorInvalidValue;
        }
    }
    if (split != 1) return cudaErrorInvalidValue;
    switch (tile_cfg) {
    case kDirectTile64x16: return launch_nk<64, 16, 1>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
    case kDirectTile64x32: return launch_nk<64, 32, 1>(nk, src, dst, weights, spans, g, p, stream, tma, buffer);
    default: return cudaErrorInvalidValue;
    }
}

size_t direct_split_smem_bytes(int split, int nk) {
    return sizeof(float) * size_t(split - 1) * nk * DirectTile<32, 16>::kThreads * PX;
}

bool direct_tma_encode(int tile_cfg, const DirectGeometry& g, float* const fields[2], int w, int h, DirectTma& out) {
    out.on = false;
    int TW, TH;
    tile_shape(tile_cfg, TW, TH);
    const int TP = tile_pitch(TW, g.xp), TR = TH + 2 * g.r;
    // Row stride a multiple of 16 bytes; the box within the field and within
    // the 256-element limit per dimension; its rows a multiple of 16 bytes.
    if (w % 4 != 0 || TP > 256 || TR > 256 || TP > w || TR > h || (TP * 4) % 16 != 0) return false;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return false;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    for (int b = 0; b < 2; ++b) {
        if (!fields[b] || (reinterpret_cast<uintptr_t>(fields[b]) & 15u) != 0) return false;
        const cuuint64_t dims[2] = {cuuint64_t(w), cuuint64_t(h)};
        const cuuint64_t strides[1] = {cuuint64_t(w) * sizeof(float)};
        const cuuint32_t box[2] = {cuuint32_t(TP), cuuint32_t(TR)};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = encode(reinterpret_cast<CUtensorMap*>(out.map[b]), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                  fields[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    out.on = true;
    return true;
}

cudaError_t launch_direct_worlds(const DirectWorld* worlds, const int3* tiles, int ntiles, int max_r,
                                 cudaStream_t stream) {
    // 32x16 tiles (small worlds); shared memory sized for the largest radius.
    constexpr int TW = 32, TH = 16;
    DirectGeometry g;
    g.r = max_r;
    g.ksize = 2 * max_r + 1;
    g.xp = (max_r + 3) / 4 * 4;
    g.wp = 2 * g.xp + 8;
    const size_t smem = direct_smem_bytes(kDirectTile32x16, 1, g);
    auto fn = direct_worlds_kernel<TW, TH>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    fn<<<ntiles, DirectTile<TW, TH>::kThreads, smem, stream>>>(worlds, tiles);
    return cudaGetLastError();
}

}  // namespace lenia
