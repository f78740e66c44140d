// life_simulation_b200/csrc/lenia_direct.cu -- direct toroidal convolution +
// growth + clip, fused in one pass (the work of leniaStep,
// Shaders/Field/Lenia.metal:63-128, generalised to up to 4 kernel LUTs with
// the leniaGrowthMulti epilogue, Lenia.metal:161-232).
//
// Design (FP32 CUDA cores; the op is 2*nnz FLOP per pixel against 8 bytes
// of state, so it is compute-bound):
//   * a CTA owns a TW x TH output tile; the (TH+2R) x (TW+2R) halo tile is
//     staged once in shared memory with toroidal wrap folded into the load;
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
#include <cuda_runtime.h>

#include <cstdint>

#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

namespace {

constexpr int PX = 8;  // outputs per thread along x

template <int TW, int TH>
struct DirectTile {
    static constexpr int kThreads = (TW / PX) * TH;
};

// Per-kernel-row chunk plan, filled on the host: for row dy (0..2R), the first
// 8-tap chunk starts at dx = start (relative to -XP... see host) and `count`
// chunks follow. Packed as (start + 128) | (count << 16).
__device__ __forceinline__ void unpack_span(uint32_t v, int& start, int& count) {
    start = int(v & 0xFFFFu) - 128;
    count = int(v >> 16);
}

// One output tile at (x0, y0) of one world.
template <int TW, int TH, int NK>
__device__ __forceinline__ void direct_tile(const float* __restrict__ src, float* __restrict__ dst,
                                            const float* __restrict__ weights,  // [NK][2R+1][WP], zero padded
                                            const uint32_t* __restrict__ spans, // [NK][2R+1]
                                            const DirectGeometry& g, const StepParams& p, int x0, int y0) {
    extern __shared__ __align__(16) float smem[];
    const int TP = TW + 2 * g.xp + 8;          // tile pitch (floats), multiple of 4
    const int TR = TH + 2 * g.r;               // tile rows
    float* tile = smem;                        // [TR][TP]
    float* wts = tile + TR * TP;               // [NK][2R+1][WP]
    uint32_t* sp = reinterpret_cast<uint32_t*>(wts + NK * g.ksize * g.wp);

    const int W = int(p.width), H = int(p.height);
    const int tid = threadIdx.x;
    constexpr int NT = DirectTile<TW, TH>::kThreads;

    // Stage the halo tile: tile[r][c] = A[(y0 - R + r) mod H][(x0 - XP + c) mod W].
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
    const int nw = NK * g.ksize * g.wp;
    for (int i = tid; i < nw; i += NT) wts[i] = __ldg(weights + i);
    for (int i = tid; i < NK * g.ksize; i += NT) sp[i] = __ldg(spans + i);
    __syncthreads();

    const int tx = tid % (TW / PX), ty = tid / (TW / PX);
    const int ox = tx * PX;  // first output column within the tile
    float acc[NK][PX];
#pragma unroll
    for (int k = 0; k < NK; ++k)
#pragma unroll
        for (int j = 0; j < PX; ++j) acc[k][j] = 0.0f;

#pragma unroll
    for (int k = 0; k < NK; ++k) {
        for (int dyi = 0; dyi < g.ksize; ++dyi) {
            int start, count;
            unpack_span(sp[k * g.ksize + dyi], start, count);
            // Input row for kernel row dy = dyi - R of output row ty.
            const float* in_row = tile + (ty + dyi) * TP + ox + g.xp;
            const float* w_row = wts + (k * g.ksize + dyi) * g.wp + g.xp;
            for (int c = 0; c < count; ++c) {
                const int d0 = start + c * PX;  // multiple of 4
                const float4* ip = reinterpret_cast<const float4*>(in_row + d0);
                const float4* wp = reinterpret_cast<const float4*>(w_row + d0);
                float4 a0 = ip[0], a1 = ip[1], a2 = ip[2], a3 = ip[3];
                float4 w0 = wp[0], w1 = wp[1];
                const float in[16] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w,
                                      a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
                const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                for (int i = 0; i < PX; ++i)
#pragma unroll
                    for (int j = 0; j < PX; ++j) acc[k][j] = fmaf(wv[i], in[i + j], acc[k][j]);
            }
        }
    }

    const int gy = y0 + ty;
    if (gy >= H) return;
    const float* arow = tile + (ty + g.r) * TP + ox + g.xp;
#pragma unroll
    for (int j = 0; j < PX; ++j) {
        const int gx = x0 + ox + j;
        if (gx >= W) break;
        const float A = arow[j];
        const float muJ = mu_jitter_shift(p, uint32_t(gx), uint32_t(gy));
        GrowthAcc ga;
#pragma unroll
        for (int k = 0; k < NK; ++k) ga.add(p.weight[k], bell(acc[k][j], p.mu[k] + muJ, p.sigma[k]));
        dst[size_t(gy) * W + gx] = growth_finish(p, A, ga, uint32_t(gx), uint32_t(gy));
    }
}

template <int TW, int TH, int NK>
__global__ void __launch_bounds__(DirectTile<TW, TH>::kThreads)
    direct_step_kernel(const float* __restrict__ src, float* __restrict__ dst,
                       const float* __restrict__ weights, const uint32_t* __restrict__ spans,
                       DirectGeometry g, StepParams p) {
    direct_tile<TW, TH, NK>(src, dst, weights, spans, g, p, blockIdx.x * TW, blockIdx.y * TH);
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
    direct_tile<TW, TH, 1>(w.src, w.dst, w.weights, w.spans, w.g, w.p, t.y * TW, t.z * TH);
}

template <int TW, int TH, int NK>
cudaError_t launch_t(const float* src, float* dst, const float* weights, const uint32_t* spans,
                     const DirectGeometry& g, const StepParams& p, cudaStream_t stream) {
    const int TP = TW + 2 * g.xp + 8;
    const size_t smem = sizeof(float) * (size_t(TH + 2 * g.r) * TP + size_t(NK) * g.ksize * g.wp) +
                        sizeof(uint32_t) * NK * g.ksize;
    auto fn = direct_step_kernel<TW, TH, NK>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((p.width + TW - 1) / TW, (p.height + TH - 1) / TH);
    fn<<<grid, DirectTile<TW, TH>::kThreads, smem, stream>>>(src, dst, weights, spans, g, p);
    return cudaGetLastError();
}

template <int TW, int TH>
cudaError_t launch_nk(int nk, const float* src, float* dst, const float* weights,
                      const uint32_t* spans, const DirectGeometry& g, const StepParams& p,
                      cudaStream_t s) {
    switch (nk) {
    case 1: return launch_t<TW, TH, 1>(src, dst, weights, spans, g, p, s);
    case 2: return launch_t<TW, TH, 2>(src, dst, weights, spans, g, p, s);
    case 3: return launch_t<TW, TH, 3>(src, dst, weights, spans, g, p, s);
    case 4: return launch_t<TW, TH, 4>(src, dst, weights, spans, g, p, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

size_t direct_smem_bytes(int tile_cfg, int nk, const DirectGeometry& g) {
    int TW = 64, TH = 16;
    if (tile_cfg == kDirectTile32x16) { TW = 32; TH = 16; }
    if (tile_cfg == kDirectTile64x32) { TW = 64; TH = 32; }
    const int TP = TW + 2 * g.xp + 8;
    return sizeof(float) * (size_t(TH + 2 * g.r) * TP + size_t(nk) * g.ksize * g.wp) +
           sizeof(uint32_t) * nk * g.ksize;
}

cudaError_t launch_direct_step(int tile_cfg, int nk, const float* src, float* dst,
                               const float* weights, const uint32_t* spans,
                               const DirectGeometry& g, const StepParams& p,
                               cudaStream_t stream) {
    switch (tile_cfg) {
    case kDirectTile32x16: return launch_nk<32, 16>(nk, src, dst, weights, spans, g, p, stream);
    case kDirectTile64x16: return launch_nk<64, 16>(nk, src, dst, weights, spans, g, p, stream);
    case kDirectTile64x32: return launch_nk<64, 32>(nk, src, dst, weights, spans, g, p, stream);
    default: return cudaErrorInvalidValue;
    }
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
