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

#include "direct_tile.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

namespace {

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
