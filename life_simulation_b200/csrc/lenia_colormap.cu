// life_simulation_b200/csrc/lenia_colormap.cu -- the Lenia module's colour
// map: the state field to an RGBA16F layer through a cosine palette
// (Shaders/Render/ColorMap.metal colorMapField / colorMapFieldScaled, run by
// the module after its substeps, Modules/FieldModules/Lenia.cpp:646-652):
//   t   = clamp(v[channel] * inputScale + inputBias, 0, 1)
//   rgb = max(a + b cos(2 pi (c t + d)), 0) * exposure,   alpha = t
// v is the field as a one-channel texture reads: (A, 0, 0, 1). When the
// output size differs from the field's, v is a bilinear sample with wrapping
// at the output pixel's centre, (x + 1/2) / W_out in normalised coordinates.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "colormap.cuh"
#include "lenia_kernels.h"

namespace lenia {
namespace {

__global__ void colormap_kernel(const float* __restrict__ field, int w, int h, ColorMapParams p,
                                ushort4* __restrict__ out, int ow, int oh) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    float v;
    if (ow == w && oh == h) {
        v = channel_of(__ldg(field + size_t(y) * w + x), p.channel);
    } else {
        // Texel space of the field: u * W - 1/2; four wrapped neighbours.
        // (Every step rounded separately, no fused multiply-adds, as the
        // reference's arithmetic.)
        const float fx = __fsub_rn(__fmul_rn((float(x) + 0.5f) / float(ow), float(w)), 0.5f);
        const float fy = __fsub_rn(__fmul_rn((float(y) + 0.5f) / float(oh), float(h)), 0.5f);
        const float x0 = floorf(fx), y0 = floorf(fy);
        const float ax = fx - x0, ay = fy - y0;
        const int xa = ((int(x0) % w) + w) % w, xb = (((int(x0) + 1) % w) + w) % w;
        const int ya = ((int(y0) % h) + h) % h, yb = (((int(y0) + 1) % h) + h) % h;
        const float t00 = channel_of(__ldg(field + size_t(ya) * w + xa), p.channel);
        const float t10 = channel_of(__ldg(field + size_t(ya) * w + xb), p.channel);
        const float t01 = channel_of(__ldg(field + size_t(yb) * w + xa), p.channel);
        const float t11 = channel_of(__ldg(field + size_t(yb) * w + xb), p.channel);
        const float top = __fadd_rn(t00, __fmul_rn(t10 - t00, ax));
        const float bot = __fadd_rn(t01, __fmul_rn(t11 - t01, ax));
        v = __fadd_rn(top, __fmul_rn(bot - top, ay));
    }
    __half rgba[4];
    palette_rgba16f(p, v, rgba);
    out[size_t(y) * ow + x] = make_ushort4(__half_as_ushort(rgba[0]), __half_as_ushort(rgba[1]),
                                           __half_as_ushort(rgba[2]), __half_as_ushort(rgba[3]));
}

}  // namespace

cudaError_t launch_colormap(const float* field, int w, int h, const ColorMapParams& p, void* rgba16f, int ow,
                            int oh, cudaStream_t s) {
    const dim3 block(32, 8);
    const dim3 grid((ow + 31) / 32, (oh + 7) / 8);
    colormap_kernel<<<grid, block, 0, s>>>(field, w, h, p, static_cast<ushort4*>(rgba16f), ow, oh);
    return cudaGetLastError();
}

}  // namespace lenia
