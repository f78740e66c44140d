// oracle/ref_shim/ref_kernels.cpp -- the reference's hot-path Metal kernels,
// compiled for the host CPU through the metal_stdlib shim.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/, never shipped, never on
// the product path). The four shader files are included from the reference
// tree at build time (the Makefile passes -I<reference root>); nothing of
// them is copied into this repository. (Five files with ColorMap.metal.) They are compiled in FP32, exactly as
// written, and every texel of a dispatch grid runs the kernel body once, in
// parallel over rows (the kernels write only their own output texels, or, for
// the FFT stages, the two autosort destinations that no other thread writes).
//
// Kernels exposed (reference file:line):
//   leniaInit        Shaders/Field/Lenia.metal:43-61
//   leniaStep        Shaders/Field/Lenia.metal:63-128
//   leniaGrowthMulti Shaders/Field/Lenia.metal:161-232
//   leniaStampInit   Shaders/Field/Lenia.metal:267-303
//   fftStageX/Y      Shaders/Common/FFT.metal:65-121
//   complexMulScale  Shaders/Common/FFT.metal:131-142
//   realToComplex    Shaders/Common/FFT.metal:145-152
//   complexToReal    Shaders/Common/FFT.metal:157-164
//   clearR32F        Shaders/Common/FFT.metal:172-177
//   colorMapField    Shaders/Render/ColorMap.metal:17-36
//   colorMapFieldScaled Shaders/Render/ColorMap.metal:50-
#include <metal_stdlib>

#include <cstring>
#include <string>

namespace refmsl {
#include "Shaders/Common/CommonTypes.metal"
#include "Shaders/Common/Random.metal"
#include "Shaders/Common/FFT.metal"
#include "Shaders/Field/Lenia.metal"
#include "Shaders/Render/ColorMap.metal"
}  // namespace refmsl

#include "ref_kernels.h"

namespace {

using metal::access;
using metal::CpuImage;
using RTex = metal::texture2d<float, access::read>;
using WTex = metal::texture2d<float, access::write>;

// Rows [g_y0, g_y1) of the grid run (the whole grid unless a row window is
// set for a bounded timing sample).
thread_local uint g_y0 = 0, g_y1 = ~0u;

template <typename F>
void grid2D(uint w, uint h, F&& f) {
    const long y0 = long(g_y0), y1 = long(std::min(h, g_y1));
#pragma omp parallel for schedule(static)
    for (long y = y0; y < y1; ++y)
        for (uint x = 0; x < w; ++x) f(uint2(x, uint(y)));
}

template <typename T>
const T& as(const void* p, size_t n, const char* what) {
    if (!p || n != sizeof(T)) {
        std::fprintf(stderr, "[ref] uniform size mismatch for %s (%zu vs %zu)\n", what, n,
                     sizeof(T));
        std::abort();
    }
    return *static_cast<const T*>(p);
}

}  // namespace

uint32_t ref_pcg_hash(uint32_t v) { return refmsl::pcg_hash(v); }
float ref_rand01(uint32_t px, uint32_t py, uint32_t tag, uint32_t seed) {
    return refmsl::rand01(uint2(px, py), tag, seed);
}

bool ref_dispatch(const std::string& fn, CpuImage* const* tex, const void* const* bytes,
                  const size_t* nbytes, uint32_t w, uint32_t h, uint32_t y0, uint32_t y1) {
    using namespace refmsl;
    g_y0 = y0;
    g_y1 = y1;
    if (fn == "leniaInit") {
        const auto& p = as<LeniaParams>(bytes[0], nbytes[0], "LeniaParams");
        WTex dst(tex[0]);
        grid2D(w, h, [&](uint2 g) { leniaInit(dst, p, g); });
    } else if (fn == "leniaStep") {
        const auto& p = as<LeniaParams>(bytes[0], nbytes[0], "LeniaParams");
        const auto& a = as<AudioUniforms>(bytes[1], nbytes[1], "AudioUniforms");
        RTex src(tex[0]);
        WTex dst(tex[1]);
        RTex kern(tex[2]);
        grid2D(w, h, [&](uint2 g) { leniaStep(src, dst, kern, p, a, g); });
    } else if (fn == "leniaGrowthMulti") {
        const auto& p = as<LeniaMultiParams>(bytes[0], nbytes[0], "LeniaMultiParams");
        const auto& a = as<AudioUniforms>(bytes[1], nbytes[1], "AudioUniforms");
        RTex src(tex[0]);
        WTex dst(tex[1]);
        RTex p0(tex[2]), p1(tex[3]), p2(tex[4]), p3(tex[5]);
        grid2D(w, h, [&](uint2 g) { leniaGrowthMulti(src, dst, p0, p1, p2, p3, p, a, g); });
    } else if (fn == "leniaStampInit") {
        const auto& p = as<LeniaStampParams>(bytes[0], nbytes[0], "LeniaStampParams");
        WTex dst(tex[0]);
        RTex org(tex[1]);
        grid2D(w, h, [&](uint2 g) { leniaStampInit(dst, org, p, g); });
    } else if (fn == "fftStageX" || fn == "fftStageY") {
        const auto& p = as<FFTParams>(bytes[0], nbytes[0], "FFTParams");
        RTex src(tex[0]);
        WTex dst(tex[1]);
        if (fn == "fftStageX")
            grid2D(w, h, [&](uint2 g) { fftStageX(src, dst, p, g); });
        else
            grid2D(w, h, [&](uint2 g) { fftStageY(src, dst, p, g); });
    } else if (fn == "complexMulScale") {
        const auto& p = as<FFTParams>(bytes[0], nbytes[0], "FFTParams");
        RTex a(tex[0]), b(tex[1]);
        WTex dst(tex[2]);
        grid2D(w, h, [&](uint2 g) { complexMulScale(a, b, dst, p, g); });
    } else if (fn == "realToComplex" || fn == "complexToReal") {
        const auto& p = as<FFTParams>(bytes[0], nbytes[0], "FFTParams");
        RTex src(tex[0]);
        WTex dst(tex[1]);
        if (fn == "realToComplex")
            grid2D(w, h, [&](uint2 g) { realToComplex(src, dst, p, g); });
        else
            grid2D(w, h, [&](uint2 g) { complexToReal(src, dst, p, g); });
    } else if (fn == "colorMapField") {
        const auto& p = as<ColorMapParams>(bytes[0], nbytes[0], "ColorMapParams");
        RTex src(tex[0]);
        WTex dst(tex[1]);
        grid2D(w, h, [&](uint2 g) { colorMapField(src, dst, p, g); });
    } else if (fn == "colorMapFieldScaled") {
        const auto& p = as<ColorMapParams>(bytes[0], nbytes[0], "ColorMapParams");
        const auto& sp = as<ColorMapScaledParams>(bytes[1], nbytes[1], "ColorMapScaledParams");
        metal::texture2d<float, access::sample> src(tex[0]);
        WTex dst(tex[1]);
        grid2D(w, h, [&](uint2 g) { colorMapFieldScaled(src, dst, p, sp, g); });
    } else if (fn == "clearR32F") {
        const auto& p = as<FFTParams>(bytes[0], nbytes[0], "FFTParams");
        WTex dst(tex[0]);
        grid2D(w, h, [&](uint2 g) { clearR32F(dst, p, g); });
    } else {
        return false;
    }
    return true;
}
