// oracle/ref_shim/cpu_image.h -- CPU image behind a shim texture binding
// (test infrastructure only). `channels` interleaved doubles per texel: 1 for
// R32F, 2 for RG32F, 4 for RGBA. A double holds every float value exactly.
#pragma once

namespace metal {
struct CpuImage {
    unsigned int width = 0, height = 0, channels = 1;
    double* data = nullptr;
};
}  // namespace metal
