// oracle/ref_shim/ref_kernels.h -- dispatch entry into the CPU-compiled
// reference shaders (test infrastructure only; see ref_kernels.cpp).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

#include "cpu_image.h"

// Runs pipeline `fn` over a w x h grid. tex[i] is the image bound at
// [[texture(i)]], bytes[i]/nbytes[i] the uniform block bound at [[buffer(i)]].
// Only grid rows [y0, y1) run (0, ~0u: all). Returns false for a pipeline
// name this shim does not know.
bool ref_dispatch(const std::string& fn, metal::CpuImage* const* tex, const void* const* bytes,
                  const size_t* nbytes, uint32_t w, uint32_t h, uint32_t y0, uint32_t y1);

uint32_t ref_pcg_hash(uint32_t v);
float ref_rand01(uint32_t px, uint32_t py, uint32_t tag, uint32_t seed);
