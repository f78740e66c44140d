// life_simulation_b200/csrc/npy_io.h -- NumPy .npy v1.0 files of float32 in C
// order: the reference's state exchange format (LifeCore/IO/NpyWriter.h).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lenia {

// Writes `count` floats with `shape` (their product must be `count`). The
// header is "{'descr': '<f4', 'fortran_order': False, 'shape': (...), }"
// padded with spaces to a 64-byte preamble ending in '\n', as the
// reference's writer makes it.
bool write_npy_f32(const std::string& path, const float* data, size_t count, const std::vector<uint32_t>& shape,
                   std::string& error);

// Reads a file whose shape must be `expected` (non-empty): the payload is
// sized from `expected`, never from the file's header, and a bad magic, a
// truncated header or payload, a dtype other than little-endian float32, a
// Fortran-order array or a different shape is an error (no partial data).
bool read_npy_f32(const std::string& path, const std::vector<uint32_t>& expected, std::vector<float>& out,
                  std::string& error);

}  // namespace lenia
