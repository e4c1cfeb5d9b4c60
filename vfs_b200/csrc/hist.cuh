#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace vfs {
// Equalise the histogram of an 8-bit image of n pixels (src -> dst; may alias).
// hist_scratch: 256 unsigned ints, lut_scratch: 256 bytes, both device memory.
void launch_equalize_hist(const uint8_t* src, uint8_t* dst, size_t n, unsigned int* hist_scratch,
                          uint8_t* lut_scratch, cudaStream_t st);
}  // namespace vfs
