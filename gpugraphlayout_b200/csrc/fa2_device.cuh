// fa2_device.cuh -- small device helpers shared by the kernel files.
#pragma once

#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

constexpr unsigned kFullMask = 0xffffffffu;

// Common leading quadrant digits of two 32-digit Morton keys (32 if equal).
__device__ __forceinline__ int lcp_digits(uint64_t a, uint64_t b) {
    const uint64_t x = a ^ b;
    return x == 0 ? kLevels : (__clzll(x) >> 1);
}

// Tree node meta word: next index (node after the subtree) << 6 | level code.
__device__ __forceinline__ int meta_level(int meta) { return meta & 63; }
__device__ __forceinline__ uint32_t meta_next(int meta) { return (uint32_t)meta >> kMetaShift; }
__device__ __forceinline__ float make_meta(uint32_t next, int level) {
    return __int_as_float((int)((next << kMetaShift) | (uint32_t)level));
}

}  // namespace fa2
