// Project-written stand-in for the un-vendored libmorton submodule
// (Wehrdo/libmorton, .gitmodules:1-3 of the reference). It provides the two
// functions the reference calls (src/MortonUtils.cu:18,24) with libmorton's
// standard convention: 21 bits per axis, bit b of x at bit 3b, of y at 3b+1,
// of z at 3b+2. Written from that definition (magic-number bit spreading).
// Used only by oracle/build_ref.sh.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

__host__ __device__ inline uint64_t shapex_shim_spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__host__ __device__ inline uint32_t shapex_shim_gather3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return (uint32_t)v;
}

__host__ __device__ inline uint64_t morton3D_64_encode(uint32_t x, uint32_t y, uint32_t z) {
    return shapex_shim_spread3(x) | (shapex_shim_spread3(y) << 1) | (shapex_shim_spread3(z) << 2);
}

__host__ __device__ inline void morton3D_64_decode(uint64_t m, uint32_t& x, uint32_t& y, uint32_t& z) {
    x = shapex_shim_gather3(m);
    y = shapex_shim_gather3(m >> 1);
    z = shapex_shim_gather3(m >> 2);
}
