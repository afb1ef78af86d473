// Shared device helpers for the sm_100a normal-estimation kernels.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace shapex {

// NVTX range for the host side of one API call or build stage (header-only
// NVTX 3: a no-op unless a profiler is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Error bits kernels OR into the context's device error word.
enum : uint32_t {
    ERRBIT_NONFINITE = 1u << 0,     // NaN/Inf input coordinate
    ERRBIT_LOOKBACK = 1u << 1,      // a decoupled look-back wait gave up
    ERRBIT_BOUNDS = 1u << 2,        // an index failed a kernel's bounds check
    ERRBIT_SEARCH_LIMIT = 1u << 3,  // kNN traversal hit its step cap
    ERRBIT_STACK = 1u << 4,         // kNN traversal stack overflow
    ERRBIT_OCT_CAPACITY = 1u << 5,  // octree larger than its buffer (host regrows)
};

// Iteration cap for every spin-wait on another block's flag (the default;
// a context's debug_wait_limit option can lower it for tests).
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bit) { atomicOr(err, bit); }

__host__ __device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

// ---- Morton codes (libmorton convention: x at bit 0, y at 1, z at 2) -------
__host__ __device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ __forceinline__ uint32_t gather3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return (uint32_t)v;
}

__host__ __device__ __forceinline__ uint32_t bitscale_of(int code_bits) { return 0xFFFFFFFFu >> (32 - code_bits / 3); }

// pointToCode (reference src/MortonUtils.cu:7-19): IEEE divide, multiply, truncate.
__device__ __forceinline__ uint64_t point_to_code(float x, float y, float z, float mn, float range, int code_bits) {
    const uint32_t bs = bitscale_of(code_bits);
    const float fbs = (float)bs;
    const uint32_t xc = __float2uint_rz(__fmul_rn(fbs, __fdiv_rn(__fsub_rn(x, mn), range)));
    const uint32_t yc = __float2uint_rz(__fmul_rn(fbs, __fdiv_rn(__fsub_rn(y, mn), range)));
    const uint32_t zc = __float2uint_rz(__fmul_rn(fbs, __fdiv_rn(__fsub_rn(z, mn), range)));
    return spread3(xc & bs) | (spread3(yc & bs) << 1) | (spread3(zc & bs) << 2);
}

// codeToPoint (reference src/MortonUtils.cu:21-29), with the FMA nvcc forms there.
__device__ __forceinline__ float3 code_to_point(uint64_t code, float mn, float range, int code_bits) {
    const float fbs = (float)bitscale_of(code_bits);
    float3 p;
    p.x = __fmaf_rn(__fdiv_rn((float)gather3(code), fbs), range, mn);
    p.y = __fmaf_rn(__fdiv_rn((float)gather3(code >> 1), fbs), range, mn);
    p.z = __fmaf_rn(__fdiv_rn((float)gather3(code >> 2), fbs), range, mn);
    return p;
}

// delta (reference src/RadixTree.cu:62-69) for codes packed right in code_bits.
__device__ __forceinline__ int delta_codes(uint64_t a, uint64_t b, int code_bits) {
    return __clzll((long long)(a ^ b)) - (64 - code_bits);
}

// Shifts with PTX clamping semantics made explicit (out-of-range amounts give 0).
__device__ __forceinline__ uint64_t shr_clamp(uint64_t v, int s) { return (s < 0 || s >= 64) ? 0ull : (v >> s); }
__device__ __forceinline__ uint64_t shl_clamp(uint64_t v, int s) { return (s < 0 || s >= 64) ? 0ull : (v << s); }
__device__ __forceinline__ int one_shl(int s) { return (s < 0 || s >= 32) ? 0 : (1 << s); }

// Canonical exact-kNN squared distance (bit-identical to the CPU oracle).
__device__ __forceinline__ float dist2(float qx, float qy, float qz, float px, float py, float pz) {
    const float dx = __fsub_rn(qx, px), dy = __fsub_rn(qy, py), dz = __fsub_rn(qz, pz);
    return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}

// dist2 for two points at once with sm_100's packed FP32 instructions: each
// 64-bit operand holds two floats (the first point in the low half), and each
// half is rounded exactly as the scalar instruction rounds it, so both halves
// of the result equal dist2 bit for bit. qq* hold the query coordinate twice.
__device__ __forceinline__ uint64_t dist2_pair(uint64_t qqx, uint64_t qqy, uint64_t qqz, uint64_t x, uint64_t y,
                                               uint64_t z) {
    uint64_t dx, dy, dz, s;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dx) : "l"(qqx), "l"(x));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dy) : "l"(qqy), "l"(y));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dz) : "l"(qqz), "l"(z));
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(s) : "l"(dz), "l"(dz));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(s) : "l"(dy), "l"(dy), "l"(s));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(s) : "l"(dx), "l"(dx), "l"(s));
    return s;
}
__device__ __forceinline__ uint64_t twice(float v) {
    const uint64_t b = __float_as_uint(v);
    return (b << 32) | b;
}
__device__ __forceinline__ float lo_half(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float hi_half(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }

// Squared distance from q to a box with the same rounding chain; never larger
// than dist2 to any point inside the box (rounding is monotonic).
__device__ __forceinline__ float box_dist2(float qx, float qy, float qz, float lx, float ly, float lz, float hx,
                                           float hy, float hz) {
    const float gx = qx < lx ? __fsub_rn(lx, qx) : (qx > hx ? __fsub_rn(qx, hx) : 0.0f);
    const float gy = qy < ly ? __fsub_rn(ly, qy) : (qy > hy ? __fsub_rn(qy, hy) : 0.0f);
    const float gz = qz < lz ? __fsub_rn(lz, qz) : (qz > hz ? __fsub_rn(qz, hz) : 0.0f);
    return __fmaf_rn(gx, gx, __fmaf_rn(gy, gy, __fmul_rn(gz, gz)));
}

// Relaxed GPU-scope loads/stores for cross-block flags.
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Monotonic float <-> uint32 mapping for atomic min/max on floats.
__device__ __forceinline__ uint32_t f2ord(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t o) {
    const uint32_t b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

}  // namespace shapex
