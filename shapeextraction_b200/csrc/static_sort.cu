// se_sort_keys_static: a device sort of 64-bit keys that allocates nothing.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory budget (the host application owns and pools all device
// memory, so a stray cudaMalloc can fail or fragment its pool), and
// latency-critical loops where cudaMalloc/cudaFree are banned because they can
// synchronise the whole device. For them this entry point sorts with scratch
// memory that is a file-scope static device array, reserved once per GPU when
// the library's kernels are loaded on that GPU and held until the process
// exits. The caller passes only the input and output key arrays.
//
// Scratch layout (one array, shared by every call on a device):
//   [0, 8 MiB)       second key buffer for the ping-pong radix passes
//   [8 MiB, +512 KiB) decoupled look-back words (512 per 4096-key tile)
//   then              the sort's small device state (histograms, counters)

#include <cstdint>

#include "pipeline.cuh"
#include "shapex.h"

using namespace shapex;

namespace {

constexpr int64_t kMaxKeys = SE_STATIC_SORT_MAX_KEYS;
constexpr size_t kKeyBytes = (size_t)kMaxKeys * sizeof(uint64_t);
constexpr size_t kLookbackBytes = (size_t)((kMaxKeys + kSortTile - 1) / kSortTile) * kSortBins * sizeof(uint32_t);
constexpr size_t kStateOffset = kKeyBytes + kLookbackBytes;
constexpr size_t kScratchBytes = SE_STATIC_SORT_BYTES;
static_assert(kKeyBytes % 256 == 0 && kLookbackBytes % 256 == 0, "scratch regions stay 256-byte aligned");
static_assert(kStateOffset + sizeof(DevState) <= kScratchBytes, "scratch layout exceeds SE_STATIC_SORT_BYTES");

// The scratch. In host code this name is only a stand-in for the symbol, not a
// device address: the address is looked up with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// Device address of the scratch in the current context. It is looked up on
// every call, not cached: after cudaDeviceReset, or when the caller makes
// another driver context current on the same device, the library's module is
// loaded again and the array can move, so a cached address could point at
// memory the array no longer owns.
int scratch_address(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return SE_ERR_CUDA;
    }
    *out = p;
    return SE_OK;
}

}  // namespace

extern "C" int se_sort_keys_static(const uint64_t* d_keys_in, uint64_t* d_keys_out, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!d_keys_in || !d_keys_out))) return SE_ERR_INVALID_ARG;
    if (n > kMaxKeys) return SE_ERR_INVALID_ARG;  // beyond SE_STATIC_SORT_MAX_KEYS
    int device = 0, sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return SE_ERR_CUDA;
    }
    void* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    unsigned char* b = static_cast<unsigned char*>(base);
    uint64_t* tmp = reinterpret_cast<uint64_t*>(b);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(b + kKeyBytes);
    DevState* st = reinterpret_cast<DevState*>(b + kStateOffset);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (n > 0 && d_keys_out != d_keys_in)
        e = cudaMemcpyAsync(d_keys_out, d_keys_in, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s);
    // enqueue_sort_keys clears the state and every look-back region it uses
    // before use: the scratch keeps whatever the previous call left in it.
    if (e == cudaSuccess) e = enqueue_sort_keys(d_keys_out, tmp, n, lookback, st, s, sms);
    uint32_t err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &st->err, sizeof(err), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return SE_ERR_CUDA;
    }
    if (err & ERRBIT_LOOKBACK) return SE_ERR_SYNC_TIMEOUT;
    if (err) return SE_ERR_DEVICE_CHECK;
    return SE_OK;
}
