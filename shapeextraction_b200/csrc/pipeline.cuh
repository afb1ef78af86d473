// Internal interface between the C ABI layer (capi.cu) and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace shapex {

// LSD radix sort of 64-bit keys in 9-bit digits: 7 passes cover the 63 bits of
// a Morton code; the 8th (bit 63 alone) is trivial for codes and skipped.
constexpr int kSortBits = 9;
constexpr int kSortBins = 1 << kSortBits;
constexpr int kSortPasses = 8;
constexpr int kSortThreads = 512;
constexpr int kSortIpt = 8;
constexpr int kSortTile = kSortThreads * kSortIpt;  // 4096 keys per tile
constexpr int kDedupThreads = 256;
constexpr int kDedupIpt = 16;
constexpr int kDedupTile = kDedupThreads * kDedupIpt;
constexpr int kScanThreads = 256;
constexpr int kScanIpt = 16;
constexpr int kScanTile = kScanThreads * kScanIpt;

// Query counters: fp64 solves, nodes visited, buckets scanned, candidates,
// merge steps, inserts.
enum { CNT_FP64 = 0, CNT_NODES, CNT_BUCKETS, CNT_CANDIDATES, CNT_MERGE, CNT_INSERTS, CNT_LEARNED_MISS,
       CNT_CELL_WARPS, CNT_CELL_FALLBACK, CNT_CELL_LOOKUPS, CNT_CELL_POINTS, kQueryCounters };

// Small device-resident state of one build (zeroed at the start of each build).
struct DevState {
    uint32_t err;
    uint32_t min_ord;  // ordered-uint encodings (f2ord) of the bbox min / max
    uint32_t max_ord;
    uint32_t pad0;
    float min_coord, max_coord, range;
    int32_t n_active;                       // non-trivial sort passes
    int32_t pass_active[kSortPasses];
    int32_t pass_parity[kSortPasses];
    uint32_t tile_counter[16];              // dynamic tile ids: sort passes, dedup, octree scan
    uint32_t hist[kSortPasses][kSortBins];       // per-digit histograms of the codes
    uint32_t digit_off[kSortPasses][kSortBins];  // exclusive digit offsets
    unsigned long long u;                   // unique codes
    unsigned long long n_oct;               // octree nodes
    int32_t root_level;
    // fixed-root description used by the search hierarchy (node 0)
    int32_t sroot_gamma;
    int32_t sroot_hl, sroot_hr;
    // query counters, in the order of se_stats
    unsigned long long counters[kQueryCounters];
};

// Byte layout of OT::OTNode (reference src/Octree.hpp:19-36), 56 bytes.
struct OtNode {
    int32_t children[8];
    float corner[3];
    float cell_size;
    int32_t child_node_mask;
    int32_t child_leaf_mask;
};
static_assert(sizeof(OtNode) == 56, "OTNode layout");

// Search hierarchy node: internal node of the binary radix tree (root range
// always [0, u-1]) holding both children's tight point boxes. A child with at
// most `bucket` points is a bucket: ref = first point index, points
// [ref, ref + cnt) are contiguous in Morton order. Otherwise ref = node index.
struct __align__(16) SNode {
    float4 lo_l;  // .w: ref of the left child (int bits)
    float4 hi_l;  // .w: point count of the left child (int bits)
    float4 lo_r;
    float4 hi_r;
};

struct BuildBufs {
    int64_t cap;  // capacity in points
    const float* x;
    const float* y;
    const float* z;
    uint64_t* keys0;
    uint64_t* keys1;
    uint32_t* lookback;  // sort/dedup look-back words
    unsigned long long* lookback64;  // octree-scan look-back words
    uint64_t* codes;     // unique sorted codes
    float4* pts4;        // decoded points, padded for 16-byte loads
    float* pts3;         // decoded points, AoS xyz
    // radix tree as exported (RT::Nodes)
    int32_t* left_child;
    int32_t* parent;
    uint8_t* prefix_n;
    uint8_t* has_leaf_left;
    uint8_t* has_leaf_right;
    // search hierarchy
    int32_t* sparent;
    int32_t* leaf_parent;
    int32_t* range_end;
    uint32_t* visit;
    float4* node_box;  // 2 per node: lo, hi
    SNode* snodes;
    // octree
    int32_t* oct_counts;
    int32_t* oct_offsets;  // cap + 1
    void* oct_nodes;       // se_otnode[oct_cap]
    int64_t oct_cap;
    DevState* st;
};

struct BuildParams {
    int64_t n;
    int code_bits;
    int root_compat;
    int build_octree;
    int bucket;
    int spin_limit = kSpinLimit;  // polls before a look-back wait gives up
    int stall_first_tile = 0;     // test hook: the first sort tile never publishes its prefix
};

// Stage events of one build: [0] start, then after bbox, encode, sort, dedup,
// radix tree, search boxes, octree.
constexpr int kBuildEvents = 8;

// Enqueue the whole build on `s`. Reads x/y/z from bufs; results stay on the
// device. `ev` (kBuildEvents events, may be null) are recorded between stages;
// *launches receives the number of kernels launched.
cudaError_t enqueue_build(const BuildBufs& b, const BuildParams& p, cudaStream_t s, int num_sms, cudaEvent_t* ev,
                          int* launches);
// Enqueue only the octree stage (used to redo it after a capacity regrow).
cudaError_t enqueue_octree(const BuildBufs& b, const BuildParams& p, cudaStream_t s, int num_sms, int* launches);

// ---- learned search-radius proposal (mlp.cu) --------------------------------
constexpr int kMlpF = 32;  // features per point
constexpr int kMlpH = 64;  // hidden width
// FP32 master parameters, one flat array.
struct MlpLayout {
    static constexpr int W1 = 0;                   // [kMlpF][kMlpH], input-major
    static constexpr int B1 = W1 + kMlpF * kMlpH;  // [kMlpH]
    static constexpr int W2 = B1 + kMlpH;          // [kMlpH][kMlpH], input-major
    static constexpr int B2 = W2 + kMlpH * kMlpH;  // [kMlpH]
    static constexpr int W3 = B2 + kMlpH;          // [kMlpH]
    static constexpr int B3 = W3 + kMlpH;          // scalar
    static constexpr int N = B3 + 1;
};
constexpr int kMlpParams = MlpLayout::N;

// Training work arrays for n samples.
struct MlpWork {
    float* yhat;  // n
    float* h1;    // n x kMlpH
    float* h2;    // n x kMlpH
    float* dy;    // n
    float* dh1;   // n x kMlpH
    float* dh2;   // n x kMlpH
};

cudaError_t enqueue_features(const BuildBufs& b, int64_t u, int code_bits, int64_t start, int64_t count, float* out,
                             cudaStream_t s);
cudaError_t enqueue_predict_radius(const BuildBufs& b, const float* params, float margin, int64_t u, int code_bits,
                                   int64_t start, int64_t count, float* r2_out, float* yhat_out, cudaStream_t s);
cudaError_t enqueue_mlp_forward(const float* params, const float* X, int64_t n, float* yhat, float* h1, float* h2,
                                cudaStream_t s);
cudaError_t enqueue_mlp_grad(const float* params, const float* X, const float* y, int64_t n, float tau, MlpWork& w,
                             float* grads, float* loss, cudaStream_t s);
cudaError_t enqueue_adam(float* params, const float* grads, float* m, float* v, float lr, int step, cudaStream_t s);

// Sort n 64-bit keys in place in `keys` (ascending) with the onesweep passes;
// `tmp` (n keys), `lookback` (kSortBins words per 4096-key tile) and `st` are scratch.
cudaError_t enqueue_sort_keys(uint64_t* keys, uint64_t* tmp, int64_t n, uint32_t* lookback, DevState* st,
                              cudaStream_t s, int num_sms);

struct QueryParams {
    int k;
    int64_t start;      // first query (self queries)
    int64_t count;      // number of queries
    int64_t u;          // tree points
    const float* ext_queries;  // AoS xyz external queries or nullptr (self queries)
    int32_t* out_idx;   // count*k or nullptr
    float* out_d2;      // count*k or nullptr
    float* out_normals; // count*3 or nullptr
    float vx, vy, vz;
    float eigengap_fp64;
    int code_bits;
    int bucket;
    int seed_halo;
    const float* learned_r2;  // per query: starting bound from the learned radius, or nullptr
    int learned_skip_seed;    // with learned_r2: skip the Morton-window seed
    int device_count;         // 1: query all u points of the build, u read on the device; `count`
                              // is then an upper bound used only to size the grid
    int compat;               // 1: the reference's approximate octree search and FP32 covariance
    int64_t n_octree;         // octree nodes (compat search)
    int step_limit = 0;       // > 0: node visits per warp before the walk gives up (test hook)
    // learned cell scan: the code-range table of this build (null: the learned
    // attempt walks the tree with the cap), its per-axis shift, and the most
    // points a warp scans before it falls back to the walk
    const uint32_t* cell_lut = nullptr;
    int lut_shift = 0;
    int cell_pmax = 0;
    int cell_span = 3;
    // persistent batch launches: resident blocks per SM (0: as many as fit)
    // and warps per block (0: the per-k default; 2 or 4)
    int batch_blocks_per_sm = 0;
    int batch_warps_per_block = 0;
};

// Code-range table of a build for the learned cell scan: lut[j] = the number
// of unique codes below j << (3 * (bits per axis - level)), j = 0 .. 8^level
// (lut[8^level] = u). Level between 1 and the bits per axis.
cudaError_t enqueue_cell_lut(const BuildBufs& b, int code_bits, int level, uint32_t* lut, cudaStream_t s,
                             int num_sms);

cudaError_t enqueue_query(const BuildBufs& b, const QueryParams& q, cudaStream_t s, int num_sms);

// One cloud of a batched query: its own points, search hierarchy and build
// state (u is read there on the device), its output, and the index of its
// first 32-query item in the launch.
struct BatchCloud {
    const float4* pts;
    const SNode* snodes;
    DevState* st;
    float* out_normals;
    int64_t item0;
};

// Normals of many clouds that share q.k in one persistent launch (grid = the
// kernel's resident blocks on every SM). `clouds` is a device array of
// n_clouds entries, `counter` a device word this call resets. q supplies k,
// viewpoint, eigengap threshold, bucket and seed halo.
// u and the error word of every cloud of a batch (states st[0..n)) into
// u_out / err_out.
cudaError_t enqueue_batch_collect(const DevState* st, int n, unsigned long long* u_out, uint32_t* err_out,
                                  cudaStream_t s);

cudaError_t enqueue_query_batch(const BatchCloud* clouds, int n_clouds, int64_t n_items, unsigned long long* counter,
                                const QueryParams& q, cudaStream_t s, int num_sms);
// Reference-compatible search over the OTNode array (enqueue_query forwards
// to it when q.compat is set).
cudaError_t enqueue_query_compat(const BuildBufs& b, const QueryParams& q, cudaStream_t s);

}  // namespace shapex
