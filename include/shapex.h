/*
 * shapex.h -- C ABI of the B200-native normal-estimation path.
 *
 * Drop-in boundary for the reference's C++ entry points (Wehrdo/ShapeExtraction,
 * paths relative to its project root). Every entry point cites the reference
 * interface it replaces. Plain pointers and sizes only; every call returns an
 * se_status. A context owns its device memory and one CUDA stream; use one
 * context per host thread.
 *
 * Memory arguments (`mem`): SE_MEM_HOST means the pointer is host memory (the
 * call copies through the context's stream and returns after the copy ends);
 * SE_MEM_DEVICE means device memory on the context's device (the call only
 * enqueues work, except where stated).
 */
#ifndef SHAPEX_H
#define SHAPEX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SE_ABI_VERSION 2 /* 2: se_options and se_stats gained the cell-scan fields */

/* The library exports exactly the functions below; everything else in it is
 * hidden. */
#if defined(__GNUC__)
#define SE_API __attribute__((visibility("default")))
#else
#define SE_API
#endif

typedef enum se_status {
    SE_OK = 0,
    SE_ERR_INVALID_ARG = 1,   /* bad pointer, size, k or option */
    SE_ERR_CUDA = 2,          /* a CUDA runtime call failed (text in se_last_error) */
    SE_ERR_OOM = 3,           /* device allocation failed */
    SE_ERR_NOT_BUILT = 4,     /* query before a successful se_build */
    SE_ERR_NONFINITE = 5,     /* NaN or Inf among the input coordinates */
    SE_ERR_SEARCH_LIMIT = 6,  /* a kNN traversal hit its iteration or stack cap */
    SE_ERR_DEVICE_CHECK = 7,  /* a kernel's own bounds check fired */
    SE_ERR_SYNC_TIMEOUT = 8,  /* a cross-block wait (scan look-back) gave up */
    SE_ERR_UNSUPPORTED = 9    /* e.g. a k outside {1..32}, or no sm_100 device */
} se_status;

typedef enum se_mem { SE_MEM_HOST = 0, SE_MEM_DEVICE = 1 } se_mem;

typedef struct se_ctx se_ctx;

/* Options. se_options_init fills the reference's behaviour. */
typedef struct se_options {
    int32_t code_bits;     /* 63 (21 bits/axis, src/MortonUtils.hpp:10) or 30 (10 bits/axis) */
    int32_t root_compat;   /* 1: radix root covers [0, u-2] as src/RadixTree.cu:128-130
                              with N = u-1 (src/RadixTree.cu:353-362); 0: full [0, u-1] */
    int32_t build_octree;  /* 1: build the OTNode array (OT::Octree); 0: radix tree only */
    float viewpoint[3];    /* orientation viewpoint, src/NormalEstimation.hpp:318-319 */
    float eigengap_fp64;   /* relative eigengap (l1-l0)/l2 below which the 3x3
                              eigensolve is redone in FP64 on the GPU */
    int32_t leaf_bucket;   /* kNN bucket size: subtrees of <= this many points are
                              scanned directly, 32 at a time (1..128; 0 or the
                              default: 96) */
    int32_t device;        /* CUDA device ordinal */
    void* stream;          /* cudaStream_t to use; NULL: the context creates one */
    int32_t seed_halo;     /* kNN: points offered on each side of a warp's 32 queries
                              before the tree walk (0..48); -1 (the default) picks
                              per k: 16 up to k = 16, 32 above (measured best) */
    int32_t learned;       /* 1: queries start from the learned radius (se_mlp_*);
                              queries it underestimates are searched again without it.
                              Applies to the tree's own points (se_knn_self,
                              se_normals), not to se_knn or se_normals_batch */
    int32_t learned_skip_seed; /* with learned: skip the Morton-window seed */
    int32_t search_compat; /* 1: se_knn, se_knn_self and se_normals run the reference's
                              own approximate search (knnSearchKernel<k>,
                              src/Octree.hpp:136-193: face-plane node distance,
                              32-slot bounded node heap, k-slot result heap) and its
                              FP32 covariance (src/NormalEstimation.hpp:96-120),
                              reproducing its neighbour lists bit for bit; needs the
                              octree (build_octree = 1); not with se_normals_batch */
    int32_t batch_graph;   /* 1: se_normals_batch records its launches once as a CUDA
                              graph and replays it while the batch layout, the k's and
                              the buffers repeat (inputs in device or pinned host
                              memory); 0: plain stream launches every call */
    /* Test hooks for the failure paths (all off by default; not for production
     * use). The reference only prints its CUDA errors (src/CudaCommon.hpp:23-76);
     * these make each bounded wait and each status path here reachable in a test
     * without faulting or hanging a GPU. */
    int32_t debug_wait_limit; /* 0: cross-block look-back waits give up after
                                 2^22 polls; > 0: after this many */
    int32_t debug_inject;     /* SE_DEBUG_* bits; each fires once, on the next call
                                 that reaches it, and is then cleared */
    int32_t learned_cell_scan; /* with learned and learned_skip_seed: 1 runs the learned
                                  attempt as a direct scan of the Morton cells that cover
                                  each query's predicted ball (no tree walk; warps whose
                                  cells are too many walk the tree); 0 (the default) walks
                                  the tree with the predicted bound as a cap, which
                                  measured faster on every cloud tried */
    int32_t cell_span;         /* cell scan: at most this many cells per axis cover one
                                  query's predicted ball (2..4; 0: the default, 3) */
    int32_t cell_max_points;   /* cell scan: a warp whose cells hold more points walks the
                                  tree instead (0: the default, 4096) */
    /* se_normals_batch scheduling (0: the default of each); se_tune_batch
     * measures and sets them, with leaf_bucket and seed_halo. */
    int32_t batch_lanes;           /* streams the clouds' builds are spread over (1..16;
                                      default 8) */
    int32_t batch_lane_min_points; /* clouds of at least this many points are queried on
                                      their stream right after their build, the others in
                                      the shared persistent launches (default 65536) */
    int32_t batch_blocks_per_sm;   /* resident blocks per SM of the persistent launches
                                      (default: as many as fit) */
    int32_t batch_warps_per_block; /* warps per block of the persistent launches: 2 or 4
                                      (default: 4 up to k = 16, 2 above) */
} se_options;

/* se_options.debug_inject bits. */
#define SE_DEBUG_STALL_SORT_TILE 1 /* next se_build: the first radix-sort tile never
                                      publishes its prefix, so its successors' waits run
                                      out: SE_ERR_SYNC_TIMEOUT, nothing else is written */
#define SE_DEBUG_SEARCH_LIMIT 2    /* next kNN call: each warp's tree walk gives up
                                      after one node visit: SE_ERR_SEARCH_LIMIT */
#define SE_DEBUG_ALLOC_FAIL 4      /* next growth of the build buffers fails as a failed
                                      cudaMalloc would: SE_ERR_OOM */

/* Sizes after se_build (RT::RadixTree / OT::Octree public fields). */
typedef struct se_info {
    int64_t n_input;   /* points given to se_build */
    int64_t n_points;  /* unique codes u (RadixTree::n_pts after dedup, src/RadixTree.cu:290) */
    int64_t n_radix;   /* u-1 internal nodes (RadixTree::n_nodes, src/RadixTree.cu:353) */
    int64_t n_octree;  /* octree nodes (Octree::n_nodes, src/Octree.cu:247) */
    float min_coord;   /* RadixTree::min_coord, src/RadixTree.cu:241 */
    float max_coord;   /* RadixTree::max_coord, src/RadixTree.cu:240 */
    int32_t code_bits;
    int32_t root_level; /* prefixN[0] / 3, src/Octree.cu:258 */
} se_info;

/* Byte-compatible with OT::OTNode, src/Octree.hpp:19-36 (56 bytes). */
typedef struct se_otnode {
    int32_t children[8];
    float corner[3];
    float cell_size;
    int32_t child_node_mask;
    int32_t child_leaf_mask;
} se_otnode;

/* Device pointers owned by the context (valid until the next se_build or
 * se_destroy). Layouts: codes u64[u]; points float[3u] (AoS `Point`,
 * src/PointCloud.hpp:21-36); octree se_otnode[n_octree]; radix arrays as
 * RT::Nodes (src/RadixTree.hpp:17-34). */
typedef struct se_device_views {
    const uint64_t* codes;
    const float* points;
    const se_otnode* octree;
    const int32_t* left_child;
    const int32_t* parent;
    const uint8_t* prefix_n;
    const uint8_t* has_leaf_left;
    const uint8_t* has_leaf_right;
} se_device_views;

SE_API int se_options_init(se_options* opt);
SE_API const char* se_status_string(int status);
SE_API int se_abi_version(void);

/* Context lifetime. Replaces the implicit global state of the reference
 * (default stream, per-call cudaMallocManaged). */
SE_API int se_create(se_ctx** ctx, const se_options* opt);
SE_API int se_destroy(se_ctx* ctx);
SE_API const char* se_last_error(const se_ctx* ctx);

/* Replaces RT::RadixTree::RadixTree(const PointCloud<float>&)
 * (src/RadixTree.hpp:38, src/RadixTree.cu:305-382) followed by
 * OT::Octree::Octree(const RT::RadixTree&) (src/Octree.hpp:95,
 * src/Octree.cu:213-319): bbox, Morton encode, sort, dedup, Karras radix tree,
 * octree, decode. x, y, z are the SoA coordinate arrays of PointCloud<float>
 * (src/PointCloud.hpp:105-122). Returns after the build has finished. */
SE_API int se_build(se_ctx* ctx, const float* x, const float* y, const float* z, int64_t n, int mem);

/* RadixTree::n_pts/n_nodes/min_coord/max_coord, Octree::n_pts/n_nodes. */
SE_API int se_get_info(const se_ctx* ctx, se_info* info);
/* Device pointers to the built arrays (RadixTree::d_tree, Octree::u_nodes, Octree::u_points). */
SE_API int se_get_device_views(const se_ctx* ctx, se_device_views* views);

/* Copies of the build stages for parity checks. */
/* RT::Nodes::mortonCode after dedup (src/RadixTree.cu:294-296): u codes, ascending. */
SE_API int se_get_codes(se_ctx* ctx, uint64_t* out, int mem);
/* RT::Nodes arrays, src/RadixTree.cu:344-362: n_radix entries each; parent has
 * u entries (entries never written by the tree, e.g. parent[0], are 0). */
SE_API int se_get_radix(se_ctx* ctx, int32_t* left_child, int32_t* parent, uint8_t* prefix_n,
                 uint8_t* has_leaf_left, uint8_t* has_leaf_right, int mem);
/* Octree::u_nodes, src/Octree.cu:250-282: n_octree nodes. */
SE_API int se_get_octree(se_ctx* ctx, se_otnode* out, int mem);
/* Octree::u_points / h_points, src/Octree.cu:305-318: u points, AoS xyz. */
SE_API int se_get_points(se_ctx* ctx, float* out_xyz, int mem);

/* Replaces Octree::deviceKnnSearch<k>(d_query, d_nn, N, eps) (src/Octree.hpp:106-107,
 * 199-212) with the tree's own points [start, start+count) as queries, as
 * NormalEstimation::estimateNormals does (src/NormalEstimation.hpp:204,211).
 * Exact kNN, rows ascending by (squared distance, index); out_idx count*k
 * int32, out_d2 (optional, may be NULL) count*k float. 1 <= k <= 32. */
SE_API int se_knn_self(se_ctx* ctx, int k, int64_t start, int64_t count, int32_t* out_idx, float* out_d2, int mem);

/* Replaces Octree::knnSearch<k>(points, eps) (src/Octree.hpp:102-103, 214-242)
 * for arbitrary query points (AoS xyz, n_queries of them), with the
 * reference's N/eps argument swap (src/Octree.hpp:232) not reproduced. */
SE_API int se_knn(se_ctx* ctx, int k, const float* queries_xyz, int64_t n_queries, int32_t* out_idx, float* out_d2,
           int mem);

/* Replaces NormalEstimation::estimateNormals<k>(octree, start_idx, n)
 * (src/NormalEstimation.hpp:16-19, 196-335): exact kNN, covariance, 3x3
 * symmetric eigensolve, orientation towards the viewpoint, fused in one
 * kernel. out_xyz: count normals, AoS xyz (std::vector<Point> layout). */
SE_API int se_normals(se_ctx* ctx, int k, int64_t start, int64_t count, float* out_xyz, int mem);

/* Batched normal estimation over n_clouds independent clouds; no counterpart
 * in the reference (one cloud per call there). The clouds are concatenated
 * SoA: cloud c is points [offsets[c], offsets[c+1]) of x, y, z, with its own
 * k = ks[c] (1..32). Every cloud's build (bbox, codes, sort, dedup, radix
 * tree, search hierarchy; no octree) runs with device-side sizes, spread
 * largest-first over the context's internal streams with no host
 * synchronisation between clouds; then one persistent kNN + normals launch
 * per distinct k serves all clouds with that k, warps taking 32-query items
 * of the largest clouds first. With options.batch_graph the whole sequence is
 * captured once as a CUDA graph and replayed by later calls with the same
 * layout. out_normals holds
 * offsets[n_clouds] rows of xyz: cloud c's u_c normals (its unique points in
 * Morton order) start at row offsets[c]; out_u[c] = u_c. offsets, ks and out_u
 * are host arrays; x, y, z and out_normals follow `mem`. */
SE_API int se_normals_batch(se_ctx* ctx, const float* x, const float* y, const float* z, const int64_t* offsets,
                     int n_clouds, const int32_t* ks, float* out_normals, int64_t* out_u, int mem);

/* Batch tuning: the bucket size, seed halo and scheduling that
 * se_normals_batch uses (the options of the same names). No counterpart in
 * the reference, which runs one cloud at a time and hard-codes 512 threads
 * per block (src/CudaCommon.hpp:78). */
typedef struct se_batch_tuning {
    int32_t leaf_bucket;
    int32_t seed_halo;
    int32_t lanes;
    int32_t lane_min_points;
    int32_t blocks_per_sm;   /* 0: as many as fit */
    int32_t warps_per_block; /* 0: per k */
} se_batch_tuning;
SE_API int se_get_batch_tuning(const se_ctx* ctx, se_batch_tuning* tuning);
SE_API int se_set_batch_tuning(se_ctx* ctx, const se_batch_tuning* tuning);

/* Autotuner for se_normals_batch: times the given batch (the same arguments
 * as se_normals_batch, outputs to internal memory) with CUDA events under
 * candidate tunings, one parameter at a time over two rounds (bucket 48..128,
 * halo, lanes 4..16, lane cut-off 2^15..2^18, resident blocks, 2- or 4-warp
 * blocks), `reps` timed calls each (median), and leaves the fastest set on
 * the context. best and best_ms (optional) receive it and its time. */
SE_API int se_tune_batch(se_ctx* ctx, const float* x, const float* y, const float* z, const int64_t* offsets,
                  int n_clouds, const int32_t* ks, int mem, int reps, se_batch_tuning* best, float* best_ms);

/* Work counters of the last se_normals/se_knn/se_knn_self call (diagnostics). */
typedef struct se_stats {
    int64_t fp64_solves;     /* queries whose eigensolve took the FP64 path */
    int64_t nodes_visited;   /* search-hierarchy nodes visited, summed over warps */
    int64_t buckets_scanned; /* point buckets streamed, summed over warps */
    int64_t candidates;      /* points that reached a query's bound, summed over queries */
    int64_t merge_steps;     /* candidate-buffer merge steps, summed over warps */
    int64_t inserts;         /* insertions into the k-best lists, summed over queries */
    int64_t learned_misses;  /* queries whose learned radius was too small (searched again) */
    int64_t cell_warps;      /* warps whose learned attempt scanned Morton cells (no tree walk) */
    int64_t cell_fallbacks;  /* warps whose cells were too many: the learned attempt walked the tree */
    int64_t cell_lookups;    /* cells whose code range was looked up, summed over warps */
    int64_t cell_points;     /* points in the cells a warp scanned, summed over warps */
} se_stats;
SE_API int se_get_stats(const se_ctx* ctx, se_stats* stats);

/* Device timings of the last se_build and query call, from CUDA events
 * recorded on the context's stream around each stage, and the number of
 * kernels each call launched. build_ms: bbox, encode (+ sort histograms),
 * radix sort, dedup + decode, radix tree, search boxes, octree, total. */
typedef struct se_profile {
    float build_ms[8];
    float query_ms;
    int32_t build_launches;
    int32_t query_launches;
} se_profile;
SE_API int se_get_profile(se_ctx* ctx, se_profile* prof);

/* ---- Learned search radius. No counterpart in the reference (the north
 * star's learned stage): a 32 -> 64 -> 64 -> 1 MLP with BF16 weights and FP32
 * accumulation predicts, per tree point, y = log2(r_k^2 / range^2) from
 * occupancy features of the built tree; the search starts from
 * r^2 = range^2 * 2^(y + margin) and stays exact (queries it underestimates
 * are searched again without it). Parameters live in the context. */
#define SE_MLP_FEATURES 32
#define SE_MLP_PARAMS 6337
/* Features of tree points [start, start+count): count x SE_MLP_FEATURES floats. */
SE_API int se_features(se_ctx* ctx, int64_t start, int64_t count, float* out, int mem);
/* Random initialisation (uniform He scaling), biases zero. */
SE_API int se_mlp_init(se_ctx* ctx, uint64_t seed);
/* Copy the FP32 master parameters out (set = 0) or in (set = 1). */
SE_API int se_mlp_params(se_ctx* ctx, float* params, int set, int mem);
/* Turn the learned starting bound on/off for later queries (se_options.learned
 * and .learned_skip_seed at run time). */
SE_API int se_mlp_enable(se_ctx* ctx, int learned, int skip_seed);
/* Log-margin added to predictions to make them upper bounds. */
SE_API int se_mlp_set_margin(se_ctx* ctx, float margin_log2);
/* Training loss of se_mlp_train and se_mlp_grad: quantile 0 (the default) is
 * the mean squared error of log2(r_k^2 / range^2); a quantile in (0, 1) is
 * the pinball loss of that quantile, so that the network predicts a per-point
 * upper bound (the margin then covers only what it still misses). No
 * counterpart in the reference. */
SE_API int se_mlp_set_loss(se_ctx* ctx, float quantile);
/* Forward pass of the training path (CUDA cores): out[n] = y-hat. */
SE_API int se_mlp_forward(se_ctx* ctx, const float* features, int64_t n, float* out, int mem);
/* Tensor-core inference fused with the features, on tree points
 * [start, start+count): y-hat and/or the search bound r^2 (either may be NULL). */
SE_API int se_mlp_predict(se_ctx* ctx, int64_t start, int64_t count, float* yhat, float* r2, int mem);
/* Mean squared error and its gradient w.r.t. every parameter (SE_MLP_PARAMS floats). */
SE_API int se_mlp_grad(se_ctx* ctx, const float* features, const float* targets, int64_t n, float* grads, float* loss,
                int mem);
/* Adam on the MSE over `steps` consecutive mini-batches of `batch` rows
 * (cycling over the n rows); losses (optional, `steps` floats) per step. */
SE_API int se_mlp_train(se_ctx* ctx, const float* features, const float* targets, int64_t n, int steps, int batch, float lr,
                 float* losses, int mem);
/* Parameters + margin to / from a file (magic "SXMLP1", F, H, params, margin). */
SE_API int se_mlp_save(se_ctx* ctx, const char* path);
SE_API int se_mlp_load(se_ctx* ctx, const char* path);

/* Sorts n 64-bit keys (e.g. Morton codes) ascending on the current device
 * WITHOUT ALLOCATING. It has no counterpart in the reference.
 * For callers that cannot call cudaMalloc: code running inside another
 * framework's memory budget (the host application owns all device memory) and
 * latency-critical loops where cudaMalloc/cudaFree, which can synchronise the
 * device, are not allowed. d_keys_in and d_keys_out are caller-owned device
 * arrays of n keys (they may be the same array); every other byte it needs is
 * one file-scope static device array inside the library (SE_STATIC_SORT_BYTES
 * on every GPU that loads the library, held until the process exits).
 * - n may not exceed SE_STATIC_SORT_MAX_KEYS: larger n returns
 *   SE_ERR_INVALID_ARG and touches nothing.
 * - Every call looks up the scratch's device address in the current context
 *   (cudaGetSymbolAddress), so it stays right after cudaDeviceReset or a
 *   change of driver context.
 * - All calls on one device share the scratch: calls that overlap on the GPU
 *   (different streams or host threads, without ordering) race on it. Each
 *   call clears the parts of the scratch that must start at zero.
 * - Synchronous: it runs on `stream` (a cudaStream_t, NULL for the legacy
 *   default stream), reads the kernels' error word back and waits for the
 *   stream before it returns. It must never be called while a stream is being
 *   captured into a CUDA graph. */
#define SE_STATIC_SORT_MAX_KEYS (1 << 20)
#define SE_STATIC_SORT_BYTES (8u * (1u << 20) + 512u * 1024u + 36864u)
SE_API int se_sort_keys_static(const uint64_t* d_keys_in, uint64_t* d_keys_out, int64_t n, void* stream);

/* Waits for all work queued on the context's stream. */
SE_API int se_synchronize(se_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SHAPEX_H */
