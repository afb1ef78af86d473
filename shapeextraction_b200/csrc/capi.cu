// C ABI of the normal-estimation path: context, device memory, entry points.
// Declarations and the reference interface each entry point replaces are in
// include/shapex.h.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "pipeline.cuh"
#include "shapex.h"

using namespace shapex;

// One independent pipeline of the batched path: its own stream, buffers and
// device state, so that clouds on different lanes overlap on the GPU.
struct BatchLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<cudaEvent_t> group_done;  // the lane's builds of k group g are done
    BuildBufs b{};
    int64_t cap = 0;
};

// A recorded batched sequence and the layout it was recorded for.
struct BatchGraph {
    std::vector<int64_t> key;
    cudaGraphExec_t exec = nullptr;
    BatchCloud* desc = nullptr;  // the cloud descriptors its kNN launches read
    int launches = 0;
};

inline void release_graph(BatchGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.desc) cudaFree(g.desc);
    g.exec = nullptr;
    g.desc = nullptr;
}

struct se_ctx {
    se_options opt;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;

    int64_t cap = 0;      // point capacity of the build buffers
    int64_t oct_cap = 0;  // node capacity of the octree buffer
    int64_t out_cap = 0;  // float capacity of the query staging buffer
    int64_t idx_cap = 0;  // int capacity of the kNN staging buffer
    int64_t q_cap = 0;    // float capacity of the external-query staging buffer
    BuildBufs b{};
    float* in_xyz = nullptr;    // staging for host inputs (3 * cap)
    float* out_buf = nullptr;   // staging for host outputs
    int32_t* idx_buf = nullptr;
    float* d2_buf = nullptr;
    float* q_buf = nullptr;
    DevState* h_st = nullptr;   // pinned mirror of the device state

    bool built = false;
    se_info info{};
    int64_t last_counters[kQueryCounters] = {};

    // learned search radius
    float* mlp = nullptr;  // FP32 master parameters
    float* mlp_m = nullptr;
    float* mlp_v = nullptr;
    float* mlp_g = nullptr;
    float* mlp_loss = nullptr;
    int mlp_step = 0;
    float mlp_margin = 0.0f;
    bool mlp_ready = false;
    MlpWork mw{};
    int64_t mw_cap = 0;
    float* r2_buf = nullptr;
    int64_t r2_cap = 0;
    float* xs_buf = nullptr;  // staging of host features / targets / outputs
    int64_t xs_cap = 0;

    // batched path
    std::vector<BatchLane> lanes;
    cudaEvent_t batch_in_ready = nullptr;
    float* batch_in = nullptr;   // staged host coordinates (3 x total)
    float* batch_out = nullptr;  // staged normals for host output
    int64_t batch_cap = 0;
    unsigned long long* batch_u = nullptr;  // u per cloud
    uint32_t* batch_err = nullptr;          // error word per cloud
    unsigned long long* h_batch_u = nullptr;
    uint32_t* h_batch_err = nullptr;
    int batch_clouds_cap = 0;
    // build outputs the batched kNN reads, one slice per cloud, and per-cloud state
    float4* batch_pts4 = nullptr;
    SNode* batch_snodes = nullptr;
    int64_t batch_pts_cap = 0;
    DevState* batch_st = nullptr;
    BatchCloud* batch_desc = nullptr;    // per k group, clouds largest first
    BatchCloud* h_batch_desc = nullptr;  // pinned host copy
    unsigned long long* batch_counter = nullptr;  // work counter per k group (32)
    int batch_st_cap = 0;
    // graph of the batched sequence and the layout it was recorded for
    cudaStream_t graph_stream = nullptr;
    cudaEvent_t batch_ev_in = nullptr, batch_ev_out = nullptr;
    std::vector<BatchGraph> batch_graphs;  // most recently used last (at most 4)
    uint64_t batch_epoch = 1;  // bumped whenever a buffer a recorded graph may use moves

    cudaEvent_t build_ev[kBuildEvents] = {};
    cudaEvent_t query_ev[2] = {};
    bool have_build_times = false, have_query_times = false;
    int build_launches = 0, query_launches = 0;
};

namespace {

int fail(se_ctx* c, int status, const std::string& msg) {
    if (c) c->last_error = msg;
    return status;
}

int cuda_fail(se_ctx* c, cudaError_t e, const char* where) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(c, SE_ERR_OOM, std::string(where) + ": out of device memory");
    return fail(c, SE_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define SE_CUDA(c, call, where)                         \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return cuda_fail(c, _e, where); \
    } while (0)

template <typename T>
cudaError_t regrow(T*& p, int64_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count <= 0) return cudaSuccess;
    return cudaMalloc((void**)&p, sizeof(T) * (size_t)count);
}

void free_build(se_ctx* c) {
    BuildBufs& b = c->b;
    void* ptrs[] = {b.keys0,     b.keys1,     b.lookback,    b.lookback64, b.codes,     b.pts4,
                    b.pts3,      b.left_child, b.parent,     b.prefix_n,   b.has_leaf_left, b.has_leaf_right,
                    b.sparent,   b.leaf_parent, b.range_end, b.visit,      b.node_box,  b.snodes,
                    b.oct_counts, b.oct_offsets, c->in_xyz};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    DevState* st = b.st;
    void* oct = b.oct_nodes;
    b = BuildBufs{};
    b.st = st;
    b.oct_nodes = oct;
    b.oct_cap = c->oct_cap;
    c->in_xyz = nullptr;
    c->cap = 0;
}

int ensure_build_capacity(se_ctx* c, int64_t n) {
    if (n <= c->cap && c->b.keys0) return SE_OK;
    free_build(c);
    const int64_t cap = n < 1024 ? 1024 : n;
    BuildBufs& b = c->b;
    const int64_t sort_tiles = (cap + kSortTile - 1) / kSortTile;
    const int64_t scan_tiles = (cap + kScanTile - 1) / kScanTile;
    SE_CUDA(c, regrow(b.keys0, cap), "alloc keys");
    SE_CUDA(c, regrow(b.keys1, cap), "alloc keys");
    SE_CUDA(c, regrow(b.lookback, sort_tiles * 256 + 64), "alloc lookback");
    SE_CUDA(c, regrow(b.lookback64, scan_tiles + 64), "alloc lookback");
    SE_CUDA(c, regrow(b.codes, cap), "alloc codes");
    SE_CUDA(c, regrow(b.pts4, cap), "alloc points");
    SE_CUDA(c, regrow(b.pts3, 3 * cap), "alloc points");
    SE_CUDA(c, regrow(b.left_child, cap), "alloc radix");
    SE_CUDA(c, regrow(b.parent, cap), "alloc radix");
    SE_CUDA(c, regrow(b.prefix_n, cap), "alloc radix");
    SE_CUDA(c, regrow(b.has_leaf_left, cap), "alloc radix");
    SE_CUDA(c, regrow(b.has_leaf_right, cap), "alloc radix");
    SE_CUDA(c, regrow(b.sparent, cap), "alloc search");
    SE_CUDA(c, regrow(b.leaf_parent, cap), "alloc search");
    SE_CUDA(c, regrow(b.range_end, cap), "alloc search");
    SE_CUDA(c, regrow(b.visit, cap), "alloc search");
    SE_CUDA(c, regrow(b.node_box, 2 * cap), "alloc search");
    SE_CUDA(c, regrow(b.snodes, cap), "alloc search");
    SE_CUDA(c, regrow(b.oct_counts, cap), "alloc octree");
    SE_CUDA(c, regrow(b.oct_offsets, cap + 1), "alloc octree");
    SE_CUDA(c, regrow(c->in_xyz, 3 * cap), "alloc staging");
    b.cap = cap;
    c->cap = cap;
    return SE_OK;
}

int ensure_oct_capacity(se_ctx* c, int64_t m) {
    if (m <= c->oct_cap && c->b.oct_nodes) return SE_OK;
    if (c->b.oct_nodes) cudaFree(c->b.oct_nodes);
    c->b.oct_nodes = nullptr;
    const int64_t cap = m < 1024 ? 1024 : m;
    SE_CUDA(c, cudaMalloc(&c->b.oct_nodes, sizeof(OtNode) * (size_t)cap), "alloc octree nodes");
    c->oct_cap = cap;
    c->b.oct_cap = cap;
    return SE_OK;
}

int check_err_bits(se_ctx* c, uint32_t err) {
    if (!err) return SE_OK;
    if (err & ERRBIT_NONFINITE) return fail(c, SE_ERR_NONFINITE, "input coordinates contain NaN or Inf");
    if (err & ERRBIT_LOOKBACK) return fail(c, SE_ERR_SYNC_TIMEOUT, "a scan look-back wait gave up");
    if (err & (ERRBIT_SEARCH_LIMIT | ERRBIT_STACK))
        return fail(c, SE_ERR_SEARCH_LIMIT, "kNN traversal exceeded its step or stack cap");
    if (err & ERRBIT_BOUNDS) return fail(c, SE_ERR_DEVICE_CHECK, "a kernel bounds check fired");
    return fail(c, SE_ERR_DEVICE_CHECK, "device error word set");
}

int read_state(se_ctx* c) {
    SE_CUDA(c, cudaMemcpyAsync(c->h_st, c->b.st, sizeof(DevState), cudaMemcpyDeviceToHost, c->stream), "read state");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

cudaMemcpyKind kind_out(int mem) { return mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice; }

int prologue(se_ctx* c) {
    if (!c) return SE_ERR_INVALID_ARG;
    SE_CUDA(c, cudaSetDevice(c->opt.device), "cudaSetDevice");
    return SE_OK;
}

int check_mem(se_ctx* c, int mem) {
    if (mem != SE_MEM_HOST && mem != SE_MEM_DEVICE) return fail(c, SE_ERR_INVALID_ARG, "mem must be SE_MEM_HOST or SE_MEM_DEVICE");
    return SE_OK;
}

int run_query(se_ctx* c, int k, int64_t start, int64_t count, const float* ext, int32_t* out_idx, float* out_d2,
              float* out_normals, int mem) {
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "query before a successful se_build");
    if (k < 1 || k > 32) return fail(c, SE_ERR_UNSUPPORTED, "k must be in [1, 32]");
    if (count < 0) return fail(c, SE_ERR_INVALID_ARG, "negative count");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t u = c->info.n_points;
    if (!ext && (start < 0 || start + count > u)) return fail(c, SE_ERR_INVALID_ARG, "query range outside [0, u)");
    if (count == 0) return SE_OK;
    if (u == 0) return fail(c, SE_ERR_INVALID_ARG, "empty tree");
    if ((out_idx == nullptr) && (out_normals == nullptr)) return fail(c, SE_ERR_INVALID_ARG, "no output pointer");
    if (count > (int64_t)1 << 30) return fail(c, SE_ERR_INVALID_ARG, "too many queries in one call");
    QueryParams q{};
    q.k = k;
    q.start = start;
    q.count = count;
    q.u = u;
    q.vx = c->opt.viewpoint[0];
    q.vy = c->opt.viewpoint[1];
    q.vz = c->opt.viewpoint[2];
    q.eigengap_fp64 = c->opt.eigengap_fp64;
    q.code_bits = c->opt.code_bits;
    q.bucket = c->opt.leaf_bucket;
    q.seed_halo = c->opt.seed_halo;
    q.compat = c->opt.search_compat ? 1 : 0;
    q.n_octree = c->info.n_octree;
    if (q.compat && q.n_octree < 1)
        return fail(c, SE_ERR_UNSUPPORTED, "the reference-compatible search needs the octree (build_octree = 1, u >= 2)");
    const bool use_learned = c->opt.learned && !ext && c->mlp_ready && !q.compat;
    if (use_learned && c->r2_cap < count) {
        SE_CUDA(c, regrow(c->r2_buf, count), "alloc learned bounds");
        c->r2_cap = count;
    }
    q.learned_r2 = use_learned ? c->r2_buf : nullptr;
    q.learned_skip_seed = c->opt.learned_skip_seed;
    const bool host = mem == SE_MEM_HOST;
    if (ext) {
        if (host) {
            if (c->q_cap < 3 * count) {
                SE_CUDA(c, regrow(c->q_buf, 3 * count), "alloc queries");
                c->q_cap = 3 * count;
            }
            SE_CUDA(c, cudaMemcpyAsync(c->q_buf, ext, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, c->stream),
                    "copy queries");
            q.ext_queries = c->q_buf;
        } else {
            q.ext_queries = ext;
        }
    }
    // Pinned host outputs are written by the kernel itself (mapped host
    // memory), so the results cross PCIe while the kernel runs instead of in
    // a copy after it. Other host outputs go through device staging.
    auto mapped = [&](void* p) -> void* {
        if (!host || !p) return nullptr;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
    };
    void* m_idx = mapped(out_idx);
    void* m_d2 = mapped(out_d2);
    void* m_nrm = mapped(out_normals);
    if (out_idx) {
        if (host) {
            if (c->idx_cap < (int64_t)k * count) {
                SE_CUDA(c, regrow(c->idx_buf, (int64_t)k * count), "alloc knn staging");
                SE_CUDA(c, regrow(c->d2_buf, (int64_t)k * count), "alloc knn staging");
                c->idx_cap = (int64_t)k * count;
            }
            q.out_idx = m_idx ? static_cast<int32_t*>(m_idx) : c->idx_buf;
            q.out_d2 = out_d2 ? (m_d2 ? static_cast<float*>(m_d2) : c->d2_buf) : nullptr;
        } else {
            q.out_idx = out_idx;
            q.out_d2 = out_d2;
        }
    }
    if (out_normals) {
        if (host) {
            if (c->out_cap < 3 * count) {
                SE_CUDA(c, regrow(c->out_buf, 3 * count), "alloc normals staging");
                c->out_cap = 3 * count;
            }
            q.out_normals = m_nrm ? static_cast<float*>(m_nrm) : c->out_buf;
        } else {
            q.out_normals = out_normals;
        }
    }
    // clear the error word and counters of the previous call
    SE_CUDA(c, cudaMemsetAsync(&c->b.st->err, 0, sizeof(uint32_t), c->stream), "reset");
    SE_CUDA(c, cudaMemsetAsync(c->b.st->counters, 0, sizeof(c->b.st->counters), c->stream), "reset");
    c->have_query_times = false;
    SE_CUDA(c, cudaEventRecord(c->query_ev[0], c->stream), "event");
    if (use_learned)
        SE_CUDA(c, enqueue_predict_radius(c->b, c->mlp, c->mlp_margin, u, c->opt.code_bits, start, count, c->r2_buf,
                                          nullptr, c->stream),
                "launch radius prediction");
    SE_CUDA(c, enqueue_query(c->b, q, c->stream, c->num_sms), "launch query");
    SE_CUDA(c, cudaEventRecord(c->query_ev[1], c->stream), "event");
    if (host) {
        if (out_idx && q.out_idx == c->idx_buf)
            SE_CUDA(c, cudaMemcpyAsync(out_idx, q.out_idx, sizeof(int32_t) * k * count, cudaMemcpyDeviceToHost, c->stream),
                    "copy knn");
        if (out_idx && out_d2 && q.out_d2 == c->d2_buf)
            SE_CUDA(c, cudaMemcpyAsync(out_d2, q.out_d2, sizeof(float) * k * count, cudaMemcpyDeviceToHost, c->stream),
                    "copy knn");
        if (out_normals && q.out_normals == c->out_buf)
            SE_CUDA(c, cudaMemcpyAsync(out_normals, q.out_normals, sizeof(float) * 3 * count, cudaMemcpyDeviceToHost,
                                       c->stream),
                    "copy normals");
    }
    c->query_launches = use_learned ? 2 : 1;
    c->have_query_times = true;
    SE_CUDA(c, cudaMemcpyAsync(&c->h_st->err, &c->b.st->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
            "read state");
    SE_CUDA(c, cudaMemcpyAsync(c->h_st->counters, c->b.st->counters, sizeof(c->b.st->counters),
                               cudaMemcpyDeviceToHost, c->stream),
            "read state");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    for (int i = 0; i < kQueryCounters; ++i) c->last_counters[i] = (int64_t)c->h_st->counters[i];
    return check_err_bits(c, c->h_st->err);
}

}  // namespace

extern "C" {

int se_abi_version(void) { return SE_ABI_VERSION; }

int se_options_init(se_options* o) {
    if (!o) return SE_ERR_INVALID_ARG;
    std::memset(o, 0, sizeof(*o));
    o->code_bits = 63;
    o->root_compat = 1;
    o->build_octree = 1;
    o->viewpoint[0] = o->viewpoint[1] = o->viewpoint[2] = 0.0f;
    o->eigengap_fp64 = 1e-4f;
    o->leaf_bucket = 32;
    o->device = 0;
    o->stream = nullptr;
    o->seed_halo = 16;
    o->learned = 0;
    o->learned_skip_seed = 0;
    o->search_compat = 0;
    o->batch_graph = 1;
    return SE_OK;
}

const char* se_status_string(int s) {
    switch (s) {
        case SE_OK: return "SE_OK";
        case SE_ERR_INVALID_ARG: return "SE_ERR_INVALID_ARG";
        case SE_ERR_CUDA: return "SE_ERR_CUDA";
        case SE_ERR_OOM: return "SE_ERR_OOM";
        case SE_ERR_NOT_BUILT: return "SE_ERR_NOT_BUILT";
        case SE_ERR_NONFINITE: return "SE_ERR_NONFINITE";
        case SE_ERR_SEARCH_LIMIT: return "SE_ERR_SEARCH_LIMIT";
        case SE_ERR_DEVICE_CHECK: return "SE_ERR_DEVICE_CHECK";
        case SE_ERR_SYNC_TIMEOUT: return "SE_ERR_SYNC_TIMEOUT";
        case SE_ERR_UNSUPPORTED: return "SE_ERR_UNSUPPORTED";
        default: return "unknown status";
    }
}

int se_create(se_ctx** out, const se_options* opt) {
    if (!out) return SE_ERR_INVALID_ARG;
    *out = nullptr;
    se_options o;
    if (opt) o = *opt; else se_options_init(&o);
    if (o.code_bits != 63 && o.code_bits != 30) return SE_ERR_INVALID_ARG;
    if (o.leaf_bucket == 0) o.leaf_bucket = 32;
    if (o.leaf_bucket < 1 || o.leaf_bucket > 32) return SE_ERR_INVALID_ARG;
    if (o.seed_halo < 0) o.seed_halo = 16;
    if (o.seed_halo > 48) return SE_ERR_INVALID_ARG;
    if (!(o.eigengap_fp64 >= 0.0f)) return SE_ERR_INVALID_ARG;
    se_ctx* c = new se_ctx();
    c->opt = o;
    cudaError_t e = cudaSetDevice(o.device);
    int major = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, o.device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, o.device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return SE_ERR_CUDA;
    }
    if (major != 10) {
        delete c;
        return SE_ERR_UNSUPPORTED;  // kernels are built for sm_100a only
    }
    if (o.stream) {
        c->stream = (cudaStream_t)o.stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return SE_ERR_CUDA;
        }
        c->own_stream = true;
    }
    if (cudaMalloc(&c->b.st, sizeof(DevState)) != cudaSuccess ||
        cudaMallocHost(&c->h_st, sizeof(DevState)) != cudaSuccess) {
        se_destroy(c);
        return SE_ERR_OOM;
    }
    for (auto& e : c->build_ev) cudaEventCreate(&e);
    for (auto& e : c->query_ev) cudaEventCreate(&e);
    *out = c;
    return SE_OK;
}

int se_destroy(se_ctx* c) {
    if (!c) return SE_OK;
    cudaSetDevice(c->opt.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_build(c);
    if (c->b.oct_nodes) cudaFree(c->b.oct_nodes);
    if (c->b.st) cudaFree(c->b.st);
    if (c->h_st) cudaFreeHost(c->h_st);
    if (c->out_buf) cudaFree(c->out_buf);
    if (c->idx_buf) cudaFree(c->idx_buf);
    if (c->d2_buf) cudaFree(c->d2_buf);
    if (c->q_buf) cudaFree(c->q_buf);
    float* mlp_bufs[] = {c->mlp, c->mlp_m, c->mlp_v, c->mlp_g, c->mlp_loss, c->r2_buf, c->xs_buf,
                         c->mw.yhat, c->mw.h1, c->mw.h2, c->mw.dy, c->mw.dh1, c->mw.dh2};
    for (float* p : mlp_bufs)
        if (p) cudaFree(p);
    for (BatchLane& l : c->lanes) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        void* ptrs[] = {l.b.keys0, l.b.keys1, l.b.lookback, l.b.lookback64, l.b.codes, l.b.pts4, l.b.pts3,
                        l.b.left_child, l.b.parent, l.b.prefix_n, l.b.has_leaf_left, l.b.has_leaf_right, l.b.sparent,
                        l.b.leaf_parent, l.b.range_end, l.b.visit, l.b.node_box, l.b.snodes, l.b.st};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        if (l.done) cudaEventDestroy(l.done);
        for (cudaEvent_t e : l.group_done) cudaEventDestroy(e);
        if (l.stream) cudaStreamDestroy(l.stream);
    }
    for (BatchGraph& bg : c->batch_graphs) release_graph(bg);
    if (c->graph_stream) {
        cudaStreamSynchronize(c->graph_stream);
        cudaStreamDestroy(c->graph_stream);
    }
    if (c->batch_ev_in) cudaEventDestroy(c->batch_ev_in);
    if (c->batch_ev_out) cudaEventDestroy(c->batch_ev_out);
    void* bptrs[] = {c->batch_pts4, c->batch_snodes, c->batch_st, c->batch_desc, c->batch_counter};
    for (void* p : bptrs)
        if (p) cudaFree(p);
    if (c->h_batch_desc) cudaFreeHost(c->h_batch_desc);
    if (c->batch_in_ready) cudaEventDestroy(c->batch_in_ready);
    if (c->batch_in) cudaFree(c->batch_in);
    if (c->batch_out) cudaFree(c->batch_out);
    if (c->batch_u) cudaFree(c->batch_u);
    if (c->batch_err) cudaFree(c->batch_err);
    if (c->h_batch_u) cudaFreeHost(c->h_batch_u);
    if (c->h_batch_err) cudaFreeHost(c->h_batch_err);
    for (auto& e : c->build_ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->query_ev)
        if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return SE_OK;
}

const char* se_last_error(const se_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

int se_build(se_ctx* c, const float* x, const float* y, const float* z, int64_t n, int mem) {
    if (int rc = prologue(c)) return rc;
    c->built = false;
    if (int rc = check_mem(c, mem)) return rc;
    if (n < 0) return fail(c, SE_ERR_INVALID_ARG, "negative point count");
    if (n > ((int64_t)1 << 30) - 1) return fail(c, SE_ERR_INVALID_ARG, "more than 2^30 - 1 points");
    if (n > 0 && (!x || !y || !z)) return fail(c, SE_ERR_INVALID_ARG, "null coordinate pointer");
    if (int rc = ensure_build_capacity(c, n)) return rc;
    if (int rc = ensure_oct_capacity(c, n + 1024)) return rc;
    BuildBufs& b = c->b;
    if (mem == SE_MEM_HOST && n > 0) {
        SE_CUDA(c, cudaMemcpyAsync(c->in_xyz, x, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "copy x");
        SE_CUDA(c, cudaMemcpyAsync(c->in_xyz + c->cap, y, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "copy y");
        SE_CUDA(c, cudaMemcpyAsync(c->in_xyz + 2 * c->cap, z, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream),
                "copy z");
        b.x = c->in_xyz;
        b.y = c->in_xyz + c->cap;
        b.z = c->in_xyz + 2 * c->cap;
    } else {
        b.x = x;
        b.y = y;
        b.z = z;
    }
    BuildParams p{n, c->opt.code_bits, c->opt.root_compat, c->opt.build_octree, c->opt.leaf_bucket};
    c->have_build_times = false;
    SE_CUDA(c, enqueue_build(b, p, c->stream, c->num_sms, c->build_ev, &c->build_launches), "launch build");
    if (int rc = read_state(c)) return rc;
    c->have_build_times = true;
    if (c->h_st->err & ERRBIT_OCT_CAPACITY) {
        const int64_t m = (int64_t)c->h_st->n_oct;
        if (int rc = ensure_oct_capacity(c, m)) return rc;
        SE_CUDA(c, cudaMemsetAsync(&b.st->err, 0, sizeof(uint32_t), c->stream), "reset");
        SE_CUDA(c, enqueue_octree(b, p, c->stream, c->num_sms, &c->build_launches), "launch octree");
        if (int rc = read_state(c)) return rc;
        c->have_build_times = false;
    }
    if (int rc = check_err_bits(c, c->h_st->err)) return rc;
    const DevState& h = *c->h_st;
    c->info.n_input = n;
    c->info.n_points = (int64_t)h.u;
    c->info.n_radix = h.u > 0 ? (int64_t)h.u - 1 : 0;
    c->info.n_octree = c->opt.build_octree ? (int64_t)h.n_oct : 0;
    c->info.min_coord = n > 0 ? h.min_coord : 0.0f;
    c->info.max_coord = n > 0 ? h.max_coord : 0.0f;
    c->info.code_bits = c->opt.code_bits;
    c->info.root_level = h.root_level;
    c->built = true;
    return SE_OK;
}

int se_get_info(const se_ctx* c, se_info* info) {
    if (!c || !info) return SE_ERR_INVALID_ARG;
    if (!c->built) return SE_ERR_NOT_BUILT;
    *info = c->info;
    return SE_OK;
}

int se_get_device_views(const se_ctx* c, se_device_views* v) {
    if (!c || !v) return SE_ERR_INVALID_ARG;
    if (!c->built) return SE_ERR_NOT_BUILT;
    v->codes = c->b.codes;
    v->points = c->b.pts3;
    v->octree = (const se_otnode*)c->b.oct_nodes;
    v->left_child = c->b.left_child;
    v->parent = c->b.parent;
    v->prefix_n = c->b.prefix_n;
    v->has_leaf_left = c->b.has_leaf_left;
    v->has_leaf_right = c->b.has_leaf_right;
    return SE_OK;
}

int se_get_codes(se_ctx* c, uint64_t* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t u = c->info.n_points;
    if (u == 0) return SE_OK;
    if (!out) return fail(c, SE_ERR_INVALID_ARG, "null output");
    SE_CUDA(c, cudaMemcpyAsync(out, c->b.codes, sizeof(uint64_t) * u, kind_out(mem), c->stream), "copy codes");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_get_radix(se_ctx* c, int32_t* left_child, int32_t* parent, uint8_t* prefix_n, uint8_t* hll, uint8_t* hlr,
                 int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t nr = c->info.n_radix, u = c->info.n_points;
    const cudaMemcpyKind k = kind_out(mem);
    if (nr > 0) {
        if (left_child) SE_CUDA(c, cudaMemcpyAsync(left_child, c->b.left_child, 4 * nr, k, c->stream), "copy radix");
        if (prefix_n) SE_CUDA(c, cudaMemcpyAsync(prefix_n, c->b.prefix_n, nr, k, c->stream), "copy radix");
        if (hll) SE_CUDA(c, cudaMemcpyAsync(hll, c->b.has_leaf_left, nr, k, c->stream), "copy radix");
        if (hlr) SE_CUDA(c, cudaMemcpyAsync(hlr, c->b.has_leaf_right, nr, k, c->stream), "copy radix");
    }
    if (u > 0 && parent) SE_CUDA(c, cudaMemcpyAsync(parent, c->b.parent, 4 * u, k, c->stream), "copy radix");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_get_octree(se_ctx* c, se_otnode* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t m = c->info.n_octree;
    if (m == 0) return SE_OK;
    if (!out) return fail(c, SE_ERR_INVALID_ARG, "null output");
    SE_CUDA(c, cudaMemcpyAsync(out, c->b.oct_nodes, sizeof(OtNode) * m, kind_out(mem), c->stream), "copy octree");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_get_points(se_ctx* c, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t u = c->info.n_points;
    if (u == 0) return SE_OK;
    if (!out) return fail(c, SE_ERR_INVALID_ARG, "null output");
    SE_CUDA(c, cudaMemcpyAsync(out, c->b.pts3, sizeof(float) * 3 * u, kind_out(mem), c->stream), "copy points");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_knn_self(se_ctx* c, int k, int64_t start, int64_t count, int32_t* out_idx, float* out_d2, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!out_idx && count > 0) return fail(c, SE_ERR_INVALID_ARG, "null output");
    return run_query(c, k, start, count, nullptr, out_idx, out_d2, nullptr, mem);
}

int se_knn(se_ctx* c, int k, const float* queries, int64_t nq, int32_t* out_idx, float* out_d2, int mem) {
    if (int rc = prologue(c)) return rc;
    if (nq > 0 && (!queries || !out_idx)) return fail(c, SE_ERR_INVALID_ARG, "null pointer");
    if (nq == 0) return SE_OK;
    return run_query(c, k, 0, nq, queries, out_idx, out_d2, nullptr, mem);
}

int se_normals(se_ctx* c, int k, int64_t start, int64_t count, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!out && count > 0) return fail(c, SE_ERR_INVALID_ARG, "null output");
    return run_query(c, k, start, count, nullptr, nullptr, nullptr, out, mem);
}

int se_get_stats(const se_ctx* c, se_stats* out) {
    if (!c || !out) return SE_ERR_INVALID_ARG;
    static_assert(sizeof(se_stats) == sizeof(int64_t) * kQueryCounters, "se_stats layout");
    std::memcpy(out, c->last_counters, sizeof(*out));
    return SE_OK;
}

int se_get_profile(se_ctx* c, se_profile* prof) {
    if (!c || !prof) return SE_ERR_INVALID_ARG;
    std::memset(prof, 0, sizeof(*prof));
    if (int rc = prologue(c)) return rc;
    if (c->have_build_times) {
        for (int i = 1; i < kBuildEvents; ++i)
            SE_CUDA(c, cudaEventElapsedTime(&prof->build_ms[i - 1], c->build_ev[i - 1], c->build_ev[i]), "event time");
        SE_CUDA(c, cudaEventElapsedTime(&prof->build_ms[7], c->build_ev[0], c->build_ev[kBuildEvents - 1]),
                "event time");
    }
    if (c->have_query_times)
        SE_CUDA(c, cudaEventElapsedTime(&prof->query_ms, c->query_ev[0], c->query_ev[1]), "event time");
    prof->build_launches = c->build_launches;
    prof->query_launches = c->query_launches;
    return SE_OK;
}

// ---- learned search radius ---------------------------------------------------

namespace {

int mlp_alloc(se_ctx* c) {
    if (c->mlp) return SE_OK;
    SE_CUDA(c, regrow(c->mlp, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_m, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_v, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_g, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_loss, 1), "alloc mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    c->mlp_step = 0;
    return SE_OK;
}

int mlp_work(se_ctx* c, int64_t n) {
    if (n <= c->mw_cap) return SE_OK;
    SE_CUDA(c, regrow(c->mw.yhat, n), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.h1, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.h2, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dy, n), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dh1, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dh2, n * kMlpH), "alloc mlp work");
    c->mw_cap = n;
    return SE_OK;
}

// Device pointer for n floats given by the caller: host data goes through the
// context's staging buffer at float offset `off` (the buffer holds `total`).
int stage_in(se_ctx* c, const float* src, int64_t n, int mem, int64_t off, int64_t total, const float** out) {
    if (mem == SE_MEM_DEVICE || n == 0) {
        *out = src;
        return SE_OK;
    }
    if (c->xs_cap < total) {
        SE_CUDA(c, regrow(c->xs_buf, total), "alloc staging");
        c->xs_cap = total;
    }
    SE_CUDA(c, cudaMemcpyAsync(c->xs_buf + off, src, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "copy in");
    *out = c->xs_buf + off;
    return SE_OK;
}

uint64_t xorshift(uint64_t& s) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

}  // namespace

int se_features(se_ctx* c, int64_t start, int64_t count, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t u = c->info.n_points;
    if (start < 0 || count < 0 || start + count > u) return fail(c, SE_ERR_INVALID_ARG, "range outside [0, u)");
    if (count == 0) return SE_OK;
    if (!out) return fail(c, SE_ERR_INVALID_ARG, "null output");
    float* dst = out;
    if (mem == SE_MEM_HOST) {
        if (c->xs_cap < count * kMlpF) {
            SE_CUDA(c, regrow(c->xs_buf, count * kMlpF), "alloc staging");
            c->xs_cap = count * kMlpF;
        }
        dst = c->xs_buf;
    }
    SE_CUDA(c, enqueue_features(c->b, u, c->opt.code_bits, start, count, dst, c->stream), "launch features");
    if (mem == SE_MEM_HOST)
        SE_CUDA(c, cudaMemcpyAsync(out, dst, sizeof(float) * count * kMlpF, cudaMemcpyDeviceToHost, c->stream),
                "copy features");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_init(se_ctx* c, uint64_t seed) {
    if (int rc = prologue(c)) return rc;
    if (int rc = mlp_alloc(c)) return rc;
    float h[kMlpParams] = {};
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull;
    if (!s) s = 1;
    auto uni = [&](float a) { return a * (2.0f * (float)((xorshift(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0f); };
    const float a1 = sqrtf(6.0f / kMlpF), a2 = sqrtf(6.0f / kMlpH);
    for (int i = 0; i < kMlpF * kMlpH; ++i) h[MlpLayout::W1 + i] = uni(a1);
    for (int i = 0; i < kMlpH * kMlpH; ++i) h[MlpLayout::W2 + i] = uni(a2);
    for (int i = 0; i < kMlpH; ++i) h[MlpLayout::W3 + i] = uni(a2) * 0.1f;
    SE_CUDA(c, cudaMemcpyAsync(c->mlp, h, sizeof(h), cudaMemcpyHostToDevice, c->stream), "upload mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    c->mlp_step = 0;
    c->mlp_ready = true;
    return SE_OK;
}

int se_mlp_params(se_ctx* c, float* params, int set, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!params) return fail(c, SE_ERR_INVALID_ARG, "null params");
    if (int rc = mlp_alloc(c)) return rc;
    const cudaMemcpyKind k = set ? (mem == SE_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice)
                                 : (mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
    if (set) {
        SE_CUDA(c, cudaMemcpyAsync(c->mlp, params, sizeof(float) * kMlpParams, k, c->stream), "set params");
        SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "reset adam");
        SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "reset adam");
        c->mlp_step = 0;
        c->mlp_ready = true;
    } else {
        SE_CUDA(c, cudaMemcpyAsync(params, c->mlp, sizeof(float) * kMlpParams, k, c->stream), "get params");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_enable(se_ctx* c, int learned, int skip_seed) {
    if (!c) return SE_ERR_INVALID_ARG;
    if (learned && !c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    c->opt.learned = learned ? 1 : 0;
    c->opt.learned_skip_seed = skip_seed ? 1 : 0;
    return SE_OK;
}

int se_mlp_set_margin(se_ctx* c, float margin_log2) {
    if (!c) return SE_ERR_INVALID_ARG;
    if (!(margin_log2 > -64.0f && margin_log2 < 64.0f)) return fail(c, SE_ERR_INVALID_ARG, "margin out of range");
    c->mlp_margin = margin_log2;
    return SE_OK;
}

int se_mlp_forward(se_ctx* c, const float* features, int64_t n, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 0) return fail(c, SE_ERR_INVALID_ARG, "negative n");
    if (n == 0) return SE_OK;
    if (!features || !out) return fail(c, SE_ERR_INVALID_ARG, "null pointer");
    const float* X;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    float* Y = mem == SE_MEM_HOST ? c->xs_buf + n * kMlpF : out;
    SE_CUDA(c, enqueue_mlp_forward(c->mlp, X, n, Y, nullptr, nullptr, c->stream), "launch forward");
    if (mem == SE_MEM_HOST)
        SE_CUDA(c, cudaMemcpyAsync(out, Y, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream), "copy out");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_predict(se_ctx* c, int64_t start, int64_t count, float* yhat, float* r2, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    const int64_t u = c->info.n_points;
    if (start < 0 || count < 0 || start + count > u) return fail(c, SE_ERR_INVALID_ARG, "range outside [0, u)");
    if (count == 0) return SE_OK;
    float *dy = yhat, *dr = r2;
    if (mem == SE_MEM_HOST) {
        if (c->xs_cap < 2 * count) {
            SE_CUDA(c, regrow(c->xs_buf, 2 * count), "alloc staging");
            c->xs_cap = 2 * count;
        }
        dy = yhat ? c->xs_buf : nullptr;
        dr = r2 ? c->xs_buf + count : nullptr;
    }
    SE_CUDA(c, enqueue_predict_radius(c->b, c->mlp, c->mlp_margin, u, c->opt.code_bits, start, count, dr, dy,
                                      c->stream),
            "launch prediction");
    if (mem == SE_MEM_HOST) {
        if (yhat) SE_CUDA(c, cudaMemcpyAsync(yhat, dy, sizeof(float) * count, cudaMemcpyDeviceToHost, c->stream), "copy");
        if (r2) SE_CUDA(c, cudaMemcpyAsync(r2, dr, sizeof(float) * count, cudaMemcpyDeviceToHost, c->stream), "copy");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_grad(se_ctx* c, const float* features, const float* targets, int64_t n, float* grads, float* loss,
                int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 1 || !features || !targets) return fail(c, SE_ERR_INVALID_ARG, "bad arguments");
    if (int rc = mlp_work(c, n)) return rc;
    const float *X, *Y;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    if (int rc = stage_in(c, targets, n, mem, n * kMlpF, n * kMlpF + n, &Y)) return rc;
    SE_CUDA(c, enqueue_mlp_grad(c->mlp, X, Y, n, c->mw, c->mlp_g, c->mlp_loss, c->stream), "launch grad");
    const cudaMemcpyKind k = mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (grads) SE_CUDA(c, cudaMemcpyAsync(grads, c->mlp_g, sizeof(float) * kMlpParams, k, c->stream), "copy grads");
    if (loss) SE_CUDA(c, cudaMemcpyAsync(loss, c->mlp_loss, sizeof(float), k, c->stream), "copy loss");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_train(se_ctx* c, const float* features, const float* targets, int64_t n, int steps, int batch, float lr,
                 float* losses, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 1 || steps < 0 || batch < 1 || !features || !targets || !(lr > 0.0f))
        return fail(c, SE_ERR_INVALID_ARG, "bad arguments");
    if (batch > n) batch = (int)n;
    if (int rc = mlp_work(c, batch)) return rc;
    const float *X, *Y;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    if (int rc = stage_in(c, targets, n, mem, n * kMlpF, n * kMlpF + n, &Y)) return rc;
    float* dloss = nullptr;
    if (losses) {
        SE_CUDA(c, regrow(dloss, steps > 0 ? steps : 1), "alloc losses");
    }
    int64_t row = 0;
    for (int it = 0; it < steps; ++it) {
        if (row + batch > n) row = 0;
        SE_CUDA(c, enqueue_mlp_grad(c->mlp, X + row * kMlpF, Y + row, batch, c->mw, c->mlp_g,
                                    dloss ? dloss + it : c->mlp_loss, c->stream),
                "launch grad");
        SE_CUDA(c, enqueue_adam(c->mlp, c->mlp_g, c->mlp_m, c->mlp_v, lr, ++c->mlp_step, c->stream), "launch adam");
        row += batch;
    }
    if (dloss) {
        cudaError_t e = cudaMemcpyAsync(losses, dloss, sizeof(float) * steps, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        cudaFree(dloss);
        if (e != cudaSuccess) return cuda_fail(c, e, "copy losses");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_save(se_ctx* c, const char* path) {
    if (!c || !path) return SE_ERR_INVALID_ARG;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    float h[kMlpParams];
    if (int rc = se_mlp_params(c, h, 0, SE_MEM_HOST)) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(c, SE_ERR_INVALID_ARG, std::string("cannot write ") + path);
    const int32_t dims[2] = {kMlpF, kMlpH};
    bool ok = std::fwrite("SXMLP1\0\0", 1, 8, f) == 8 && std::fwrite(dims, 4, 2, f) == 2 &&
              std::fwrite(h, 4, kMlpParams, f) == (size_t)kMlpParams && std::fwrite(&c->mlp_margin, 4, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SE_OK : fail(c, SE_ERR_INVALID_ARG, std::string("write failed: ") + path);
}

int se_mlp_load(se_ctx* c, const char* path) {
    if (!c || !path) return SE_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(c, SE_ERR_INVALID_ARG, std::string("cannot read ") + path);
    char magic[8];
    int32_t dims[2];
    float h[kMlpParams];
    float margin = 0.0f;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SXMLP1", 6) == 0 &&
              std::fread(dims, 4, 2, f) == 2 && dims[0] == kMlpF && dims[1] == kMlpH &&
              std::fread(h, 4, kMlpParams, f) == (size_t)kMlpParams && std::fread(&margin, 4, 1, f) == 1;
    std::fclose(f);
    if (!ok) return fail(c, SE_ERR_INVALID_ARG, std::string("not a model file of this layout: ") + path);
    if (int rc = se_mlp_params(c, h, 1, SE_MEM_HOST)) return rc;
    c->mlp_margin = margin;
    return SE_OK;
}

// ---- batched path --------------------------------------------------------------

namespace {

int lane_capacity(se_ctx* c, BatchLane& l, int64_t n) {
    if (!l.stream) {
        SE_CUDA(c, cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking), "lane stream");
        SE_CUDA(c, cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming), "lane event");
        SE_CUDA(c, cudaMalloc(&l.b.st, sizeof(DevState)), "lane state");
    }
    if (n <= l.cap && l.b.keys0) return SE_OK;
    ++c->batch_epoch;
    BuildBufs& b = l.b;
    const int64_t cap = n < 1024 ? 1024 : n;
    const int64_t sort_tiles = (cap + kSortTile - 1) / kSortTile;
    const int64_t scan_tiles = (cap + kScanTile - 1) / kScanTile;
    SE_CUDA(c, regrow(b.keys0, cap), "alloc lane");
    SE_CUDA(c, regrow(b.keys1, cap), "alloc lane");
    SE_CUDA(c, regrow(b.lookback, sort_tiles * 256 + 64), "alloc lane");
    SE_CUDA(c, regrow(b.lookback64, scan_tiles + 64), "alloc lane");
    SE_CUDA(c, regrow(b.codes, cap), "alloc lane");
    SE_CUDA(c, regrow(b.pts3, 3 * cap), "alloc lane");
    SE_CUDA(c, regrow(b.left_child, cap), "alloc lane");
    SE_CUDA(c, regrow(b.parent, cap), "alloc lane");
    SE_CUDA(c, regrow(b.prefix_n, cap), "alloc lane");
    SE_CUDA(c, regrow(b.has_leaf_left, cap), "alloc lane");
    SE_CUDA(c, regrow(b.has_leaf_right, cap), "alloc lane");
    SE_CUDA(c, regrow(b.sparent, cap), "alloc lane");
    SE_CUDA(c, regrow(b.leaf_parent, cap), "alloc lane");
    SE_CUDA(c, regrow(b.range_end, cap), "alloc lane");
    SE_CUDA(c, regrow(b.visit, cap), "alloc lane");
    SE_CUDA(c, regrow(b.node_box, 2 * cap), "alloc lane");
    b.cap = cap;
    l.cap = cap;
    return SE_OK;
}

}  // namespace

namespace {

// What one se_normals_batch call enqueues: per-lane build queues, k groups.
struct BatchPlan {
    int n_lanes = 0;
    std::vector<std::vector<int>> queue;  // clouds per lane: group by group, largest first in each
    std::vector<std::vector<int>> group_end;  // per lane: end of each group's run in `queue`
    std::vector<char> lane_query;         // per cloud: queried on its lane right after its build
    int n_lane_queries = 0;
    std::vector<int> group_k;             // distinct k of the other clouds, one persistent launch each
    std::vector<int> group_first;         // first descriptor of each group (+ end)
    std::vector<int64_t> group_items;     // 32-query items per group
};

bool device_reachable(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeManaged;
}

extern "C++" {
template <typename T>
int grow_batch(se_ctx* c, T*& p, int64_t count, const char* what) {
    ++c->batch_epoch;
    SE_CUDA(c, regrow(p, count), what);
    return SE_OK;
}
}

// Enqueue the whole batched sequence on c->graph_stream (recorded into a
// graph, or run directly): host-input copies, per-cloud builds on the lanes,
// one persistent kNN + normals launch per k group, the per-cloud u / error
// words, the host-output copies.
int enqueue_batch(se_ctx* c, const BatchPlan& plan, const BatchCloud* d_desc, const float* x, const float* y,
                  const float* z, const int64_t* offsets, int n_clouds, const int32_t* ks, float* out_normals,
                  float* bout, bool host, int& launches) {
    const int64_t total = offsets[n_clouds];
    cudaStream_t g = c->graph_stream;
    const float *bx = x, *by = y, *bz = z;
    if (host && total > 0) {
        SE_CUDA(c, cudaMemcpyAsync(c->batch_in, x, 4 * total, cudaMemcpyHostToDevice, g), "copy x");
        SE_CUDA(c, cudaMemcpyAsync(c->batch_in + total, y, 4 * total, cudaMemcpyHostToDevice, g), "copy y");
        SE_CUDA(c, cudaMemcpyAsync(c->batch_in + 2 * total, z, 4 * total, cudaMemcpyHostToDevice, g), "copy z");
        bx = c->batch_in;
        by = c->batch_in + total;
        bz = c->batch_in + 2 * total;
    }
    for (int ci = 0; ci < n_clouds; ++ci)
        if (offsets[ci + 1] == offsets[ci]) {  // empty cloud: no build clears its state
            SE_CUDA(c, cudaMemsetAsync(&c->batch_st[ci].u, 0, sizeof(unsigned long long), g), "reset batch");
            SE_CUDA(c, cudaMemsetAsync(&c->batch_st[ci].err, 0, sizeof(uint32_t), g), "reset batch");
        }
    SE_CUDA(c, cudaEventRecord(c->batch_in_ready, g), "event");
    launches = 0;
    for (int l = 0; l < plan.n_lanes; ++l) {
        BatchLane& lane = c->lanes[l];
        SE_CUDA(c, cudaStreamWaitEvent(lane.stream, c->batch_in_ready, 0), "wait");
        size_t gi = 0;
        for (int qi = 0; qi <= (int)plan.queue[l].size(); ++qi) {
            while (gi < plan.group_k.size() && plan.group_end[l][gi] == qi) {
                SE_CUDA(c, cudaEventRecord(lane.group_done[gi], lane.stream), "event");
                ++gi;
            }
            if (qi == (int)plan.queue[l].size()) break;
            const int ci = plan.queue[l][qi];
            const int64_t off = offsets[ci], n = offsets[ci + 1] - offsets[ci];
            BuildBufs b = lane.b;
            b.x = bx + off;
            b.y = by + off;
            b.z = bz + off;
            b.pts4 = c->batch_pts4 + off;
            b.snodes = c->batch_snodes + off;
            b.st = c->batch_st + ci;
            BuildParams p{n, c->opt.code_bits, 0, 0, c->opt.leaf_bucket};
            int nl = 0;
            SE_CUDA(c, enqueue_build(b, p, lane.stream, c->num_sms, nullptr, &nl), "launch batch build");
            launches += nl;
            if (plan.lane_query[ci]) {
                QueryParams q{};
                q.k = ks[ci];
                q.count = n;  // upper bound (grid size); u is read on the device
                q.u = n;
                q.device_count = 1;
                q.out_normals = bout + 3 * off;
                q.vx = c->opt.viewpoint[0];
                q.vy = c->opt.viewpoint[1];
                q.vz = c->opt.viewpoint[2];
                q.eigengap_fp64 = c->opt.eigengap_fp64;
                q.code_bits = c->opt.code_bits;
                q.bucket = c->opt.leaf_bucket;
                q.seed_halo = c->opt.seed_halo;
                SE_CUDA(c, enqueue_query(b, q, lane.stream, c->num_sms), "launch batch query");
                ++launches;
            }
        }
        SE_CUDA(c, cudaEventRecord(lane.done, lane.stream), "event");
        SE_CUDA(c, cudaStreamWaitEvent(g, lane.done, 0), "join");
    }
    for (size_t gi = 0; gi < plan.group_k.size(); ++gi) {
        for (int l = 0; l < plan.n_lanes; ++l)
            SE_CUDA(c, cudaStreamWaitEvent(g, c->lanes[l].group_done[gi], 0), "wait");
        QueryParams q{};
        q.k = plan.group_k[gi];
        q.vx = c->opt.viewpoint[0];
        q.vy = c->opt.viewpoint[1];
        q.vz = c->opt.viewpoint[2];
        q.eigengap_fp64 = c->opt.eigengap_fp64;
        q.code_bits = c->opt.code_bits;
        q.bucket = c->opt.leaf_bucket;
        q.seed_halo = c->opt.seed_halo;
        const int first = plan.group_first[gi], count = plan.group_first[gi + 1] - first;
        SE_CUDA(c, enqueue_query_batch(d_desc + first, count, plan.group_items[gi], c->batch_counter + gi, q, g,
                                       c->num_sms),
                "launch batch query");
        ++launches;
    }
    SE_CUDA(c, enqueue_batch_collect(c->batch_st, n_clouds, c->batch_u, c->batch_err, g), "launch batch collect");
    ++launches;
    if (host && total > 0 && bout == c->batch_out)  // staged (pageable) host output
        SE_CUDA(c, cudaMemcpyAsync(out_normals, bout, sizeof(float) * 3 * total, cudaMemcpyDeviceToHost, g),
                "copy normals");
    SE_CUDA(c, cudaMemcpyAsync(c->h_batch_u, c->batch_u, sizeof(unsigned long long) * n_clouds, cudaMemcpyDeviceToHost,
                               g),
            "read u");
    SE_CUDA(c, cudaMemcpyAsync(c->h_batch_err, c->batch_err, sizeof(uint32_t) * n_clouds, cudaMemcpyDeviceToHost, g),
            "read errors");
    return SE_OK;
}

}  // namespace

int se_normals_batch(se_ctx* c, const float* x, const float* y, const float* z, const int64_t* offsets, int n_clouds,
                     const int32_t* ks, float* out_normals, int64_t* out_u, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (n_clouds < 0 || (n_clouds > 0 && (!offsets || !ks || !out_u)))
        return fail(c, SE_ERR_INVALID_ARG, "bad batch description");
    if (n_clouds == 0) return SE_OK;
    if (offsets[0] != 0) return fail(c, SE_ERR_INVALID_ARG, "offsets[0] must be 0");
    if (c->opt.search_compat)
        return fail(c, SE_ERR_UNSUPPORTED, "the reference-compatible search is not available in batches");
    for (int i = 0; i < n_clouds; ++i) {
        if (offsets[i + 1] < offsets[i]) return fail(c, SE_ERR_INVALID_ARG, "offsets must not decrease");
        if (ks[i] < 1 || ks[i] > 32) return fail(c, SE_ERR_UNSUPPORTED, "k must be in [1, 32]");
    }
    const int64_t total = offsets[n_clouds];
    if (total > ((int64_t)1 << 30)) return fail(c, SE_ERR_INVALID_ARG, "more than 2^30 points in one batch");
    if (total > 0 && (!x || !y || !z || !out_normals)) return fail(c, SE_ERR_INVALID_ARG, "null pointer");
    const bool host = mem == SE_MEM_HOST;

    // ---- buffers (every move of one invalidates a recorded graph) ----
    if (c->batch_clouds_cap < n_clouds) {
        ++c->batch_epoch;
        if (c->batch_u) cudaFree(c->batch_u);
        if (c->batch_err) cudaFree(c->batch_err);
        if (c->batch_st) cudaFree(c->batch_st);
        if (c->batch_desc) cudaFree(c->batch_desc);
        if (c->h_batch_u) cudaFreeHost(c->h_batch_u);
        if (c->h_batch_err) cudaFreeHost(c->h_batch_err);
        if (c->h_batch_desc) cudaFreeHost(c->h_batch_desc);
        c->batch_u = nullptr;
        c->batch_err = nullptr;
        c->batch_st = nullptr;
        c->batch_desc = nullptr;
        c->h_batch_u = nullptr;
        c->h_batch_err = nullptr;
        c->h_batch_desc = nullptr;
        c->batch_clouds_cap = 0;
        SE_CUDA(c, cudaMalloc(&c->batch_u, sizeof(unsigned long long) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMalloc(&c->batch_err, sizeof(uint32_t) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMalloc(&c->batch_st, sizeof(DevState) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMalloc(&c->batch_desc, sizeof(BatchCloud) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMallocHost(&c->h_batch_u, sizeof(unsigned long long) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMallocHost(&c->h_batch_err, sizeof(uint32_t) * n_clouds), "alloc batch");
        SE_CUDA(c, cudaMallocHost(&c->h_batch_desc, sizeof(BatchCloud) * n_clouds), "alloc batch");
        c->batch_clouds_cap = n_clouds;
    }
    if (!c->batch_counter) SE_CUDA(c, cudaMalloc(&c->batch_counter, sizeof(unsigned long long) * 32), "alloc batch");
    if (!c->batch_in_ready) SE_CUDA(c, cudaEventCreateWithFlags(&c->batch_in_ready, cudaEventDisableTiming), "event");
    if (!c->batch_ev_in) SE_CUDA(c, cudaEventCreateWithFlags(&c->batch_ev_in, cudaEventDisableTiming), "event");
    if (!c->batch_ev_out) SE_CUDA(c, cudaEventCreateWithFlags(&c->batch_ev_out, cudaEventDisableTiming), "event");
    if (!c->graph_stream) SE_CUDA(c, cudaStreamCreateWithFlags(&c->graph_stream, cudaStreamNonBlocking), "stream");
    if (c->batch_pts_cap < total) {
        if (int rc = grow_batch(c, c->batch_pts4, total, "alloc batch points")) return rc;
        if (int rc = grow_batch(c, c->batch_snodes, total, "alloc batch hierarchy")) return rc;
        c->batch_pts_cap = total;
    }
    if (host && total > 0 && c->batch_cap < total) {
        if (int rc = grow_batch(c, c->batch_in, 3 * total, "alloc batch staging")) return rc;
        if (int rc = grow_batch(c, c->batch_out, 3 * total, "alloc batch staging")) return rc;
        c->batch_cap = total;
    }

    // ---- plan ----
    // Clouds of at least kLaneQueryMin points are queried on their lane right
    // after their build (a launch of their own fills enough of the GPU). The
    // rest share one persistent launch per k, after their builds; their k
    // groups go largest k first, so the costliest queries start while the
    // lanes still build later groups. Lanes take the large clouds first, then
    // the small ones group by group; largest cloud first, each to the lane
    // with the least queued work.
    constexpr int64_t kLaneQueryMin = 65536;
    BatchPlan plan;
    plan.lane_query.assign(n_clouds, 0);
    plan.n_lanes = std::min(n_clouds, 8);
    if ((int)c->lanes.size() < plan.n_lanes) c->lanes.resize(plan.n_lanes);
    std::vector<int> order(n_clouds);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return offsets[a + 1] - offsets[a] > offsets[b + 1] - offsets[b];
    });
    for (int ci : order) {
        const int64_t n = offsets[ci + 1] - offsets[ci];
        if (n == 0) continue;
        if (n >= kLaneQueryMin) {
            plan.lane_query[ci] = 1;
            ++plan.n_lane_queries;
        } else if (std::find(plan.group_k.begin(), plan.group_k.end(), ks[ci]) == plan.group_k.end()) {
            plan.group_k.push_back(ks[ci]);
        }
    }
    std::sort(plan.group_k.begin(), plan.group_k.end(), [](int a, int b) { return a > b; });
    plan.queue.assign(plan.n_lanes, {});
    plan.group_end.assign(plan.n_lanes, {});
    std::vector<int64_t> load(plan.n_lanes, 0), need(plan.n_lanes, 0);
    for (int ci : order) {
        if (!plan.lane_query[ci]) continue;
        const int64_t n = offsets[ci + 1] - offsets[ci];
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        plan.queue[l].push_back(ci);
        load[l] += 2 * n;  // build and query
        need[l] = std::max(need[l], n);
    }
    for (int k : plan.group_k) {
        for (int ci : order) {
            const int64_t n = offsets[ci + 1] - offsets[ci];
            if (n == 0 || ks[ci] != k || plan.lane_query[ci]) continue;
            const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            plan.queue[l].push_back(ci);
            load[l] += n + 4096;  // fixed cost per cloud
            need[l] = std::max(need[l], n);
        }
        for (int l = 0; l < plan.n_lanes; ++l) plan.group_end[l].push_back((int)plan.queue[l].size());
    }
    for (int l = 0; l < plan.n_lanes; ++l) {
        if (int rc = lane_capacity(c, c->lanes[l], need[l])) return rc;
        BatchLane& lane = c->lanes[l];
        while (lane.group_done.size() < plan.group_k.size()) {
            cudaEvent_t e = nullptr;
            SE_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "lane event");
            lane.group_done.push_back(e);
        }
    }
    std::vector<BatchCloud> desc;
    // a pinned host output is written by the kernels directly (mapped memory)
    float* bout = out_normals;
    if (host && total > 0) {
        bout = c->batch_out;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, out_normals) == cudaSuccess) {
            if (at.type == cudaMemoryTypeHost && at.devicePointer) bout = static_cast<float*>(at.devicePointer);
        } else {
            cudaGetLastError();
        }
    }
    for (int k : plan.group_k) {
        plan.group_first.push_back((int)desc.size());
        int64_t items = 0;
        for (int ci : order) {
            const int64_t off = offsets[ci], n = offsets[ci + 1] - offsets[ci];
            if (n == 0 || ks[ci] != k || plan.lane_query[ci]) continue;
            desc.push_back(BatchCloud{c->batch_pts4 + off, c->batch_snodes + off, c->batch_st + ci, bout + 3 * off, items});
            items += (n + 31) / 32;
        }
        plan.group_items.push_back(items);
    }
    plan.group_first.push_back((int)desc.size());

    // ---- graph key: layout, k's, buffers; a recorded graph replays only for the same key ----
    std::vector<int64_t> key;
    key.reserve(2 * n_clouds + 8);
    key.push_back(n_clouds);
    key.push_back(mem);
    key.push_back((int64_t)(uintptr_t)x);
    key.push_back((int64_t)(uintptr_t)y);
    key.push_back((int64_t)(uintptr_t)z);
    key.push_back((int64_t)(uintptr_t)out_normals);
    key.push_back((int64_t)c->batch_epoch);
    key.insert(key.end(), offsets, offsets + n_clouds + 1);
    key.insert(key.end(), ks, ks + n_clouds);
    const bool graphable = c->opt.batch_graph && total > 0 &&
                           (!host || (device_reachable(x) && device_reachable(y) && device_reachable(z) &&
                                      device_reachable(out_normals)));
    int hit = -1;
    for (int i = 0; i < (int)c->batch_graphs.size(); ++i)
        if (c->batch_graphs[i].key == key) hit = i;
    const bool replay = graphable && hit >= 0;

    // order after the caller's stream; the caller's stream waits for the result
    SE_CUDA(c, cudaEventRecord(c->batch_ev_in, c->stream), "event");
    SE_CUDA(c, cudaStreamWaitEvent(c->graph_stream, c->batch_ev_in, 0), "wait");
    int launches = 0;
    if (!replay) {
        // descriptors: the context's buffer for plain launches; a buffer of
        // its own for a recorded graph, so that other layouts cannot change it
        BatchCloud* d_desc = c->batch_desc;
        BatchGraph bg;
        if (graphable) {
            // keep the 3 most recent graphs whose buffers have not moved
            std::vector<BatchGraph> keep;
            for (BatchGraph& old : c->batch_graphs) {
                if (old.key[6] == (int64_t)c->batch_epoch) keep.push_back(old);
                else release_graph(old);
            }
            while (keep.size() > 3) {
                release_graph(keep.front());
                keep.erase(keep.begin());
            }
            c->batch_graphs = keep;
            bg.key = key;
            SE_CUDA(c, cudaMalloc(&bg.desc, sizeof(BatchCloud) * (desc.empty() ? 1 : desc.size())), "alloc batch");
            d_desc = bg.desc;
        }
        if (!desc.empty()) {
            std::memcpy(c->h_batch_desc, desc.data(), sizeof(BatchCloud) * desc.size());
            const cudaError_t e = cudaMemcpyAsync(d_desc, c->h_batch_desc, sizeof(BatchCloud) * desc.size(),
                                                  cudaMemcpyHostToDevice, c->graph_stream);
            if (e != cudaSuccess) {
                release_graph(bg);
                return cuda_fail(c, e, "copy batch descriptors");
            }
        }
        if (graphable) {
            cudaError_t ce = cudaStreamBeginCapture(c->graph_stream, cudaStreamCaptureModeThreadLocal);
            if (ce != cudaSuccess) {
                release_graph(bg);
                return cuda_fail(c, ce, "begin capture");
            }
            const int rc =
                enqueue_batch(c, plan, d_desc, x, y, z, offsets, n_clouds, ks, out_normals, bout, host, launches);
            cudaGraph_t graph = nullptr;
            ce = cudaStreamEndCapture(c->graph_stream, &graph);
            if (rc == SE_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&bg.exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (rc != SE_OK || ce != cudaSuccess) {
                release_graph(bg);
                return rc != SE_OK ? rc : cuda_fail(c, ce, "record batch graph");
            }
            bg.launches = launches;
            c->batch_graphs.push_back(bg);
            SE_CUDA(c, cudaGraphLaunch(bg.exec, c->graph_stream), "launch batch graph");
        } else {
            if (int rc =
                    enqueue_batch(c, plan, d_desc, x, y, z, offsets, n_clouds, ks, out_normals, bout, host, launches))
                return rc;
        }
    } else {
        BatchGraph bg = c->batch_graphs[hit];  // move to the most-recent end
        c->batch_graphs.erase(c->batch_graphs.begin() + hit);
        c->batch_graphs.push_back(bg);
        launches = bg.launches;
        SE_CUDA(c, cudaGraphLaunch(bg.exec, c->graph_stream), "launch batch graph");
    }
    SE_CUDA(c, cudaEventRecord(c->batch_ev_out, c->graph_stream), "event");
    SE_CUDA(c, cudaStreamWaitEvent(c->stream, c->batch_ev_out, 0), "wait");
    SE_CUDA(c, cudaStreamSynchronize(c->graph_stream), "synchronize");
    c->query_launches = plan.n_lane_queries + (int)plan.group_k.size() + 1;
    c->build_launches = launches - c->query_launches;
    c->have_build_times = false;
    c->have_query_times = false;
    uint32_t err = 0;
    for (int i = 0; i < n_clouds; ++i) {
        out_u[i] = (int64_t)c->h_batch_u[i];
        err |= c->h_batch_err[i];
    }
    return check_err_bits(c, err);
}

int se_synchronize(se_ctx* c) {
    if (int rc = prologue(c)) return rc;
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

}  // extern "C"
