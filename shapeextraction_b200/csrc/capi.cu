// C ABI of the normal-estimation path: context lifetime, build, getters and
// queries. The learned-radius entry points are in capi_mlp.cu, the batched
// path in capi_batch.cu. Declarations and the reference interface each entry
// point replaces are in include/shapex.h.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "context.cuh"

using namespace shapex;
using namespace shapex::capi;

namespace shapex {
namespace capi {

int fail(se_ctx* c, int status, const std::string& msg) {
    if (c) c->last_error = msg;
    return status;
}

int cuda_fail(se_ctx* c, cudaError_t e, const char* where) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(c, SE_ERR_OOM, std::string(where) + ": out of device memory");
    return fail(c, SE_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
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

int prologue(se_ctx* c) {
    if (!c) return SE_ERR_INVALID_ARG;
    SE_CUDA(c, cudaSetDevice(c->opt.device), "cudaSetDevice");
    return SE_OK;
}

int seed_halo_for(const se_ctx* c, int k) {
    // a larger window pays once the list is long: at k = 32 a 32-point halo
    // was 15% faster than 16 on a 2M-point scene; at k <= 16 the two tie
    if (c->opt.seed_halo >= 0) return c->opt.seed_halo;
    return k > 16 ? 32 : 16;
}

int check_mem(se_ctx* c, int mem) {
    if (mem != SE_MEM_HOST && mem != SE_MEM_DEVICE) return fail(c, SE_ERR_INVALID_ARG, "mem must be SE_MEM_HOST or SE_MEM_DEVICE");
    return SE_OK;
}

}  // namespace capi
}  // namespace shapex

namespace {

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
    if (c->debug_pending & SE_DEBUG_ALLOC_FAIL) {  // test hook: this growth fails as cudaMalloc would
        c->debug_pending &= ~SE_DEBUG_ALLOC_FAIL;
        return cuda_fail(c, cudaErrorMemoryAllocation, "alloc keys (injected by SE_DEBUG_ALLOC_FAIL)");
    }
    const int64_t cap = n < 1024 ? 1024 : n;
    BuildBufs& b = c->b;
    const int64_t sort_tiles = (cap + kSortTile - 1) / kSortTile;
    const int64_t scan_tiles = (cap + kScanTile - 1) / kScanTile;
    SE_CUDA(c, regrow(b.keys0, cap), "alloc keys");
    SE_CUDA(c, regrow(b.keys1, cap), "alloc keys");
    SE_CUDA(c, regrow(b.lookback, sort_tiles * kSortBins + 64), "alloc lookback");
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


int read_state(se_ctx* c) {
    SE_CUDA(c, cudaMemcpyAsync(c->h_st, c->b.st, sizeof(DevState), cudaMemcpyDeviceToHost, c->stream), "read state");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

cudaMemcpyKind kind_out(int mem) { return mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice; }



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
    q.seed_halo = seed_halo_for(c, k);
    q.compat = c->opt.search_compat ? 1 : 0;
    q.n_octree = c->info.n_octree;
    if (c->debug_pending & SE_DEBUG_SEARCH_LIMIT) {  // test hook: one node visit per warp
        c->debug_pending &= ~SE_DEBUG_SEARCH_LIMIT;
        q.step_limit = 1;
    }
    if (q.compat && q.n_octree < 1)
        return fail(c, SE_ERR_UNSUPPORTED, "the reference-compatible search needs the octree (build_octree = 1, u >= 2)");
    const bool use_learned = c->opt.learned && !ext && c->mlp_ready && !q.compat;
    if (use_learned && c->r2_cap < count) {
        SE_CUDA(c, regrow(c->r2_buf, count), "alloc learned bounds");
        c->r2_cap = count;
    }
    q.learned_r2 = use_learned ? c->r2_buf : nullptr;
    q.learned_skip_seed = c->opt.learned_skip_seed;
    // with learned_cell_scan the learned attempt scans Morton cells directly
    // (no tree walk); it needs the seed skipped
    const bool cells = use_learned && c->opt.learned_skip_seed && c->opt.learned_cell_scan;
    bool lut_launched = false;
    if (cells && c->lut_level == 0) {
        // table level: at least 2 codes per entry on average, 8^7 entries (8 MB) at most
        const int bpa = c->opt.code_bits / 3;
        int level = 1;
        while (level < bpa && level < 7 && ((int64_t)8 << (3 * level)) * 2 <= u) ++level;
        const int64_t n_ent = ((int64_t)1 << (3 * level)) + 1;
        if (c->lut_cap < n_ent) {
            SE_CUDA(c, regrow(c->lut_buf, n_ent), "alloc cell table");
            c->lut_cap = n_ent;
        }
        SE_CUDA(c, enqueue_cell_lut(c->b, c->opt.code_bits, level, c->lut_buf, c->stream, c->num_sms),
                "launch cell table");
        c->lut_level = level;
        lut_launched = true;
    }
    if (cells) {
        q.cell_lut = c->lut_buf;
        q.lut_shift = c->opt.code_bits / 3 - c->lut_level;
        q.cell_pmax = c->opt.cell_max_points > 0 ? c->opt.cell_max_points : 4096;
        q.cell_span = c->opt.cell_span > 0 ? c->opt.cell_span : 3;
    }
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
    c->query_launches = (use_learned ? 2 : 1) + (lut_launched ? 1 : 0);
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
    o->leaf_bucket = 96;
    o->device = 0;
    o->stream = nullptr;
    o->seed_halo = -1;
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
    if (o.leaf_bucket == 0) o.leaf_bucket = 96;
    if (o.leaf_bucket < 1 || o.leaf_bucket > 128) return SE_ERR_INVALID_ARG;
    if (o.seed_halo < 0) o.seed_halo = -1;  // per-k default, resolved by seed_halo_for
    if (o.seed_halo > 48) return SE_ERR_INVALID_ARG;
    if (!(o.eigengap_fp64 >= 0.0f)) return SE_ERR_INVALID_ARG;
    if (o.debug_wait_limit < 0) return SE_ERR_INVALID_ARG;
    if (o.learned_cell_scan != 0 && o.learned_cell_scan != 1) return SE_ERR_INVALID_ARG;
    if (o.cell_span != 0 && (o.cell_span < 2 || o.cell_span > 4)) return SE_ERR_INVALID_ARG;
    if (o.cell_max_points < 0) return SE_ERR_INVALID_ARG;
    if (o.batch_lanes < 0 || o.batch_lanes > 16 || o.batch_lane_min_points < 0 || o.batch_blocks_per_sm < 0 ||
        o.batch_blocks_per_sm > 32 ||
        (o.batch_warps_per_block != 0 && o.batch_warps_per_block != 2 && o.batch_warps_per_block != 4))
        return SE_ERR_INVALID_ARG;
    if (o.debug_inject & ~(SE_DEBUG_STALL_SORT_TILE | SE_DEBUG_SEARCH_LIMIT | SE_DEBUG_ALLOC_FAIL))
        return SE_ERR_INVALID_ARG;
    se_ctx* c = new se_ctx();
    c->opt = o;
    c->debug_pending = o.debug_inject;
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
    if (c->lut_buf) cudaFree(c->lut_buf);
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
    NvtxRange nvtx("shapex.se_build");
    if (int rc = prologue(c)) return rc;
    c->built = false;
    c->lut_level = 0;
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
    if (c->opt.debug_wait_limit > 0) p.spin_limit = c->opt.debug_wait_limit;
    if (c->debug_pending & SE_DEBUG_STALL_SORT_TILE) {  // test hook: the first sort tile never publishes
        c->debug_pending &= ~SE_DEBUG_STALL_SORT_TILE;
        p.stall_first_tile = 1;
    }
    c->have_build_times = false;
    SE_CUDA(c, enqueue_build(b, p, c->stream, c->num_sms, c->build_ev, &c->build_launches), "launch build");
    if (int rc = read_state(c)) return rc;
    c->have_build_times = true;
    // any other failure first: the octree count of a failed build means nothing
    if (int rc = check_err_bits(c, c->h_st->err & ~(uint32_t)ERRBIT_OCT_CAPACITY)) return rc;
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
    NvtxRange nvtx("shapex.se_knn_self");
    if (int rc = prologue(c)) return rc;
    if (!out_idx && count > 0) return fail(c, SE_ERR_INVALID_ARG, "null output");
    return run_query(c, k, start, count, nullptr, out_idx, out_d2, nullptr, mem);
}

int se_knn(se_ctx* c, int k, const float* queries, int64_t nq, int32_t* out_idx, float* out_d2, int mem) {
    NvtxRange nvtx("shapex.se_knn");
    if (int rc = prologue(c)) return rc;
    if (nq > 0 && (!queries || !out_idx)) return fail(c, SE_ERR_INVALID_ARG, "null pointer");
    if (nq == 0) return SE_OK;
    return run_query(c, k, 0, nq, queries, out_idx, out_d2, nullptr, mem);
}

int se_normals(se_ctx* c, int k, int64_t start, int64_t count, float* out, int mem) {
    NvtxRange nvtx("shapex.se_normals");
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

int se_synchronize(se_ctx* c) {
    if (int rc = prologue(c)) return rc;
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

}  // extern "C"
