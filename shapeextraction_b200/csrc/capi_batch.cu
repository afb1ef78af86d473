// C ABI: batched normals over many clouds (se_normals_batch). Declarations
// are in include/shapex.h.

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "context.cuh"

using namespace shapex;
using namespace shapex::capi;

extern "C" {

// ---- batched path --------------------------------------------------------------

namespace {

int batch_lanes(const se_ctx* c) { return c->opt.batch_lanes > 0 ? c->opt.batch_lanes : 8; }
int64_t batch_lane_min(const se_ctx* c) {
    return c->opt.batch_lane_min_points > 0 ? (int64_t)c->opt.batch_lane_min_points : 65536;
}

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
    SE_CUDA(c, regrow(b.lookback, sort_tiles * kSortBins + 64), "alloc lane");
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
                q.seed_halo = seed_halo_for(c, q.k);
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
        q.seed_halo = seed_halo_for(c, q.k);
        q.batch_blocks_per_sm = c->opt.batch_blocks_per_sm;
        q.batch_warps_per_block = c->opt.batch_warps_per_block;
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
    NvtxRange nvtx("shapex.se_normals_batch");
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
    const int64_t kLaneQueryMin = batch_lane_min(c);
    BatchPlan plan;
    plan.lane_query.assign(n_clouds, 0);
    plan.n_lanes = std::min(n_clouds, batch_lanes(c));
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
    // the tuning changes the launches
    key.push_back(c->opt.leaf_bucket);
    key.push_back(c->opt.seed_halo);
    key.push_back(batch_lanes(c));
    key.push_back(kLaneQueryMin);
    key.push_back(c->opt.batch_blocks_per_sm);
    key.push_back(c->opt.batch_warps_per_block);
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

int se_get_batch_tuning(const se_ctx* c, se_batch_tuning* t) {
    if (!c || !t) return SE_ERR_INVALID_ARG;
    t->leaf_bucket = c->opt.leaf_bucket;
    t->seed_halo = c->opt.seed_halo;
    t->lanes = batch_lanes(c);
    t->lane_min_points = (int32_t)batch_lane_min(c);
    t->blocks_per_sm = c->opt.batch_blocks_per_sm;
    t->warps_per_block = c->opt.batch_warps_per_block;
    return SE_OK;
}

int se_set_batch_tuning(se_ctx* c, const se_batch_tuning* t) {
    if (!c || !t) return SE_ERR_INVALID_ARG;
    if (t->leaf_bucket < 1 || t->leaf_bucket > 128 || t->seed_halo < -1 || t->seed_halo > 48 || t->lanes < 0 ||
        t->lanes > 16 || t->lane_min_points < 0 || t->blocks_per_sm < 0 || t->blocks_per_sm > 32 ||
        (t->warps_per_block != 0 && t->warps_per_block != 2 && t->warps_per_block != 4))
        return fail(c, SE_ERR_INVALID_ARG, "batch tuning out of range");
    c->opt.leaf_bucket = t->leaf_bucket;
    c->opt.seed_halo = t->seed_halo;
    c->opt.batch_lanes = t->lanes;
    c->opt.batch_lane_min_points = t->lane_min_points;
    c->opt.batch_blocks_per_sm = t->blocks_per_sm;
    c->opt.batch_warps_per_block = t->warps_per_block;
    return SE_OK;
}

int se_tune_batch(se_ctx* c, const float* x, const float* y, const float* z, const int64_t* offsets, int n_clouds,
                  const int32_t* ks, int mem, int reps, se_batch_tuning* best, float* best_ms) {
    NvtxRange nvtx("shapex.se_tune_batch");
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (n_clouds < 1 || !offsets || !ks) return fail(c, SE_ERR_INVALID_ARG, "bad batch description");
    if (reps < 1) reps = 1;
    const int64_t total = offsets[n_clouds];
    if (total < 0 || total > ((int64_t)1 << 30)) return fail(c, SE_ERR_INVALID_ARG, "bad batch size");
    // outputs like the caller's: device memory, or pinned host memory
    float* out = nullptr;
    const bool host = mem == SE_MEM_HOST;
    const size_t out_bytes = sizeof(float) * 3 * (size_t)(total > 0 ? total : 1);
    cudaError_t e = host ? cudaMallocHost(&out, out_bytes) : cudaMalloc(&out, out_bytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "alloc tuner output");
    std::vector<int64_t> u(n_clouds);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    se_batch_tuning orig{}, cur{};
    se_get_batch_tuning(c, &orig);
    cur = orig;
    int rc = SE_OK;
    // median over reps of one configuration (a first untimed call records its graph)
    auto measure = [&](const se_batch_tuning& t, float& ms) -> int {
        if (int r = se_set_batch_tuning(c, &t)) return r;
        if (int r = se_normals_batch(c, x, y, z, offsets, n_clouds, ks, out, u.data(), mem)) return r;
        std::vector<float> ts;
        for (int i = 0; i < reps; ++i) {
            cudaEventRecord(e0, c->stream);
            if (int r = se_normals_batch(c, x, y, z, offsets, n_clouds, ks, out, u.data(), mem)) return r;
            cudaEventRecord(e1, c->stream);
            const cudaError_t ce = cudaEventSynchronize(e1);
            if (ce != cudaSuccess) return cuda_fail(c, ce, "time batch");
            float t_ms = 0.0f;
            cudaEventElapsedTime(&t_ms, e0, e1);
            ts.push_back(t_ms);
        }
        std::sort(ts.begin(), ts.end());
        ms = ts[ts.size() / 2];
        return SE_OK;
    };
    float cur_ms = 0.0f;
    rc = measure(cur, cur_ms);
    // coordinate descent, two rounds: each parameter over its values, the others fixed
    static const int kBucket[] = {48, 64, 96, 128};
    static const int kHalo[] = {-1, 8, 16, 32};
    static const int kLanes[] = {4, 8, 16};
    static const int kLaneMin[] = {32768, 65536, 131072, 262144};
    static const int kBlocks[] = {0, 2, 3, 4};
    static const int kWarps[] = {2, 4};
    for (int round = 0; round < 2 && rc == SE_OK; ++round) {
        for (int dim = 0; dim < 6 && rc == SE_OK; ++dim) {
            const int* vals;
            int nv;
            int32_t se_batch_tuning::*field;
            switch (dim) {
                case 0: vals = kBucket; nv = 4; field = &se_batch_tuning::leaf_bucket; break;
                case 1: vals = kHalo; nv = 4; field = &se_batch_tuning::seed_halo; break;
                case 2: vals = kLanes; nv = 3; field = &se_batch_tuning::lanes; break;
                case 3: vals = kLaneMin; nv = 4; field = &se_batch_tuning::lane_min_points; break;
                case 4: vals = kBlocks; nv = 4; field = &se_batch_tuning::blocks_per_sm; break;
                default: vals = kWarps; nv = 2; field = &se_batch_tuning::warps_per_block; break;
            }
            for (int vi = 0; vi < nv && rc == SE_OK; ++vi) {
                if (cur.*field == vals[vi]) continue;
                se_batch_tuning t = cur;
                t.*field = vals[vi];
                float ms = 0.0f;
                rc = measure(t, ms);
                if (rc == SE_OK && ms < cur_ms) {
                    cur = t;
                    cur_ms = ms;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (host) cudaFreeHost(out);
    else cudaFree(out);
    if (rc != SE_OK) {
        const std::string msg = c->last_error;
        se_set_batch_tuning(c, &orig);
        c->last_error = msg;
        return rc;
    }
    se_set_batch_tuning(c, &cur);
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return SE_OK;
}

}  // extern "C"
