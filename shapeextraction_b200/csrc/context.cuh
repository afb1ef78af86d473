// The context behind the C ABI (se_ctx) and the helpers its entry points
// share: status mapping, CUDA error checks, buffer regrowth. Included by the
// translation units of the ABI: capi.cu (context, build, queries), capi_mlp.cu
// (learned search radius) and capi_batch.cu (batched normals).
#pragma once

#include <cstdint>
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
    int debug_pending = 0;  // SE_DEBUG_* test hooks not fired yet (from options.debug_inject)
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
    float mlp_tau = 0.0f;  // training loss: 0 squared error, else the pinball loss of this quantile
    bool mlp_ready = false;
    MlpWork mw{};
    int64_t mw_cap = 0;
    float* r2_buf = nullptr;
    int64_t r2_cap = 0;
    // code-range table of the current build for the learned cell scan
    uint32_t* lut_buf = nullptr;
    int64_t lut_cap = 0;
    int lut_level = 0;  // 0: not built for the current build
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

namespace shapex {
namespace capi {

// Record the message in the context and return the status.
int fail(se_ctx* c, int status, const std::string& msg);
// SE_ERR_OOM for an allocation failure, SE_ERR_CUDA otherwise; clears the CUDA error.
int cuda_fail(se_ctx* c, cudaError_t e, const char* where);
// Status for the device error word of a build or query.
int check_err_bits(se_ctx* c, uint32_t err);
// Makes the context's device current.
int prologue(se_ctx* c);
int check_mem(se_ctx* c, int mem);
// The seed halo a query of k neighbours uses (the option, or its per-k default).
int seed_halo_for(const se_ctx* c, int k);

#define SE_CUDA(c, call, where)                                          \
    do {                                                                 \
        cudaError_t _e = (call);                                         \
        if (_e != cudaSuccess) return ::shapex::capi::cuda_fail(c, _e, where); \
    } while (0)

// Free p and allocate count elements (nothing for count <= 0).
template <typename T>
cudaError_t regrow(T*& p, int64_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count <= 0) return cudaSuccess;
    return cudaMalloc((void**)&p, sizeof(T) * (size_t)count);
}

}  // namespace capi
}  // namespace shapex
