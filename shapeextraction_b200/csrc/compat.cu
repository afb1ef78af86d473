// Reference-compatible kNN search and normals.
//
// Reproduces the reference's approximate search bit-exactly on the GPU:
// knnSearchKernel<k> (src/Octree.hpp:136-193) walks the OTNode array best
// first with a bounded search heap of 32 node slots (SEARCH_Q_SIZE,
// src/Octree.hpp:17) and a result heap of k point slots, both the bounded
// min-max heap of src/dequeue.hpp:55-289 (a full heap drops its largest
// priority when the new one is not larger, src/dequeue.hpp:60-67). Node
// priority is nodeBoxDistance (src/Octree.cu:326-352): 0 inside the cube,
// else the smallest distance to one of its six face planes. Point priority is
// Point::distance2 (src/PointCloud.hpp:30-35) as nvcc contracts it,
// fma(dz, dz, fma(dx, dx, dy*dy)). The search runs until the node heap is
// empty (the early stop of src/Octree.hpp:152-155 never fires because its
// bound is never updated). Results leave the result heap in remove-min order;
// a query with fewer than k results repeats its first one
// (src/Octree.hpp:181-191).
//
// The normals of this mode follow estimateNormals (src/NormalEstimation.hpp:
// 96-192): centroid as a plain FP32 sum divided by k, covariance as FP32 fmas
// of the centred points divided by k-1, in the neighbours' output order; the
// 3x3 eigensolve, done by a closed library in the reference, is the FP64
// Jacobi of the exact mode on that FP32 matrix; orientation towards the
// viewpoint.
//
// Layout: one thread per query. Both heaps live in shared memory as
// [slot][thread] arrays, so the threads of a warp touch 32 distinct banks
// whatever slots they address. Queries are the tree's Morton-ordered points
// (or caller queries), so neighbouring threads walk similar paths.

#include <cstdint>

#include "eig3.cuh"
#include "pipeline.cuh"

namespace shapex {

namespace {

constexpr int kCompatThreads = 128;
constexpr int kSearchSlots = 32;  // SEARCH_Q_SIZE, src/Octree.hpp:17

// Bounded min-max heap over one thread's column of [slot][thread] arrays.
// Even levels are min levels, odd levels max levels (src/dequeue.hpp:55-289).
struct ColumnHeap {
    float* pri;     // pri[slot * kCompatThreads]
    int32_t* item;  // item[slot * kCompatThreads]
    int size;
    int cap;

    __device__ __forceinline__ float P(int i) const { return pri[i * kCompatThreads]; }
    __device__ __forceinline__ void swp(int a, int b) {
        const float pa = pri[a * kCompatThreads];
        const int32_t ia = item[a * kCompatThreads];
        pri[a * kCompatThreads] = pri[b * kCompatThreads];
        item[a * kCompatThreads] = item[b * kCompatThreads];
        pri[b * kCompatThreads] = pa;
        item[b * kCompatThreads] = ia;
    }
    static __device__ __forceinline__ int par(int i) { return (i - 1) / 2; }
    static __device__ __forceinline__ int lc(int i) { return 2 * i + 1; }
    static __device__ __forceinline__ int rc(int i) { return 2 * i + 2; }
    static __device__ __forceinline__ bool min_level(int i) { return ((31 - __clz(i + 1)) & 1) == 0; }

    __device__ __forceinline__ int largest() const {
        if (size >= 2) {
            if (size == 2) return 1;
            return P(1) > P(2) ? 1 : 2;
        }
        return 0;
    }
    __device__ void up_min(int i) {
        while (i >= 3) {
            const int g = par(par(i));
            if (P(i) < P(g)) {
                swp(i, g);
                i = g;
            } else {
                break;
            }
        }
    }
    __device__ void up_max(int i) {
        while (i >= 3) {
            const int g = par(par(i));
            if (P(i) > P(g)) {
                swp(i, g);
                i = g;
            } else {
                break;
            }
        }
    }
    __device__ void bubble_up(int i) {
        if (min_level(i)) {
            if (i > 0 && P(i) > P(par(i))) {
                swp(i, par(i));
                up_max(par(i));
            } else {
                up_min(i);
            }
        } else {
            if (i > 0 && P(i) < P(par(i))) {
                swp(i, par(i));
                up_min(par(i));
            } else {
                up_max(i);
            }
        }
    }
    // smallest (MIN) or largest (!MIN) of i's children and grandchildren,
    // first in the order lc, rc, lc(lc), rc(lc), lc(rc), rc(rc) on ties
    template <bool MIN>
    __device__ __forceinline__ int pick(int i) const {
        int m = lc(i);
        float pm = P(m);
        const int desc[5] = {rc(i), lc(lc(i)), rc(lc(i)), lc(rc(i)), rc(rc(i))};
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            if (desc[d] < size) {
                const float pd = P(desc[d]);
                if (MIN ? pd < pm : pd > pm) {
                    m = desc[d];
                    pm = pd;
                }
            }
        }
        return m;
    }
    template <bool MIN>
    __device__ void down(int i) {
        while (lc(i) < size) {
            const int m = pick<MIN>(i);
            if (m > rc(i)) {  // a grandchild
                if (MIN ? P(m) < P(i) : P(m) > P(i)) {
                    swp(i, m);
                    if (MIN ? P(m) > P(par(m)) : P(m) < P(par(m))) swp(par(m), m);
                    i = m;
                } else {
                    break;
                }
            } else {  // a child
                if (MIN ? P(m) < P(i) : P(m) > P(i)) swp(i, m);
                break;
            }
        }
    }
    __device__ __forceinline__ void percolate(int i) {
        if (min_level(i)) down<true>(i);
        else down<false>(i);
    }
    __device__ __forceinline__ void remove_min(float& p, int32_t& it) {
        p = P(0);
        it = item[0];
        --size;
        pri[0] = P(size);
        item[0] = item[size * kCompatThreads];
        percolate(0);
    }
    __device__ __forceinline__ void remove_max() {
        const int l = largest();
        --size;
        pri[l * kCompatThreads] = P(size);
        item[l * kCompatThreads] = item[size * kCompatThreads];
        percolate(l);
    }
    __device__ __forceinline__ void insert(int32_t it, float w) {
        if (size == cap) {
            if (P(largest()) >= w) remove_max();
            else return;
        }
        ++size;
        pri[(size - 1) * kCompatThreads] = w;
        item[(size - 1) * kCompatThreads] = it;
        bubble_up(size - 1);
    }
};

// nodeBoxDistance, src/Octree.cu:326-352
__device__ __forceinline__ float face_distance(float qx, float qy, float qz, const OtNode& n) {
    const float x1 = n.corner[0], x2 = __fadd_rn(n.corner[0], n.cell_size);
    const float y1 = n.corner[1], y2 = __fadd_rn(n.corner[1], n.cell_size);
    const float z1 = n.corner[2], z2 = __fadd_rn(n.corner[2], n.cell_size);
    if (qx > x1 && qx < x2 && qy > y1 && qy < y2 && qz > z1 && qz < z2) return 0.0f;
    float m = fabsf(__fsub_rn(qx, x1));
    m = fminf(m, fabsf(__fsub_rn(qx, x2)));
    m = fminf(m, fabsf(__fsub_rn(qy, y1)));
    m = fminf(m, fabsf(__fsub_rn(qy, y2)));
    m = fminf(m, fabsf(__fsub_rn(qz, z1)));
    m = fminf(m, fabsf(__fsub_rn(qz, z2)));
    return m;
}

// Point::distance2 as the reference build contracts it
__device__ __forceinline__ float ref_distance2(float qx, float qy, float qz, float4 p) {
    const float dx = __fsub_rn(qx, p.x), dy = __fsub_rn(qy, p.y), dz = __fsub_rn(qz, p.z);
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

struct CompatArgs {
    int k;
    int64_t start, count, u, m;
    const float* ext;
    int32_t* out_idx;
    float* out_d2;
    float* out_normals;
    float vx, vy, vz;
};

template <bool EXT, bool NORMALS>
__global__ void __launch_bounds__(kCompatThreads)
    k_knn_compat(const OtNode* __restrict__ nodes, const float4* __restrict__ pts, CompatArgs a, DevState* st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    float* s_pri = reinterpret_cast<float*>(smem_raw);
    int32_t* s_item = reinterpret_cast<int32_t*>(s_pri + kSearchSlots * kCompatThreads);
    float* r_pri = reinterpret_cast<float*>(s_item + kSearchSlots * kCompatThreads);
    int32_t* r_item = reinterpret_cast<int32_t*>(r_pri + a.k * kCompatThreads);
    const int64_t qi = (int64_t)blockIdx.x * kCompatThreads + tid;
    if (qi >= a.count) return;
    float qx, qy, qz;
    if (EXT) {
        qx = a.ext[3 * qi];
        qy = a.ext[3 * qi + 1];
        qz = a.ext[3 * qi + 2];
    } else {
        const float4 q = pts[a.start + qi];
        qx = q.x;
        qy = q.y;
        qz = q.z;
    }
    ColumnHeap sq{s_pri + tid, s_item + tid, 0, kSearchSlots};
    ColumnHeap rq{r_pri + tid, r_item + tid, 0, a.k};
    uint32_t err = 0;
    sq.insert(0, 0.0f);
    // every node enters the heap at most once (children of a popped node), so
    // a walk of more than m pops means a malformed octree
    int64_t pops = 0;
    while (sq.size > 0) {
        float pr;
        int32_t ni;
        sq.remove_min(pr, ni);
        if (++pops > a.m) {
            err |= ERRBIT_SEARCH_LIMIT;
            break;
        }
        const OtNode& nd = nodes[ni];
        const int leaf_mask = nd.child_leaf_mask, node_mask = nd.child_node_mask;
        if (leaf_mask) {
#pragma unroll 1
            for (int c = 0; c < 8; ++c) {
                if (leaf_mask & (1 << c)) {
                    const int32_t li = nd.children[c];
                    if (li < 0 || li >= a.u) {
                        err |= ERRBIT_BOUNDS;
                        continue;
                    }
                    rq.insert(li, ref_distance2(qx, qy, qz, __ldg(pts + li)));
                }
            }
        }
#pragma unroll 1
        for (int c = 0; c < 8; ++c) {
            if (node_mask & (1 << c)) {
                const int32_t ci = nd.children[c];
                if (ci < 0 || ci >= a.m) {
                    err |= ERRBIT_BOUNDS;
                    continue;
                }
                sq.insert(ci, face_distance(qx, qy, qz, nodes[ci]));
            }
        }
    }
    // results in remove-min order, written back into the (empty) node heap's
    // column so that the covariance reads them in that order
    int32_t* order = s_item + tid;
    float* order_d2 = s_pri + tid;
    int32_t first = -1;
    float first_d2 = __int_as_float(0x7f800000);
    for (int c = 0; c < a.k; ++c) {
        int32_t it;
        float p;
        if (rq.size == 0) {
            it = first;
            p = first_d2;
        } else {
            rq.remove_min(p, it);
        }
        if (c == 0) {
            first = it;
            first_d2 = p;
        }
        order[c * kCompatThreads] = it;
        order_d2[c * kCompatThreads] = p;
    }
    if (a.out_idx) {
        for (int c = 0; c < a.k; ++c) a.out_idx[qi * a.k + c] = order[c * kCompatThreads];
        if (a.out_d2)
            for (int c = 0; c < a.k; ++c) a.out_d2[qi * a.k + c] = order_d2[c * kCompatThreads];
    }
    if (NORMALS) {
        float* out = a.out_normals + 3 * qi;
        if (first < 0) {
            out[0] = out[1] = out[2] = __int_as_float(0x7fc00000);
        } else {
            // calculateCovariance<k>, src/NormalEstimation.hpp:96-120
            float cx = 0.0f, cy = 0.0f, cz = 0.0f;
            for (int c = 0; c < a.k; ++c) {
                const float4 p = __ldg(pts + order[c * kCompatThreads]);
                cx = __fadd_rn(cx, p.x);
                cy = __fadd_rn(cy, p.y);
                cz = __fadd_rn(cz, p.z);
            }
            const float fk = (float)a.k;
            cx = __fdiv_rn(cx, fk);
            cy = __fdiv_rn(cy, fk);
            cz = __fdiv_rn(cz, fk);
            float cv[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            for (int c = 0; c < a.k; ++c) {
                const float4 p = __ldg(pts + order[c * kCompatThreads]);
                const float m0 = __fsub_rn(p.x, cx), m1 = __fsub_rn(p.y, cy), m2 = __fsub_rn(p.z, cz);
                cv[0] = __fmaf_rn(m0, m0, cv[0]);
                cv[1] = __fmaf_rn(m0, m1, cv[1]);
                cv[2] = __fmaf_rn(m0, m2, cv[2]);
                cv[3] = __fmaf_rn(m1, m1, cv[3]);
                cv[4] = __fmaf_rn(m1, m2, cv[4]);
                cv[5] = __fmaf_rn(m2, m2, cv[5]);
            }
            const float den = (float)(a.k - 1);
            double C[6];
#pragma unroll
            for (int e = 0; e < 6; ++e) C[e] = (double)__fdiv_rn(cv[e], den);
            double w[3], nv[3];
            eig3<double>(C, w, nv);
            float nx = (float)nv[0], ny = (float)nv[1], nz = (float)nv[2];
            // normalsFromEigenVectors, src/NormalEstimation.hpp:158-192
            const float dot = (a.vx - qx) * nx + (a.vy - qy) * ny + (a.vz - qz) * nz;
            if (dot < 0.0f) {
                nx = -nx;
                ny = -ny;
                nz = -nz;
            }
            out[0] = nx;
            out[1] = ny;
            out[2] = nz;
        }
    }
    if (err) atomicOr(&st->err, err);
}

template <bool EXT, bool NORMALS>
cudaError_t launch_compat(const BuildBufs& b, const CompatArgs& a, cudaStream_t s) {
    const int smem = (kSearchSlots + a.k) * kCompatThreads * 8;
    cudaError_t e = cudaFuncSetAttribute(k_knn_compat<EXT, NORMALS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((a.count + kCompatThreads - 1) / kCompatThreads);
    k_knn_compat<EXT, NORMALS><<<blocks, kCompatThreads, smem, s>>>(static_cast<const OtNode*>(b.oct_nodes), b.pts4,
                                                                    a, b.st);
    return cudaGetLastError();
}

}  // namespace

cudaError_t enqueue_query_compat(const BuildBufs& b, const QueryParams& q, cudaStream_t s) {
    if (q.count <= 0) return cudaSuccess;
    if (q.k < 1 || q.k > 32 || q.n_octree < 1 || !b.oct_nodes) return cudaErrorInvalidValue;
    CompatArgs a;
    a.k = q.k;
    a.start = q.start;
    a.count = q.count;
    a.u = q.u;
    a.m = q.n_octree;
    a.ext = q.ext_queries;
    a.out_idx = q.out_idx;
    a.out_d2 = q.out_d2;
    a.out_normals = q.out_normals;
    a.vx = q.vx;
    a.vy = q.vy;
    a.vz = q.vz;
    if (a.ext) return launch_compat<true, false>(b, a, s);
    if (a.out_normals) return launch_compat<false, true>(b, a, s);
    return launch_compat<false, false>(b, a, s);
}

}  // namespace shapex
