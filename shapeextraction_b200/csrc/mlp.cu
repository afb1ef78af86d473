// Learned search-radius proposal: per-point occupancy features and a 3-layer
// MLP (32 -> 64 -> 64 -> 1, BF16 weights and activations, FP32 accumulation)
// that predicts log2(r_k^2 / range^2), the squared distance to a point's k-th
// neighbour in units of the cloud's extent. Training (forward, backward,
// weight-gradient reductions, Adam) and inference are kernels of this file;
// inference runs the two hidden layers on the tensor cores (mma.sync
// m16n8k16, BF16 in, FP32 accumulate), fused with the feature computation.
// The exact kNN search uses the prediction only as a starting bound and falls
// back to the plain search for any query whose k-th neighbour lies beyond it.

#include <cstdint>
#include <cuda_bf16.h>

#include "pipeline.cuh"

namespace shapex {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// ---------------------------------------------------------------------------
// Features of query qi (a tree point), all scale-free:
//   0..11  log2(d2 to the Morton neighbours at +-1, 2, 4, 8, 16, 32) - log2(range^2), / 16
//   12..27 for the leaf's first 8 ancestors in the search hierarchy (parent
//          first): log2(points under the node) / 21, then its code-prefix
//          length / 63; past the root the root's values repeat. A node of s
//          points with a p-bit prefix spans a cube of side range * 2^(-p/3),
//          so each pair measures the local density at one scale.
//   28     log2(u) / 30
//   29     1 (bias)
//   30..31 0
// Eight dependent ancestor steps cover the scales around k. A walk over 16
// occupancy levels (up to ~40 steps) predicted about as well (residual spread
// within 5%) at several times the cost.
// ---------------------------------------------------------------------------
__device__ void point_features(int64_t qi, const float4* __restrict__ pts, const int32_t* __restrict__ leaf_parent,
                               const int32_t* __restrict__ sparent, const uint8_t* __restrict__ prefix_n,
                               const int32_t* __restrict__ range_end, const uint64_t* __restrict__ codes, int64_t u,
                               int code_bits, float log2_range2, float (&f)[kMlpF]) {
#pragma unroll
    for (int j = 0; j < kMlpF; ++j) f[j] = 0.0f;
    f[29] = 1.0f;
    f[28] = __log2f((float)u) * (1.0f / 30.0f);
    const float4 p = __ldg(pts + qi);
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int64_t j = 1 << s;
        int64_t a = qi + j, b = qi - j;
        if (a >= u) a = b >= 0 ? b : qi;
        if (b < 0) b = a;
        const float4 pa = __ldg(pts + a), pb = __ldg(pts + b);
        const float da = dist2(p.x, p.y, p.z, pa.x, pa.y, pa.z), db = dist2(p.x, p.y, p.z, pb.x, pb.y, pb.z);
        f[2 * s] = (__log2f(da + 1e-30f) - log2_range2) * (1.0f / 16.0f);
        f[2 * s + 1] = (__log2f(db + 1e-30f) - log2_range2) * (1.0f / 16.0f);
    }
    if (u < 2) return;
    const int root_pn = __clzll((long long)(codes[0] ^ codes[u - 1])) - (64 - code_bits);
    int64_t node = leaf_parent[qi];
    float size = 1.0f, pn = (float)code_bits;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (node >= 0 && node < u - 1) {
            pn = (float)(node == 0 ? root_pn : (int)prefix_n[node]);
            const int64_t e = range_end[node];
            size = (float)((e > node ? e - node : node - e) + 1);
            node = node == 0 ? -1 : sparent[node];
        }
        f[12 + 2 * a] = __log2f(size) * (1.0f / 21.0f);
        f[13 + 2 * a] = pn * (1.0f / 63.0f);
    }
}

__global__ void __launch_bounds__(256) k_features(const float4* __restrict__ pts, const int32_t* __restrict__ leaf_parent,
                                                  const int32_t* __restrict__ sparent,
                                                  const uint8_t* __restrict__ prefix_n,
                                                  const int32_t* __restrict__ range_end,
                                                  const uint64_t* __restrict__ codes, int64_t u, int code_bits,
                                                  int64_t start, int64_t count, float* __restrict__ out,
                                                  const DevState* st) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= count) return;
    const float log2_range2 = 2.0f * __log2f(st->range);
    float f[kMlpF];
    point_features(start + t, pts, leaf_parent, sparent, prefix_n, range_end, codes, u, code_bits, log2_range2, f);
#pragma unroll
    for (int j = 0; j < kMlpF; ++j) out[t * kMlpF + j] = f[j];
}

// ---------------------------------------------------------------------------
// Training path (CUDA cores, FP32 accumulation over BF16-rounded weights,
// inputs and activations: the same numbers the tensor-core inference uses).
// Parameter layout (FP32 master copy): see MlpLayout in pipeline.cuh.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X,
                                                     int64_t n, float* __restrict__ yhat, float* __restrict__ h1_out,
                                                     float* __restrict__ h2_out) {
    __shared__ float sW1[kMlpF * kMlpH], sW2[kMlpH * kMlpH], sb1[kMlpH], sb2[kMlpH], sw3[kMlpH];
    for (int i = threadIdx.x; i < kMlpF * kMlpH; i += blockDim.x) sW1[i] = bf16r(params[MlpLayout::W1 + i]);
    for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) sW2[i] = bf16r(params[MlpLayout::W2 + i]);
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        sb1[i] = params[MlpLayout::B1 + i];
        sb2[i] = params[MlpLayout::B2 + i];
        sw3[i] = bf16r(params[MlpLayout::W3 + i]);
    }
    __syncthreads();
    const float b3 = params[MlpLayout::B3];
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    float x[kMlpF];
#pragma unroll
    for (int j = 0; j < kMlpF; ++j) x[j] = bf16r(X[r * kMlpF + j]);
    float h1[kMlpH];
#pragma unroll 4
    for (int i = 0; i < kMlpH; ++i) {
        float a = sb1[i];
#pragma unroll
        for (int j = 0; j < kMlpF; ++j) a = fmaf(x[j], sW1[j * kMlpH + i], a);
        h1[i] = bf16r(fmaxf(a, 0.0f));
    }
    float y = b3;
    for (int i = 0; i < kMlpH; ++i) {
        float a = sb2[i];
#pragma unroll
        for (int j = 0; j < kMlpH; ++j) a = fmaf(h1[j], sW2[j * kMlpH + i], a);
        const float h2 = bf16r(fmaxf(a, 0.0f));
        if (h2_out) h2_out[r * kMlpH + i] = h2;
        y = fmaf(h2, sw3[i], y);
    }
    if (h1_out)
        for (int i = 0; i < kMlpH; ++i) h1_out[r * kMlpH + i] = h1[i];
    yhat[r] = y;
}

// Per-sample output and hidden-layer gradients of the mean squared error
// loss = mean((yhat - y)^2); accumulates the bias gradients and the loss.
__global__ void __launch_bounds__(128) k_mlp_backward_rows(const float* __restrict__ params,
                                                           const float* __restrict__ yhat,
                                                           const float* __restrict__ y, const float* __restrict__ h1,
                                                           const float* __restrict__ h2, int64_t n,
                                                           float* __restrict__ dy_out, float* __restrict__ dh1_out,
                                                           float* __restrict__ dh2_out, float* __restrict__ grads,
                                                           float* __restrict__ loss) {
    __shared__ float sW2[kMlpH * kMlpH], sw3[kMlpH], sdb1[kMlpH], sdb2[kMlpH];
    __shared__ float sdb3, sloss;
    for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) sW2[i] = bf16r(params[MlpLayout::W2 + i]);
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        sw3[i] = bf16r(params[MlpLayout::W3 + i]);
        sdb1[i] = 0.0f;
        sdb2[i] = 0.0f;
    }
    if (threadIdx.x == 0) { sdb3 = 0.0f; sloss = 0.0f; }
    __syncthreads();
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n) {
        const float e = yhat[r] - y[r];
        const float dy = 2.0f * e / (float)n;
        dy_out[r] = dy;
        atomicAdd(&sloss, e * e / (float)n);
        atomicAdd(&sdb3, dy);
        float dh2[kMlpH];
#pragma unroll 8
        for (int i = 0; i < kMlpH; ++i) {
            dh2[i] = h2[r * kMlpH + i] > 0.0f ? dy * sw3[i] : 0.0f;
            dh2_out[r * kMlpH + i] = dh2[i];
            atomicAdd(&sdb2[i], dh2[i]);
        }
        for (int j = 0; j < kMlpH; ++j) {
            float a = 0.0f;
            if (h1[r * kMlpH + j] > 0.0f) {
#pragma unroll 8
                for (int i = 0; i < kMlpH; ++i) a = fmaf(sW2[j * kMlpH + i], dh2[i], a);
            }
            dh1_out[r * kMlpH + j] = a;
            atomicAdd(&sdb1[j], a);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        atomicAdd(&grads[MlpLayout::B1 + i], sdb1[i]);
        atomicAdd(&grads[MlpLayout::B2 + i], sdb2[i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grads[MlpLayout::B3], sdb3);
        atomicAdd(loss, sloss);
    }
}

// Weight gradient G[a][b] += sum_r A[r][a] * D[r][b] (A: n x na, D: n x nb),
// one thread per output entry, rows split over blocks along y.
__global__ void __launch_bounds__(256) k_mlp_outer(const float* __restrict__ A, int na, const float* __restrict__ D,
                                                   int nb, int64_t n, bool bf16_a, float* __restrict__ G) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= na * nb) return;
    const int ia = idx / nb, ib = idx % nb;
    const int64_t rows_per = (n + gridDim.y - 1) / gridDim.y;
    const int64_t r0 = blockIdx.y * rows_per, r1 = min64(n, r0 + rows_per);
    float acc = 0.0f;
    for (int64_t r = r0; r < r1; ++r) {
        const float a = A[r * na + ia];
        acc = fmaf(bf16_a ? bf16r(a) : a, D[r * nb + ib], acc);
    }
    atomicAdd(&G[idx], acc);
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters.
__global__ void k_adam(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                       float* __restrict__ v, int np, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float g = grads[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---------------------------------------------------------------------------
// Inference on the tensor cores: one warp = 32 query points. Features are
// computed per lane and staged as a 32 x 32 BF16 tile; both hidden layers are
// mma.sync.m16n8k16 (BF16 x BF16 -> FP32) over fragments read from shared
// memory; the output layer is a dot product reduced across each quad.
// Writes the bound r^2 = range^2 * 2^(yhat + margin) per query.
// ---------------------------------------------------------------------------
struct MlpSmem {
    __nv_bfloat16 w1t[kMlpH][kMlpF + 8];  // W1 transposed: [out][in], padded rows
    __nv_bfloat16 w2t[kMlpH][kMlpH + 8];
    float b1[kMlpH], b2[kMlpH], w3[kMlpH];
    __nv_bfloat16 x[4][32][kMlpF + 8];    // per warp: features
    __nv_bfloat16 h[4][32][kMlpH + 8];    // per warp: hidden activations
};

__device__ __forceinline__ uint32_t ld_b32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// out[32 x kMlpH] = act(in[32 x KIN] * W^T + bias), with W stored [kMlpH][KIN+8].
template <int KIN>
__device__ __forceinline__ void mma_layer(const __nv_bfloat16 (*in)[KIN + 8], const __nv_bfloat16 (*wt)[KIN + 8],
                                          int lane, float (&acc)[2][8][4]) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int nb = 0; nb < 8; ++nb)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mb][nb][e] = 0.0f;
#pragma unroll
    for (int kb = 0; kb < KIN / 16; ++kb) {
        const int k0 = kb * 16 + 2 * t;
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
            const int r0 = mb * 16 + g;
            const uint32_t a[4] = {ld_b32(&in[r0][k0]), ld_b32(&in[r0 + 8][k0]), ld_b32(&in[r0][k0 + 8]),
                                   ld_b32(&in[r0 + 8][k0 + 8])};
#pragma unroll
            for (int nb = 0; nb < 8; ++nb) {
                const int n0 = nb * 8 + g;
                const uint32_t b[2] = {ld_b32(&wt[n0][k0]), ld_b32(&wt[n0][k0 + 8])};
                mma_bf16_16816(acc[mb][nb], a, b);
            }
        }
    }
}

__global__ void __launch_bounds__(128) k_predict_radius(const float* __restrict__ params, float margin,
                                                        const float4* __restrict__ pts,
                                                        const int32_t* __restrict__ leaf_parent,
                                                        const int32_t* __restrict__ sparent,
                                                        const uint8_t* __restrict__ prefix_n,
                                                        const int32_t* __restrict__ range_end,
                                                        const uint64_t* __restrict__ codes, int64_t u, int code_bits,
                                                        int64_t start, int64_t count, float* __restrict__ r2_out,
                                                        float* __restrict__ yhat_out, const DevState* st) {
    __shared__ MlpSmem S;
    for (int i = threadIdx.x; i < kMlpF * kMlpH; i += blockDim.x) {
        const int in = i / kMlpH, out = i % kMlpH;
        S.w1t[out][in] = __float2bfloat16_rn(params[MlpLayout::W1 + i]);
    }
    for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) {
        const int in = i / kMlpH, out = i % kMlpH;
        S.w2t[out][in] = __float2bfloat16_rn(params[MlpLayout::W2 + i]);
    }
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        S.b1[i] = params[MlpLayout::B1 + i];
        S.b2[i] = params[MlpLayout::B2 + i];
        S.w3[i] = bf16r(params[MlpLayout::W3 + i]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float b3 = params[MlpLayout::B3];
    // the block keeps its weights in shared memory and walks 128-query chunks
    for (int64_t chunk = blockIdx.x;; chunk += gridDim.x) {
    const int64_t q0 = (chunk * 4 + warp) * 32;
    if (q0 >= count) break;
    const int64_t qo = q0 + lane;
    const bool active = qo < count;
    const float range = st->range;
    const float log2_range2 = 2.0f * __log2f(range);
    {
        float f[kMlpF];
        point_features(start + (active ? qo : q0), pts, leaf_parent, sparent, prefix_n, range_end, codes, u, code_bits,
                       log2_range2, f);
#pragma unroll
        for (int j = 0; j < kMlpF; ++j) S.x[warp][lane][j] = __float2bfloat16_rn(f[j]);
    }
    __syncwarp();
    const int g = lane >> 2, t = lane & 3;
    float acc[2][8][4];
    mma_layer<kMlpF>(S.x[warp], S.w1t, lane, acc);
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int nb = 0; nb < 8; ++nb) {
            const int c = nb * 8 + 2 * t;
            S.h[warp][mb * 16 + g][c] = __float2bfloat16_rn(fmaxf(acc[mb][nb][0] + S.b1[c], 0.0f));
            S.h[warp][mb * 16 + g][c + 1] = __float2bfloat16_rn(fmaxf(acc[mb][nb][1] + S.b1[c + 1], 0.0f));
            S.h[warp][mb * 16 + g + 8][c] = __float2bfloat16_rn(fmaxf(acc[mb][nb][2] + S.b1[c], 0.0f));
            S.h[warp][mb * 16 + g + 8][c + 1] = __float2bfloat16_rn(fmaxf(acc[mb][nb][3] + S.b1[c + 1], 0.0f));
        }
    __syncwarp();
    mma_layer<kMlpH>(S.h[warp], S.w2t, lane, acc);
    // output layer: rows g, g+8 of each 16-row block; reduce the 4 lanes of a quad
    float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int nb = 0; nb < 8; ++nb) {
            const int c = nb * 8 + 2 * t;
            y[mb][0] = fmaf(bf16r(fmaxf(acc[mb][nb][0] + S.b2[c], 0.0f)), S.w3[c], y[mb][0]);
            y[mb][0] = fmaf(bf16r(fmaxf(acc[mb][nb][1] + S.b2[c + 1], 0.0f)), S.w3[c + 1], y[mb][0]);
            y[mb][1] = fmaf(bf16r(fmaxf(acc[mb][nb][2] + S.b2[c], 0.0f)), S.w3[c], y[mb][1]);
            y[mb][1] = fmaf(bf16r(fmaxf(acc[mb][nb][3] + S.b2[c + 1], 0.0f)), S.w3[c + 1], y[mb][1]);
        }
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            y[mb][h] += __shfl_xor_sync(FULL, y[mb][h], 1);
            y[mb][h] += __shfl_xor_sync(FULL, y[mb][h], 2);
        }
    // lane t == 0 of quad g holds rows g, g+8, g+16, g+24
    if (t == 0) {
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = mb * 16 + g + 8 * h;
                const int64_t o = q0 + row;
                if (o < count) {
                    const float yh = y[mb][h] + b3;
                    if (yhat_out) yhat_out[o] = yh;
                    if (r2_out) r2_out[o] = range * range * exp2f(yh + margin);
                }
            }
    }
    __syncwarp();  // S.x / S.h of this warp are rewritten by its next chunk
    }
}

inline unsigned blocks_for(int64_t work, int threads) { return (unsigned)((work + threads - 1) / threads); }

}  // namespace

cudaError_t enqueue_features(const BuildBufs& b, int64_t u, int code_bits, int64_t start, int64_t count, float* out,
                             cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_features<<<blocks_for(count, 256), 256, 0, s>>>(b.pts4, b.leaf_parent, b.sparent, b.prefix_n, b.range_end,
                                                      b.codes, u, code_bits, start, count, out, b.st);
    return cudaGetLastError();
}

cudaError_t enqueue_predict_radius(const BuildBufs& b, const float* params, float margin, int64_t u, int code_bits,
                                   int64_t start, int64_t count, float* r2_out, float* yhat_out, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    // the resident blocks only, each loading the weights once
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_predict_radius, 128, 0);
    if (e != cudaSuccess) return e;
    const int64_t resident = (int64_t)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    const int64_t want = (int64_t)blocks_for((count + 31) / 32, 4);
    const unsigned blocks = (unsigned)(want < resident ? want : resident);
    k_predict_radius<<<blocks, 128, 0, s>>>(params, margin, b.pts4, b.leaf_parent, b.sparent, b.prefix_n, b.range_end,
                                            b.codes, u, code_bits, start, count, r2_out, yhat_out, b.st);
    return cudaGetLastError();
}

cudaError_t enqueue_mlp_forward(const float* params, const float* X, int64_t n, float* yhat, float* h1, float* h2,
                                cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_mlp_forward<<<blocks_for(n, 128), 128, 0, s>>>(params, X, n, yhat, h1, h2);
    return cudaGetLastError();
}

cudaError_t enqueue_mlp_grad(const float* params, const float* X, const float* y, int64_t n, MlpWork& w, float* grads,
                             float* loss, cudaStream_t s) {
    cudaMemsetAsync(grads, 0, sizeof(float) * kMlpParams, s);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    if (n <= 0) return cudaGetLastError();
    k_mlp_forward<<<blocks_for(n, 128), 128, 0, s>>>(params, X, n, w.yhat, w.h1, w.h2);
    k_mlp_backward_rows<<<blocks_for(n, 128), 128, 0, s>>>(params, w.yhat, y, w.h1, w.h2, n, w.dy, w.dh1, w.dh2, grads,
                                                           loss);
    const unsigned ysplit = (unsigned)min64(64, (n + 255) / 256);
    k_mlp_outer<<<dim3(blocks_for(kMlpF * kMlpH, 256), ysplit), 256, 0, s>>>(X, kMlpF, w.dh1, kMlpH, n, true,
                                                                            grads + MlpLayout::W1);
    k_mlp_outer<<<dim3(blocks_for(kMlpH * kMlpH, 256), ysplit), 256, 0, s>>>(w.h1, kMlpH, w.dh2, kMlpH, n, false,
                                                                            grads + MlpLayout::W2);
    k_mlp_outer<<<dim3(1, ysplit), 256, 0, s>>>(w.h2, kMlpH, w.dy, 1, n, false, grads + MlpLayout::W3);
    return cudaGetLastError();
}

cudaError_t enqueue_adam(float* params, const float* grads, float* m, float* v, float lr, int step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<blocks_for(kMlpParams, 256), 256, 0, s>>>(params, grads, m, v, kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace shapex
