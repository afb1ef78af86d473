// Learned search-radius proposal: per-point occupancy features and a 3-layer
// MLP (32 -> 64 -> 64 -> 1, BF16 weights and activations, FP32 accumulation)
// that predicts log2(r_k^2 / range^2), the squared distance to a point's k-th
// neighbour in units of the cloud's extent. Training (a fused forward,
// backward and weight-gradient step, then Adam) and inference are kernels of
// this file; both run their contractions on the tensor cores (mma.sync
// m16n8k16, BF16 in, FP32 accumulate); inference is fused with the feature
// computation.
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
// Forward on the CUDA cores (FP32 accumulation in a fixed fmaf order over
// BF16-rounded weights, inputs and activations), for se_mlp_forward: the
// calibration of the margin and the oracle check use it. Parameter layout
// (FP32 master copy): see MlpLayout in pipeline.cuh.
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

// ---------------------------------------------------------------------------
// Training step on the tensor cores: forward, backward and weight gradients of
// the loss (mean squared error, or with tau > 0 the pinball loss of quantile
// tau) for one batch in one kernel. A warp takes 32 rows at
// a time: both hidden layers, dh1 = (h1 > 0) * (dh2 W2^T) and the weight
// gradients dW1 = X^T dh1 and dW2 = h1^T dh2 (K = the 32 rows) are
// mma.sync.m16n8k16 products over BF16 tiles in shared memory (row-major tiles
// for the layers, transposed ones for the gradients) with FP32 accumulation;
// dh1 and dh2 enter the weight gradients rounded to BF16, the bias gradients
// unrounded. Each warp's gradient tiles are added to the FP32 gradient
// vector with reductions; the bias, w3 and loss terms are reduced across the
// warp first.
// ---------------------------------------------------------------------------
struct MlpTrainSmem {
    __nv_bfloat16 w1t[kMlpH][kMlpF + 8];  // forward layer 1: [out][in]
    __nv_bfloat16 w2t[kMlpH][kMlpH + 8];  // forward layer 2: [out][in]
    __nv_bfloat16 w2n[kMlpH][kMlpH + 8];  // backward: W2 as stored, [in][out]
    float b1[kMlpH], b2[kMlpH], w3[kMlpH];
    struct Warp {
        __nv_bfloat16 x[32][kMlpF + 8];   // [row][feature]
        __nv_bfloat16 xt[kMlpF][32 + 8];  // [feature][row]
        __nv_bfloat16 h1[32][kMlpH + 8];  // [row][unit]
        __nv_bfloat16 h1t[kMlpH][32 + 8]; // [unit][row]
        __nv_bfloat16 d2[32][kMlpH + 8];  // dh2 [row][unit]
        __nv_bfloat16 d2t[kMlpH][32 + 8];
        __nv_bfloat16 d1t[kMlpH][32 + 8]; // dh1 [unit][row]
        float sums[3][kMlpH];             // this warp's b1, b2 and w3 gradient sums
    } w[4];
};

// Sum v over the 8 row groups of the lanes (lanes with the same t), and add
// the total of each column nb * 8 + 2t + b to dst[col] on the lanes of group 0.
__device__ __forceinline__ void add_columns(float (&v)[16], float* __restrict__ dst, int lane) {
#pragma unroll
    for (int i = 0; i < 16; ++i)
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) v[i] += __shfl_xor_sync(FULL, v[i], o);
    if ((lane >> 2) == 0) {
        const int t = lane & 3;
#pragma unroll
        for (int nb = 0; nb < 8; ++nb)
#pragma unroll
            for (int b = 0; b < 2; ++b) dst[nb * 8 + 2 * t + b] += v[nb * 2 + b];
    }
}

// grads[base + row * kMlpH + col] += acc (the 32 x 64 product of mma_layer),
// rows offset by row0.
__device__ __forceinline__ void add_tile(float* __restrict__ grads, int base, int row0, const float (&acc)[2][8][4],
                                         int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int nb = 0; nb < 8; ++nb)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = row0 + mb * 16 + g + 8 * (e >> 1), col = nb * 8 + 2 * t + (e & 1);
                atomicAdd(grads + base + row * kMlpH + col, acc[mb][nb][e]);
            }
}

__global__ void __launch_bounds__(128, 1) k_mlp_train_tc(const float* __restrict__ params,
                                                         const float* __restrict__ X, const float* __restrict__ Y,
                                                         int64_t n, float tau, float* __restrict__ grads,
                                                         float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char mlp_smem[];
    MlpTrainSmem& S = *reinterpret_cast<MlpTrainSmem*>(mlp_smem);
    for (int i = threadIdx.x; i < kMlpF * kMlpH; i += blockDim.x) {
        const int in = i / kMlpH, out = i % kMlpH;
        S.w1t[out][in] = __float2bfloat16_rn(params[MlpLayout::W1 + i]);
    }
    for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) {
        const int in = i / kMlpH, out = i % kMlpH;
        const __nv_bfloat16 v = __float2bfloat16_rn(params[MlpLayout::W2 + i]);
        S.w2t[out][in] = v;
        S.w2n[in][out] = v;
    }
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        S.b1[i] = params[MlpLayout::B1 + i];
        S.b2[i] = params[MlpLayout::B2 + i];
        S.w3[i] = bf16r(params[MlpLayout::W3 + i]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    MlpTrainSmem::Warp& T = S.w[warp];
    const float b3 = params[MlpLayout::B3];
    const float inv_n = 1.0f / (float)n;
    for (int i = lane; i < 3 * kMlpH; i += 32) (&T.sums[0][0])[i] = 0.0f;
    __syncwarp();
    float db3 = 0.0f, lsum = 0.0f;
    for (int64_t chunk = blockIdx.x;; chunk += gridDim.x) {
        const int64_t q0 = (chunk * 4 + warp) * 32;
        if (q0 >= n) break;
        {
            const int64_t r = q0 + lane;
            const bool valid = r < n;
#pragma unroll 8
            for (int j = 0; j < kMlpF; ++j) {
                const __nv_bfloat16 b = __float2bfloat16_rn(valid ? __ldg(X + r * kMlpF + j) : 0.0f);
                T.x[lane][j] = b;
                T.xt[j][lane] = b;
            }
        }
        __syncwarp();
        float acc[2][8][4];
        mma_layer<kMlpF>(T.x, S.w1t, lane, acc);
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int nb = 0; nb < 8; ++nb)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int row = mb * 16 + g + 8 * (e >> 1), col = nb * 8 + 2 * t + (e & 1);
                    const __nv_bfloat16 h = __float2bfloat16_rn(fmaxf(acc[mb][nb][e] + S.b1[col], 0.0f));
                    T.h1[row][col] = h;
                    T.h1t[col][row] = h;
                }
        __syncwarp();
        mma_layer<kMlpH>(T.h1, S.w2t, lane, acc);
        float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int nb = 0; nb < 8; ++nb)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int col = nb * 8 + 2 * t + (e & 1);
                    const float h2 = bf16r(fmaxf(acc[mb][nb][e] + S.b2[col], 0.0f));
                    acc[mb][nb][e] = h2;
                    y[mb][e >> 1] = fmaf(h2, S.w3[col], y[mb][e >> 1]);
                }
        float dy[2][2];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float v = y[mb][h];
                v += __shfl_xor_sync(FULL, v, 1);
                v += __shfl_xor_sync(FULL, v, 2);
                const int64_t o = q0 + mb * 16 + g + 8 * h;
                const float err = o < n ? v + b3 - __ldg(Y + o) : 0.0f;
                float l;
                if (tau > 0.0f) {  // pinball loss at quantile tau: tau (y - yhat)+ + (1 - tau) (yhat - y)+
                    dy[mb][h] = (err > 0.0f ? 1.0f - tau : (err < 0.0f ? -tau : 0.0f)) * inv_n;
                    l = (err > 0.0f ? (1.0f - tau) * err : -tau * err) * inv_n;
                } else {  // mean squared error
                    dy[mb][h] = 2.0f * err * inv_n;
                    l = err * err * inv_n;
                }
                if (t == 0) {
                    lsum += l;
                    db3 += dy[mb][h];
                }
            }
        // dh2 = (h2 > 0) * dy * w3; w3 and b2 gradients (per lane: columns nb * 8 + 2t + b)
        float db2[16], dw3[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) db2[i] = dw3[i] = 0.0f;
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int nb = 0; nb < 8; ++nb)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int row = mb * 16 + g + 8 * (e >> 1), col = nb * 8 + 2 * t + (e & 1);
                    const float h2 = acc[mb][nb][e], d = dy[mb][e >> 1];
                    const float d2 = h2 > 0.0f ? d * S.w3[col] : 0.0f;
                    db2[nb * 2 + (e & 1)] += d2;
                    dw3[nb * 2 + (e & 1)] = fmaf(d, h2, dw3[nb * 2 + (e & 1)]);
                    const __nv_bfloat16 b = __float2bfloat16_rn(d2);
                    T.d2[row][col] = b;
                    T.d2t[col][row] = b;
                }
        add_columns(db2, T.sums[1], lane);
        add_columns(dw3, T.sums[2], lane);
        __syncwarp();
        // dh1 = (h1 > 0) * (dh2 W2^T)
        mma_layer<kMlpH>(T.d2, S.w2n, lane, acc);
        float db1[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) db1[i] = 0.0f;
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int nb = 0; nb < 8; ++nb)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int row = mb * 16 + g + 8 * (e >> 1), col = nb * 8 + 2 * t + (e & 1);
                    const float d1 = __bfloat162float(T.h1[row][col]) > 0.0f ? acc[mb][nb][e] : 0.0f;
                    db1[nb * 2 + (e & 1)] += d1;
                    T.d1t[col][row] = __float2bfloat16_rn(d1);
                }
        add_columns(db1, T.sums[0], lane);
        __syncwarp();
        // weight gradients of these 32 rows
        mma_layer<32>(T.xt, T.d1t, lane, acc);
        add_tile(grads, MlpLayout::W1, 0, acc, lane);
        mma_layer<32>(T.h1t, T.d2t, lane, acc);
        add_tile(grads, MlpLayout::W2, 0, acc, lane);
        mma_layer<32>(T.h1t + 32, T.d2t, lane, acc);
        add_tile(grads, MlpLayout::W2, 32, acc, lane);
        __syncwarp();  // this warp's tiles are rewritten by its next chunk
    }
    // this warp's column sums: one reduction per column
    __syncwarp();
    for (int i = lane; i < kMlpH; i += 32) {
        atomicAdd(grads + MlpLayout::B1 + i, T.sums[0][i]);
        atomicAdd(grads + MlpLayout::B2 + i, T.sums[1][i]);
        atomicAdd(grads + MlpLayout::W3 + i, T.sums[2][i]);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        db3 += __shfl_xor_sync(FULL, db3, o);
        lsum += __shfl_xor_sync(FULL, lsum, o);
    }
    if (lane == 0) {
        atomicAdd(grads + MlpLayout::B3, db3);
        atomicAdd(loss, lsum);
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

cudaError_t enqueue_mlp_grad(const float* params, const float* X, const float* y, int64_t n, float tau,
                             MlpWork& /*w*/, float* grads, float* loss, cudaStream_t s) {
    cudaMemsetAsync(grads, 0, sizeof(float) * kMlpParams, s);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    if (n <= 0) return cudaGetLastError();
    constexpr int smem = (int)sizeof(MlpTrainSmem);
    cudaError_t e = cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int64_t want = (n + 127) / 128;  // 4 warps x 32 rows per block and pass
    const unsigned blocks = (unsigned)(want < sms ? want : (sms > 0 ? sms : 1));
    k_mlp_train_tc<<<blocks, 128, smem, s>>>(params, X, y, n, tau, grads, loss);
    return cudaGetLastError();
}

cudaError_t enqueue_adam(float* params, const float* grads, float* m, float* v, float lr, int step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<blocks_for(kMlpParams, 256), 256, 0, s>>>(params, grads, m, v, kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace shapex
