// Build stages of the normal-estimation path on sm_100a:
//   bbox -> Morton encode (+ digit histograms) -> onesweep LSD radix sort ->
//   dedup + decode -> Karras radix tree -> search boxes -> octree.
// Each kernel cites the reference stage it replaces (paths relative to the
// reference project root).

#include <cfloat>
#include <cstdint>

#include "pipeline.cuh"

namespace shapex {

namespace {

constexpr uint32_t LB_AGG = 1u << 30;
constexpr uint32_t LB_PRE = 2u << 30;
constexpr uint32_t LB_VAL = (1u << 30) - 1;
constexpr unsigned long long LB64_AGG = 1ull << 62;
constexpr unsigned long long LB64_PRE = 2ull << 62;
constexpr unsigned long long LB64_VAL = (1ull << 62) - 1;

__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan (blockDim.x = NT, multiple of 32). Returns the
// thread's exclusive prefix; *total receives the block sum.
template <int NT, typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* smem_warp, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31) smem_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = (lane < NT / 32) ? smem_warp[lane] : T(0);
        T wi = warp_incl_scan(w);
        if (lane < NT / 32) smem_warp[lane] = wi - w;
        if (lane == NT / 32 - 1) smem_warp[NT / 32] = wi;
    }
    __syncthreads();
    T r = inc - v + smem_warp[warp];
    *total = smem_warp[NT / 32];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// bbox: replaces 3x DeviceReduce::Max + 3x DeviceReduce::Min and the host
// min/max of src/RadixTree.cu:218-241 with one pass over x, y, z producing a
// single isotropic [min, max]. Also rejects NaN/Inf.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_bbox(const float* __restrict__ x, const float* __restrict__ y,
                                              const float* __restrict__ z, int64_t n, DevState* st) {
    float lo = FLT_MAX, hi = -FLT_MAX;
    bool bad = false;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    auto take = [&](float v) {
        bad |= !isfinite(v);
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    };
    const bool vec = (((uintptr_t)x | (uintptr_t)y | (uintptr_t)z) & 15) == 0;
    int64_t done = 0;
    if (vec) {
        const int64_t n4 = n >> 2;
        const float4* x4 = reinterpret_cast<const float4*>(x);
        const float4* y4 = reinterpret_cast<const float4*>(y);
        const float4* z4 = reinterpret_cast<const float4*>(z);
        for (int64_t i = tid; i < n4; i += stride) {
            const float4 a = __ldcs(x4 + i), b = __ldcs(y4 + i), c = __ldcs(z4 + i);
            take(a.x); take(a.y); take(a.z); take(a.w);
            take(b.x); take(b.y); take(b.z); take(b.w);
            take(c.x); take(c.y); take(c.z); take(c.w);
        }
        done = n4 << 2;
    }
    for (int64_t i = done + tid; i < n; i += stride) {
        take(x[i]); take(y[i]); take(z[i]);
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    __shared__ float s_lo[8], s_hi[8];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    if (bad) s_bad = 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s_lo[warp] = lo; s_hi[warp] = hi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { lo = fminf(lo, s_lo[w]); hi = fmaxf(hi, s_hi[w]); }
        // min is kept inverted so that both words start at 0 and use atomicMax
        atomicMax(&st->min_ord, ~f2ord(lo));
        atomicMax(&st->max_ord, f2ord(hi));
        if (s_bad) set_err(&st->err, ERRBIT_NONFINITE);
    }
}

__device__ __forceinline__ void load_bbox(const DevState* st, float& mn, float& range) {
    mn = ord2f(~st->min_ord);
    const float mx = ord2f(st->max_ord);
    range = __fsub_rn(mx, mn);  // float tree_range = max - min, src/RadixTree.cu:246
}

// ---------------------------------------------------------------------------
// encode: replaces makeCodes (src/RadixTree.cu:21-39, 244-248); also builds
// the digit histograms of the onesweep sort's passes in the same pass.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_encode(const float* __restrict__ x, const float* __restrict__ y,
                                                const float* __restrict__ z, int64_t n, int code_bits,
                                                uint64_t* __restrict__ keys, DevState* st) {
    __shared__ uint32_t s_h[kSortPasses][kSortBins];
    for (int i = threadIdx.x; i < kSortPasses * kSortBins; i += blockDim.x) (&s_h[0][0])[i] = 0;
    __syncthreads();
    float mn, range;
    load_bbox(st, mn, range);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->min_coord = mn;
        st->max_coord = ord2f(st->max_ord);
        st->range = range;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t c = point_to_code(__ldcs(x + i), __ldcs(y + i), __ldcs(z + i), mn, range, code_bits);
        keys[i] = c;
#pragma unroll
        for (int p = 0; p < kSortPasses; ++p) atomicAdd(&s_h[p][(c >> (kSortBits * p)) & (kSortBins - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortPasses * kSortBins; i += blockDim.x) {
        const uint32_t v = (&s_h[0][0])[i];
        if (v) atomicAdd(&(&st->hist[0][0])[i], v);
    }
}

// Digit offsets, trivial-pass detection and ping-pong parity, on one block.
__global__ void __launch_bounds__(kSortBins) k_sort_prep(int64_t n, DevState* st) {
    __shared__ uint32_t s_w[kSortBins / 32 + 1];
    __shared__ int s_triv[kSortPasses];
    const int d = threadIdx.x;
    for (int p = 0; p < kSortPasses; ++p) {
        const uint32_t h = st->hist[p][d];
        uint32_t tot;
        const uint32_t ex = block_excl_scan<kSortBins, uint32_t>(h, s_w, &tot);
        st->digit_off[p][d] = ex;
        if (d == 0) s_triv[p] = 0;
        __syncthreads();
        if ((int64_t)h == n) s_triv[p] = 1;
        __syncthreads();
    }
    if (d == 0) {
        int act = 0;
        for (int p = 0; p < kSortPasses; ++p) {
            st->pass_active[p] = !s_triv[p];
            st->pass_parity[p] = act & 1;
            act += !s_triv[p];
        }
        st->n_active = act;
    }
}

// ---------------------------------------------------------------------------
// Onesweep LSD radix sort pass over 64-bit keys (Adinets & Merrill,
// "Onesweep: A Faster Least Significant Digit Radix Sort for GPUs", 2022):
// warp-level multi-split ranking with ballot peer masks, decoupled look-back
// over per-tile digit counts, scatter through shared memory. Replaces
// DeviceRadixSort::SortKeys (src/RadixTree.cu:316-337). Stable.
//
// 9-bit digits (512 bins, one per thread), so a 63-bit Morton code takes 7
// passes instead of 8. A tile publishes its digit counts as soon as it has
// ranked its keys, scatters them into shared memory, and only then reads its
// predecessors' counts. Three blocks per SM (the whole shared-memory
// carveout).
// ---------------------------------------------------------------------------
constexpr int kSortWarps = kSortThreads / 32;
static_assert(kSortThreads == kSortBins, "one digit per thread");

struct SortSmem {
    uint32_t hist[kSortWarps][kSortBins];  // per-warp digit counts, then per-warp offsets
    uint64_t keys[kSortTile];
    uint32_t local_start[kSortBins];  // first slot of each digit in the tile
    int32_t goff[kSortBins];          // global position of the digit's run minus local_start
    uint32_t scan_w[kSortWarps + 1];
    uint32_t tile_id;
};

__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(uint64_t* buf0, uint64_t* buf1, int64_t n, int pass,
                                                           uint32_t* __restrict__ lookback, DevState* st,
                                                           int spin_limit, int stall_first_tile) {
    // a look-back of this build gave up: its key order is lost, write nothing
    if (!st->pass_active[pass] || (st->err & ERRBIT_LOOKBACK)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int parity = st->pass_parity[pass];
    const uint64_t* __restrict__ in = parity ? buf1 : buf0;
    uint64_t* __restrict__ out = parity ? buf0 : buf1;
    const int shift = kSortBits * pass;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int i = tid; i < kSortWarps * kSortBins; i += kSortThreads) (&S.hist[0][0])[i] = 0;
    if (tid == 0) S.tile_id = atomicAdd(&st->tile_counter[pass], 1u);
    __syncthreads();
    const uint32_t tile = S.tile_id;
    const int64_t base = (int64_t)tile * kSortTile;

    uint64_t key[kSortIpt];
    uint32_t rank[kSortIpt];
    const int64_t wbase = base + (int64_t)warp * 32 * kSortIpt;
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const int64_t idx = wbase + i * 32 + lane;
        key[i] = idx < n ? in[idx] : 0ull;
    }
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const int64_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = (uint32_t)(key[i] >> shift) & (kSortBins - 1);
        // lanes holding the same digit: one ballot for validity, one per digit
        // bit (measured slightly faster than __match_any_sync)
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
        if (!valid) peers = ~peers;
#pragma unroll
        for (int bb = 0; bb < kSortBits; ++bb) {
            const uint32_t v = __ballot_sync(0xffffffffu, (d >> bb) & 1u);
            peers &= ((d >> bb) & 1u) ? v : ~v;
        }
        uint32_t b = 0;
        if (valid) b = S.hist[warp][d];
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) S.hist[warp][d] = b + __popc(peers);
        __syncwarp();
        rank[i] = b + __popc(peers & lanemask_lt());
    }
    __syncthreads();

    // digit `tid`: exclusive prefix over warps and the tile's count, published
    // at once so that successors' look-backs find it early
    const int dg = tid;
    uint32_t cnt = 0;
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = S.hist[w][dg];
        S.hist[w][dg] = cnt;
        cnt += c;
    }
    if (tile == 0) {
        if (!stall_first_tile) st_relaxed(lookback + dg, LB_PRE | cnt);
    } else {
        st_relaxed(lookback + (size_t)tile * kSortBins + dg, LB_AGG | cnt);
    }
    {
        uint32_t tot;
        S.local_start[dg] = block_excl_scan<kSortThreads, uint32_t>(cnt, S.scan_w, &tot);
    }
    __syncthreads();
    // keys into shared memory in digit order
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const int64_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (uint32_t)(key[i] >> shift) & (kSortBins - 1);
            S.keys[S.local_start[d] + S.hist[warp][d] + rank[i]] = key[i];
        }
    }
    // decoupled look-back on digit `dg`, after the scatter: by then most
    // predecessors have published (reading them earlier, or several at a time,
    // measured slower: the polls compete with the tiles still ranking)
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t p = (int64_t)tile - 1;
        int spins = 0;
        while (p >= 0) {
            const uint32_t v = ld_relaxed(lookback + (size_t)p * kSortBins + dg);
            const uint32_t f = v >> 30;
            if (f == 0) {
                if (++spins > spin_limit) {
                    set_err(&st->err, ERRBIT_LOOKBACK);
                    break;
                }
                continue;
            }
            excl += v & LB_VAL;
            if (f == 2) break;
            --p;
        }
        st_relaxed(lookback + (size_t)tile * kSortBins + dg, LB_PRE | (excl + cnt));
    }
    S.goff[dg] = (int32_t)(st->digit_off[pass][dg] + excl) - (int32_t)S.local_start[dg];
    __syncthreads();
    const int tile_n = (int)min64(kSortTile, n - base);
    for (int j = tid; j < tile_n; j += kSortThreads) {
        const uint64_t k = S.keys[j];
        const uint32_t d = (uint32_t)(k >> shift) & (kSortBins - 1);
        const int64_t pos = (int64_t)S.goff[d] + j;
        if (pos >= 0 && pos < n) out[pos] = k;
        else set_err(&st->err, ERRBIT_BOUNDS);
    }
}

// ---------------------------------------------------------------------------
// dedup + decode: replaces findDups + InclusiveSum + moveDups
// (src/RadixTree.cu:71-97, 258-303) and decodePoints (src/Octree.cu:14-24,
// 305-315) with one pass: flag, block scan, decoupled look-back, compact, and
// decode of each surviving code.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kDedupThreads) k_dedup(const uint64_t* buf0, const uint64_t* buf1, int64_t n,
                                                         int code_bits, uint64_t* __restrict__ codes_out,
                                                         float4* __restrict__ pts4, float* __restrict__ pts3,
                                                         uint32_t* __restrict__ lookback, DevState* st,
                                                         int spin_limit) {
    // a sort look-back gave up: no order to dedup; u stays 0 and later stages do nothing
    if (st->err & ERRBIT_LOOKBACK) return;
    constexpr int kWarps = kDedupThreads / 32;
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ uint32_t s_wcnt[kWarps];
    __shared__ uint32_t s_tile, s_excl;
    const uint64_t* __restrict__ keys = (st->n_active & 1) ? buf1 : buf0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&st->tile_counter[kSortPasses], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    // Warp-striped: a warp's 32 * kDedupIpt keys are contiguous and element i
    // of lane l is key wbase + 32 i + l, so loads and the compacted stores of
    // each step are coalesced. Flags are kept as one ballot per step.
    const int64_t wbase = (int64_t)tile * kDedupTile + (int64_t)warp * 32 * kDedupIpt;
    uint64_t k[kDedupIpt];
    uint32_t m[kDedupIpt];
    uint64_t last = (wbase > 0 && wbase - 1 < n) ? keys[wbase - 1] : 0ull;  // the key before this step's
    uint32_t wcnt = 0;
#pragma unroll
    for (int i = 0; i < kDedupIpt; ++i) {
        const int64_t j = wbase + 32 * i + lane;
        k[i] = j < n ? keys[j] : 0ull;
        uint64_t prev = __shfl_up_sync(kFull, k[i], 1);
        if (lane == 0) prev = last;
        last = __shfl_sync(kFull, k[i], 31);
        m[i] = __ballot_sync(kFull, j < n && (j == 0 || k[i] != prev));
        wcnt += __popc(m[i]);
    }
    if (lane == 0) s_wcnt[warp] = wcnt;
    __syncthreads();
    uint32_t woff = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = s_wcnt[w];
        woff += w < warp ? c : 0u;
        tot += c;
    }
    // Decoupled look-back by warp 0, 32 predecessors per step: lane i reads
    // tile p - i. The walk ends at the nearest tile with an inclusive prefix
    // (tile 0 always publishes one); it needs every tile up to that one ready.
    if (warp == 0) {
        uint32_t excl = 0;
        if (tile == 0) {
            if (lane == 0) st_relaxed(lookback, LB_PRE | tot);
        } else {
            if (lane == 0) st_relaxed(lookback + tile, LB_AGG | tot);
            int64_t p = (int64_t)tile - 1;
            int spins = 0;
            for (;;) {
                const int64_t q = p - lane;
                const uint32_t v = q >= 0 ? ld_relaxed(lookback + q) : LB_PRE;
                const uint32_t f = v >> 30;
                const uint32_t pre = __ballot_sync(kFull, f == 2);
                const uint32_t need = pre ? (((pre & (0u - pre)) << 1) - 1u) : kFull;  // lanes up to the first prefix
                if (__ballot_sync(kFull, f == 0) & need) {
                    if (++spins > spin_limit) {
                        if (lane == 0) set_err(&st->err, ERRBIT_LOOKBACK);
                        break;
                    }
                    continue;
                }
                excl += __reduce_add_sync(kFull, ((need >> lane) & 1u) ? (v & LB_VAL) : 0u);
                if (pre) break;
                p -= 32;
            }
            if (lane == 0) st_relaxed(lookback + tile, LB_PRE | (excl + tot));
        }
        if (lane == 0) {
            s_excl = excl;
            if ((int64_t)(tile + 1) * kDedupTile >= n) st->u = (unsigned long long)(excl + tot);
        }
    }
    __syncthreads();
    const float mn = st->min_coord, range = st->range;
    uint32_t base = s_excl + woff;
#pragma unroll
    for (int i = 0; i < kDedupIpt; ++i) {
        if ((m[i] >> lane) & 1u) {
            const uint32_t pos = base + __popc(m[i] & lanemask_lt());
            if ((int64_t)pos >= n) {
                set_err(&st->err, ERRBIT_BOUNDS);
            } else {
                codes_out[pos] = k[i];
                const float3 p = code_to_point(k[i], mn, range, code_bits);
                pts4[pos] = make_float4(p.x, p.y, p.z, 0.0f);
                pts3[3 * (size_t)pos + 0] = p.x;
                pts3[3 * (size_t)pos + 1] = p.y;
                pts3[3 * (size_t)pos + 2] = p.z;
            }
        }
        base += __popc(m[i]);
    }
}

// ---------------------------------------------------------------------------
// Karras radix tree: replaces constructTree (src/RadixTree.cu:99-194,
// launched at :351-364). One thread per internal node, same search steps and
// integer semantics as the reference, so topology is bit-exact. Node 0 is
// computed twice: with the reference's root range l = N-1 (:128-130) for the
// exported arrays when root_compat is set, and with the full range for the
// search hierarchy. Also records each leaf's parent and each node's range end
// for the search hierarchy.
// ---------------------------------------------------------------------------
struct KNode {
    int64_t j;
    int64_t gamma;
    int dnode;
    bool hl, hr;
};

__device__ __forceinline__ KNode karras_node(const uint64_t* __restrict__ codes, int64_t i, int64_t N, int cb,
                                             bool compat_root) {
    const uint64_t ci = codes[i];
    int d;
    if (i == 0) {
        d = 1;
    } else {
        const int dd = delta_codes(ci, codes[i + 1], cb) - delta_codes(ci, codes[i - 1], cb);
        d = (dd > 0) - (dd < 0);
    }
    int64_t l = 0;
    if (i == 0) {
        l = compat_root ? N - 1 : N;
    } else {
        const int dmin = delta_codes(ci, codes[i - d], cb);
        int64_t lmax = 2;
        while (i + lmax * d >= 0 && i + lmax * d <= N && delta_codes(ci, codes[i + lmax * d], cb) > dmin) lmax *= 2;
        const int64_t lcut = (d == -1) ? i : N - i;
        // t = lmax / 2, lmax / 4, ... (powers-of-two divisions as shifts: 64-bit
        // divisions made the radix stage 22% slower on 13M codes)
        for (int sh = 1; (lmax >> sh) >= 1; ++sh) {
            const int64_t t = lmax >> sh;
            if (l + t <= lcut && delta_codes(ci, codes[i + (l + t) * d], cb) > dmin) l += t;
        }
    }
    KNode r;
    r.j = i + l * d;
    r.dnode = delta_codes(codes[i], codes[r.j], cb);
    int64_t s = 0;
    if (l >= 1) {
        const int nlow = 63 - __clzll((long long)l);
        const int lc = nlow + ((uint64_t)l > (uint64_t)one_shl(nlow));  // ceil(log2 l)
        const int64_t scut = (d == -1) ? i - 1 : N - i - 1;
        // t = ceil(l / 2), ceil(l / 4), ... up to 2^lc (shifts, not divisions)
        for (int sh = 1; sh <= lc; ++sh) {
            const int64_t t = (l + ((int64_t)1 << sh) - 1) >> sh;
            if (s + t <= scut && delta_codes(ci, codes[i + (s + t) * d], cb) > r.dnode) s += t;
        }
    }
    r.gamma = i + s * d + min(d, 0);
    r.hl = min(i, r.j) == r.gamma;
    r.hr = max(i, r.j) == r.gamma + 1;
    return r;
}

__global__ void __launch_bounds__(256) k_karras(const uint64_t* __restrict__ codes, int code_bits, int root_compat,
                                                int32_t* __restrict__ left_child, int32_t* __restrict__ parent,
                                                uint8_t* __restrict__ prefix_n, uint8_t* __restrict__ hll,
                                                uint8_t* __restrict__ hlr, int32_t* __restrict__ sparent,
                                                int32_t* __restrict__ leaf_parent, int32_t* __restrict__ range_end,
                                                DevState* st) {
    const int64_t u = (int64_t)st->u;
    const int64_t N = u - 1;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const KNode f = karras_node(codes, i, N, code_bits, false);
    // search hierarchy (full root range)
    range_end[i] = (int32_t)f.j;
    if (f.hl) leaf_parent[f.gamma] = (int32_t)i; else sparent[f.gamma] = (int32_t)i;
    if (f.hr) leaf_parent[f.gamma + 1] = (int32_t)i; else sparent[f.gamma + 1] = (int32_t)i;
    KNode e = f;
    if (i == 0) {
        st->sroot_gamma = (int32_t)f.gamma;
        st->sroot_hl = f.hl;
        st->sroot_hr = f.hr;
        if (root_compat) e = karras_node(codes, 0, N, code_bits, true);
    }
    left_child[i] = (int32_t)e.gamma;
    prefix_n[i] = (uint8_t)e.dnode;
    hll[i] = e.hl;
    hlr[i] = e.hr;
    // The compat root's parent claims are written after this kernel (k_root_parent)
    // so that, in a tree the compat root breaks, they win deterministically.
    if (i != 0 || !root_compat) {
        if (!e.hl) parent[e.gamma] = (int32_t)i;
        if (!e.hr) parent[e.gamma + 1] = (int32_t)i;
    }
}

__global__ void k_root_parent(const int32_t* __restrict__ left_child, int32_t* __restrict__ parent,
                              const uint8_t* __restrict__ hll, const uint8_t* __restrict__ hlr, DevState* st) {
    const int64_t u = (int64_t)st->u;
    if (u < 2) return;
    const int32_t g = left_child[0];
    if (g < 0 || g + 1 >= u) { set_err(&st->err, ERRBIT_BOUNDS); return; }
    if (!hll[0]) parent[g] = 0;
    if (!hlr[0]) parent[g + 1] = 0;
}

// ---------------------------------------------------------------------------
// Search boxes: bottom-up over the full-range radix tree (Karras 2012 sec. 4:
// second arrival at a node merges). Only nodes the kNN traversal visits need
// an SNode: the root and every node of more than `bucket` points. A subtree
// of at most `bucket` points is a bucket, read as a point range, so its inner
// nodes get nothing. Thread i looks at node i: a bucket root (at most
// `bucket` points, parent the root or larger) has its contiguous points
// reduced to a box by the whole warp (coalesced loads, shuffles), and its
// thread enters the merge protocol at the parent. Thread i also looks at
// leaf i: a leaf whose parent is the root or larger than a bucket is a bucket
// of one point and enters the merge at that parent. (An earlier version had
// every leaf climb to its bucket root and one thread read each bucket's
// points serially: 0.91 ms against 0.52 ms for this one on 13M unique points.)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_boxes(const float4* __restrict__ pts, const int32_t* __restrict__ left_child,
                                               const uint8_t* __restrict__ hll, const uint8_t* __restrict__ hlr,
                                               const int32_t* __restrict__ sparent,
                                               const int32_t* __restrict__ leaf_parent,
                                               const int32_t* __restrict__ range_end, uint32_t* __restrict__ visit,
                                               float4* __restrict__ node_box, SNode* __restrict__ snodes, int bucket,
                                               DevState* st) {
    const int64_t u = (int64_t)st->u;
    if (u < 2) return;
    const int64_t N = u - 1;  // internal nodes
    const int lane = threadIdx.x & 31;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // a node index and a leaf index
    auto size_of = [&](int64_t c) {
        const int64_t e = range_end[c];
        return (c > e ? c - e : e - c) + 1;
    };
    // (a) thread i as internal node i: a bucket root is a node of at most
    // `bucket` points below the root whose parent is the root or larger
    int64_t f = 0, l = 0, par = -1;
    bool root = false;
    if (i > 0 && i < N) {
        const int64_t e = range_end[i];
        f = min(i, e);
        l = max(i, e);
        if (l - f + 1 <= bucket) {
            par = sparent[i];
            if (par < 0 || par >= N) {
                set_err(&st->err, ERRBIT_BOUNDS);
            } else {
                root = par == 0 || size_of(par) > bucket;
            }
        }
    }
    // the warp reduces each of its bucket roots' contiguous points together
    uint32_t roots = __ballot_sync(0xffffffffu, root);
    while (roots) {
        const int r = __ffs(roots) - 1;
        roots &= roots - 1;
        const int64_t rf = __shfl_sync(0xffffffffu, f, r), rl = __shfl_sync(0xffffffffu, l, r);
        float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
        for (int64_t q = rf + lane; q <= rl; q += 32) {
            const float4 v = __ldg(pts + q);
            lx = fminf(lx, v.x); ly = fminf(ly, v.y); lz = fminf(lz, v.z);
            hx = fmaxf(hx, v.x); hy = fmaxf(hy, v.y); hz = fmaxf(hz, v.z);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
            ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
            lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
            hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
            hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
            hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
        }
        if (lane == r) {
            node_box[2 * i] = make_float4(lx, ly, lz, 0.f);
            node_box[2 * i + 1] = make_float4(hx, hy, hz, 0.f);
        }
    }
    // (b) thread i as leaf i: a leaf whose parent is the root or larger than a
    // bucket is a bucket of one point and enters the merge at that parent
    int64_t leaf_start = -1;
    if (i < u) {
        const int64_t lp = leaf_parent[i];
        if (lp < 0 || lp >= N) {
            set_err(&st->err, ERRBIT_BOUNDS);
        } else if (lp == 0 || size_of(lp) > bucket) {
            leaf_start = lp;
        }
    }
    // Merge protocol over the nodes the traversal visits (Karras 2012 sec. 4):
    // the second arrival at a node builds its SNode from both children and
    // goes on to the parent. Arrivals come from bucket roots and one-point
    // buckets; each thread runs at most two climbs.
#pragma unroll 1
    for (int climb = 0; climb < 2; ++climb) {
        int64_t node = climb == 0 ? (root ? par : -1) : leaf_start;
        if (node < 0) continue;
        int it = 0;
        for (; it < 130; ++it) {
            if (node < 0 || node >= N) {
                set_err(&st->err, ERRBIT_BOUNDS);
                break;
            }
            __threadfence();
            if (atomicAdd(&visit[node], 1u) == 0) break;
            __threadfence();
            int64_t g;
            bool l_leaf, r_leaf;
            if (node == 0) {
                g = st->sroot_gamma;
                l_leaf = st->sroot_hl;
                r_leaf = st->sroot_hr;
            } else {
                g = left_child[node];
                l_leaf = hll[node];
                r_leaf = hlr[node];
            }
            float4 lo[2], hi[2];
            int32_t ref[2], cnt[2];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int64_t ch = g + side;
                const bool leaf = side ? r_leaf : l_leaf;
                if (leaf) {
                    const float4 q = pts[ch];
                    lo[side] = q;
                    hi[side] = q;
                    ref[side] = (int32_t)ch;
                    cnt[side] = 1;
                } else {
                    lo[side] = __ldcg(node_box + 2 * ch);
                    hi[side] = __ldcg(node_box + 2 * ch + 1);
                    const int64_t e = range_end[ch];
                    const int64_t cf = min(ch, e), cl = max(ch, e);
                    cnt[side] = (int32_t)(cl - cf + 1);
                    ref[side] = cnt[side] <= bucket ? (int32_t)cf : (int32_t)ch;
                }
            }
            SNode sn;
            sn.lo_l = make_float4(lo[0].x, lo[0].y, lo[0].z, __int_as_float(ref[0]));
            sn.hi_l = make_float4(hi[0].x, hi[0].y, hi[0].z, __int_as_float(cnt[0]));
            sn.lo_r = make_float4(lo[1].x, lo[1].y, lo[1].z, __int_as_float(ref[1]));
            sn.hi_r = make_float4(hi[1].x, hi[1].y, hi[1].z, __int_as_float(cnt[1]));
            snodes[node] = sn;
            node_box[2 * node] =
                make_float4(fminf(lo[0].x, lo[1].x), fminf(lo[0].y, lo[1].y), fminf(lo[0].z, lo[1].z), 0.f);
            node_box[2 * node + 1] =
                make_float4(fmaxf(hi[0].x, hi[1].x), fmaxf(hi[0].y, hi[1].y), fmaxf(hi[0].z, hi[1].z), 0.f);
            if (node == 0) break;
            node = sparent[node];
        }
        if (it == 130) set_err(&st->err, ERRBIT_BOUNDS);
    }
}

// ---------------------------------------------------------------------------
// Octree: replaces calcEdgeCounts + InclusiveSum (src/Octree.cu:38-50,
// 215-247) with one counting + decoupled look-back scan kernel writing the
// exclusive offsets and the node total.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kScanThreads) k_oct_scan(const uint8_t* __restrict__ prefix_n,
                                                           const int32_t* __restrict__ parent,
                                                           int32_t* __restrict__ counts,
                                                           int32_t* __restrict__ offsets,
                                                           unsigned long long* __restrict__ lookback,
                                                           DevState* st, int spin_limit) {
    __shared__ long long s_w[kScanThreads / 32 + 1];
    __shared__ uint32_t s_tile;
    __shared__ long long s_excl;
    const int64_t N = (int64_t)st->u - 1;
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(&st->tile_counter[kSortPasses + 1], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t first = (int64_t)tile * kScanTile + (int64_t)tid * kScanIpt;
    int32_t c[kScanIpt];
    long long sum = 0;
    const int root_level = N > 0 ? prefix_n[0] / 3 : 0;
#pragma unroll
    for (int i = 0; i < kScanIpt; ++i) {
        const int64_t j = first + i;
        int32_t v = 0;
        if (j == 0) {
            v = 1;  // the root (src/Octree.cu:217-218)
        } else if (j < N) {
            const int32_t pp = parent[j];
            v = prefix_n[j] / 3 - ((pp >= 0 && pp < N) ? prefix_n[pp] / 3 : root_level);
        }
        c[i] = v;
        if (j < N) counts[j] = v;
        sum += v;
    }
    // Counts can be negative only in a tree broken by the compat root; values
    // travel through the look-back as 62-bit two's complement.
    auto sx62 = [](unsigned long long v) { return (long long)(v << 2) >> 2; };
    long long tot;
    const long long toff = block_excl_scan<kScanThreads, long long>(sum, s_w, &tot);
    if (tid == 0) {
        unsigned long long* mine = lookback + tile;
        long long excl = 0;
        if (tile == 0) {
            st_relaxed64(mine, LB64_PRE | ((unsigned long long)tot & LB64_VAL));
        } else {
            st_relaxed64(mine, LB64_AGG | ((unsigned long long)tot & LB64_VAL));
            int64_t p = (int64_t)tile - 1;
            int spins = 0;
            while (p >= 0) {
                const unsigned long long v = ld_relaxed64(lookback + p);
                const unsigned long long f = v >> 62;
                if (f == 0) {
                    if (++spins > spin_limit) { set_err(&st->err, ERRBIT_LOOKBACK); break; }
                    continue;
                }
                excl += sx62(v & LB64_VAL);
                if (f == 2) break;
                --p;
            }
            st_relaxed64(mine, LB64_PRE | ((unsigned long long)(excl + tot) & LB64_VAL));
        }
        s_excl = excl;
        if ((int64_t)(tile + 1) * kScanTile >= N) {
            const long long total = excl + tot;
            st->n_oct = (N > 0 && total > 0) ? (unsigned long long)total : 0ull;
            st->root_level = root_level;
        }
    }
    __syncthreads();
    long long run = s_excl + toff;
#pragma unroll
    for (int i = 0; i < kScanIpt; ++i) {
        const int64_t j = first + i;
        if (j <= N) offsets[j] = (int32_t)run;
        run += c[i];
    }
}

// Zero the node array (src/Octree.cu:250-253). The root's corner and size are
// written by k_oct_make's thread 0 (src/Octree.cu:257-261).
__global__ void __launch_bounds__(256) k_oct_zero(OtNode* __restrict__ nodes, int64_t cap, DevState* st) {
    const int64_t m = (int64_t)st->n_oct;
    if (m > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_err(&st->err, ERRBIT_OCT_CAPACITY);
        return;
    }
    uint2* w = reinterpret_cast<uint2*>(nodes);  // 56 B = 7 x 8 B per node
    const int64_t words = m * 7;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += stride) w[i] = make_uint2(0u, 0u);
}

__device__ __forceinline__ int64_t oct_walk_up(int64_t r, const int32_t* __restrict__ counts,
                                               const int32_t* __restrict__ parent, int64_t N, DevState* st) {
    for (int it = 0; it < 130; ++it) {
        if (r < 0 || r >= N) { set_err(&st->err, ERRBIT_BOUNDS); return -1; }
        if (counts[r] != 0) return r;
        r = parent[r];
    }
    set_err(&st->err, ERRBIT_BOUNDS);
    return -1;
}

// makeNodes, src/Octree.cu:114-161: each radix node emits its chain of
// counts[i] octree nodes (deepest first) and links the chain's top under the
// bottom node of its nearest contributing ancestor.
__global__ void __launch_bounds__(256) k_oct_make(OtNode* __restrict__ nodes, int64_t cap,
                                                  const int32_t* __restrict__ offsets,
                                                  const int32_t* __restrict__ counts,
                                                  const uint64_t* __restrict__ codes,
                                                  const uint8_t* __restrict__ prefix_n,
                                                  const int32_t* __restrict__ parent, int code_bits, DevState* st) {
    const int64_t m = (int64_t)st->n_oct;
    if (m > cap || m < 1) return;
    const int64_t N = (int64_t)st->u - 1;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float mn = st->min_coord, range = st->range;
    const int CL = code_bits;
    const int root_level = st->root_level;
    auto cell = [&](int level) { return __fdiv_rn(range, (float)one_shl(level - root_level)); };
    auto put_corner = [&](int64_t o, uint64_t pre, int level) {
        const float3 c = code_to_point(shl_clamp(pre, CL - 3 * level), mn, range, CL);
        nodes[o].corner[0] = c.x;
        nodes[o].corner[1] = c.y;
        nodes[o].corner[2] = c.z;
        nodes[o].cell_size = cell(level);
    };
    if (i == 0) {
        const uint64_t rp = shr_clamp(codes[0], CL - 3 * root_level);
        const float3 c = code_to_point(shl_clamp(rp, CL - 3 * root_level), mn, range, CL);
        nodes[0].corner[0] = c.x;
        nodes[0].corner[1] = c.y;
        nodes[0].corner[2] = c.z;
        nodes[0].cell_size = range;
        return;
    }
    int64_t oct = offsets[i];
    const int nn = counts[i];
    const int lvl_i = prefix_n[i] / 3;
    const uint64_t ci = codes[i];
    for (int j = 0; j < nn - 1; ++j) {
        const int level = lvl_i - j;
        const uint64_t pre = shr_clamp(ci, CL - 3 * level);
        const int64_t par = oct + 1;
        if (par >= 0 && par < m && oct >= 0 && oct < m) {
            nodes[par].children[pre & 7] = (int32_t)oct;
            atomicOr(&nodes[par].child_node_mask, 1 << (pre & 7));
            put_corner(oct, pre, level);
        } else {
            set_err(&st->err, ERRBIT_BOUNDS);
        }
        oct = par;
    }
    if (nn > 0) {
        const int64_t rp = oct_walk_up(parent[i], counts, parent, N, st);
        if (rp < 0) return;
        const int64_t op = offsets[rp];
        const int top = lvl_i - nn + 1;
        const uint64_t pre = shr_clamp(ci, CL - 3 * top);
        if (op >= 0 && op < m && oct >= 0 && oct < m) {
            nodes[op].children[pre & 7] = (int32_t)oct;
            atomicOr(&nodes[op].child_node_mask, 1 << (pre & 7));
            put_corner(oct, pre, top);
        } else {
            set_err(&st->err, ERRBIT_BOUNDS);
        }
    }
}

// linkLeafNodes, src/Octree.cu:65-112: each leaf child of a radix node goes
// into the bottom octree node of the nearest contributing ancestor.
__global__ void __launch_bounds__(256) k_oct_link(OtNode* __restrict__ nodes, int64_t cap,
                                                  const int32_t* __restrict__ offsets,
                                                  const int32_t* __restrict__ counts,
                                                  const uint64_t* __restrict__ codes,
                                                  const uint8_t* __restrict__ hll, const uint8_t* __restrict__ hlr,
                                                  const uint8_t* __restrict__ prefix_n,
                                                  const int32_t* __restrict__ parent,
                                                  const int32_t* __restrict__ left_child, int code_bits,
                                                  DevState* st) {
    const int64_t m = (int64_t)st->n_oct;
    if (m > cap) return;
    const int64_t u = (int64_t)st->u;
    const int64_t N = u - 1;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const bool sides[2] = {hll[i] != 0, hlr[i] != 0};
    if (!sides[0] && !sides[1]) return;
    const int lvl = prefix_n[i] / 3 + 1;
    const int64_t rn = oct_walk_up(i, counts, parent, N, st);
    if (rn < 0) return;
    const int64_t node = offsets[rn];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        if (!sides[side]) continue;
        const int64_t leaf = (int64_t)left_child[i] + side;
        if (leaf < 0 || leaf >= u || node < 0 || node >= m) { set_err(&st->err, ERRBIT_BOUNDS); continue; }
        const uint64_t pre = shr_clamp(codes[leaf], code_bits - 3 * lvl);
        nodes[node].children[pre & 7] = (int32_t)leaf;
        atomicOr(&nodes[node].child_leaf_mask, 1 << (pre & 7));
    }
}

// Digit histograms of given keys (the histogram half of k_encode), for
// sorting keys that were not produced by k_encode.
__global__ void __launch_bounds__(256) k_hist_keys(const uint64_t* __restrict__ keys, int64_t n, DevState* st) {
    __shared__ uint32_t s_h[kSortPasses][kSortBins];
    for (int i = threadIdx.x; i < kSortPasses * kSortBins; i += blockDim.x) (&s_h[0][0])[i] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t c = keys[i];
#pragma unroll
        for (int p = 0; p < kSortPasses; ++p) atomicAdd(&s_h[p][(c >> (kSortBits * p)) & (kSortBins - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortPasses * kSortBins; i += blockDim.x) {
        const uint32_t v = (&s_h[0][0])[i];
        if (v) atomicAdd(&(&st->hist[0][0])[i], v);
    }
}

// After the sort passes the result sits in buf1 when an odd number of passes
// ran; copy it back into buf0.
__global__ void __launch_bounds__(256) k_copy_if_odd(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                                     int64_t n, const DevState* st) {
    if (!(st->n_active & 1)) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
}

inline unsigned grid_for(int64_t work, int threads, int64_t cap_blocks) {
    int64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (cap_blocks > 0 && b > cap_blocks) b = cap_blocks;
    return (unsigned)b;
}

}  // namespace

// Onesweep's shared memory (68 KB per block) with the whole carveout for
// shared memory, so that the 3 blocks its registers allow fit on an SM.
static cudaError_t set_onesweep_attributes() {
    cudaError_t e = cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(SortSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_onesweep, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    return e;
}

cudaError_t enqueue_sort_keys(uint64_t* keys, uint64_t* tmp, int64_t n, uint32_t* lookback, DevState* st,
                              cudaStream_t s, int num_sms) {
    cudaError_t e = set_onesweep_attributes();
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(st, 0, sizeof(DevState), s);
    if (n <= 0) return cudaGetLastError();
    k_hist_keys<<<grid_for(n, 256, num_sms * 4), 256, 0, s>>>(keys, n, st);
    k_sort_prep<<<1, kSortBins, 0, s>>>(n, st);
    const int64_t sort_tiles = (n + kSortTile - 1) / kSortTile;
    for (int pass = 0; pass < kSortPasses; ++pass) {
        cudaMemsetAsync(lookback, 0, sizeof(uint32_t) * kSortBins * sort_tiles, s);
        k_onesweep<<<(unsigned)sort_tiles, kSortThreads, sizeof(SortSmem), s>>>(keys, tmp, n, pass, lookback, st,
                                                                                 kSpinLimit, 0);
    }
    k_copy_if_odd<<<grid_for(n, 256, num_sms * 4), 256, 0, s>>>(tmp, keys, n, st);
    return cudaGetLastError();
}

cudaError_t enqueue_octree(const BuildBufs& b, const BuildParams& p, cudaStream_t s, int num_sms, int* launches) {
    const int64_t n = p.n;
    const int64_t scan_tiles = (n + kScanTile - 1) / kScanTile;
    cudaMemsetAsync(b.lookback64, 0, sizeof(unsigned long long) * scan_tiles, s);
    cudaMemsetAsync(&b.st->tile_counter[kSortPasses + 1], 0, sizeof(uint32_t), s);
    k_oct_scan<<<(unsigned)scan_tiles, kScanThreads, 0, s>>>(b.prefix_n, b.parent, b.oct_counts, b.oct_offsets,
                                                             b.lookback64, b.st, p.spin_limit);
    k_oct_zero<<<grid_for(b.oct_cap * 7, 256, num_sms * 8), 256, 0, s>>>((OtNode*)b.oct_nodes, b.oct_cap, b.st);
    k_oct_make<<<grid_for(n, 256, 0), 256, 0, s>>>((OtNode*)b.oct_nodes, b.oct_cap, b.oct_offsets, b.oct_counts,
                                                   b.codes, b.prefix_n, b.parent, p.code_bits, b.st);
    k_oct_link<<<grid_for(n, 256, 0), 256, 0, s>>>((OtNode*)b.oct_nodes, b.oct_cap, b.oct_offsets, b.oct_counts,
                                                   b.codes, b.has_leaf_left, b.has_leaf_right, b.prefix_n, b.parent,
                                                   b.left_child, p.code_bits, b.st);
    if (launches) *launches += 4;
    return cudaGetLastError();
}

cudaError_t enqueue_build(const BuildBufs& b, const BuildParams& p, cudaStream_t s, int num_sms, cudaEvent_t* ev,
                          int* launches) {
    int nl = 0;
    // stage i runs between events i and i+1; each stage is also an NVTX range
    static const char* const kStageNames[kBuildEvents - 1] = {
        "shapex.build.bbox", "shapex.build.encode", "shapex.build.sort", "shapex.build.dedup",
        "shapex.build.radix_tree", "shapex.build.search_boxes", "shapex.build.octree"};
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], s);
        if (i > 0) nvtxRangePop();
        if (i < kBuildEvents - 1) nvtxRangePushA(kStageNames[i]);
    };
    {
        // per device and cheap: set on every build
        cudaError_t e = set_onesweep_attributes();
        if (e != cudaSuccess) return e;
    }
    const int64_t n = p.n;
    mark(0);
    cudaMemsetAsync(b.st, 0, sizeof(DevState), s);
    if (n <= 0) {
        for (int i = 1; i < kBuildEvents; ++i) mark(i);
        if (launches) *launches = 0;
        return cudaGetLastError();
    }
    k_bbox<<<grid_for((n + 3) / 4, 256, num_sms * 4), 256, 0, s>>>(b.x, b.y, b.z, n, b.st);
    mark(1);
    k_encode<<<grid_for(n, 256, num_sms * 4), 256, 0, s>>>(b.x, b.y, b.z, n, p.code_bits, b.keys0, b.st);
    k_sort_prep<<<1, kSortBins, 0, s>>>(n, b.st);
    mark(2);
    nl += 3;
    const int64_t sort_tiles = (n + kSortTile - 1) / kSortTile;
    for (int pass = 0; pass < kSortPasses; ++pass) {
        cudaMemsetAsync(b.lookback, 0, sizeof(uint32_t) * kSortBins * sort_tiles, s);
        k_onesweep<<<(unsigned)sort_tiles, kSortThreads, sizeof(SortSmem), s>>>(b.keys0, b.keys1, n, pass,
                                                                                 b.lookback, b.st, p.spin_limit,
                                                                                 p.stall_first_tile);
        ++nl;
    }
    mark(3);
    const int64_t dd_tiles = (n + kDedupTile - 1) / kDedupTile;
    cudaMemsetAsync(b.lookback, 0, sizeof(uint32_t) * dd_tiles, s);
    k_dedup<<<(unsigned)dd_tiles, kDedupThreads, 0, s>>>(b.keys0, b.keys1, n, p.code_bits, b.codes, b.pts4, b.pts3,
                                                         b.lookback, b.st, p.spin_limit);
    ++nl;
    mark(4);
    cudaMemsetAsync(b.parent, 0, sizeof(int32_t) * n, s);
    cudaMemsetAsync(b.visit, 0, sizeof(uint32_t) * n, s);
    cudaMemsetAsync(b.sparent, 0xff, sizeof(int32_t) * n, s);
    cudaMemsetAsync(b.leaf_parent, 0xff, sizeof(int32_t) * n, s);
    k_karras<<<grid_for(n, 256, 0), 256, 0, s>>>(b.codes, p.code_bits, p.root_compat, b.left_child, b.parent,
                                                 b.prefix_n, b.has_leaf_left, b.has_leaf_right, b.sparent,
                                                 b.leaf_parent, b.range_end, b.st);
    ++nl;
    if (p.root_compat) {
        k_root_parent<<<1, 1, 0, s>>>(b.left_child, b.parent, b.has_leaf_left, b.has_leaf_right, b.st);
        ++nl;
    }
    mark(5);
    k_boxes<<<grid_for(n, 256, 0), 256, 0, s>>>(b.pts4, b.left_child, b.has_leaf_left, b.has_leaf_right, b.sparent,
                                                b.leaf_parent, b.range_end, b.visit, b.node_box, b.snodes, p.bucket,
                                                b.st);
    ++nl;
    mark(6);
    if (p.build_octree) {
        cudaError_t e = enqueue_octree(b, p, s, num_sms, &nl);
        if (e != cudaSuccess) {
            nvtxRangePop();  // the octree stage's range
            return e;
        }
    }
    mark(7);
    if (launches) *launches = nl;
    return cudaGetLastError();
}

}  // namespace shapex
