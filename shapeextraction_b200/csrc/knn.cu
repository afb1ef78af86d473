// Exact kNN over the search hierarchy, fused with covariance, 3x3 symmetric
// eigensolve and orientation (sm_100a).
//
// Replaces, from the reference (paths relative to its project root):
//   knnSearchKernel<k> + nodeBoxDistance + PriorityQueue
//       src/Octree.hpp:136-212, src/Octree.cu:326-352, src/dequeue.hpp
//   findCovariancesKernel<k>            src/NormalEstimation.hpp:96-156
//   cusolverDnSsyevjBatched             src/NormalEstimation.hpp:235-301
//   normalsFromEigenVectors             src/NormalEstimation.hpp:158-192
//
// One warp serves 32 consecutive queries (Morton-ordered, so spatially
// coherent); lane i owns query i. Each lane keeps its k best (squared
// distance, index) keys as a sorted list in registers, whose last entry is
// the lane's pruning bound. The warp first offers the Morton window around its
// queries, then walks the search hierarchy depth first with a shared stack: a
// child is entered when any lane's bound reaches its box, nearer child first
// by lane vote. Bucket points (contiguous runs of at most `bucket` points) are
// staged in shared memory and read by broadcast. A point that reaches a lane's
// bound goes to that lane's candidate buffer; buffers are merged into the
// lists in batches, so that the warp pays for one list update per buffered
// slot rather than one per point any lane accepts. Pruning uses the box
// distance with the same rounding chain as the point distance, so the result
// is exact, ties broken by point index.

#include <cfloat>
#include <climits>
#include <cstdint>

#include "pipeline.cuh"
#include "eig3.cuh"

namespace shapex {

namespace {

constexpr int kStackDepth = 96;
// Per-k tile shape, measured on B200 (2M scene and 5M mixture clouds): small
// lists leave registers for more resident warps, which pays for itself up to
// k = 16. The 24- and 32-key lists need more registers, so they keep the
// larger buffer and run in 2-warp blocks: 7 resident blocks (14 warps) where
// 4-warp blocks fit only 3 (12 warps); k = 32 ran 2.7% faster. k = 24 fits
// 128 registers without spills and is asked for 8 blocks (16 warps): at 130
// registers (7 blocks) it ran 11% slower on the 2M scene. k = 32 asks for 6
// so that ptxas does not cap its registers (a cap of 7 x 64 threads forced
// 128 registers and spills). Registers, not shared
// memory, hold k <= 16 at 5 blocks, so its buffer grew from 48 to 56 slots
// (fewer flushes; the learned search ran 3% faster). 64 slots shrank the L1
// cache enough to cost 3-4%.
template <int K>
struct KnnCfg {
    static constexpr int buf = K <= 8 ? 40 : (K <= 16 ? 56 : 64);  // candidate buffer slots per lane
    static constexpr int threads = K <= 16 ? 128 : 64;              // block size
    static constexpr int warps = threads / 32;
    static constexpr int min_blocks = K <= 8 ? 6 : (K <= 16 ? 5 : (K <= 24 ? 8 : 6));  // resident blocks per SM asked of ptxas
};
constexpr int kMaxHalo = 48;            // seed points on each side of a warp's queries
constexpr int kWindowMax = 32 + 2 * kMaxHalo;
constexpr unsigned FULL = 0xffffffffu;

// (squared distance, index) packed so that one unsigned compare orders by
// distance then index; distances are >= 0, so their IEEE bits are monotonic.
__device__ __forceinline__ unsigned long long pack_key(float d, int64_t i) {
    return ((unsigned long long)__float_as_uint(d) << 32) | (uint32_t)i;
}
constexpr unsigned long long kEmptyKey = (0x7f800000ull << 32) | 0xffffffffull;  // (+inf, max index)
__device__ __forceinline__ int32_t key_idx(unsigned long long k) { return (int32_t)(uint32_t)k; }
__device__ __forceinline__ float key_d(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }

// key[i] for a run-time i, as a masked OR over all entries, so that the list
// stays in registers (a direct key[i] would move it to local memory).
template <int K>
__device__ __forceinline__ unsigned long long pick(const unsigned long long (&key)[K], int i) {
    unsigned long long acc = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) acc |= key[j] & (0ull - (unsigned long long)(j == i));
    return acc;
}

// The k best keys of one query, ascending, in registers. Insertion compares
// the new key with every entry independently and shifts in one step (no
// serial chain). With EXACT = false the list is longer than k and the bound
// is entry k-1.
template <int K, bool EXACT>
struct TopK {
    static_assert(K % 2 == 0, "list sizes are even");
    unsigned long long key[K];
    unsigned long long bk;  // entry k-1: the pruning bound
    int kk;
    __device__ __forceinline__ void init(int k) {
#pragma unroll
        for (int j = 0; j < K; ++j) key[j] = kEmptyKey;
        bk = kEmptyKey;
        kk = k;
    }
    __device__ __forceinline__ float tau() const { return key_d(bk); }
    // After key[0..K) was filled with arbitrary keys: sort ascending with an
    // odd-even transposition network (K passes of independent
    // compare-exchanges) and set the bound.
    __device__ __forceinline__ void sort_filled() {
        if constexpr (K == 4 || K == 8 || K == 16) {
            // power-of-two lists: a bitonic network, fully unrolled (80
            // compare-exchanges at K = 16 against 120 for the transposition
            // network below, in about as much code)
#pragma unroll
            for (int k = 2; k <= K; k <<= 1)
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
                    for (int i = 0; i < K; ++i) {
                        const int l = i ^ j;
                        if (l > i) {
                            const unsigned long long a = key[i], b = key[l];
                            const bool up = (i & k) == 0;
                            const bool sw = up ? (b < a) : (a < b);
                            key[i] = sw ? b : a;
                            key[l] = sw ? a : b;
                        }
                    }
        } else {
            // K passes as K/2 rolled (even, odd) pairs: the same exchanges as
            // a fully unrolled network in K instead of K*K/2 instructions'
            // worth of code, which keeps large-k kernels inside the
            // instruction cache
#pragma unroll 1
            for (int pass = 0; pass < K; pass += 2) {
#pragma unroll
                for (int j = 0; j + 1 < K; j += 2) {
                    const unsigned long long a = key[j], b = key[j + 1];
                    key[j] = a < b ? a : b;
                    key[j + 1] = a < b ? b : a;
                }
#pragma unroll
                for (int j = 1; j + 1 < K; j += 2) {
                    const unsigned long long a = key[j], b = key[j + 1];
                    key[j] = a < b ? a : b;
                    key[j + 1] = a < b ? b : a;
                }
            }
        }
        if (EXACT) {
            bk = key[K - 1];
        } else {
            bk = pick(key, kk - 1);
        }
    }
    // insert() for a key that lands in the last K - H entries (nk > key[H - 1]):
    // the first H stay, so only the rest is compared and shifted.
    template <int H>
    __device__ __forceinline__ void insert_upper(unsigned long long nk) {  // requires key[H-1] < nk < bk
        bool lt[K];
#pragma unroll
        for (int j = H; j < K; ++j) lt[j] = key[j] < nk;
#pragma unroll
        for (int j = K - 1; j >= H + 1; --j) key[j] = lt[j] ? key[j] : (lt[j - 1] ? nk : key[j - 1]);
        key[H] = lt[H] ? key[H] : nk;
        if (EXACT) {
            bk = key[K - 1];
        } else {
            bk = pick(key, kk - 1);
        }
    }
    // One merge step of the warp (lists of up to 16 keys): lanes with `ins`
    // insert nk; when every inserting lane's key lands in the upper half of
    // its list (most late insertions), the warp takes the half-width
    // insertion. Plain kNN 1.5-3.7% faster at k = 16. Lists of 24 and 32 keys
    // keep the full insertion: the second one's registers cost them
    // occupancy (k = 32 1-4% slower).
    __device__ __forceinline__ void merge_step(unsigned long long nk, bool ins) {
        if (!__any_sync(0xffffffffu, ins)) return;
        if (__all_sync(0xffffffffu, !ins || nk > key[K / 2 - 1])) {
            if (ins) insert_upper<K / 2>(nk);
        } else {
            if (ins) insert(nk);
        }
    }
    __device__ __forceinline__ void insert(unsigned long long nk) {  // requires nk < bk
        bool lt[K];
#pragma unroll
        for (int j = 0; j < K; ++j) lt[j] = key[j] < nk;
#pragma unroll
        for (int j = K - 1; j >= 1; --j) key[j] = lt[j] ? key[j] : (lt[j - 1] ? nk : key[j - 1]);
        key[0] = lt[0] ? key[0] : nk;
        if (EXACT) {
            bk = key[K - 1];
        } else {
            bk = pick(key, kk - 1);
        }
    }
};

// Per-warp shared scratch: traversal stack, staged points, candidate buffers
// ([slot][lane] so that a warp's accesses to one slot fall in distinct banks).
template <int B>
struct WarpSmem {
    int32_t stack[kStackDepth];
    float4 pts[kWindowMax];
    int32_t buf[B][32];
};

// Ordered widest first so that the struct packs into 128 bytes: one more
// padded word (144 bytes) made ptxas give the k = 32 kernels 161-163
// registers instead of 142, one resident block per SM fewer.
struct QArgs {
    int64_t start, count, u;
    const float* ext;
    int32_t* out_idx;
    float* out_d2;
    float* out_normals;
    const float* learned_r2;
    const uint32_t* cell_lut;  // learned cell scan: code-range table (null: tree walk with the cap)
    float vx, vy, vz;
    float gap;
    int k;
    int code_bits;
    int bucket;
    int seed_halo;
    int learned_skip_seed;
    int device_count;  // 1: u = count = the build's unique-point count, read on the device (start 0)
    int step_limit;    // > 0: node visits per warp before the walk gives up (test hook)
    int lut_shift;     // per-axis shift of the table's level (bits per axis - level)
    int cell_pmax;     // cell scan: most points per warp before it falls back to the walk
    int cell_span;     // cell scan: most cells per axis covering one lane's ball (2..4)
};
static_assert(sizeof(QArgs) == 128, "QArgs grew past 128 bytes");

struct Counters {
    int cand = 0, ins = 0, merge = 0, buckets = 0, lmiss = 0, cells = 0, cell_fallback = 0, cell_lookups = 0,
        cell_points = 0;
};

// Merge every lane's buffered candidates into its list; the warp steps
// through max-over-lanes slots together.
template <int K, bool EXACT, class WS>
__device__ __forceinline__ void flush(TopK<K, EXACT>& tk, int& bc, WS& W, int lane, Counters& ct,
                                      const float4* __restrict__ pts, float qx, float qy, float qz) {
    const int maxc = (int)__reduce_max_sync(FULL, (unsigned)bc);
    ct.merge += maxc;
    ct.cand += bc;
    if (K > 8) {
        // the next candidate's point is loaded before this one's insertion,
        // hiding its latency behind the list update (about 1% at k >= 16;
        // slower at k = 8, whose insertions are too short to hide it)
        int32_t idx_n = bc > 0 ? W.buf[0][lane] : 0;
        float4 p_n = bc > 0 ? __ldg(pts + idx_n) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int j = 0; j < maxc; ++j) {
            const int32_t idx = idx_n;
            const float4 p = p_n;
            if (j + 1 < bc) {
                idx_n = W.buf[j + 1][lane];
                p_n = __ldg(pts + idx_n);
            }
            if constexpr (K <= 16) {
                const unsigned long long nk = pack_key(dist2(qx, qy, qz, p.x, p.y, p.z), idx);
                const bool ins = j < bc && nk < tk.bk;
                tk.merge_step(nk, ins);
                ct.ins += ins;
            } else {
                if (j < bc) {
                    const unsigned long long nk = pack_key(dist2(qx, qy, qz, p.x, p.y, p.z), idx);
                    if (nk < tk.bk) {
                        tk.insert(nk);
                        ++ct.ins;
                    }
                }
            }
        }
    } else {
        for (int j = 0; j < maxc; ++j) {
            const bool in = j < bc;
            const int32_t idx = in ? W.buf[j][lane] : 0;
            const float4 p = __ldg(pts + idx);
            const unsigned long long nk = pack_key(dist2(qx, qy, qz, p.x, p.y, p.z), idx);
            const bool ins = in && nk < tk.bk;
            tk.merge_step(nk, ins);
            ct.ins += ins;
        }
    }
    bc = 0;
}

// Stage points [first, first + cnt) (cnt <= 32) in shared memory and append
// every one whose distance reaches the lane's bound to the lane's buffer.
// Points of the seed window [w0, w1) are skipped (they were already offered).
// The caller guarantees that bc + cnt fits the buffer.
// The points are staged in pairs for dist2_pair: floats [4j, 4j + 4) hold
// x and y of points 2j and 2j + 1, floats [64 + 2j, 64 + 2j + 2) their z; a
// slot past cnt holds a NaN x, whose distance passes no bound.
template <class WS>
__device__ __forceinline__ void scan_chunk(int32_t first, int cnt, bool need, float qx, float qy, float qz,
                                           float tau, int& bc, WS& W, const float4* __restrict__ pts,
                                           int32_t w0, int32_t w1, int lane) {
    float* f = reinterpret_cast<float*>(W.pts);
    {
        const float4 p = lane < cnt ? __ldg(pts + first + lane) : make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
        const int o = 4 * (lane >> 1) + (lane & 1);
        f[o] = p.x;
        f[o + 2] = p.y;
        f[64 + lane] = p.z;
    }
    __syncwarp();
    if (need) {
        const uint64_t qqx = twice(qx), qqy = twice(qy), qqz = twice(qz);
        if (first < w1 && first + cnt > w0) {  // overlaps the seed window: skip its points
            for (int t = 0; t < cnt; t += 2) {
                const ulonglong2 xy = *reinterpret_cast<const ulonglong2*>(f + 2 * t);
                const uint64_t d = dist2_pair(qqx, qqy, qqz, xy.x, xy.y, *reinterpret_cast<const uint64_t*>(f + 64 + t));
                const int32_t idx = first + t;
                if (lo_half(d) <= tau && (idx < w0 || idx >= w1)) W.buf[bc++][lane] = idx;
                if (hi_half(d) <= tau && (idx + 1 < w0 || idx + 1 >= w1)) W.buf[bc++][lane] = idx + 1;
            }
        } else {
            for (int t = 0; t < cnt; t += 2) {
                const ulonglong2 xy = *reinterpret_cast<const ulonglong2*>(f + 2 * t);
                const uint64_t d = dist2_pair(qqx, qqy, qqz, xy.x, xy.y, *reinterpret_cast<const uint64_t*>(f + 64 + t));
                if (lo_half(d) <= tau) W.buf[bc++][lane] = first + t;
                if (hi_half(d) <= tau) W.buf[bc++][lane] = first + t + 1;
            }
        }
    }
    __syncwarp();
}

// Same as scan_chunk when few lanes need the bucket (`mask`): each lane holds
// one point of the bucket and the warp steps over the needing queries, so the
// cost follows the number of needing lanes rather than the bucket size. Hits
// are appended to the needing lane's buffer in ballot order.
template <class WS>
__device__ __forceinline__ void scan_sparse(int32_t first, int cnt, uint32_t mask, float qx, float qy, float qz,
                                            float tau, int& bc, WS& W, const float4* __restrict__ pts,
                                            int32_t w0, int32_t w1, int lane) {
    const int32_t idx = first + lane;
    const bool has = lane < cnt && (idx < w0 || idx >= w1);
    const float4 p = lane < cnt ? __ldg(pts + idx) : make_float4(0.f, 0.f, 0.f, 0.f);
    while (mask) {
        const int i = __ffs(mask) - 1;
        mask &= mask - 1;
        const float xi = __shfl_sync(FULL, qx, i), yi = __shfl_sync(FULL, qy, i), zi = __shfl_sync(FULL, qz, i);
        const float ti = __shfl_sync(FULL, tau, i);
        const int base = __shfl_sync(FULL, bc, i);
        const bool pass = has && dist2(xi, yi, zi, p.x, p.y, p.z) <= ti;
        const uint32_t pm = __ballot_sync(FULL, pass);
        if (pass) W.buf[base + __popc(pm & lanemask_lt())][i] = idx;
        if (lane == i) bc += __popc(pm);
    }
    __syncwarp();
}

// Position of set bit number n (from 0) of w; w has more than n set bits.
__device__ __forceinline__ int nth_set_bit(uint32_t w, int n) {
    int pos = 0;
#pragma unroll
    for (int width = 16; width >= 1; width >>= 1) {
        const int c = __popc(w & ((1u << width) - 1u));
        if (n >= c) {
            n -= c;
            w >>= width;
            pos += width;
        }
    }
    return pos;
}

// First index in codes[lo, hi) whose code is >= key (hi when none).
__device__ __forceinline__ uint32_t lower_bound_codes(const uint64_t* __restrict__ codes, uint32_t lo, uint32_t hi,
                                                      uint64_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(codes + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Bounds of the decoded coordinates X0..X1 of one axis, for pruning: the
// decode (codeToPoint: fma(X / M, range, min)) is evaluated with a multiply by
// 1/M instead of the division and widened by `pad`, which exceeds the
// difference between the two evaluations (at most range * 2^-22 + max|coord| *
// 2^-23), so every decoded point of the range lies inside [lo, hi].
__device__ __forceinline__ void axis_bounds(uint32_t X0, uint32_t X1, float inv_m, float mn, float range, float pad,
                                            float& lo, float& hi) {
    lo = __fmaf_rn((float)X0 * inv_m, range, mn) - pad;
    hi = __fmaf_rn((float)X1 * inv_m, range, mn) + pad;
}

// Integer code-coordinate box [lo, hi] (per axis, clamped to [0, M]) that
// holds every tree point within squared distance r2 of the tree point whose
// code is `code`: |x_p - x_q| <= R for every point p with dist2 <= r2
// (dist2's rounding costs far less than the 1e-6 added to R), and in code
// units the decode adds at most 1/4 + 2^-23 * M * max|coordinate| / range on
// each side. r2 must be finite and >= 0; a degenerate range gives the whole
// cube.
__device__ __forceinline__ void ball_box(uint64_t code, float r2, uint32_t M, float mn, float range, uint32_t (&lo)[3],
                                         uint32_t (&hi)[3]) {
    const float fbs = (float)M;
    const float R = __fmul_ru(__fsqrt_ru(r2), 1.000001f);
    const float ru = __fmul_ru(R, __fdiv_ru(fbs, range));
    const float big = fmaxf(fabsf(mn), fabsf(mn + range));
    const float slack = __fadd_ru(__fmul_ru(__fmul_ru(1.1920929e-7f, fbs), __fdiv_ru(big, range)), 0.25f);
    const float ext = __fadd_ru(ru, slack) + 1.0f;
    const int64_t e = ext < 4.0e9f ? (int64_t)ceilf(ext) : ((int64_t)1 << 40);  // NaN: whole cube
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int64_t X = (int64_t)gather3(code >> ax);
        lo[ax] = (uint32_t)max64(0, X - e);
        hi[ax] = (uint32_t)min64((int64_t)M, X + e);
    }
}

constexpr int kCellBits = 1024;   // cells of a warp's union grid: one bit each, in stack[0, 32)
constexpr int kCellRanges = 64;   // nonempty cells a warp scans: listed in pts[32, 96), order keys after

// Learned attempt as a direct scan of Morton cells, with no tree walk.
//
// Each lane's predicted ball (radius sqrt(cap) around its query) is covered by
// an integer box of code coordinates, widened by the decode rounding, and the
// warp picks the finest level at which every lane's box spans at most
// cell_span cells per axis. The union of the lanes' cells is marked in a
// shared bitmap; each marked cell is the contiguous run of sorted codes under
// its prefix, found with the build's code-range table and a short binary
// search. The nonempty cells are taken nearest first (box distance to the
// warp's first query); a cell that no lane's current bound reaches any more is
// skipped, and the points of the others are packed into 32-point chunks that
// every lane tests against its own bound (dense: no per-lane loops). Every
// point within a lane's cap lies in one of its cells and is offered to it
// unless the lane's bound already excludes the cell's box, so a lane whose
// k-th distance ends within its cap has its exact k best; the caller searches
// the others again. Returns false, having offered nothing, when the warp's
// cells are too many (queries spread across distant regions) or hold more
// than cell_pmax points; the caller then walks the tree with the cap.
template <int K, bool EXACT, class WS>
__device__ __forceinline__ bool cell_scan(TopK<K, EXACT>& tk, int& bc, WS& W, int lane, Counters& ct,
                                          const float4* __restrict__ pts, const uint64_t* __restrict__ codes,
                                          const QArgs& a, const DevState* st, bool act, int64_t qi, float qx,
                                          float qy, float qz, float cap) {
    constexpr int kBuf = KnnCfg<K>::buf;
    const int bpa = a.code_bits / 3;
    const uint32_t M = bitscale_of(a.code_bits);
    const float fbs = (float)M;
    const float mn = st->min_coord, range = st->range;
    const bool ok = act && cap >= 0.0f && cap < INFINITY;  // false for NaN
    uint32_t lo[3] = {0u, 0u, 0u}, hi[3] = {0u, 0u, 0u};
    int s = 0;
    if (ok) {
        ball_box(__ldg(codes + qi), cap, M, mn, range, lo, hi);
        uint32_t dmax = 0;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) dmax = max(dmax, hi[ax] - lo[ax]);
        // the finest level at which the box spans at most cell_span cells per
        // axis: (hi >> s) - (lo >> s) <= (dmax >> s) + 1 <= cell_span - 1
        while ((int)(dmax >> s) > a.cell_span - 2) ++s;
    }
    const uint32_t okm = __ballot_sync(FULL, ok);
    if (!okm) return true;  // no lane has a usable cap: every active lane is searched again
    s = (int)__reduce_max_sync(FULL, (unsigned)(ok ? s : 0));
    uint32_t A[3], g[3];
    for (int tries = 0;; ++tries) {
        uint64_t cells = 1;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            A[ax] = __reduce_min_sync(FULL, ok ? (lo[ax] >> s) : 0xffffffffu);
            const uint32_t b = __reduce_max_sync(FULL, ok ? (hi[ax] >> s) : 0u);
            g[ax] = b - A[ax] + 1;
            cells *= g[ax];
        }
        if (cells <= (uint64_t)kCellBits) break;
        if (tries == 2 || s >= bpa) {
            ++ct.cell_fallback;
            return false;
        }
        ++s;
    }
    // mark the union of the lanes' cells
    uint32_t* bits = reinterpret_cast<uint32_t*>(W.stack);  // words [0, 32); inclusive prefixes at [32, 64)
    __syncwarp();
    bits[lane] = 0u;
    __syncwarp();
    if (ok) {
        for (uint32_t z = (lo[2] >> s) - A[2]; z <= (hi[2] >> s) - A[2]; ++z)
            for (uint32_t y = (lo[1] >> s) - A[1]; y <= (hi[1] >> s) - A[1]; ++y)
                for (uint32_t x = (lo[0] >> s) - A[0]; x <= (hi[0] >> s) - A[0]; ++x) {
                    const uint32_t b = (z * g[1] + y) * g[0] + x;
                    atomicOr(&bits[b >> 5], 1u << (b & 31));
                }
    }
    __syncwarp();
    const uint32_t word = bits[lane];
    int incl = __popc(word);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    uint32_t* pre = bits + 32;
    pre[lane] = (uint32_t)incl;
    __syncwarp();
    // one cell per lane per round: its code range and its order key
    int4* list = reinterpret_cast<int4*>(&W.pts[32]);                         // (first, count, prefix lo, hi)
    uint32_t* okeys = reinterpret_cast<uint32_t*>(&W.pts[32 + kCellRanges]);  // scan order keys
    const uint32_t* lut = a.cell_lut;
    const int ls = a.lut_shift;
    const float inv_m = 1.0f / fbs;
    const float big = fmaxf(fabsf(mn), fabsf(mn + range));
    const float pad = __fadd_ru(__fmul_ru(big, 4.76837158e-7f), __fmul_ru(range, 9.53674316e-7f));  // 2^-21, 2^-20
    // order reference: the warp's first query with a usable cap
    const int ref = __ffs(okm) - 1;
    const float rx = __shfl_sync(FULL, qx, ref), ry = __shfl_sync(FULL, qy, ref), rz = __shfl_sync(FULL, qz, ref);
    int nr = 0;
    int64_t ptotal = 0;
    ct.cell_lookups += total;
    for (int r0 = 0; r0 < total; r0 += 32) {
        const int idx = r0 + lane;
        uint32_t first = 0, cnt = 0;
        uint64_t P = 0;
        float key = 0.0f;
        if (idx < total) {
            int w = 0;  // the word holding marked cell number idx
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1)
                if ((int)pre[w + step - 1] <= idx) w += step;
            const int before = w > 0 ? (int)pre[w - 1] : 0;
            const uint32_t b = (uint32_t)(w * 32 + nth_set_bit(bits[w], idx - before));
            const uint32_t C[3] = {A[0] + b % g[0], A[1] + (b / g[0]) % g[1], A[2] + b / (g[0] * g[1])};
            P = spread3(C[0]) | (spread3(C[1]) << 1) | (spread3(C[2]) << 2);
            uint32_t last;
            if (s >= ls) {
                const int d = 3 * (s - ls);
                first = __ldg(lut + (P << d));
                last = __ldg(lut + ((P + 1) << d));
            } else {
                const uint64_t j = P >> (3 * (ls - s));
                const uint32_t l0 = __ldg(lut + j), l1 = __ldg(lut + j + 1);
                first = lower_bound_codes(codes, l0, l1, P << (3 * s));
                last = lower_bound_codes(codes, first, l1, (P + 1) << (3 * s));
            }
            cnt = last - first;
            float bl[3], bh[3];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax)
                axis_bounds(C[ax] << s, (uint32_t)min64((int64_t)M, ((int64_t)(C[ax] + 1) << s) - 1), inv_m, mn, range,
                            pad, bl[ax], bh[ax]);
            key = box_dist2(rx, ry, rz, bl[0], bl[1], bl[2], bh[0], bh[1], bh[2]);
        }
        const bool keep = cnt > 0;
        const uint32_t km = __ballot_sync(FULL, keep);
        if (keep) {
            const int pos = nr + __popc(km & lanemask_lt());
            if (pos < kCellRanges) {
                list[pos] = make_int4((int)first, (int)cnt, (int)(uint32_t)P, (int)(uint32_t)(P >> 32));
                okeys[pos] = (__float_as_uint(key) & ~0x7fu) | (uint32_t)pos;  // distance bits, entry number
            }
        }
        nr += __popc(km);
        ptotal += (int64_t)__reduce_add_sync(FULL, keep ? min(cnt, 1u << 26) : 0u);
    }
    if (nr > kCellRanges || ptotal > (int64_t)a.cell_pmax) {
        ++ct.cell_fallback;
        return false;
    }
    __syncwarp();
    ++ct.cells;
    ct.cell_points += (int)ptotal;
    // Cells nearest first, so that the bounds tighten early. Lane l holds the
    // order keys of entries l and l + 32. A cell goes on only if some lane's
    // current bound (its k-th distance so far, at most its cap) reaches the
    // cell's box; its points are appended to the staging chunk pts[0, 32)
    // (index in .w), and each full chunk is tested by every lane.
    uint32_t ok0 = lane < nr ? okeys[lane] : 0xffffffffu;
    uint32_t ok1 = lane + 32 < nr ? okeys[lane + 32] : 0xffffffffu;
    int fill = 0;
    bool merged = false;
    auto test_chunk = [&](int n) {
        __syncwarp();
        if (__any_sync(FULL, bc + n > kBuf)) flush(tk, bc, W, lane, ct, pts, qx, qy, qz);
        if (ok) {
            const float b2 = fminf(tk.tau(), cap);
            for (int t = 0; t < n; ++t) {
                const float4 p = W.pts[t];
                if (dist2(qx, qy, qz, p.x, p.y, p.z) <= b2) W.buf[bc++][lane] = __float_as_int(p.w);
            }
        }
        __syncwarp();
        if (!merged) {  // the nearest points usually hold most of each list: merge them at once
            merged = true;
            flush(tk, bc, W, lane, ct, pts, qx, qy, qz);
        }
    };
    for (int it = 0; it < nr; ++it) {
        const uint32_t m = __reduce_min_sync(FULL, min(ok0, ok1));
        if (ok0 == m) ok0 = 0xffffffffu;
        if (ok1 == m) ok1 = 0xffffffffu;
        const int4 r = list[m & 0x7fu];
        const uint64_t P = (uint64_t)(uint32_t)r.z | ((uint64_t)(uint32_t)r.w << 32);
        float bl[3], bh[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const uint32_t Cax = gather3(P >> ax);
            axis_bounds(Cax << s, (uint32_t)min64((int64_t)M, ((int64_t)(Cax + 1) << s) - 1), inv_m, mn, range, pad,
                        bl[ax], bh[ax]);
        }
        const bool need = ok && box_dist2(qx, qy, qz, bl[0], bl[1], bl[2], bh[0], bh[1], bh[2]) <= fminf(tk.tau(), cap);
        if (!__any_sync(FULL, need)) continue;
        ++ct.buckets;
        for (int off = 0; off < r.y;) {
            const int take = min(r.y - off, 32 - fill);
            if (lane < take) {
                const int32_t pi = r.x + off + lane;
                float4 p = __ldg(pts + pi);
                p.w = __int_as_float(pi);
                W.pts[fill + lane] = p;
            }
            fill += take;
            off += take;
            if (fill == 32) {
                test_chunk(32);
                fill = 0;
            }
        }
    }
    if (fill > 0) test_chunk(fill);
    return true;
}

__device__ __forceinline__ void neu_add(float& s, float& c, float x) {
    const float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// Normal of one query from its k neighbours, ascending, whose indices are in
// nbr[0], nbr[32], ... (the lane's column of the candidate buffer, free once
// the search is done; rolled loops keep the code small for large k):
// centred covariance with compensated FP32 sums, FP32 Jacobi, FP64 redo when
// the relative eigengap (l1 - l0) / l2 is below `gap`, orientation towards
// the viewpoint (src/NormalEstimation.hpp:184-189).
__device__ __forceinline__ void estimate_normal(const int32_t* nbr, int k, const float4* __restrict__ pts,
                                                float qx, float qy, float qz, const QArgs& a, float* out,
                                                DevState* st) {
    float s[3] = {0.f, 0.f, 0.f}, c[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
    for (int j = 0; j < k; ++j) {
        const float4 p = __ldg(pts + nbr[32 * j]);
        neu_add(s[0], c[0], p.x - qx);
        neu_add(s[1], c[1], p.y - qy);
        neu_add(s[2], c[2], p.z - qz);
    }
    const float inv_k = 1.0f / (float)k;
    const float m0 = (s[0] + c[0]) * inv_k, m1 = (s[1] + c[1]) * inv_k, m2 = (s[2] + c[2]) * inv_k;
    float cs[6] = {0, 0, 0, 0, 0, 0}, cc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int j = 0; j < k; ++j) {
        const float4 p = __ldg(pts + nbr[32 * j]);
        const float r0 = (p.x - qx) - m0, r1 = (p.y - qy) - m1, r2 = (p.z - qz) - m2;
        neu_add(cs[0], cc[0], r0 * r0);
        neu_add(cs[1], cc[1], r0 * r1);
        neu_add(cs[2], cc[2], r0 * r2);
        neu_add(cs[3], cc[3], r1 * r1);
        neu_add(cs[4], cc[4], r1 * r2);
        neu_add(cs[5], cc[5], r2 * r2);
    }
    const float inv_den = 1.0f / (float)(k > 1 ? k - 1 : 1);
    float C[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) C[e] = (cs[e] + cc[e]) * inv_den;
    float w[3], nv[3];
    eig3<float>(C, w, nv);
    float nx = nv[0], ny = nv[1], nz = nv[2];
    const float gap = (w[1] - w[0]) / fmaxf(fabsf(w[2]), FLT_MIN);
    if (!(gap >= a.gap)) {
        // near-degenerate neighbourhood: redo covariance and eigensolve in FP64
        double sd[3] = {0, 0, 0};
#pragma unroll 1
        for (int j = 0; j < k; ++j) {
            const float4 p = __ldg(pts + nbr[32 * j]);
            sd[0] += (double)p.x - (double)qx;
            sd[1] += (double)p.y - (double)qy;
            sd[2] += (double)p.z - (double)qz;
        }
        const double md[3] = {sd[0] / k, sd[1] / k, sd[2] / k};
        double Cd[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
        for (int j = 0; j < k; ++j) {
            const float4 p = __ldg(pts + nbr[32 * j]);
            const double r0 = ((double)p.x - (double)qx) - md[0];
            const double r1 = ((double)p.y - (double)qy) - md[1];
            const double r2 = ((double)p.z - (double)qz) - md[2];
            Cd[0] += r0 * r0; Cd[1] += r0 * r1; Cd[2] += r0 * r2;
            Cd[3] += r1 * r1; Cd[4] += r1 * r2; Cd[5] += r2 * r2;
        }
        const double dd = (double)(k > 1 ? k - 1 : 1);
#pragma unroll
        for (int e = 0; e < 6; ++e) Cd[e] /= dd;
        double wd[3], nd[3];
        eig3<double>(Cd, wd, nd);
        nx = (float)nd[0];
        ny = (float)nd[1];
        nz = (float)nd[2];
        atomicAdd(&st->counters[CNT_FP64], 1ull);
    }
    const float dot = (a.vx - qx) * nx + (a.vy - qy) * ny + (a.vz - qz) * nz;
    if (dot < 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
    out[0] = nx;
    out[1] = ny;
    out[2] = nz;
}

// The 32 queries [q0, q0 + 32) of one warp: search, then the outputs.
// CELLS: the learned attempt may run the cell scan (a separate instantiation,
// launched only when the caller turned the cell scan on: compiled into the
// default kernels, its code alone slowed them by about 8%).
template <int K, bool EXACT, bool EXT, bool NORMALS, bool CELLS>
__device__ __forceinline__ void knn_warp(const float4* __restrict__ pts, const SNode* __restrict__ snodes,
                                         const uint64_t* __restrict__ codes, const QArgs& a, DevState* st,
                                         int64_t q0, WarpSmem<KnnCfg<K>::buf>& W, int lane) {
    constexpr int kBuf = KnnCfg<K>::buf;
    static_assert(K <= kBuf, "the neighbour list is staged in the candidate buffer");
    const int64_t u = a.device_count ? (int64_t)st->u : a.u;
    const int64_t count = a.device_count ? u : a.count;
    if (q0 >= count) return;  // whole warp
    const int64_t qo = q0 + lane;
    const bool active = qo < count;
    float qx, qy, qz;
    int64_t center;  // tree index of the warp's first query (or its code position)
    if (EXT) {
        const int64_t src = active ? qo : q0;
        qx = __ldg(a.ext + 3 * src);
        qy = __ldg(a.ext + 3 * src + 1);
        qz = __ldg(a.ext + 3 * src + 2);
        const float lx = __shfl_sync(FULL, qx, 0), ly = __shfl_sync(FULL, qy, 0), lz = __shfl_sync(FULL, qz, 0);
        const float mn = st->min_coord, range = st->range;
        const float fbs = (float)bitscale_of(a.code_bits);
        auto q1 = [&](float v) {
            float f = __fmul_rn(fbs, __fdiv_rn(__fsub_rn(v, mn), range));
            f = fminf(fmaxf(f, 0.0f), fbs);
            return __float2uint_rz(f);
        };
        const uint64_t code = spread3(q1(lx)) | (spread3(q1(ly)) << 1) | (spread3(q1(lz)) << 2);
        int64_t lo = 0, hi = u;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (__ldg(codes + mid) < code) lo = mid + 1; else hi = mid;
        }
        center = lo - 16;
    } else {
        const float4 p = __ldg(pts + a.start + (active ? qo : q0));
        qx = p.x;
        qy = p.y;
        qz = p.z;
        center = a.start + q0;
    }
    const int64_t w0 = max64(0, center - a.seed_halo);
    const int64_t w1 = min64(u, center + 32 + a.seed_halo);
    const int S = (int)(w1 - w0);

    TopK<K, EXACT> tk;
    tk.init(a.k);
    Counters ct;
    uint32_t steps = 0;
    // With a learned radius, attempt 0 searches with the predicted bound as a
    // cap; a lane whose k-th neighbour lies beyond its cap (the cap pruned
    // points that could belong to its k best) is searched again without it.
    const bool learned = a.learned_r2 != nullptr;
    const float cap0 = (learned && active) ? __ldg(a.learned_r2 + qo) : INFINITY;
    bool act = active;
    for (int attempt = learned ? 0 : 1; attempt < 2; ++attempt) {
        const float cap = attempt == 0 ? cap0 : INFINITY;
        const bool seed = attempt == 1 || !a.learned_skip_seed;
        const int64_t sw0 = seed ? w0 : 0, sw1 = seed ? w1 : 0;  // points offered by the seed
        if (act) tk.init(a.k);
        int bc = 0;  // buffered candidates of this lane
        // learned attempt as a cell scan (falls back to the capped tree walk)
        const bool scanned = CELLS && attempt == 0 && a.cell_lut != nullptr &&
                             cell_scan<K, EXACT>(tk, bc, W, lane, ct, pts, codes, a, st, act,
                                                 a.start + (active ? qo : q0), qx, qy, qz, cap);
        __syncwarp();
        if (seed) {
            // Seed: each lane walks the Morton window outwards from its own
            // position (0, +1, -1, +2, ...), so its first candidates are its
            // index neighbours.
            __syncwarp();
            for (int i = lane; i < S; i += 32) W.pts[i] = __ldg(pts + w0 + i);
            __syncwarp();
            const int p = EXT ? (int)(center + 16 - w0) : (int)(center + lane - w0);
            const int reach = max(p, S - 1 - p);
            const int nsteps = 2 * (int)__reduce_max_sync(FULL, (unsigned)(act ? reach : 0)) + 1;
            // the first K spiral candidates fill the list directly, then one sort
            if (act) {
#pragma unroll
                for (int t = 0; t < K; ++t) {
                    const int off = (t & 1) ? (t + 1) >> 1 : -(t >> 1);
                    const int iw = p + off;
                    unsigned long long kv = kEmptyKey;
                    if (iw >= 0 && iw < S) {
                        const float4 q = W.pts[iw];
                        kv = pack_key(dist2(qx, qy, qz, q.x, q.y, q.z), w0 + iw);
                    }
                    tk.key[t] = kv;
                }
                tk.sort_filled();
            }
            // the rest of the window in runs of at most kBuf steps (a step
            // buffers at most one point per lane), one merge after each run
            float tau = fminf(tk.tau(), cap);
            int t = K;
            do {
                const int lim = min(nsteps, t + kBuf);
                for (; t < lim; ++t) {
                    const int off = (t & 1) ? (t + 1) >> 1 : -(t >> 1);
                    const int iw = p + off;
                    if (act && iw >= 0 && iw < S) {
                        const float4 q = W.pts[iw];
                        if (dist2(qx, qy, qz, q.x, q.y, q.z) <= tau) W.buf[bc++][lane] = (int32_t)(w0 + iw);
                    }
                }
                flush(tk, bc, W, lane, ct, pts, qx, qy, qz);
                tau = fminf(tk.tau(), cap);
            } while (t < nsteps);
        }

        if (!scanned && u >= 2 && (sw0 > 0 || sw1 < u)) {
            int sp = 1;
            if (lane == 0) W.stack[0] = 0;
            __syncwarp();
            const uint32_t step_cap =
                a.step_limit > 0 ? (uint32_t)a.step_limit : (uint32_t)min64(2 * u + 64, 0x7fffffff);
            while (sp > 0) {
                --sp;
                const int32_t node = W.stack[sp];
                __syncwarp();
                if (++steps > step_cap || node < 0 || node >= u - 1) {
                    if (lane == 0) set_err(&st->err, steps > step_cap ? ERRBIT_SEARCH_LIMIT : ERRBIT_BOUNDS);
                    break;
                }
                const SNode* sn = snodes + node;
                const float4 lo_l = __ldg(&sn->lo_l), hi_l = __ldg(&sn->hi_l);
                const float4 lo_r = __ldg(&sn->lo_r), hi_r = __ldg(&sn->hi_r);
                const int32_t refl = __float_as_int(lo_l.w), refr = __float_as_int(lo_r.w);
                const int32_t cntl = __float_as_int(hi_l.w), cntr = __float_as_int(hi_r.w);
                const uint32_t u32 = (uint32_t)u;
                const bool okl = cntl <= a.bucket ? (cntl >= 1 && (uint32_t)refl <= u32 - (uint32_t)cntl)
                                                  : (uint32_t)refl < u32 - 1;
                const bool okr = cntr <= a.bucket ? (cntr >= 1 && (uint32_t)refr <= u32 - (uint32_t)cntr)
                                                  : (uint32_t)refr < u32 - 1;
                if (!(okl && okr)) {
                    if (lane == 0) set_err(&st->err, ERRBIT_BOUNDS);
                    break;
                }
                const float tau = fminf(tk.tau(), cap);
                const float dl = box_dist2(qx, qy, qz, lo_l.x, lo_l.y, lo_l.z, hi_l.x, hi_l.y, hi_l.z);
                const float dr = box_dist2(qx, qy, qz, lo_r.x, lo_r.y, lo_r.z, hi_r.x, hi_r.y, hi_r.z);
                const uint32_t bl = __ballot_sync(FULL, act && dl <= tau);
                const uint32_t br = __ballot_sync(FULL, act && dr <= tau);
                if (!(bl | br)) continue;
                const uint32_t vote = __ballot_sync(FULL, act && dl <= dr);
                const int nact = __popc(__ballot_sync(FULL, act));
                const bool leftFirst = 2 * __popc(vote) >= nact;
                // rolled: one copy of the scan and merge code serves both
                // children (a copy per child cost 4-8% in instruction fetch)
#pragma unroll 1
                for (int o = 0; o < 2; ++o) {
                    const bool left = (o == 0) == leftFirst;
                    const int32_t cnt = left ? cntl : cntr;
                    if (cnt > a.bucket) continue;
                    const int32_t first = left ? refl : refr;
                    if (first >= sw0 && first + cnt <= sw1) continue;  // all of it was in the seed window
                    const float bnd = fminf(tk.tau(), cap);
                    const bool need = act && (left ? dl : dr) <= bnd;
                    const uint32_t needm = __ballot_sync(FULL, need);
                    if (!needm) continue;
                    ++ct.buckets;
                    // buckets of more than 32 points go in 32-point chunks
                    for (int c0 = 0; c0 < cnt; c0 += 32) {
                        const int32_t f = first + c0;
                        const int n = min(32, cnt - c0);
                        if (f >= sw0 && f + n <= sw1) continue;  // this chunk was in the seed window
                        if (__any_sync(FULL, bc + n > kBuf)) flush(tk, bc, W, lane, ct, pts, qx, qy, qz);
                        const float b2 = fminf(tk.tau(), cap);
                        if (3 * __popc(needm) < 2 * n)
                            scan_sparse(f, n, needm, qx, qy, qz, b2, bc, W, pts, (int32_t)sw0, (int32_t)sw1, lane);
                        else
                            scan_chunk(f, n, need, qx, qy, qz, b2, bc, W, pts, (int32_t)sw0, (int32_t)sw1, lane);
                    }
                }
#pragma unroll
                for (int o = 1; o >= 0; --o) {
                    const bool left = (o == 0) == leftFirst;
                    if ((left ? cntl : cntr) <= a.bucket || !(left ? bl : br)) continue;
                    if (sp >= kStackDepth) {
                        if (lane == 0) set_err(&st->err, ERRBIT_STACK);
                        continue;
                    }
                    if (lane == 0) W.stack[sp] = left ? refl : refr;
                    ++sp;
                }
                __syncwarp();
            }
        }
        flush(tk, bc, W, lane, ct, pts, qx, qy, qz);
        if (attempt == 0) {
            // a lane the cell scan could not serve (its cap is +inf or not a
            // number) was offered nothing: search it again as a miss
            const bool unserved = scanned && !(cap >= 0.0f && cap < INFINITY);
            const bool miss = act && (unserved || !(tk.tau() <= cap));
            ct.lmiss += miss;
            act = miss;
            if (!__any_sync(FULL, act)) break;
        }
    }
    {
        const unsigned cand = __reduce_add_sync(FULL, (unsigned)ct.cand);
        const unsigned ins = __reduce_add_sync(FULL, (unsigned)ct.ins);
        const unsigned lmiss = __reduce_add_sync(FULL, (unsigned)ct.lmiss);
        if (lane == 0) {
            if (ct.cells) atomicAdd(&st->counters[CNT_CELL_WARPS], (unsigned long long)ct.cells);
            if (ct.cell_fallback) atomicAdd(&st->counters[CNT_CELL_FALLBACK], (unsigned long long)ct.cell_fallback);
            if (ct.cell_lookups) atomicAdd(&st->counters[CNT_CELL_LOOKUPS], (unsigned long long)ct.cell_lookups);
            if (ct.cell_points) atomicAdd(&st->counters[CNT_CELL_POINTS], (unsigned long long)ct.cell_points);
            atomicAdd(&st->counters[CNT_NODES], (unsigned long long)steps);
            atomicAdd(&st->counters[CNT_BUCKETS], (unsigned long long)ct.buckets);
            atomicAdd(&st->counters[CNT_MERGE], (unsigned long long)ct.merge);
            atomicAdd(&st->counters[CNT_CANDIDATES], (unsigned long long)cand);
            atomicAdd(&st->counters[CNT_INSERTS], (unsigned long long)ins);
            if (lmiss) atomicAdd(&st->counters[CNT_LEARNED_MISS], (unsigned long long)lmiss);
        }
    }
    if (!active) return;

    // fewer than k points in the tree: repeat entry 0 (src/Octree.hpp:181-191)
    int32_t nbr[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (j > 0 && tk.key[j] == kEmptyKey) tk.key[j] = tk.key[0];
        nbr[j] = key_idx(tk.key[j]);
    }
    if (a.out_idx) {
        int32_t* o = a.out_idx + qo * a.k;
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (j < a.k) o[j] = nbr[j];
    }
    if (a.out_d2) {
        float* o = a.out_d2 + qo * a.k;
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (j < a.k) o[j] = key_d(tk.key[j]);
    }
    if (NORMALS) {
#pragma unroll
        for (int j = 0; j < K; ++j) W.buf[j][lane] = nbr[j];  // this lane's column only
        estimate_normal(&W.buf[0][lane], a.k, pts, qx, qy, qz, a, a.out_normals + 3 * qo, st);
    }
}

template <int K, bool EXACT, bool EXT, bool NORMALS, bool CELLS>
__global__ void __launch_bounds__(KnnCfg<K>::threads, KnnCfg<K>::min_blocks)
    k_knn(const float4* __restrict__ pts, const SNode* __restrict__ snodes,
                                                     const uint64_t* __restrict__ codes, QArgs a, DevState* st) {
    extern __shared__ __align__(16) unsigned char knn_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    using WS = WarpSmem<KnnCfg<K>::buf>;
    WS& W = reinterpret_cast<WS*>(knn_smem)[warp];
    const int64_t q0 = ((int64_t)blockIdx.x * KnnCfg<K>::warps + warp) * 32;
    knn_warp<K, EXACT, EXT, NORMALS, CELLS>(pts, snodes, codes, a, st, q0, W, lane);
}

// Persistent kernel over many clouds that share k: each warp takes the next
// 32-query item from a global counter until all are taken. Items are laid out
// cloud by cloud in the order of `clouds` (largest first), so the large clouds
// start first and the small ones fill the tail. Each cloud's size is read on
// the device from its own build state.
// Block shape of the persistent launch: W warps per block, with the
// resident-block target scaled so that ptxas gets the same register budget
// per thread as the per-k default shape (KnnCfg).
template <int K, int W>
struct BatchCfg {
    static constexpr int threads = 32 * W;
    static constexpr int min_blocks =
        (KnnCfg<K>::min_blocks * KnnCfg<K>::warps) / W > 0 ? (KnnCfg<K>::min_blocks * KnnCfg<K>::warps) / W : 1;
};

template <int K, bool EXACT, int NW>
__global__ void __launch_bounds__(BatchCfg<K, NW>::threads, BatchCfg<K, NW>::min_blocks)
    k_knn_batch(const BatchCloud* __restrict__ clouds, int n_clouds,
                                                           int64_t n_items, unsigned long long* counter, QArgs a) {
    extern __shared__ __align__(16) unsigned char knn_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    using WS = WarpSmem<KnnCfg<K>::buf>;
    WS& W = reinterpret_cast<WS*>(knn_smem)[warp];
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(counter, 1ull);
        item = __shfl_sync(FULL, item, 0);
        if (item >= (unsigned long long)n_items) break;
        int lo = 0, hi = n_clouds - 1;  // last cloud whose first item is <= item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if ((unsigned long long)__ldg(&clouds[mid].item0) <= item) lo = mid;
            else hi = mid - 1;
        }
        const BatchCloud d = clouds[lo];
        QArgs ca = a;
        ca.out_normals = d.out_normals;
        ca.start = 0;
        ca.device_count = 1;
        knn_warp<K, EXACT, false, true, false>(d.pts, d.snodes, nullptr, ca, d.st, ((int64_t)item - d.item0) * 32,
                                               W, lane);
        __syncwarp();
    }
}

template <int K, bool EXACT, bool EXT, bool NORMALS, bool CELLS = false>
cudaError_t launch_one(const BuildBufs& b, const QArgs& a, unsigned blocks, cudaStream_t s) {
    constexpr int smem = (int)sizeof(WarpSmem<KnnCfg<K>::buf>) * KnnCfg<K>::warps;
    cudaError_t e = cudaFuncSetAttribute(k_knn<K, EXACT, EXT, NORMALS, CELLS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_knn<K, EXACT, EXT, NORMALS, CELLS><<<blocks, KnnCfg<K>::threads, smem, s>>>(b.pts4, b.snodes, b.codes, a,
                                                                                   b.st);
    return cudaGetLastError();
}

template <int K, bool EXACT>
cudaError_t launch_k(const BuildBufs& b, const QArgs& a, bool ext, bool normals, cudaStream_t s) {
    const int64_t warps = (a.count + 31) / 32;
    const unsigned blocks = (unsigned)((warps + KnnCfg<K>::warps - 1) / KnnCfg<K>::warps);
    if (ext) return launch_one<K, EXACT, true, false>(b, a, blocks, s);
    if (a.cell_lut) {
        if (normals) return launch_one<K, EXACT, false, true, true>(b, a, blocks, s);
        return launch_one<K, EXACT, false, false, true>(b, a, blocks, s);
    }
    if (normals) return launch_one<K, EXACT, false, true>(b, a, blocks, s);
    return launch_one<K, EXACT, false, false>(b, a, blocks, s);
}

template <int K, bool EXACT, int NW>
cudaError_t launch_batch_w(const BatchCloud* clouds, int n_clouds, int64_t n_items, unsigned long long* counter,
                           const QArgs& a, cudaStream_t s, int num_sms, int blocks_per_sm) {
    constexpr int threads = BatchCfg<K, NW>::threads;
    constexpr int smem = (int)sizeof(WarpSmem<KnnCfg<K>::buf>) * NW;
    cudaError_t e =
        cudaFuncSetAttribute(k_knn_batch<K, EXACT, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_knn_batch<K, EXACT, NW>, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
    const int64_t want = (n_items + NW - 1) / NW;
    const int64_t resident = (int64_t)per_sm * num_sms;
    const unsigned blocks = (unsigned)(want < resident ? want : resident);
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    k_knn_batch<K, EXACT, NW><<<blocks, threads, smem, s>>>(clouds, n_clouds, n_items, counter, a);
    return cudaGetLastError();
}

// The per-k default block shape, or the other one of 2 and 4 warps.
template <int K, bool EXACT>
cudaError_t launch_batch(const BatchCloud* clouds, int n_clouds, int64_t n_items, unsigned long long* counter,
                         const QArgs& a, cudaStream_t s, int num_sms, int blocks_per_sm, int warps) {
    constexpr int def = KnnCfg<K>::warps;
    constexpr int alt = def == 4 ? 2 : 4;
    if (warps == alt) return launch_batch_w<K, EXACT, alt>(clouds, n_clouds, n_items, counter, a, s, num_sms,
                                                           blocks_per_sm);
    return launch_batch_w<K, EXACT, def>(clouds, n_clouds, n_items, counter, a, s, num_sms, blocks_per_sm);
}

// lut[j] = lower bound of j << sh in the u sorted unique codes, for j in
// [0, n_ent]; the code count u is read on the device from the build state.
__global__ void __launch_bounds__(256) k_cell_lut(const uint64_t* __restrict__ codes, const DevState* st, int sh,
                                                  int64_t n_ent, uint32_t* __restrict__ lut) {
    const uint32_t u = (uint32_t)st->u;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= n_ent;
         j += (int64_t)gridDim.x * blockDim.x) {
        lut[j] = j == n_ent ? u : lower_bound_codes(codes, 0u, u, (uint64_t)j << sh);
    }
}

}  // namespace

cudaError_t enqueue_cell_lut(const BuildBufs& b, int code_bits, int level, uint32_t* lut, cudaStream_t s,
                             int num_sms) {
    const int bpa = code_bits / 3;
    if (level < 1 || level > bpa || level > 10) return cudaErrorInvalidValue;
    const int64_t n_ent = (int64_t)1 << (3 * level);
    const int64_t want = (n_ent + 256) / 256;
    const unsigned blocks = (unsigned)(want < (int64_t)num_sms * 16 ? want : (int64_t)num_sms * 16);
    k_cell_lut<<<blocks, 256, 0, s>>>(b.codes, b.st, 3 * (bpa - level), n_ent, lut);
    return cudaGetLastError();
}

__global__ void k_batch_collect(const DevState* __restrict__ st, int n, unsigned long long* __restrict__ u_out,
                                uint32_t* __restrict__ err_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u_out[i] = st[i].u;
    err_out[i] = st[i].err;
}

cudaError_t enqueue_batch_collect(const DevState* st, int n, unsigned long long* u_out, uint32_t* err_out,
                                  cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_batch_collect<<<(n + 127) / 128, 128, 0, s>>>(st, n, u_out, err_out);
    return cudaGetLastError();
}

cudaError_t enqueue_query_batch(const BatchCloud* clouds, int n_clouds, int64_t n_items, unsigned long long* counter,
                                const QueryParams& q, cudaStream_t s, int num_sms) {
    if (n_clouds <= 0 || n_items <= 0) return cudaSuccess;
    if (q.k < 1 || q.k > 32) return cudaErrorInvalidValue;
    QArgs a{};
    a.k = q.k;
    a.vx = q.vx;
    a.vy = q.vy;
    a.vz = q.vz;
    a.gap = q.eigengap_fp64;
    a.code_bits = q.code_bits;
    a.bucket = q.bucket;
    a.seed_halo = q.seed_halo < 0 ? 0 : (q.seed_halo > kMaxHalo ? kMaxHalo : q.seed_halo);
    a.device_count = 1;
    const int bps = q.batch_blocks_per_sm, wpb = q.batch_warps_per_block;
    switch (q.k) {
        case 8: return launch_batch<8, true>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
        case 10: return launch_batch<10, true>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
        case 16: return launch_batch<16, true>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
        case 32: return launch_batch<32, true>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
        default: break;
    }
    if (q.k <= 4) return launch_batch<4, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
    if (q.k <= 8) return launch_batch<8, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
    if (q.k <= 12) return launch_batch<12, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
    if (q.k <= 16) return launch_batch<16, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
    if (q.k <= 24) return launch_batch<24, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
    return launch_batch<32, false>(clouds, n_clouds, n_items, counter, a, s, num_sms, bps, wpb);
}

cudaError_t enqueue_query(const BuildBufs& b, const QueryParams& q, cudaStream_t s, int /*num_sms*/) {
    if (q.count <= 0) return cudaSuccess;
    if (q.k < 1 || q.k > 32) return cudaErrorInvalidValue;
    if (q.compat) return enqueue_query_compat(b, q, s);
    QArgs a;
    a.k = q.k;
    a.start = q.start;
    a.count = q.count;
    a.u = q.u;
    a.ext = q.ext_queries;
    a.out_idx = q.out_idx;
    a.out_d2 = q.out_d2;
    a.out_normals = q.out_normals;
    a.vx = q.vx;
    a.vy = q.vy;
    a.vz = q.vz;
    a.gap = q.eigengap_fp64;
    a.code_bits = q.code_bits;
    a.bucket = q.bucket;
    a.seed_halo = q.seed_halo;
    a.learned_r2 = q.learned_r2;
    a.learned_skip_seed = q.learned_skip_seed;
    a.device_count = q.device_count;
    a.step_limit = q.step_limit;
    a.cell_lut = q.learned_r2 ? q.cell_lut : nullptr;
    a.lut_shift = q.lut_shift;
    a.cell_pmax = q.cell_pmax;
    a.cell_span = q.cell_span < 2 ? 2 : (q.cell_span > 4 ? 4 : q.cell_span);
    if (a.seed_halo > kMaxHalo) a.seed_halo = kMaxHalo;
    if (a.seed_halo < 0) a.seed_halo = 0;
    const bool ext = q.ext_queries != nullptr;
    const bool nrm = q.out_normals != nullptr && !ext;
    switch (q.k) {
        case 8: return launch_k<8, true>(b, a, ext, nrm, s);
        case 10: return launch_k<10, true>(b, a, ext, nrm, s);
        case 16: return launch_k<16, true>(b, a, ext, nrm, s);
        case 32: return launch_k<32, true>(b, a, ext, nrm, s);
        default: break;
    }
    if (q.k <= 4) return launch_k<4, false>(b, a, ext, nrm, s);
    if (q.k <= 8) return launch_k<8, false>(b, a, ext, nrm, s);
    if (q.k <= 12) return launch_k<12, false>(b, a, ext, nrm, s);
    if (q.k <= 16) return launch_k<16, false>(b, a, ext, nrm, s);
    if (q.k <= 24) return launch_k<24, false>(b, a, ext, nrm, s);
    return launch_k<32, false>(b, a, ext, nrm, s);
}

}  // namespace shapex
