// CPU oracle for the normal-estimation path of Wehrdo/ShapeExtraction.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: the parity tests, the
// smoke check and the CPU-baseline leg of the benchmark call it. The product
// (libshapex.so) never links, loads or calls it.
//
// Every stage restates the reference's algorithm on the host, citing the
// reference file:line it follows (paths are relative to the reference's
// project root):
//   bbox            src/RadixTree.cu:218-241
//   encode          src/MortonUtils.cu:7-19 via makeCodes src/RadixTree.cu:21-39
//   sort + dedup    src/RadixTree.cu:258-337
//   Karras tree     src/RadixTree.cu:42-69, 99-194
//   octree          src/Octree.cu:26-50, 65-161, 213-304
//   decode          src/MortonUtils.cu:21-29, src/Octree.cu:14-24
//   compat kNN      src/Octree.hpp:136-193, src/Octree.cu:326-352,
//                   src/dequeue.hpp:55-289, src/dequeue.cu:4-15
//   covariance      src/NormalEstimation.hpp:96-156
//   orientation     src/NormalEstimation.hpp:158-192
// plus an exact kNN (kd-tree, ties by index) and an FP64 PCA (cyclic Jacobi,
// Golub & Van Loan, Matrix Computations, 4th ed., Alg. 8.5.2/8.5.3).
//
// Float semantics follow what nvcc emits for the reference by default:
// IEEE division, and FMA contraction in codeToPoint. The exact-kNN distance is
// the project's canonical fmaf chain, shared bit for bit with the CUDA kernels.
//
// Build: g++ -O2 -std=c++17 -fopenmp -ffp-contract=off -shared -fPIC.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#include <omp.h>
#include <parallel/algorithm>

namespace {

// ---------------------------------------------------------------------------
// Morton interleave. The reference calls libmorton's morton3D_64_encode/decode
// (src/MortonUtils.cu:3,18,24; submodule Wehrdo/libmorton, not vendored). The
// standard libmorton convention is restated: bit b of x goes to bit 3b, of y to
// 3b+1, of z to 3b+2.
// ---------------------------------------------------------------------------
inline uint64_t split3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
inline uint32_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return (uint32_t)v;
}
inline uint64_t interleave(uint32_t x, uint32_t y, uint32_t z) {
    return split3(x) | (split3(y) << 1) | (split3(z) << 2);
}

// float -> uint32 conversion with the device's cvt.rzi.u32.f32 semantics
// (NaN -> 0, saturating). Inputs on the path lie in [0, bitscale] except NaN
// from a zero range.
inline uint32_t f2u_rz(float f) {
    if (std::isnan(f) || f <= 0.0f) return 0u;
    if (f >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)f;
}

inline uint32_t bitscale_of(int code_bits) {
    return 0xFFFFFFFFu >> (32 - code_bits / 3);
}

// pointToCode, src/MortonUtils.cu:7-19.
inline uint64_t point_to_code(float x, float y, float z, float mn, float range, int code_bits) {
    const uint32_t bs = bitscale_of(code_bits);
    const float fbs = (float)bs;
    const uint32_t xc = f2u_rz(fbs * ((x - mn) / range));
    const uint32_t yc = f2u_rz(fbs * ((y - mn) / range));
    const uint32_t zc = f2u_rz(fbs * ((z - mn) / range));
    const uint32_t mask = bs;
    return interleave(xc & mask, yc & mask, zc & mask);
}

// codeToPoint, src/MortonUtils.cu:21-29; nvcc contracts `q * range + min` to fmaf.
inline void code_to_point(uint64_t code, float mn, float range, int code_bits, float* out) {
    const float fbs = (float)bitscale_of(code_bits);
    const uint32_t rx = compact3(code), ry = compact3(code >> 1), rz = compact3(code >> 2);
    out[0] = std::fmaf((float)rx / fbs, range, mn);
    out[1] = std::fmaf((float)ry / fbs, range, mn);
    out[2] = std::fmaf((float)rz / fbs, range, mn);
}

// __clzll with clzll(0) == 64.
inline int clz64(uint64_t v) { return v ? __builtin_clzll(v) : 64; }

// delta, src/RadixTree.cu:62-69, generalised to CODE_LEN bits packed right.
inline int delta(uint64_t a, uint64_t b, int code_bits) { return clz64(a ^ b) - (64 - code_bits); }

// Right shift with PTX shr.b64 clamping (amounts >= 64, or negative, give 0).
inline uint64_t shr_clamp(uint64_t v, int s) { return (s < 0 || s >= 64) ? 0ull : (v >> s); }
inline uint64_t shl_clamp(uint64_t v, int s) { return (s < 0 || s >= 64) ? 0ull : (v << s); }
// int shift `1 << s` as PTX shl.b32 (amount treated unsigned, clamped to 32).
inline int one_shl(int s) { return (s < 0 || s >= 32) ? 0 : (1 << s); }

struct OTNode {  // layout of OT::OTNode, src/Octree.hpp:19-36 (56 bytes)
    int32_t children[8];
    float corner[3];
    float cell_size;
    int32_t child_node_mask;
    int32_t child_leaf_mask;
};
static_assert(sizeof(OTNode) == 56, "OTNode layout");

// Canonical exact-kNN distance, shared bit for bit with the CUDA kernels.
inline float dist2(const float* q, const float* p) {
    const float dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
    return std::fmaf(dx, dx, std::fmaf(dy, dy, dz * dz));
}
// Conservative squared distance from q to an axis-aligned box, same chain.
inline float box_dist2(const float* q, const float* lo, const float* hi) {
    float g[3];
    for (int a = 0; a < 3; ++a) {
        if (q[a] < lo[a]) g[a] = lo[a] - q[a];
        else if (q[a] > hi[a]) g[a] = q[a] - hi[a];
        else g[a] = 0.0f;
    }
    return std::fmaf(g[0], g[0], std::fmaf(g[1], g[1], g[2] * g[2]));
}

// ---------------------------------------------------------------------------
// Bounded min-max heap restating PriorityQueue<T, MAX_Q>,
// src/dequeue.hpp:12-45 (interface) and :55-289 (algorithm), int_log2
// src/dequeue.cu:4-15. The steps are kept identical because which element
// leaves a full heap, and the order of equal priorities, decide the
// reference's kNN sets.
// ---------------------------------------------------------------------------
inline int ilog2(int x) { int r = 0; while (x >>= 1) ++r; return r; }

template <typename T>
struct MinMaxHeap {
    struct Item { T data; float pri; };
    std::vector<Item> h;
    int cap;
    int size = 0;
    explicit MinMaxHeap(int capacity) : h(capacity), cap(capacity) {}

    static int par(int i) { return (i - 1) / 2; }
    static int lc(int i) { return 2 * i + 1; }
    static int rc(int i) { return 2 * i + 2; }
    void swp(int a, int b) { std::swap(h[a], h[b]); }

    int largest() const {
        if (size >= 2) {
            if (size == 2) return 1;
            return (h[1].pri > h[2].pri) ? 1 : 2;
        }
        return 0;
    }
    void up_min(int i) {
        while (i >= 3) {
            int g = par(par(i));
            if (h[i].pri < h[g].pri) { swp(i, g); i = g; } else break;
        }
    }
    void up_max(int i) {
        while (i >= 3) {
            int g = par(par(i));
            if (h[i].pri > h[g].pri) { swp(i, g); i = g; } else break;
        }
    }
    void bubble_up(int i) {
        if (ilog2(i + 1) % 2 == 0) {
            if (par(i) >= 0 && h[i].pri > h[par(i)].pri) { swp(i, par(i)); up_max(par(i)); }
            else up_min(i);
        } else {
            if (par(i) >= 0 && h[i].pri < h[par(i)].pri) { swp(i, par(i)); up_min(par(i)); }
            else up_max(i);
        }
    }
    void down_min(int i) {
        while (lc(i) < size) {
            const int desc[5] = {rc(i), lc(lc(i)), rc(lc(i)), lc(rc(i)), rc(rc(i))};
            int m = lc(i);
            for (int d : desc) if (d < size && h[d].pri < h[m].pri) m = d;
            if (m > rc(i)) {
                if (h[m].pri < h[i].pri) {
                    swp(i, m);
                    if (h[m].pri > h[par(m)].pri) swp(par(m), m);
                    i = m;
                } else break;
            } else {
                if (h[m].pri < h[i].pri) { swp(i, m); i = m; }
                break;
            }
        }
    }
    void down_max(int i) {
        while (lc(i) < size) {
            const int desc[5] = {rc(i), lc(lc(i)), rc(lc(i)), lc(rc(i)), rc(rc(i))};
            int m = lc(i);
            for (int d : desc) if (d < size && h[d].pri > h[m].pri) m = d;
            if (m > rc(i)) {
                if (h[m].pri > h[i].pri) {
                    swp(i, m);
                    if (h[m].pri < h[par(m)].pri) swp(par(m), m);
                    i = m;
                } else break;
            } else {
                if (h[m].pri > h[i].pri) { swp(i, m); i = m; }
                break;
            }
        }
    }
    void percolate(int i) {
        if (ilog2(i + 1) % 2 == 0) down_min(i); else down_max(i);
    }
    Item remove_min() {
        Item r = h[0];
        size--;
        h[0] = h[size];
        percolate(0);
        return r;
    }
    Item remove_max() {
        int l = largest();
        Item r = h[l];
        size--;
        h[l] = h[size];
        percolate(l);
        return r;
    }
    void insert(T d, float w) {
        if (size == cap) {
            if (h[largest()].pri >= w) remove_max();
            else return;
        }
        size += 1;
        h[size - 1] = Item{d, w};
        bubble_up(size - 1);
    }
};

// nodeBoxDistance, src/Octree.cu:326-352 (face-plane distance, not Euclidean).
inline float node_box_distance(const float* q, const OTNode& n) {
    const float x1 = n.corner[0], x2 = n.corner[0] + n.cell_size;
    const float y1 = n.corner[1], y2 = n.corner[1] + n.cell_size;
    const float z1 = n.corner[2], z2 = n.corner[2] + n.cell_size;
    const bool contained = q[0] > x1 && q[0] < x2 && q[1] > y1 && q[1] < y2 && q[2] > z1 && q[2] < z2;
    if (contained) return 0.0f;
    float m = std::fabs(q[0] - x1);
    m = std::fmin(m, std::fabs(q[0] - x2));
    m = std::fmin(m, std::fabs(q[1] - y1));
    m = std::fmin(m, std::fabs(q[1] - y2));
    m = std::fmin(m, std::fabs(q[2] - z1));
    m = std::fmin(m, std::fabs(q[2] - z2));
    return m;
}

// Point::distance2 as nvcc contracts it (src/PointCloud.hpp:30-35):
// variant 0: fma(z,z, fma(y,y, x*x)); variant 1: fma(z,z, fma(x,x, y*y)).
// Variant 1 reproduces the reference build's kNN sets on every golden vector
// (tests/golden); the others differ on equal-distance lattice neighbours.
inline float ref_dist2(const float* a, const float* b, int variant) {
    const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    if (variant == 0) return std::fmaf(dz, dz, std::fmaf(dy, dy, dx * dx));
    if (variant == 1) return std::fmaf(dz, dz, std::fmaf(dx, dx, dy * dy));
    return dx * dx + dy * dy + dz * dz;
}

// ---------------------------------------------------------------------------
// Exact kNN: kd-tree over the decoded points, pruned with the conservative box
// distance; result sets ordered by (distance, index).
// ---------------------------------------------------------------------------
struct KdNode {
    float lo[3], hi[3];
    int32_t begin, end;   // range in perm
    int32_t left, right;  // children, -1 for a leaf
};

struct KdTree {
    const float* pts;
    std::vector<int32_t> perm;
    std::vector<KdNode> nodes;
    static constexpr int LEAF = 12;

    // Nodes of the subtree over m points (median splits: floor(m/2) left).
    static int64_t count(int64_t m) { return m <= LEAF ? 1 : 1 + count(m / 2) + count(m - m / 2); }

    // Subtree over perm[b, e) at node `id`, in depth-first preorder (left
    // subtree at id + 1, right after it), so the layout is fixed by the sizes
    // alone and large subtrees can be built as parallel tasks.
    void build(int64_t b, int64_t e, int64_t id) {
        KdNode nd;
        for (int a = 0; a < 3; ++a) { nd.lo[a] = INFINITY; nd.hi[a] = -INFINITY; }
        for (int64_t i = b; i < e; ++i)
            for (int a = 0; a < 3; ++a) {
                nd.lo[a] = std::min(nd.lo[a], pts[3 * perm[i] + a]);
                nd.hi[a] = std::max(nd.hi[a], pts[3 * perm[i] + a]);
            }
        nd.begin = (int32_t)b; nd.end = (int32_t)e; nd.left = nd.right = -1;
        if (e - b > LEAF) {
            int ax = 0;
            float w = nd.hi[0] - nd.lo[0];
            for (int a = 1; a < 3; ++a) if (nd.hi[a] - nd.lo[a] > w) { w = nd.hi[a] - nd.lo[a]; ax = a; }
            const int64_t mid = b + (e - b) / 2;
            std::nth_element(perm.begin() + b, perm.begin() + mid, perm.begin() + e,
                             [&](int32_t i, int32_t j) { return pts[3 * i + ax] < pts[3 * j + ax]; });
            nd.left = (int32_t)(id + 1);
            nd.right = (int32_t)(id + 1 + count(mid - b));
            if (e - b > 200000) {
#pragma omp task
                build(b, mid, nd.left);
#pragma omp task
                build(mid, e, nd.right);
#pragma omp taskwait
            } else {
                build(b, mid, nd.left);
                build(mid, e, nd.right);
            }
        }
        nodes[id] = nd;
    }
    KdTree(const float* p, int64_t n) : pts(p), perm(n) {
        std::iota(perm.begin(), perm.end(), 0);
        if (n > 0) {
            nodes.resize(count(n));
#pragma omp parallel
#pragma omp single
            build(0, n, 0);
        }
    }
};

struct TopK {
    int k, cnt = 0;
    float* d;
    int32_t* id;
    // true when (a_d, a_i) < (b_d, b_i)
    static bool less(float ad, int32_t ai, float bd, int32_t bi) { return ad < bd || (ad == bd && ai < bi); }
    void push(float dd, int32_t ii) {
        if (cnt < k) {
            int j = cnt++;
            while (j > 0 && less(dd, ii, d[j - 1], id[j - 1])) { d[j] = d[j - 1]; id[j] = id[j - 1]; --j; }
            d[j] = dd; id[j] = ii;
        } else if (less(dd, ii, d[k - 1], id[k - 1])) {
            int j = k - 1;
            while (j > 0 && less(dd, ii, d[j - 1], id[j - 1])) { d[j] = d[j - 1]; id[j] = id[j - 1]; --j; }
            d[j] = dd; id[j] = ii;
        }
    }
    float bound() const { return cnt < k ? INFINITY : d[k - 1]; }
};

void kd_search(const KdTree& t, int node, const float* q, TopK& tk) {
    const KdNode& nd = t.nodes[node];
    if (nd.left < 0) {
        for (int i = nd.begin; i < nd.end; ++i) {
            int32_t pi = t.perm[i];
            tk.push(dist2(q, t.pts + 3 * pi), pi);
        }
        return;
    }
    const KdNode& L = t.nodes[nd.left];
    const KdNode& R = t.nodes[nd.right];
    float dl = box_dist2(q, L.lo, L.hi), dr = box_dist2(q, R.lo, R.hi);
    int first = nd.left, second = nd.right;
    float d1 = dl, d2 = dr;
    if (dr < dl) { std::swap(first, second); std::swap(d1, d2); }
    if (d1 <= tk.bound()) kd_search(t, first, q, tk);
    if (d2 <= tk.bound()) kd_search(t, second, q, tk);
}

// ---------------------------------------------------------------------------
// FP64 cyclic Jacobi for a symmetric 3x3 (Golub & Van Loan, Alg. 8.5.2
// sym.schur2 and 8.5.3 cyclic Jacobi). Returns ascending eigenvalues and the
// eigenvector columns in V (row-major V[r][c], column c = eigenvector c).
// ---------------------------------------------------------------------------
void jacobi3_f64(const double A_in[3][3], double w[3], double V[3][3]) {
    double A[3][3];
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) { A[r][c] = A_in[r][c]; V[r][c] = (r == c); }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        double fro = off * 2 + A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-36 * fro || off == 0.0) break;
        for (int p = 0; p < 2; ++p) for (int q = p + 1; q < 3; ++q) {
            if (A[p][q] == 0.0) continue;
            double tau = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
            double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
            double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
            // A <- J^T A J with J = rotation in (p, q)
            for (int k = 0; k < 3; ++k) {
                double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
            }
            for (int k = 0; k < 3; ++k) {
                double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
            for (int k = 0; k < 3; ++k) {
                double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
    double ev[3] = {A[0][0], A[1][1], A[2][2]};
    int ord[3] = {0, 1, 2};
    std::sort(ord, ord + 3, [&](int a, int b) { return ev[a] < ev[b]; });
    double Vs[3][3];
    for (int c = 0; c < 3; ++c) {
        w[c] = ev[ord[c]];
        for (int r = 0; r < 3; ++r) Vs[r][c] = V[r][ord[c]];
    }
    std::memcpy(V, Vs, sizeof(Vs));
}

}  // namespace

extern "C" {

int or_version() { return 1; }

// ---- bbox: RadixTree::encodePoints, src/RadixTree.cu:218-241 -------------
void or_bbox(const float* x, const float* y, const float* z, int64_t n, float* mn_out, float* mx_out) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const float* a[3] = {x, y, z};
    for (int ax = 0; ax < 3; ++ax) {
        float lo = INFINITY, hi = -INFINITY;
#pragma omp parallel for reduction(min : lo) reduction(max : hi)
        for (int64_t i = 0; i < n; ++i) { lo = std::min(lo, a[ax][i]); hi = std::max(hi, a[ax][i]); }
        mn[ax] = lo; mx[ax] = hi;
    }
    *mn_out = std::min(mn[0], std::min(mn[1], mn[2]));
    *mx_out = std::max(mx[0], std::max(mx[1], mx[2]));
}

// ---- encode: makeCodes src/RadixTree.cu:21-39 + pointToCode ---------------
void or_encode(const float* x, const float* y, const float* z, int64_t n, float mn, float range,
               int code_bits, uint64_t* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = point_to_code(x[i], y[i], z[i], mn, range, code_bits);
}

// ---- decode: decodePoints src/Octree.cu:14-24 + codeToPoint ---------------
void or_decode(const uint64_t* codes, int64_t u, float mn, float range, int code_bits, float* out_xyz) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < u; ++i) code_to_point(codes[i], mn, range, code_bits, out_xyz + 3 * i);
}

// ---- sort + dedup: src/RadixTree.cu:316-337 (SortKeys) and :258-303 ------
// Writes the ascending unique codes to out (capacity n); returns u.
int64_t or_sort_dedup(const uint64_t* codes, int64_t n, uint64_t* out) {
    if (n <= 0) return 0;
    std::vector<uint64_t> s(codes, codes + n);
    __gnu_parallel::sort(s.begin(), s.end());
    int64_t u = 0;
    for (int64_t i = 0; i < n; ++i)
        if (i == 0 || s[i] != s[i - 1]) out[u++] = s[i];
    return u;
}

// ---- Karras radix tree: constructTree, src/RadixTree.cu:99-194 ------------
// u leaves, u-1 internal nodes. root_compat=1 keeps the reference's root range
// l = N-1 (src/RadixTree.cu:128-130 with N = u-1, launched at :353-362);
// root_compat=0 gives the root its full range [0, u-1].
// parent[] must be zero-initialised by the caller (the reference never writes
// parent[0] nor the parent of a node orphaned by the compat root).
void or_karras(const uint64_t* codes, int64_t u, int code_bits, int root_compat, int32_t* leftChild,
               int32_t* parent, uint8_t* prefixN, uint8_t* hasLeafLeft, uint8_t* hasLeafRight) {
    const int64_t N = u - 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        const uint64_t ci = codes[i];
        int d;
        if (i == 0) d = 1;
        else {
            int dd = delta(ci, codes[i + 1], code_bits) - delta(ci, codes[i - 1], code_bits);
            d = (dd > 0) - (dd < 0);
        }
        int64_t l = 0;
        if (i == 0) {
            l = root_compat ? N - 1 : N;
        } else {
            const int dmin = delta(ci, codes[i - d], code_bits);
            int64_t lmax = 2;
            while (i + lmax * d >= 0 && i + lmax * d <= N && delta(ci, codes[i + lmax * d], code_bits) > dmin)
                lmax *= 2;
            const int64_t lcut = (d == -1) ? i : N - i;
            for (int64_t t = lmax / 2, div = 2; t >= 1; div *= 2, t = lmax / div)
                if (l + t <= lcut && delta(ci, codes[i + (l + t) * d], code_bits) > dmin) l += t;
        }
        const int64_t j = i + l * d;
        const int dnode = delta(codes[i], codes[j], code_bits);
        prefixN[i] = (uint8_t)dnode;
        int64_t s = 0;
        if (l >= 1) {
            int nlow = 63 - clz64((uint64_t)l);
            int lc = nlow + ((uint64_t)l > (uint64_t)one_shl(nlow));
            const int64_t maxdiv = one_shl(lc);
            const int64_t scut = (d == -1) ? i - 1 : N - i - 1;
            for (int64_t div = 2, t = (l + 1) / 2; div <= maxdiv; div <<= 1, t = (l + div - 1) / div)
                if (s + t <= scut && delta(ci, codes[i + (s + t) * d], code_bits) > dnode) s += t;
        }
        const int64_t gamma = i + s * d + std::min(d, 0);
        leftChild[i] = (int32_t)gamma;
        const bool hl = std::min(i, j) == gamma;
        const bool hr = std::max(i, j) == gamma + 1;
        hasLeafLeft[i] = hl;
        hasLeafRight[i] = hr;
        // the compat root's parent claims are applied after all other nodes,
        // so that in a tree the compat root breaks they win deterministically
        if (i == 0 && root_compat) continue;
        if (!hl) parent[gamma] = (int32_t)i;
        if (!hr) parent[gamma + 1] = (int32_t)i;
    }
    if (N > 0 && root_compat) {
        if (!hasLeafLeft[0]) parent[leftChild[0]] = 0;
        if (!hasLeafRight[0]) parent[leftChild[0] + 1] = 0;
    }
}

// ---- octree: Octree::Octree(const RadixTree&), src/Octree.cu:213-304 -------
// Pass 1 (calcEdgeCounts :38-50 + InclusiveSum :225-247): returns the node
// count and fills offsets[0..N] (exclusive prefix of the edge counts).
int64_t or_octree_count(const uint8_t* prefixN, const int32_t* parent, int64_t n_radix, int32_t* counts,
                        int32_t* offsets) {
    const int64_t N = n_radix;
    if (N <= 0) return 0;
    counts[0] = 1;
    for (int64_t i = 1; i < N; ++i) counts[i] = prefixN[i] / 3 - prefixN[parent[i]] / 3;
    offsets[0] = 0;
    for (int64_t i = 0; i < N; ++i) offsets[i + 1] = offsets[i] + counts[i];
    return offsets[N];
}

// Pass 2: root init (:257-261), makeNodes (:114-161), linkLeafNodes (:65-112).
// nodes must hold n_oct entries and is zero-filled here (:253). makeNodes runs
// to completion before linkLeafNodes, as the reference's two launches do.
// Writes that would fall outside the arrays (possible only in trees broken by
// the compat root) are skipped and counted; the return value is that count.
int64_t or_octree_build(const uint64_t* codes, const uint8_t* prefixN, const int32_t* parent,
                        const int32_t* leftChild, const uint8_t* hasLeafLeft, const uint8_t* hasLeafRight,
                        int64_t n_radix, const int32_t* counts, const int32_t* offsets, int64_t n_oct, float mn,
                        float mx, int code_bits, void* nodes_out) {
    OTNode* nodes = (OTNode*)nodes_out;
    std::memset(nodes, 0, sizeof(OTNode) * n_oct);
    const int64_t N = n_radix;
    if (N <= 0 || n_oct <= 0) return 0;
    const int CL = code_bits;
    const float range = mx - mn;
    const int root_level = prefixN[0] / 3;
    const uint64_t root_prefix = shr_clamp(codes[0], CL - 3 * root_level);
    code_to_point(shl_clamp(root_prefix, CL - 3 * root_level), mn, range, CL, nodes[0].corner);
    nodes[0].cell_size = range;
    int64_t skipped = 0;
    auto ok = [&](int64_t node) { return node >= 0 && node < n_oct; };
    auto set_child = [&](int64_t node, int32_t child, int slot) {
        if (!ok(node)) { __atomic_fetch_add(&skipped, 1, __ATOMIC_RELAXED); return; }
        nodes[node].children[slot] = child;
        __atomic_fetch_or(&nodes[node].child_node_mask, 1 << slot, __ATOMIC_RELAXED);
    };
    auto set_leaf = [&](int64_t node, int32_t leaf, int slot) {
        if (!ok(node)) { __atomic_fetch_add(&skipped, 1, __ATOMIC_RELAXED); return; }
        nodes[node].children[slot] = leaf;
        __atomic_fetch_or(&nodes[node].child_leaf_mask, 1 << slot, __ATOMIC_RELAXED);
    };
    auto cell = [&](int level) { return range / (float)one_shl(level - root_level); };
    auto walk_up = [&](int64_t r) {  // nearest ancestor (or self) that contributes a node
        for (int it = 0; it < 128 && counts[r] == 0; ++it) r = parent[r];
        return r;
    };
#pragma omp parallel for schedule(static)
    for (int64_t i = 1; i < N; ++i) {
        int64_t oct = offsets[i];
        const int nn = counts[i];
        for (int j = 0; j < nn - 1; ++j) {
            const int level = prefixN[i] / 3 - j;
            const uint64_t pre = shr_clamp(codes[i], CL - 3 * level);
            const int slot = (int)(pre & 7);
            const int64_t par = oct + 1;
            set_child(par, (int32_t)oct, slot);
            if (ok(oct)) {
                code_to_point(shl_clamp(pre, CL - 3 * level), mn, range, CL, nodes[oct].corner);
                nodes[oct].cell_size = cell(level);
            }
            oct = par;
        }
        if (nn > 0) {
            const int64_t rp = walk_up(parent[i]);
            const int64_t op = offsets[rp];
            const int top = prefixN[i] / 3 - nn + 1;
            const uint64_t pre = shr_clamp(codes[i], CL - 3 * top);
            set_child(op, (int32_t)oct, (int)(pre & 7));
            if (ok(oct)) {
                code_to_point(shl_clamp(pre, CL - 3 * top), mn, range, CL, nodes[oct].corner);
                nodes[oct].cell_size = cell(top);
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        for (int side = 0; side < 2; ++side) {
            if (!(side == 0 ? hasLeafLeft[i] : hasLeafRight[i])) continue;
            const int32_t leaf = leftChild[i] + side;
            const int lvl = prefixN[i] / 3 + 1;
            const uint64_t pre = shr_clamp(codes[leaf], CL - 3 * lvl);
            const int64_t rn = walk_up(i);
            set_leaf(offsets[rn], leaf, (int)(pre & 7));
        }
    }
    return skipped;
}

// ---- reference-compat kNN: knnSearchKernel<k>, src/Octree.hpp:136-193 -----
// Search heap of capacity 32 (SEARCH_Q_SIZE, src/Octree.hpp:17), result heap
// of capacity k, face-plane node distance; ties and drops as the reference's
// bounded min-max heap. dist_variant selects the FMA contraction of
// Point::distance2 (see ref_dist2). pops_out (optional) receives pop counts.
void or_knn_compat(const void* nodes_in, const float* pts, const float* queries, int64_t nq, int k,
                   int dist_variant, int32_t* out, int32_t* pops_out) {
    const OTNode* nodes = (const OTNode*)nodes_in;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t qi = 0; qi < nq; ++qi) {
        const float* q = queries + 3 * qi;
        MinMaxHeap<int32_t> sq(32);
        MinMaxHeap<int32_t> rq(k);
        sq.insert(0, 0.0f);
        int pops = 0;
        // `d` is never updated in the reference (src/Octree.hpp:152-155), so
        // the loop runs until the search heap is empty.
        while (sq.size) {
            auto top = sq.remove_min();
            ++pops;
            const OTNode& nd = nodes[top.data];
            if (nd.child_leaf_mask) {
                for (int c = 0; c < 8; ++c)
                    if (nd.child_leaf_mask & (1 << c)) {
                        const int32_t li = nd.children[c];
                        rq.insert(li, ref_dist2(q, pts + 3 * li, dist_variant));
                    }
            }
            for (int c = 0; c < 8; ++c)
                if (nd.child_node_mask & (1 << c)) {
                    const int32_t ci = nd.children[c];
                    sq.insert(ci, node_box_distance(q, nodes[ci]));
                }
        }
        int32_t* o = out + qi * (int64_t)k;
        for (int c = 0; c < k; ++c) {
            if (rq.size == 0) o[c] = o[0];
            else o[c] = rq.remove_min().data;
        }
        if (pops_out) pops_out[qi] = pops;
    }
}

// ---- exact kNN (kd-tree), ties by index ------------------------------------
// Output rows ascending by (distance, index). Rows with fewer than k points
// repeat entry 0, as the reference pads (src/Octree.hpp:181-191).
void or_knn_exact(const float* pts, int64_t u, const float* queries, int64_t nq, int k, int32_t* idx,
                  float* d2) {
    KdTree t(pts, u);
#pragma omp parallel
    {
        std::vector<float> dd(k);
        std::vector<int32_t> ii(k);
#pragma omp for schedule(dynamic, 256)
        for (int64_t qi = 0; qi < nq; ++qi) {
            TopK tk{k, 0, dd.data(), ii.data()};
            if (u > 0) kd_search(t, 0, queries + 3 * qi, tk);
            for (int c = 0; c < k; ++c) {
                const int src = c < tk.cnt ? c : 0;
                idx[qi * k + c] = tk.cnt ? ii[src] : 0;
                if (d2) d2[qi * k + c] = tk.cnt ? dd[src] : 0.0f;
            }
        }
    }
}

// Brute-force exact kNN for small clouds (cross-checks the kd-tree).
void or_knn_brute(const float* pts, int64_t u, const float* queries, int64_t nq, int k, int32_t* idx,
                  float* d2) {
#pragma omp parallel
    {
        std::vector<float> dd(k);
        std::vector<int32_t> ii(k);
#pragma omp for schedule(static)
        for (int64_t qi = 0; qi < nq; ++qi) {
            TopK tk{k, 0, dd.data(), ii.data()};
            for (int64_t p = 0; p < u; ++p) tk.push(dist2(queries + 3 * qi, pts + 3 * p), (int32_t)p);
            for (int c = 0; c < k; ++c) {
                const int src = c < tk.cnt ? c : 0;
                idx[qi * k + c] = tk.cnt ? ii[src] : 0;
                if (d2) d2[qi * k + c] = tk.cnt ? dd[src] : 0.0f;
            }
        }
    }
}

// ---- FP64 PCA normals -------------------------------------------------------
// Covariance of the k listed neighbours (centroid, then sum of outer products
// over k-1: src/NormalEstimation.hpp:96-120) in double, cyclic Jacobi in
// double, eigenvector of the smallest eigenvalue, flipped when
// (viewpoint - p) . n < 0 (src/NormalEstimation.hpp:177-189).
// normals_out: nq*3 doubles; evals_out (optional): nq*3 ascending eigenvalues.
void or_normals_f64(const float* pts, const int32_t* nn, int64_t nq, int k, const float* query_pts,
                    const float* viewpoint, double* normals_out, double* evals_out) {
#pragma omp parallel for schedule(static)
    for (int64_t qi = 0; qi < nq; ++qi) {
        const int32_t* row = nn + qi * k;
        double c[3] = {0, 0, 0};
        for (int j = 0; j < k; ++j)
            for (int a = 0; a < 3; ++a) c[a] += (double)pts[3 * row[j] + a];
        for (int a = 0; a < 3; ++a) c[a] /= k;
        double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int j = 0; j < k; ++j) {
            double p[3];
            for (int a = 0; a < 3; ++a) p[a] = (double)pts[3 * row[j] + a] - c[a];
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) A[r][s] += p[r] * p[s];
        }
        const double den = (k > 1) ? (double)(k - 1) : 1.0;
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) A[r][s] /= den;
        double w[3], V[3][3];
        jacobi3_f64(A, w, V);
        double n[3] = {V[0][0], V[1][0], V[2][0]};
        const float* qp = query_pts + 3 * qi;
        double dot = 0;
        for (int a = 0; a < 3; ++a) dot += ((double)viewpoint[a] - (double)qp[a]) * n[a];
        if (dot < 0) for (int a = 0; a < 3; ++a) n[a] = -n[a];
        for (int a = 0; a < 3; ++a) normals_out[qi * 3 + a] = n[a];
        if (evals_out) for (int a = 0; a < 3; ++a) evals_out[qi * 3 + a] = w[a];
    }
}

// ---- reference FP32 covariance: findCovariancesKernel<k>,
// src/NormalEstimation.hpp:96-156 (upper triangle a,d,e,b,f,c as the
// reference stores it; nvcc contracts the accumulation into fmaf).
void or_cov_ref_f32(const float* pts, const int32_t* nn, int64_t nq, int k, float* cov_upper_out) {
#pragma omp parallel for schedule(static)
    for (int64_t qi = 0; qi < nq; ++qi) {
        const int32_t* row = nn + qi * k;
        float c[3] = {0, 0, 0};
        for (int j = 0; j < k; ++j)
            for (int a = 0; a < 3; ++a) c[a] += pts[3 * row[j] + a];
        for (int a = 0; a < 3; ++a) c[a] /= (float)k;
        float cv[6] = {0, 0, 0, 0, 0, 0};
        for (int j = 0; j < k; ++j) {
            const float* p = pts + 3 * row[j];
            const float m0 = p[0] - c[0], m1 = p[1] - c[1], m2 = p[2] - c[2];
            cv[0] = std::fmaf(m0, m0, cv[0]);
            cv[1] = std::fmaf(m0, m1, cv[1]);
            cv[2] = std::fmaf(m0, m2, cv[2]);
            cv[3] = std::fmaf(m1, m1, cv[3]);
            cv[4] = std::fmaf(m1, m2, cv[4]);
            cv[5] = std::fmaf(m2, m2, cv[5]);
        }
        for (int a = 0; a < 6; ++a) cov_upper_out[qi * 6 + a] = cv[a] / (float)(k - 1);
    }
}

// ---- the reference pipeline end to end, on the host ------------------------
// RT::RadixTree -> OT::Octree -> estimateNormals<k> (src/main.cu:80-107):
// bit-exact build stages (compat root), the reference's approximate search,
// its FP32 covariance, then the 3x3 eigensolve (FP64 Jacobi on the FP32
// covariance, in place of the closed cusolverDnSsyevjBatched) and the
// orientation rule. This is the timed CPU baseline. normals_out holds n*3
// floats; returns u (normals are written for the u unique points).
int64_t or_pipeline_reference(const float* x, const float* y, const float* z, int64_t n, int k,
                              float* normals_out) {
    if (n <= 0) return 0;
    float mn, mx;
    or_bbox(x, y, z, n, &mn, &mx);
    std::vector<uint64_t> codes(n), uq(n);
    or_encode(x, y, z, n, mn, mx - mn, 63, codes.data());
    const int64_t u = or_sort_dedup(codes.data(), n, uq.data());
    if (u < 3) return u;
    const int64_t N = u - 1;
    std::vector<int32_t> lc(N), par(u, 0), counts(N), offsets(N + 1);
    std::vector<uint8_t> pn(N), hl(N), hr(N);
    or_karras(uq.data(), u, 63, 1, lc.data(), par.data(), pn.data(), hl.data(), hr.data());
    const int64_t m = or_octree_count(pn.data(), par.data(), N, counts.data(), offsets.data());
    std::vector<OTNode> nodes(std::max<int64_t>(m, 1));
    or_octree_build(uq.data(), pn.data(), par.data(), lc.data(), hl.data(), hr.data(), N, counts.data(),
                    offsets.data(), m, mn, mx, 63, nodes.data());
    std::vector<float> pts(3 * u);
    or_decode(uq.data(), u, mn, mx - mn, 63, pts.data());
    std::vector<int32_t> nn(u * (int64_t)k);
    or_knn_compat(nodes.data(), pts.data(), pts.data(), u, k, 1, nn.data(), nullptr);
    std::vector<float> cov(6 * u);
    or_cov_ref_f32(pts.data(), nn.data(), u, k, cov.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < u; ++i) {
        const float* c = cov.data() + 6 * i;
        const double A[3][3] = {{c[0], c[1], c[2]}, {c[1], c[3], c[4]}, {c[2], c[4], c[5]}};
        double w[3], V[3][3];
        jacobi3_f64(A, w, V);
        float nv[3] = {(float)V[0][0], (float)V[1][0], (float)V[2][0]};
        const float* p = pts.data() + 3 * i;
        const float dot = (0.0f - p[0]) * nv[0] + (0.0f - p[1]) * nv[1] + (0.0f - p[2]) * nv[2];
        if (dot < 0) for (int a = 0; a < 3; ++a) nv[a] = -nv[a];
        for (int a = 0; a < 3; ++a) normals_out[3 * i + a] = nv[a];
    }
    return u;
}

// ---- learned-radius MLP (no counterpart in the reference) --------------------
// 32 -> 64 -> 64 -> 1, ReLU, parameters flat as W1[32][64], b1[64],
// W2[64][64], b2[64], w3[64], b3. With round_bf16 = 1 the forward pass
// reproduces the GPU training kernels bit for bit: inputs, weights and hidden
// activations rounded to BF16 (round to nearest even), FP32 fmaf accumulation
// in the same order. Gradients of mean((yhat - y)^2) are accumulated in
// double, treating the BF16 roundings as identity (straight-through), as the
// GPU backward does. With round_bf16 = 0 everything is plain double math (for
// finite-difference checks of the backward formulas).
static float bf16_round(float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    if ((b & 0x7f800000u) == 0x7f800000u) return v;  // inf / nan
    b += 0x7fffu + ((b >> 16) & 1u);
    b &= 0xffff0000u;
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}

int or_mlp_grad(const float* params, const float* X, const float* y, int64_t n, int round_bf16, double tau,
                double* yhat_out, double* grads, double* loss_out) {
    constexpr int F = 32, H = 64;
    constexpr int W1 = 0, B1 = W1 + F * H, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H, NP = B3 + 1;
    std::vector<double> g(NP, 0.0);
    double loss = 0.0;
    auto rw = [&](int i) { return round_bf16 ? (double)bf16_round(params[i]) : (double)params[i]; };
    for (int64_t r = 0; r < n; ++r) {
        double x[F], h1[H], h2[H];
        for (int j = 0; j < F; ++j) x[j] = round_bf16 ? (double)bf16_round(X[r * F + j]) : (double)X[r * F + j];
        for (int i = 0; i < H; ++i) {
            if (round_bf16) {
                float a = params[B1 + i];
                for (int j = 0; j < F; ++j) a = std::fmaf((float)x[j], (float)rw(W1 + j * H + i), a);
                h1[i] = (double)bf16_round(std::fmax(a, 0.0f));
            } else {
                double a = params[B1 + i];
                for (int j = 0; j < F; ++j) a += x[j] * rw(W1 + j * H + i);
                h1[i] = a > 0 ? a : 0.0;
            }
        }
        double yh;
        if (round_bf16) {
            float yy = params[B3];
            for (int i = 0; i < H; ++i) {
                float a = params[B2 + i];
                for (int j = 0; j < H; ++j) a = std::fmaf((float)h1[j], (float)rw(W2 + j * H + i), a);
                h2[i] = (double)bf16_round(std::fmax(a, 0.0f));
                yy = std::fmaf((float)h2[i], (float)rw(W3 + i), yy);
            }
            yh = yy;
        } else {
            yh = params[B3];
            for (int i = 0; i < H; ++i) {
                double a = params[B2 + i];
                for (int j = 0; j < H; ++j) a += h1[j] * rw(W2 + j * H + i);
                h2[i] = a > 0 ? a : 0.0;
                yh += h2[i] * rw(W3 + i);
            }
        }
        if (yhat_out) yhat_out[r] = yh;
        const double e = yh - (double)y[r];
        double dy;
        if (tau > 0.0) {  // pinball loss of quantile tau
            loss += (e > 0 ? (1.0 - tau) * e : -tau * e) / (double)n;
            dy = (e > 0 ? 1.0 - tau : (e < 0 ? -tau : 0.0)) / (double)n;
        } else {          // mean squared error
            loss += e * e / (double)n;
            dy = 2.0 * e / (double)n;
        }
        g[B3] += dy;
        // round_bf16 == 2 restates the tensor-core training step (k_mlp_train_tc):
        // dh2 and dh1 enter the weight gradients, and dh2 the product that
        // gives dh1, rounded to BF16; the bias gradients take them unrounded.
        const bool tc = round_bf16 == 2;
        auto rd = [&](double v) { return tc ? (double)bf16_round((float)v) : v; };
        double dh2[H], dh1[H];
        for (int i = 0; i < H; ++i) {
            g[W3 + i] += dy * h2[i];
            dh2[i] = h2[i] > 0 ? dy * rw(W3 + i) : 0.0;
            g[B2 + i] += dh2[i];
        }
        for (int j = 0; j < H; ++j) {
            double a = 0.0;
            for (int i = 0; i < H; ++i) {
                g[W2 + j * H + i] += h1[j] * rd(dh2[i]);
                a += rw(W2 + j * H + i) * rd(dh2[i]);
            }
            dh1[j] = h1[j] > 0 ? a : 0.0;
            g[B1 + j] += dh1[j];
        }
        for (int f = 0; f < F; ++f)
            for (int i = 0; i < H; ++i) g[W1 + f * H + i] += x[f] * rd(dh1[i]);
    }
    if (grads) std::copy(g.begin(), g.end(), grads);
    if (loss_out) *loss_out = loss;
    return NP;
}

// Cross-checks of the octree, after checkTree src/Octree.cu:163-177:
// every leaf's code prefix matches its slot path, and every leaf index in
// [0, u) appears exactly once. Returns 0 on success, else a negative code;
// leaf_seen (u int32) receives per-leaf occurrence counts.
int or_octree_check(const void* nodes_in, int64_t n_oct, const uint64_t* codes, int64_t u, int code_bits,
                    int root_level, int32_t* leaf_seen) {
    const OTNode* nodes = (const OTNode*)nodes_in;
    std::fill(leaf_seen, leaf_seen + u, 0);
    if (n_oct <= 0) return 0;
    struct Fr { int32_t node; uint64_t prefix; int len; };
    std::vector<Fr> st;
    st.push_back({0, shr_clamp(codes[0], code_bits - 3 * root_level), 3 * root_level});
    int bad = 0;
    int64_t visits = 0;
    while (!st.empty()) {
        Fr f = st.back(); st.pop_back();
        if (++visits > 64 * (n_oct + 1)) return -3;
        const OTNode& nd = nodes[f.node];
        for (int c = 0; c < 8; ++c) {
            const uint64_t np = (f.prefix << 3) | (uint64_t)c;
            if (nd.child_node_mask & (1 << c)) {
                int32_t ch = nd.children[c];
                if (ch < 0 || ch >= n_oct) return -2;
                st.push_back({ch, np, f.len + 3});
            }
            if (nd.child_leaf_mask & (1 << c)) {
                int32_t li = nd.children[c];
                if (li < 0 || li >= u) return -2;
                leaf_seen[li]++;
                if (shr_clamp(codes[li], code_bits - (f.len + 3)) != np) bad++;
            }
        }
    }
    return bad ? -1 : 0;
}

}  // extern "C"
