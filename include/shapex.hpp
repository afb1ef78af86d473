// shapex.hpp -- header-only C++ facade over the C ABI (shapex.h) with the
// reference's class names, scopes and signatures (Wehrdo/ShapeExtraction,
// paths relative to its project root), so that a caller written against
//   #include "PointCloud.hpp" / "RadixTree.hpp" / "Octree.hpp" / "NormalEstimation.hpp"
// compiles against this one header and links against libshapex.so:
//
//   PointCloud<float> cloud = ...;                        // src/PointCloud.hpp:105-122
//   RT::RadixTree radix_tree(cloud);                      // src/RadixTree.hpp:36-60
//   OT::Octree octree(radix_tree);                        // src/Octree.hpp:91-126
//   auto normals = NormalEstimation::estimateNormals<8>(octree);   // src/NormalEstimation.hpp:14-20
//
// Differences, on purpose: failures throw std::runtime_error (the reference
// prints in debug builds and continues, src/CudaCommon.hpp:23-76); classes
// that own device memory are move-only (the reference's copy would double
// free); kNN is exact; knnSearch<k> runs its queries (the reference swaps N
// and eps, src/Octree.hpp:232, and runs none); the octree built from host data
// (the MPI broadcast path) holds the data but cannot be queried.
#pragma once

#include <array>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "shapex.h"

// ---- Point / PointCloud, src/PointCloud.hpp:21-149 --------------------------
struct Point {
    Point() {}
    Point(float x, float y, float z) : x(x), y(y), z(z) {}
    float x, y, z;
    static float distance2(const Point& a, const Point& b) {
        const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        return dx * dx + dy * dy + dz * dz;
    }
    float dot(const Point& o) const { return x * o.x + y * o.y + z * o.z; }
    Point& operator+=(const Point& r) { x += r.x; y += r.y; z += r.z; return *this; }
    Point& operator-=(const Point& r) { x -= r.x; y -= r.y; z -= r.z; return *this; }
    Point& operator/=(float r) { x /= r; y /= r; z /= r; return *this; }
    friend Point operator+(Point a, const Point& b) { a += b; return a; }
    friend Point operator-(Point a, const Point& b) { a -= b; return a; }
};
static_assert(sizeof(Point) == 12, "Point must stay 3 packed floats");

template <typename T>
class PointCloud {
public:
    PointCloud() {}
    PointCloud(const std::shared_ptr<const std::vector<Point>>& pts, const std::vector<Point>& normals) {
        const auto& p = *pts;
        if (p.size() != normals.size()) throw std::invalid_argument("points and normals differ in length");
        for (size_t i = 0; i < p.size(); ++i) {
            x_vals.push_back(p[i].x); y_vals.push_back(p[i].y); z_vals.push_back(p[i].z);
            x_normals.push_back(normals[i].x); y_normals.push_back(normals[i].y); z_normals.push_back(normals[i].z);
        }
    }
    std::vector<T> x_vals, y_vals, z_vals;
    std::vector<T> x_normals, y_normals, z_normals;

    void setNormals(const std::vector<Point>& normals) {  // src/PointCloud.cpp:3-14
        if (normals.size() != x_vals.size()) throw std::invalid_argument("normals and points differ in length");
        x_normals.resize(normals.size()); y_normals.resize(normals.size()); z_normals.resize(normals.size());
        for (size_t i = 0; i < normals.size(); ++i) {
            x_normals[i] = normals[i].x; y_normals[i] = normals[i].y; z_normals[i] = normals[i].z;
        }
    }

    // ASCII PLY as src/PointCloud.hpp:151-190.
    bool saveAsPly(const std::string& filename) const {
        std::ofstream of(filename);
        if (!of) return false;
        const bool nrm = !x_normals.empty();
        of << "ply\nformat ascii 1.0\nelement vertex " << x_vals.size() << "\n";
        of << "property float x\nproperty float y\nproperty float z\n";
        if (nrm) of << "property float nx\nproperty float ny\nproperty float nz\n";
        of << "end_header\n";
        for (size_t i = 0; i < x_vals.size(); ++i) {
            of << x_vals[i] << " " << y_vals[i] << " " << z_vals[i];
            if (nrm) of << " " << x_normals[i] << " " << y_normals[i] << " " << z_normals[i];
            of << "\n";
        }
        return true;
    }
};

namespace shapex_detail {
inline void check(int rc, const se_ctx* c, const char* what) {
    if (rc != SE_OK) {
        std::string msg = std::string(what) + ": " + se_status_string(rc);
        if (c) msg += std::string(" (") + se_last_error(c) + ")";
        throw std::runtime_error(msg);
    }
}
struct CtxDeleter {
    void operator()(se_ctx* c) const { se_destroy(c); }
};
using CtxPtr = std::shared_ptr<se_ctx>;

// Options every facade object is built with; change before constructing a
// RadixTree to pick e.g. 30-bit codes or the full-range radix root.
inline se_options& default_options() {
    static se_options o = [] {
        se_options v;
        se_options_init(&v);
        return v;
    }();
    return o;
}
}  // namespace shapex_detail

typedef uint64_t Code_t;
constexpr int CODE_LEN = 63;  // src/MortonUtils.hpp:9-10

namespace RT {
// src/RadixTree.hpp:17-34; device pointers owned by the context.
struct Nodes {
    const Code_t* mortonCode = nullptr;
    const bool* hasLeafLeft = nullptr;
    const bool* hasLeafRight = nullptr;
    const uint8_t* prefixN = nullptr;
    const int* leftChild = nullptr;
    const int* parent = nullptr;
};

class RadixTree {
public:
    explicit RadixTree(const PointCloud<float>& cloud, const se_options* opt = nullptr) {
        se_ctx* c = nullptr;
        shapex_detail::check(se_create(&c, opt ? opt : &shapex_detail::default_options()), nullptr, "se_create");
        ctx_ = shapex_detail::CtxPtr(c, shapex_detail::CtxDeleter());
        const size_t n = cloud.x_vals.size();
        if (cloud.y_vals.size() != n || cloud.z_vals.size() != n) throw std::invalid_argument("x/y/z sizes differ");
        shapex_detail::check(se_build(c, cloud.x_vals.data(), cloud.y_vals.data(), cloud.z_vals.data(), (int64_t)n,
                                      SE_MEM_HOST),
                             c, "se_build");
        se_info info;
        shapex_detail::check(se_get_info(c, &info), c, "se_get_info");
        n_pts = (int)info.n_points;
        n_nodes = (int)info.n_radix;
        min_coord = info.min_coord;
        max_coord = info.max_coord;
        se_device_views v;
        shapex_detail::check(se_get_device_views(c, &v), c, "se_get_device_views");
        d_tree.mortonCode = v.codes;
        d_tree.hasLeafLeft = reinterpret_cast<const bool*>(v.has_leaf_left);
        d_tree.hasLeafRight = reinterpret_cast<const bool*>(v.has_leaf_right);
        d_tree.prefixN = v.prefix_n;
        d_tree.leftChild = v.left_child;
        d_tree.parent = v.parent;
    }
    RadixTree(const RadixTree&) = delete;
    RadixTree& operator=(const RadixTree&) = delete;
    RadixTree(RadixTree&&) = default;
    RadixTree& operator=(RadixTree&&) = default;

    Nodes d_tree;
    int n_pts = 0;
    int n_nodes = 0;
    float min_coord = 0, max_coord = 0;

    const shapex_detail::CtxPtr& context() const { return ctx_; }

private:
    shapex_detail::CtxPtr ctx_;
};
}  // namespace RT

namespace OT {
constexpr static int SEARCH_Q_SIZE = 32;  // src/Octree.hpp:17 (the exact search has no such cap)

// src/Octree.hpp:19-36, byte-compatible with se_otnode.
struct OTNode {
    int children[8];
    Point corner;
    float cell_size;
    int child_node_mask;
    int child_leaf_mask;
};
static_assert(sizeof(OTNode) == sizeof(se_otnode), "OTNode layout");

class Octree {
public:
    Octree() {}
    // src/Octree.cu:213-319
    explicit Octree(const RT::RadixTree& rt) : ctx_(rt.context()) {
        se_ctx* c = ctx_.get();
        se_info info;
        shapex_detail::check(se_get_info(c, &info), c, "se_get_info");
        n_pts = (int)info.n_points;
        n_nodes = (int)info.n_octree;
        se_device_views v;
        shapex_detail::check(se_get_device_views(c, &v), c, "se_get_device_views");
        u_points = reinterpret_cast<const Point*>(v.points);
        u_nodes = reinterpret_cast<const OTNode*>(v.octree);
        h_points = std::make_shared<std::vector<Point>>(n_pts);
        if (n_pts) shapex_detail::check(se_get_points(c, &(*h_points)[0].x, SE_MEM_HOST), c, "se_get_points");
    }
    // src/Octree.cu:179-192 (host data, e.g. after an MPI broadcast): holds the
    // data; kNN and normal queries need a tree built by this library.
    Octree(std::shared_ptr<std::vector<OTNode>> nodes, int n_nodes_, std::shared_ptr<std::vector<Point>> points,
           int n_pts_)
        : n_pts(n_pts_), h_points(std::move(points)), n_nodes(n_nodes_), host_nodes_(std::move(nodes)) {}
    Octree(const Octree&) = delete;
    Octree& operator=(const Octree&) = delete;
    Octree(Octree&&) = default;
    Octree& operator=(Octree&& o) = default;  // src/Octree.cu:194-211

    // src/Octree.hpp:214-242: exact kNN of arbitrary query points.
    template <int k>
    std::vector<std::array<int, k>> knnSearch(const std::vector<Point>& points, const float eps = 0.01) const {
        (void)eps;
        se_ctx* c = ctx();
        std::vector<std::array<int, k>> out(points.size());
        if (!points.empty())
            shapex_detail::check(se_knn(c, k, &points[0].x, (int64_t)points.size(), out[0].data(), nullptr,
                                        SE_MEM_HOST),
                                 c, "se_knn");
        return out;
    }

    // src/Octree.hpp:199-212: device queries, device results (N rows of k).
    // Queries that are the tree's own points take the seeded self-query path.
    template <int k>
    void deviceKnnSearch(const Point* d_query, int* d_nn_indices, const int N, const float eps) const {
        (void)eps;
        se_ctx* c = ctx();
        if (d_query >= u_points && d_query + N <= u_points + n_pts)
            shapex_detail::check(se_knn_self(c, k, (int64_t)(d_query - u_points), N, d_nn_indices, nullptr,
                                             SE_MEM_DEVICE),
                                 c, "se_knn_self");
        else
            shapex_detail::check(se_knn(c, k, &d_query[0].x, N, d_nn_indices, nullptr, SE_MEM_DEVICE), c, "se_knn");
    }

    int n_pts = 0;
    const Point* u_points = nullptr;  // device, AoS
    std::shared_ptr<std::vector<Point>> h_points;
    int n_nodes = 0;
    const OTNode* u_nodes = nullptr;  // device

    se_ctx* ctx() const {
        if (!ctx_) throw std::runtime_error("this octree holds host data only; build it from an RT::RadixTree");
        return ctx_.get();
    }
    const std::shared_ptr<std::vector<OTNode>>& host_nodes() const { return host_nodes_; }

private:
    shapex_detail::CtxPtr ctx_;
    std::shared_ptr<std::vector<OTNode>> host_nodes_;
};
}  // namespace OT

// src/NormalEstimation.hpp:14-20, 196-335
class NormalEstimation {
public:
    template <int k>
    static std::vector<Point> estimateNormals(const OT::Octree& octree) {
        return estimateNormals<k>(octree, 0, octree.n_pts);
    }
    template <int k>
    static std::vector<Point> estimateNormals(const OT::Octree& octree, const int start_idx, const int n) {
        se_ctx* c = octree.ctx();
        std::vector<Point> out(n);
        if (n > 0) shapex_detail::check(se_normals(c, k, start_idx, n, &out[0].x, SE_MEM_HOST), c, "se_normals");
        return out;
    }
};
