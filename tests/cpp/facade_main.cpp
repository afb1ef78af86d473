// The reference's driver flow (src/main.cu:50-124, single rank, no MPI) written
// against the C++ facade include/shapex.hpp. Reads a cloud file (int64 n, then
// n float32 x, y, z), builds RT::RadixTree and OT::Octree, runs
// NormalEstimation::estimateNormals<16> and Octree::knnSearch<8>, and writes
//   <out>.normals (u x 3 float32), <out>.knn (m x 8 int32 for the first m
//   points), <out>.info (u n_radix n_octree min max as text)
// so that the Python tests can compare with the C ABI.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "shapex.hpp"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: facade_main cloud.bin out_prefix\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    long long n = 0;
    if (std::fread(&n, 8, 1, f) != 1) return 2;
    PointCloud<float> cloud;
    cloud.x_vals.resize(n);
    cloud.y_vals.resize(n);
    cloud.z_vals.resize(n);
    if (std::fread(cloud.x_vals.data(), 4, n, f) != (size_t)n || std::fread(cloud.y_vals.data(), 4, n, f) != (size_t)n ||
        std::fread(cloud.z_vals.data(), 4, n, f) != (size_t)n)
        return 2;
    std::fclose(f);

    try {
        RT::RadixTree radix_tree(cloud);
        OT::Octree octree;
        octree = OT::Octree(radix_tree);  // move-assign, as src/main.cu:85
        auto normals = NormalEstimation::estimateNormals<16>(octree);
        const int m = octree.n_pts < 1000 ? octree.n_pts : 1000;
        std::vector<Point> q(octree.h_points->begin(), octree.h_points->begin() + m);
        auto knn = octree.knnSearch<8>(q);

        std::string out = argv[2];
        FILE* g = std::fopen((out + ".normals").c_str(), "wb");
        std::fwrite(normals.data(), sizeof(Point), normals.size(), g);
        std::fclose(g);
        g = std::fopen((out + ".knn").c_str(), "wb");
        std::fwrite(knn.data(), sizeof(int) * 8, knn.size(), g);
        std::fclose(g);
        g = std::fopen((out + ".info").c_str(), "w");
        std::fprintf(g, "%d %d %d %.9g %.9g\n", octree.n_pts, radix_tree.n_nodes, octree.n_nodes, radix_tree.min_coord,
                     radix_tree.max_coord);
        std::fclose(g);

        PointCloud<float> output_cloud(octree.h_points, normals);
        output_cloud.saveAsPly(out + ".ply");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
