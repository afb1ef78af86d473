// Driver for the reference's own CUDA build (test infrastructure).
//
// Calls the UNMODIFIED reference through its public C++ API, exactly as
// src/main.cu:80-107 does (RT::RadixTree ctor -> OT::Octree ctor ->
// NormalEstimation::estimateNormals<k>), on a cloud read from a file, and
// either dumps every intermediate array (golden vectors) or times the span.
// Built by oracle/build_ref.sh against the reference sources in place; the
// binary lands in oracle/_ref/.
//
//   refdriver dump  <cloud.bin> <outdir> <k>
//   refdriver bench <cloud.bin> <k> <warmup> <reps>
//   refdriver batch <list.txt> <warmup> <reps>
//       list.txt: one "<cloud.bin> <k>" per line; every rep runs the clouds
//       one after another through the same API calls (the reference has no
//       batched entry point) and reports the summed time.
//
// cloud.bin: int64 n, then n float32 x, n float32 y, n float32 z.
// Only clouds whose radix tree the CPU oracle has checked to be well formed
// (every internal node reachable from the root, u >= 3) are given to it.

#include "PointCloud.hpp"
#include "RadixTree.hpp"
#include "Octree.hpp"
#include "NormalEstimation.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static bool read_cloud(const char* path, PointCloud<float>& cloud) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    long long n = 0;
    if (std::fread(&n, sizeof(n), 1, f) != 1 || n <= 0) { std::fclose(f); return false; }
    cloud.x_vals.resize(n);
    cloud.y_vals.resize(n);
    cloud.z_vals.resize(n);
    bool ok = std::fread(cloud.x_vals.data(), 4, n, f) == (size_t)n &&
              std::fread(cloud.y_vals.data(), 4, n, f) == (size_t)n &&
              std::fread(cloud.z_vals.data(), 4, n, f) == (size_t)n;
    std::fclose(f);
    return ok;
}

static void write_file(const std::string& path, const void* data, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(3); }
    if (bytes) std::fwrite(data, 1, bytes, f);
    std::fclose(f);
}

template <int k>
static int dump(const PointCloud<float>& cloud, const std::string& out) {
    RT::RadixTree rt(cloud);
    cudaDeviceSynchronize();
    const int u = rt.n_pts, nr = rt.n_nodes;
    write_file(out + "/codes.bin", rt.d_tree.mortonCode, sizeof(Code_t) * u);
    write_file(out + "/prefixN.bin", rt.d_tree.prefixN, nr);
    write_file(out + "/leftChild.bin", rt.d_tree.leftChild, 4 * (size_t)nr);
    write_file(out + "/parent.bin", rt.d_tree.parent, 4 * (size_t)u);
    write_file(out + "/hasLeafLeft.bin", rt.d_tree.hasLeafLeft, nr);
    write_file(out + "/hasLeafRight.bin", rt.d_tree.hasLeafRight, nr);

    OT::Octree oct(rt);
    cudaDeviceSynchronize();
    write_file(out + "/nodes.bin", oct.u_nodes, sizeof(OT::OTNode) * (size_t)oct.n_nodes);
    write_file(out + "/points.bin", oct.u_points, sizeof(Point) * (size_t)oct.n_pts);

    int* nn = nullptr;
    cudaMallocManaged(&nn, sizeof(int) * (size_t)u * k);
    oct.deviceKnnSearch<k>(oct.u_points, nn, u, 0.01f);
    cudaDeviceSynchronize();
    write_file(out + "/knn.bin", nn, sizeof(int) * (size_t)u * k);
    cudaFree(nn);

    std::vector<Point> normals = NormalEstimation::estimateNormals<k>(oct);
    write_file(out + "/normals.bin", normals.data(), sizeof(Point) * normals.size());

    std::printf("REFJSON {\"n\": %zu, \"u\": %d, \"n_radix\": %d, \"n_oct\": %d, \"min\": %.9g, \"max\": %.9g, "
                "\"k\": %d, \"cuda_error\": \"%s\"}\n",
                cloud.x_vals.size(), u, nr, oct.n_nodes, rt.min_coord, rt.max_coord, k,
                cudaGetErrorString(cudaGetLastError()));
    return 0;
}

template <int k>
static int bench(const PointCloud<float>& cloud, int warmup, int reps) {
    std::vector<double> ms;
    int u = 0;
    for (int r = 0; r < warmup + reps; ++r) {
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        RT::RadixTree rt(cloud);
        OT::Octree oct(rt);
        std::vector<Point> normals = NormalEstimation::estimateNormals<k>(oct);
        cudaDeviceSynchronize();
        auto t1 = std::chrono::steady_clock::now();
        u = oct.n_pts;
        if (r >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    std::printf("REFJSON {\"n\": %zu, \"u\": %d, \"k\": %d, \"ms\": [", cloud.x_vals.size(), u, k);
    for (size_t i = 0; i < ms.size(); ++i) std::printf("%s%.4f", i ? ", " : "", ms[i]);
    std::printf("], \"cuda_error\": \"%s\"}\n", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

template <int k>
static int one_cloud(const PointCloud<float>& cloud) {
    RT::RadixTree rt(cloud);
    OT::Octree oct(rt);
    std::vector<Point> normals = NormalEstimation::estimateNormals<k>(oct);
    cudaDeviceSynchronize();
    return oct.n_pts;
}

static int batch(const char* list, int warmup, int reps) {
    std::vector<PointCloud<float>> clouds;
    std::vector<int> ks;
    FILE* f = std::fopen(list, "r");
    if (!f) return 2;
    char path[4096];
    int k = 0;
    while (std::fscanf(f, "%4095s %d", path, &k) == 2) {
        clouds.emplace_back();
        if (!read_cloud(path, clouds.back())) { std::fclose(f); return 2; }
        ks.push_back(k);
    }
    std::fclose(f);
    std::vector<double> ms;
    long long u_total = 0;
    for (int r = 0; r < warmup + reps; ++r) {
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        long long u = 0;
        for (size_t i = 0; i < clouds.size(); ++i) {
            switch (ks[i]) {
                case 8: u += one_cloud<8>(clouds[i]); break;
                case 10: u += one_cloud<10>(clouds[i]); break;
                case 16: u += one_cloud<16>(clouds[i]); break;
                case 32: u += one_cloud<32>(clouds[i]); break;
                default: return 2;
            }
        }
        auto t1 = std::chrono::steady_clock::now();
        u_total = u;
        if (r >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    std::printf("REFJSON {\"clouds\": %zu, \"u\": %lld, \"ms\": [", clouds.size(), u_total);
    for (size_t i = 0; i < ms.size(); ++i) std::printf("%s%.4f", i ? ", " : "", ms[i]);
    std::printf("], \"cuda_error\": \"%s\"}\n", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 4) { std::fprintf(stderr, "usage: see header\n"); return 2; }
    const std::string mode = argv[1];
    if (mode == "batch") {
        if (argc < 5) return 2;
        return batch(argv[2], std::atoi(argv[3]), std::atoi(argv[4]));
    }
    PointCloud<float> cloud;
    if (!read_cloud(argv[2], cloud)) { std::fprintf(stderr, "cannot read %s\n", argv[2]); return 2; }
    if (mode == "dump") {
        if (argc < 5) return 2;
        const int k = std::atoi(argv[4]);
        switch (k) {
            case 8: return dump<8>(cloud, argv[3]);
            case 10: return dump<10>(cloud, argv[3]);
            case 16: return dump<16>(cloud, argv[3]);
            case 32: return dump<32>(cloud, argv[3]);
        }
        return 2;
    }
    if (mode == "bench") {
        if (argc < 6) return 2;
        const int k = std::atoi(argv[3]), warm = std::atoi(argv[4]), reps = std::atoi(argv[5]);
        switch (k) {
            case 8: return bench<8>(cloud, warm, reps);
            case 10: return bench<10>(cloud, warm, reps);
            case 16: return bench<16>(cloud, warm, reps);
            case 32: return bench<32>(cloud, warm, reps);
        }
        return 2;
    }
    return 2;
}
