// Loads a point cloud with DataIO::loadFile (include/shapex_io.hpp) and writes
// it back as KITTI (<out>.bin), binary PLY (<out>.ply) and ASCII PLY
// (<out>.ascii.ply, PointCloud::saveAsPly); prints the point count and whether
// normals were present.
#include <cstdio>

#include "shapex_io.hpp"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: io_main <cloud file> <out prefix>\n");
        return 2;
    }
    try {
        PointCloud<float> cloud = DataIO::loadFile(argv[1]);
        const std::string out = argv[2];
        DataIO::saveKitti(cloud, out + ".bin");
        if (!DataIO::savePly(cloud, out + ".ply")) return 3;
        if (!cloud.saveAsPly(out + ".ascii.ply")) return 4;
        PointCloud<float> back = DataIO::loadFile(out + ".ply");
        if (back.x_vals != cloud.x_vals || back.z_normals != cloud.z_normals) return 5;
        std::printf("%zu %d\n", cloud.x_vals.size(), cloud.x_normals.empty() ? 0 : 1);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
