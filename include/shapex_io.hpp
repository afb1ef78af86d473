// shapex_io.hpp -- point-cloud file I/O for the facade in shapex.hpp, with the
// reference's DataIO interface (src/DataIO.hpp, src/DataIO.cpp) and a binary
// PLY reader and writer next to PointCloud::saveAsPly's ASCII one
// (src/PointCloud.hpp:151-190).
//
// Every loader reads the whole file with one fread and parses the buffer in
// place: KITTI .bin is a strided copy out of the float32 (x, y, z, reflectance)
// records; text formats (.obj vertices, Semantic3D .txt, ASCII PLY) go through
// std::from_chars, with no stream or locale machinery per value. Writers build
// the file image in memory and write it at once.
//
// Differences from the reference, on purpose: an unknown extension throws
// (src/DataIO.cpp:13-31 falls off the end of a non-void function); loadKitti
// sizes its buffer from the file, not 4x the float count (src/DataIO.cpp:33-41);
// a line that does not parse is skipped silently instead of printed
// (src/DataIO.cpp:84-86, :104-106); a trailing partial KITTI record is ignored.
#pragma once

#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "shapex.hpp"

namespace shapex_io_detail {

inline std::vector<char> read_all(const std::string& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<char> buf;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        const long len = std::ftell(f);
        if (len > 0) {
            buf.resize((size_t)len);
            std::fseek(f, 0, SEEK_SET);
            const size_t got = std::fread(buf.data(), 1, buf.size(), f);
            buf.resize(got);
        }
    }
    std::fclose(f);
    return buf;
}

inline void write_all(const std::string& path, const std::vector<char>& buf) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path + " for writing");
    const size_t put = buf.empty() ? 0 : std::fwrite(buf.data(), 1, buf.size(), f);
    const bool ok = std::fclose(f) == 0 && put == buf.size();
    if (!ok) throw std::runtime_error("short write to " + path);
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Parse up to `want` floats from [p, line_end); returns how many parsed.
inline int parse_floats(const char* p, const char* e, float* out, int want) {
    int n = 0;
    while (n < want) {
        while (p < e && is_space(*p)) ++p;
        if (p >= e) break;
        if (*p == '+') ++p;  // from_chars takes no leading '+'
        float v;
        const auto r = std::from_chars(p, e, v);
        if (r.ec != std::errc()) break;
        out[n++] = v;
        p = r.ptr;
    }
    return n;
}

template <typename F>
inline void for_each_line(const std::vector<char>& buf, size_t from, F&& f) {
    const char* p = buf.data() + from;
    const char* end = buf.data() + buf.size();
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        const char* e = nl ? nl : end;
        f(p, e);
        p = nl ? nl + 1 : end;
    }
}

inline bool little_endian() {
    const uint16_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

}  // namespace shapex_io_detail

// src/DataIO.hpp
class DataIO {
public:
    // By extension: .bin (KITTI), .obj, .txt (Semantic3D), .ply (ASCII or
    // binary little-endian). src/DataIO.cpp:13-31 plus .ply.
    static PointCloud<float> loadFile(const std::string& filepath) {
        auto ends = [&](const char* ext) {
            const size_t n = std::strlen(ext);
            return filepath.size() >= n && filepath.compare(filepath.size() - n, n, ext) == 0;
        };
        if (ends(".obj")) return loadObj(filepath);
        if (ends(".bin")) return loadKitti(filepath, std::numeric_limits<size_t>::max());
        if (ends(".txt")) return loadSemantic3D(filepath);
        if (ends(".ply")) return loadPly(filepath);
        throw std::runtime_error("unknown point-cloud file extension: " + filepath);
    }

    // KITTI velodyne scan: float32 records (x, y, z, reflectance); `num` is
    // the most floats to read (4 per point), src/DataIO.cpp:33-57.
    static PointCloud<float> loadKitti(const std::string& filepath, size_t num) {
        const std::vector<char> buf = shapex_io_detail::read_all(filepath);
        size_t floats = buf.size() / sizeof(float);
        if (num < floats) floats = num;
        const size_t n = floats / 4;
        PointCloud<float> cloud;
        cloud.x_vals.resize(n);
        cloud.y_vals.resize(n);
        cloud.z_vals.resize(n);
        const char* p = buf.data();
        for (size_t i = 0; i < n; ++i) {
            float rec[4];
            std::memcpy(rec, p + 16 * i, 16);
            cloud.x_vals[i] = rec[0];
            cloud.y_vals[i] = rec[1];
            cloud.z_vals[i] = rec[2];
        }
        return cloud;
    }

    // Reflectance 255 for every point, as src/DataIO.cpp:59-77.
    static void saveKitti(const PointCloud<float>& cloud, const std::string& filepath) {
        const size_t n = cloud.x_vals.size();
        std::vector<char> buf(16 * n);
        const float refl = 255.0f;
        for (size_t i = 0; i < n; ++i) {
            const float rec[4] = {cloud.x_vals[i], cloud.y_vals[i], cloud.z_vals[i], refl};
            std::memcpy(buf.data() + 16 * i, rec, 16);
        }
        shapex_io_detail::write_all(filepath, buf);
    }

    // Vertex lines "v x y z" of an ASCII .obj, src/DataIO.cpp:79-95.
    static PointCloud<float> loadObj(const std::string& filepath) {
        const std::vector<char> buf = shapex_io_detail::read_all(filepath);
        PointCloud<float> cloud;
        shapex_io_detail::for_each_line(buf, 0, [&](const char* p, const char* e) {
            if (e - p > 1 && p[0] == 'v' && p[1] == ' ') {
                float v[3];
                if (shapex_io_detail::parse_floats(p + 2, e, v, 3) == 3) {
                    cloud.x_vals.push_back(v[0]);
                    cloud.y_vals.push_back(v[1]);
                    cloud.z_vals.push_back(v[2]);
                }
            }
        });
        return cloud;
    }

    // Semantic3D lines "x y z intensity r g b" (the reference parses six
    // numbers and keeps x, y, z), src/DataIO.cpp:97-115.
    static PointCloud<float> loadSemantic3D(const std::string& filepath) {
        const std::vector<char> buf = shapex_io_detail::read_all(filepath);
        PointCloud<float> cloud;
        shapex_io_detail::for_each_line(buf, 0, [&](const char* p, const char* e) {
            float v[6];
            if (shapex_io_detail::parse_floats(p, e, v, 6) == 6) {
                cloud.x_vals.push_back(v[0]);
                cloud.y_vals.push_back(v[1]);
                cloud.z_vals.push_back(v[2]);
            }
        });
        return cloud;
    }

    // PLY with a float vertex element: x, y, z and optionally nx, ny, nz, in
    // ASCII or binary little-endian (what savePly and saveAsPly write).
    static PointCloud<float> loadPly(const std::string& filepath) {
        const std::vector<char> buf = shapex_io_detail::read_all(filepath);
        const char* hdr_end_tag = "end_header\n";
        const char* b = buf.data();
        const char* he = nullptr;
        for (size_t i = 0; i + 11 <= buf.size(); ++i)
            if (std::memcmp(b + i, hdr_end_tag, 11) == 0) {
                he = b + i + 11;
                break;
            }
        if (!he || buf.size() < 4 || std::memcmp(b, "ply", 3) != 0) throw std::runtime_error("not a PLY file: " + filepath);
        bool binary = false, ascii = false, in_vertex = false;
        size_t n = 0;
        std::vector<std::string> props;
        shapex_io_detail::for_each_line(std::vector<char>(b, he), 0, [&](const char* p, const char* e) {
            std::string line(p, e);
            if (!line.empty() && line.back() == '\r') line.pop_back();
            if (line.rfind("format ", 0) == 0) {
                binary = line.find("binary_little_endian") != std::string::npos;
                ascii = line.find("ascii") != std::string::npos;
            } else if (line.rfind("element ", 0) == 0) {
                in_vertex = line.rfind("element vertex ", 0) == 0;
                if (in_vertex) n = std::stoull(line.substr(15));
            } else if (in_vertex && line.rfind("property float ", 0) == 0) {
                props.push_back(line.substr(15));
            } else if (in_vertex && line.rfind("property ", 0) == 0) {
                throw std::runtime_error("PLY vertex properties other than float are not supported: " + line);
            }
        });
        if (!binary && !ascii) throw std::runtime_error("unsupported PLY format in " + filepath);
        auto col = [&](const char* name) {
            for (size_t i = 0; i < props.size(); ++i)
                if (props[i] == name) return (int)i;
            return -1;
        };
        const int ix = col("x"), iy = col("y"), iz = col("z");
        const int inx = col("nx"), iny = col("ny"), inz = col("nz");
        if (ix < 0 || iy < 0 || iz < 0) throw std::runtime_error("PLY without x, y, z: " + filepath);
        const bool nrm = inx >= 0 && iny >= 0 && inz >= 0;
        const int np = (int)props.size();
        PointCloud<float> cloud;
        cloud.x_vals.resize(n);
        cloud.y_vals.resize(n);
        cloud.z_vals.resize(n);
        if (nrm) {
            cloud.x_normals.resize(n);
            cloud.y_normals.resize(n);
            cloud.z_normals.resize(n);
        }
        std::vector<float> rec((size_t)np);
        auto put = [&](size_t i) {
            cloud.x_vals[i] = rec[ix];
            cloud.y_vals[i] = rec[iy];
            cloud.z_vals[i] = rec[iz];
            if (nrm) {
                cloud.x_normals[i] = rec[inx];
                cloud.y_normals[i] = rec[iny];
                cloud.z_normals[i] = rec[inz];
            }
        };
        const size_t off = (size_t)(he - b);
        if (binary) {
            if (!shapex_io_detail::little_endian()) throw std::runtime_error("big-endian hosts are not supported");
            const size_t stride = 4 * (size_t)np;
            if (buf.size() - off < stride * n) throw std::runtime_error("truncated PLY: " + filepath);
            for (size_t i = 0; i < n; ++i) {
                std::memcpy(rec.data(), b + off + stride * i, stride);
                put(i);
            }
        } else {
            size_t i = 0;
            shapex_io_detail::for_each_line(buf, off, [&](const char* p, const char* e) {
                if (i < n && shapex_io_detail::parse_floats(p, e, rec.data(), np) == np) put(i++);
            });
            if (i != n) throw std::runtime_error("truncated PLY: " + filepath);
        }
        return cloud;
    }

    // Binary little-endian PLY of the cloud (and its normals when set): the
    // same header as PointCloud::saveAsPly, 12 or 24 bytes per vertex.
    static bool savePly(const PointCloud<float>& cloud, const std::string& filepath) {
        const size_t n = cloud.x_vals.size();
        const bool nrm = !cloud.x_normals.empty();
        if (cloud.y_vals.size() != n || cloud.z_vals.size() != n) return false;
        if (nrm && (cloud.x_normals.size() != n || cloud.y_normals.size() != n || cloud.z_normals.size() != n))
            return false;
        if (!shapex_io_detail::little_endian()) return false;
        std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) +
                        "\nproperty float x\nproperty float y\nproperty float z\n";
        if (nrm) h += "property float nx\nproperty float ny\nproperty float nz\n";
        h += "end_header\n";
        const size_t stride = nrm ? 24 : 12;
        std::vector<char> buf(h.size() + stride * n);
        std::memcpy(buf.data(), h.data(), h.size());
        char* o = buf.data() + h.size();
        for (size_t i = 0; i < n; ++i) {
            const float rec[6] = {cloud.x_vals[i], cloud.y_vals[i], cloud.z_vals[i],
                                  nrm ? cloud.x_normals[i] : 0.0f, nrm ? cloud.y_normals[i] : 0.0f,
                                  nrm ? cloud.z_normals[i] : 0.0f};
            std::memcpy(o + stride * i, rec, stride);
        }
        try {
            shapex_io_detail::write_all(filepath, buf);
        } catch (const std::runtime_error&) {
            return false;
        }
        return true;
    }
};
