// Particle geometry on the host: the reference's particle generators, and PLY
// files in and out (host code; no device work).
//
//   vtp_generate_particles: ModelHandler::generateObjectElements
//     (Simulator/Library/Source/Model/ModelHandler.cpp:13-175) for the five
//     particle generators - genType 1 sphere, 2 cube, 3 cylinder, 4 plane,
//     5 box - with the reference's loop order and floating-point arithmetic,
//     so the particle positions are the reference's bit for bit (the float
//     running sums of cube / cylinder / plane, the double-rounded lattice of
//     box, the float lattice and squared-radius test of sphere);
//   vtp_read_ply: the particle loader ModelHandler::load_PLY_ParticleElements
//     (ModelHandler.cpp:207-228), which takes every vertex of a PLY file as a
//     particle; ASCII and binary PLY, read directly (the reference goes
//     through assimp);
//   vtp_write_ply: ExportUtil::exportAsPly (ExportUtil.cpp:28-88), the ASCII
//     format the solvers' exports use, with the directory and file name
//     joined by '/' (the reference joins them with a backslash).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "../../include/vtp.h"

namespace vtp {
int fail(int code, const std::string &msg);
}

using json = nlohmann::json;

namespace {

struct P3 {
    float x, y, z;
};

std::vector<float> f3(const json &c, const char *k) {
    auto v = c.at(k).get<std::vector<float>>();
    if (v.size() != 3) throw std::runtime_error(std::string(k) + " needs 3 values");
    return v;
}

// A loop over float values from `start` while `keep(v)`, stepping by `step`, has at most
// this many iterations here (a step too small for the extent would otherwise not end).
constexpr uint64_t kMaxLoop = 1ull << 24;

// generateParticleCubeElements (ModelHandler.cpp:43-67): z, y, x running sums from r + lb in
// steps of 2r while below lb + size.
int gen_cube(const json &c, std::vector<P3> &out) {
    const float r = c.at("particleRadius").get<float>();
    const auto lb = f3(c, "lb"), size = f3(c, "size");
    const float d = 2 * r;
    uint64_t guard = 0;
    for (float z = r + lb[2]; z < lb[2] + size[2]; z += d) {
        for (float y = r + lb[1]; y < lb[1] + size[1]; y += d) {
            for (float x = r + lb[0]; x < lb[0] + size[0]; x += d) {
                out.push_back({x, y, z});
                if (++guard > kMaxLoop * 64) return 1;
            }
        }
    }
    return 0;
}

// generateParticleCylinderElements (ModelHandler.cpp:69-96): layers from the top down, in
// each layer x across the diameter and z across the chord at that x.
int gen_cylinder(const json &c, std::vector<P3> &out) {
    const float r = c.at("particleRadius").get<float>();
    const auto center = f3(c, "center");
    const float R = c.at("bottomAreaRadius").get<float>();
    const float height = c.at("height").get<float>();
    const float d = 2 * r;
    const float tx = center[0], ty = center[1] + height / 2, tz = center[2];
    uint64_t guard = 0;
    for (float y = ty - r; y >= ty - height; y -= d) {
        for (float x = tx - R + r; x <= tx + R; x += d) {
            // fabs and sqrt of the reference's calls resolve to the C library's double functions
            // there (ModelHandler.cpp:84-86), so both expressions are evaluated in double and
            // rounded to float on assignment.
            const float m_cos = (float)(std::fabs((double)(tx - x)) / (double)R);
            const float length = (float)((double)R * std::sqrt((double)(1 - m_cos * m_cos)));
            for (float z = tz - length + r; z <= tz + length; z += d) {
                out.push_back({x, y, z});
                if (++guard > kMaxLoop * 64) return 1;
            }
        }
    }
    return 0;
}

// generateParticleSphereElements (ModelHandler.cpp:98-122): the lattice i, j, k in
// [-n, n], n = ceil(R / 2r), kept within R of the centre (squared distances in float).
int gen_sphere(const json &c, std::vector<P3> &out) {
    const float r = c.at("particleRadius").get<float>();
    const auto center = f3(c, "volumeCenter");
    const float R = c.at("volumeRadius").get<float>();
    const float gap = r * 2.0f;
    const double nd = std::ceil(R / gap);
    if (!(nd >= 0.0) || nd > 4096.0) return 1;
    const int n = (int)nd;
    for (int i = -n; i <= n; ++i)
        for (int j = -n; j <= n; ++j)
            for (int k = -n; k <= n; ++k) {
                const P3 p{float(i) * gap + center[0], float(j) * gap + center[1], float(k) * gap + center[2]};
                const float dx = p.x - center[0], dy = p.y - center[1], dz = p.z - center[2];
                if (dx * dx + dy * dy + dz * dz <= R * R) out.push_back(p);
            }
    return 0;
}

// generateParticlePlaneElements (ModelHandler.cpp:156-175): z running sum over the extent,
// `layerNum` layers in y (the layer counter is a float, as there), x running sum.
int gen_plane(const json &c, std::vector<P3> &out) {
    const float r = c.at("particleRadius").get<float>();
    const auto lb = f3(c, "lb"), size = f3(c, "size");
    const int layers = c.at("layerNum").get<int>();
    const float d = 2 * r;
    uint64_t guard = 0;
    for (float z = r + lb[2]; z < lb[2] + size[2]; z += d) {
        float y = r + lb[1];
        for (float cnt = 0; cnt < layers; y += d, cnt += 1) {
            for (float x = r + lb[0]; x < lb[0] + size[0]; x += d) {
                out.push_back({x, y, z});
                if (++guard > kMaxLoop * 64) return 1;
            }
        }
    }
    return 0;
}

// generateParticleBoxElements (ModelHandler.cpp:124-154): lattice points i = 0..n per axis,
// n = int((size + r) / (2.0 r)), at float(lb + r + 2.0 r i) evaluated in double, kept
// when within `layerNum` of a face.
int gen_box(const json &c, std::vector<P3> &out) {
    const float r = c.at("particleRadius").get<float>();
    const auto lb = f3(c, "lb"), size = f3(c, "size");
    const int L = c.at("layerNum").get<int>();
    int n[3];
    for (int a = 0; a < 3; ++a) {
        const double v = (size[a] + r) / (2.0 * r);
        if (!(v >= 0.0) || v > 1e6) return 1;
        n[a] = static_cast<int>(v);
    }
    for (int i = 0; i <= n[0]; ++i)
        for (int j = 0; j <= n[1]; ++j)
            for (int k = 0; k <= n[2]; ++k) {
                if (i < L || i >= n[0] - L || j < L || j >= n[1] - L || k < L || k >= n[2] - L) {
                    out.push_back({static_cast<float>(lb[0] + r + 2.0 * r * i),
                                   static_cast<float>(lb[1] + r + 2.0 * r * j),
                                   static_cast<float>(lb[2] + r + 2.0 * r * k)});
                }
            }
    return 0;
}

// ---------------------------------------------------------------- PLY reading

enum PlyType { T_I8, T_U8, T_I16, T_U16, T_I32, T_U32, T_F32, T_F64, T_BAD };

PlyType ply_type(const std::string &t) {
    if (t == "char" || t == "int8") return T_I8;
    if (t == "uchar" || t == "uint8") return T_U8;
    if (t == "short" || t == "int16") return T_I16;
    if (t == "ushort" || t == "uint16") return T_U16;
    if (t == "int" || t == "int32") return T_I32;
    if (t == "uint" || t == "uint32") return T_U32;
    if (t == "float" || t == "float32") return T_F32;
    if (t == "double" || t == "float64") return T_F64;
    return T_BAD;
}

int ply_size(PlyType t) {
    switch (t) {
        case T_I8: case T_U8: return 1;
        case T_I16: case T_U16: return 2;
        case T_I32: case T_U32: case T_F32: return 4;
        case T_F64: return 8;
        default: return 0;
    }
}

struct PlyProp {
    std::string name;
    PlyType type = T_BAD;
    bool list = false;
    PlyType count_type = T_BAD;
};

struct PlyElement {
    std::string name;
    uint64_t count = 0;
    std::vector<PlyProp> props;
};

double read_binary(const unsigned char *p, PlyType t, bool swap) {
    unsigned char b[8];
    const int n = ply_size(t);
    for (int i = 0; i < n; ++i) b[i] = swap ? p[n - 1 - i] : p[i];
    switch (t) {
        case T_I8: { int8_t v; std::memcpy(&v, b, 1); return v; }
        case T_U8: { uint8_t v; std::memcpy(&v, b, 1); return v; }
        case T_I16: { int16_t v; std::memcpy(&v, b, 2); return v; }
        case T_U16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
        case T_I32: { int32_t v; std::memcpy(&v, b, 4); return v; }
        case T_U32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
        case T_F32: { float v; std::memcpy(&v, b, 4); return v; }
        case T_F64: { double v; std::memcpy(&v, b, 8); return v; }
        default: return 0.0;
    }
}

bool host_little_endian() {
    const uint16_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

int read_ply(const std::string &path, std::vector<float> &xyz) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return vtp::fail(VTP_ERR_ARG, "cannot open " + path);
    std::string line;
    if (!std::getline(f, line) || line.rfind("ply", 0) != 0) return vtp::fail(VTP_ERR_ARG, path + ": not a PLY file");
    int format = -1;   // 0 ascii, 1 binary little endian, 2 binary big endian
    std::vector<PlyElement> elems;
    bool header_done = false;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream ss(line);
        std::string kw;
        ss >> kw;
        if (kw == "format") {
            std::string fmt;
            ss >> fmt;
            format = fmt == "ascii" ? 0 : fmt == "binary_little_endian" ? 1 : fmt == "binary_big_endian" ? 2 : -1;
            if (format < 0) return vtp::fail(VTP_ERR_ARG, path + ": unknown PLY format " + fmt);
        } else if (kw == "element") {
            PlyElement e;
            ss >> e.name >> e.count;
            if (ss.fail()) return vtp::fail(VTP_ERR_ARG, path + ": bad element line: " + line);
            elems.push_back(e);
        } else if (kw == "property") {
            if (elems.empty()) return vtp::fail(VTP_ERR_ARG, path + ": property before any element");
            PlyProp p;
            std::string t;
            ss >> t;
            if (t == "list") {
                std::string ct, it;
                ss >> ct >> it >> p.name;
                p.list = true;
                p.count_type = ply_type(ct);
                p.type = ply_type(it);
            } else {
                ss >> p.name;
                p.type = ply_type(t);
            }
            if (p.type == T_BAD || (p.list && p.count_type == T_BAD))
                return vtp::fail(VTP_ERR_ARG, path + ": unknown property type in: " + line);
            elems.back().props.push_back(p);
        } else if (kw == "end_header") {
            header_done = true;
            break;
        }   // comment, obj_info: ignored
    }
    if (!header_done || format < 0) return vtp::fail(VTP_ERR_ARG, path + ": incomplete PLY header");
    const bool swap = (format == 1) != host_little_endian();
    xyz.clear();
    for (const PlyElement &e : elems) {
        int ix = -1, iy = -1, iz = -1;
        for (size_t k = 0; k < e.props.size(); ++k) {
            if (e.props[k].name == "x") ix = (int)k;
            if (e.props[k].name == "y") iy = (int)k;
            if (e.props[k].name == "z") iz = (int)k;
        }
        const bool vertex = e.name == "vertex";
        if (vertex && (ix < 0 || iy < 0 || iz < 0)) return vtp::fail(VTP_ERR_ARG, path + ": vertex without x, y, z");
        if (vertex) xyz.reserve((size_t)e.count * 3);
        std::vector<double> vals(e.props.size());
        for (uint64_t r = 0; r < e.count; ++r) {
            if (format == 0) {
                if (!std::getline(f, line)) return vtp::fail(VTP_ERR_ARG, path + ": file ends inside element " + e.name);
                std::istringstream ls(line);
                for (size_t k = 0; k < e.props.size(); ++k) {
                    if (e.props[k].list) {
                        double cnt = 0;
                        ls >> cnt;
                        for (uint64_t m = 0; m < (uint64_t)cnt; ++m) {
                            double skip;
                            ls >> skip;
                        }
                    } else {
                        ls >> vals[k];
                    }
                }
                if (ls.fail()) return vtp::fail(VTP_ERR_ARG, path + ": bad " + e.name + " line: " + line);
            } else {
                for (size_t k = 0; k < e.props.size(); ++k) {
                    unsigned char buf[8];
                    if (e.props[k].list) {
                        const int cs = ply_size(e.props[k].count_type);
                        if (!f.read((char *)buf, cs)) return vtp::fail(VTP_ERR_ARG, path + ": truncated");
                        const double cnt = read_binary(buf, e.props[k].count_type, swap);
                        if (!(cnt >= 0)) return vtp::fail(VTP_ERR_ARG, path + ": negative list length");
                        f.seekg((std::streamoff)cnt * ply_size(e.props[k].type), std::ios::cur);
                    } else {
                        const int sz = ply_size(e.props[k].type);
                        if (!f.read((char *)buf, sz)) return vtp::fail(VTP_ERR_ARG, path + ": truncated");
                        vals[k] = read_binary(buf, e.props[k].type, swap);
                    }
                }
            }
            if (vertex) {
                xyz.push_back((float)vals[ix]);
                xyz.push_back((float)vals[iy]);
                xyz.push_back((float)vals[iz]);
            }
        }
        if (vertex) return VTP_OK;   // the particles are the vertices; later elements are not needed
    }
    return vtp::fail(VTP_ERR_ARG, path + ": no vertex element");
}

}  // namespace

extern "C" {

VTP_API int vtp_generate_particles(const char *config_json, float *out, uint64_t capacity, uint64_t *count) {
    if (!config_json || !count) return vtp::fail(VTP_ERR_ARG, "null argument");
    std::vector<P3> pts;
    try {
        const json c = json::parse(config_json);
        if (!c.contains("genType")) return vtp::fail(VTP_ERR_CONFIG, "No generation type specified.");
        const int t = c.at("genType").get<int>();
        int rc = 0;
        switch (t) {
            case 1: rc = gen_sphere(c, pts); break;
            case 2: rc = gen_cube(c, pts); break;
            case 3: rc = gen_cylinder(c, pts); break;
            case 4: rc = gen_plane(c, pts); break;
            case 5: rc = gen_box(c, pts); break;
            default: return vtp::fail(VTP_ERR_CONFIG, "Unknown or Unsupported generation type specified.");
        }
        if (rc) return vtp::fail(VTP_ERR_BOUNDS, "generator extent too large for the particle radius");
    } catch (const std::exception &e) {
        return vtp::fail(VTP_ERR_CONFIG, std::string("generator config: ") + e.what());
    }
    *count = pts.size();
    if (!out) return VTP_OK;
    if (capacity < pts.size()) return vtp::fail(VTP_ERR_BOUNDS, "output capacity below the particle count");
    std::memcpy(out, pts.data(), pts.size() * sizeof(P3));
    return VTP_OK;
}

VTP_API int vtp_read_ply(const char *path, float *out, uint64_t capacity, uint64_t *count) {
    if (!path || !count) return vtp::fail(VTP_ERR_ARG, "null argument");
    std::vector<float> xyz;
    int rc;
    try {
        rc = read_ply(path, xyz);
    } catch (const std::exception &e) {
        return vtp::fail(VTP_ERR_ARG, std::string("PLY read: ") + e.what());
    }
    if (rc) return rc;
    *count = xyz.size() / 3;
    if (!out) return VTP_OK;
    if (capacity < *count) return vtp::fail(VTP_ERR_BOUNDS, "output capacity below the vertex count");
    std::memcpy(out, xyz.data(), xyz.size() * sizeof(float));
    return VTP_OK;
}

VTP_API int vtp_write_ply(const char *dir, const char *name, const float *pos, uint64_t n, const float *color,
                          const float *phase, int32_t n_phase) {
    if (!dir || !name || (n && !pos) || (phase && n_phase <= 0)) return vtp::fail(VTP_ERR_ARG, "bad argument");
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return vtp::fail(VTP_ERR_ARG, std::string("cannot create ") + dir + ": " + ec.message());
    const std::string path = std::string(dir) + "/" + name + ".ply";
    std::ofstream f(path);
    if (!f) return vtp::fail(VTP_ERR_ARG, "cannot open " + path);
    f << "ply\n";
    f << "format ascii 1.0\n";
    f << "element vertex " << n << "\n";
    f << "property float x\n";
    f << "property float y\n";
    f << "property float z\n";
    if (color) {
        f << "property uchar red" << std::endl;
        f << "property uchar green" << std::endl;
        f << "property uchar blue" << std::endl;
    }
    if (phase)
        for (int k = 0; k < n_phase; ++k) f << "property float p" << k + 1 << std::endl;
    f << "end_header\n";
    for (uint64_t i = 0; i < n; ++i) {
        f << pos[3 * i] << " " << pos[3 * i + 1] << " " << pos[3 * i + 2] << " ";
        if (color) f << color[3 * i] << " " << color[3 * i + 1] << " " << color[3 * i + 2] << " ";
        if (phase)
            for (int k = 0; k < n_phase; ++k) f << phase[i * (uint64_t)n_phase + k] << " ";
        f << "\n";
    }
    f.close();
    if (!f) return vtp::fail(VTP_ERR_ARG, "write failed: " + path);
    return VTP_OK;
}

}  // extern "C"
