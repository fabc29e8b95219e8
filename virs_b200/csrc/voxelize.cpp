// Mesh input on the host; the triangle sweep runs on the GPU
// (kernels_voxelize.cu).
//
//   OBJ parsing                 replaces tinyobj::LoadObj at simulator.cpp:279
//   bounding box + nudge        simulator.cpp:288-310
//   grid sizing                 simulator.cpp:321-329
//
// Compiled with -ffp-contract=off so every float expression is evaluated as
// written (IEEE single, no fused multiply-add).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>

#include "internal.hpp"

namespace virs {

namespace {

std::string dir_of(const std::string &p)
{
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

// newmtl names of an .mtl file, in order
void read_mtl(const std::string &path, std::unordered_map<std::string, int> &ids, int &next)
{
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string tok;
        ss >> tok;
        if (tok == "newmtl") {
            std::string name;
            ss >> name;
            if (!ids.count(name)) ids[name] = next++;
        }
    }
}

} // namespace

// Wavefront OBJ: "v", "f" (v, v/t, v//n, v/t/n, negative = relative),
// "mtllib", "usemtl".  Faces with n > 3 corners are split as a fan
// (0, i, i+1); a face before any usemtl, or with an unknown material name,
// gets material id -1 (the convention of tinyobjloader, which numbers
// materials in the order the .mtl files declare them).
virs_status load_obj(const char *path, Mesh &out)
{
    std::ifstream f(path);
    if (!f) return fail(VIRS_E_IO, std::string("cannot open OBJ file: ") + path);
    out = Mesh();
    std::unordered_map<std::string, int> mat_ids;
    int next_id = 0, cur = -1;
    const std::string base = dir_of(path);
    std::string line;
    size_t lineno = 0;
    std::vector<long> corners;
    while (std::getline(f, line)) {
        ++lineno;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        const char *s = line.c_str();
        while (*s == ' ' || *s == '\t') ++s;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            char *e = nullptr;
            const char *q = s + 2;
            float xyz[3];
            for (int a = 0; a < 3; ++a) {
                const double v = std::strtod(q, &e);
                if (e == q) return fail(VIRS_E_IO, "bad vertex at line " + std::to_string(lineno));
                xyz[a] = (float)v;
                q = e;
            }
            out.verts.insert(out.verts.end(), xyz, xyz + 3);
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            corners.clear();
            const char *q = s + 2;
            while (*q) {
                while (*q == ' ' || *q == '\t') ++q;
                if (!*q) break;
                char *e = nullptr;
                const long v = std::strtol(q, &e, 10);
                if (e == q) return fail(VIRS_E_IO, "bad face at line " + std::to_string(lineno));
                const long nv = (long)(out.verts.size() / 3);
                const long idx = v > 0 ? v - 1 : nv + v;
                if (idx < 0 || idx >= nv) return fail(VIRS_E_IO, "face index out of range at line " + std::to_string(lineno));
                corners.push_back(idx);
                q = e;
                while (*q && *q != ' ' && *q != '\t') ++q; // skip /t/n
            }
            for (size_t i = 1; i + 1 < corners.size(); ++i) {
                out.tris.push_back((uint32_t)corners[0]);
                out.tris.push_back((uint32_t)corners[i]);
                out.tris.push_back((uint32_t)corners[i + 1]);
                out.tri_mat.push_back(cur);
            }
        } else if (!std::strncmp(s, "mtllib", 6)) {
            std::istringstream ss(s + 6);
            std::string name;
            while (ss >> name) read_mtl(base + "/" + name, mat_ids, next_id);
        } else if (!std::strncmp(s, "usemtl", 6)) {
            std::istringstream ss(s + 6);
            std::string name;
            ss >> name;
            auto it = mat_ids.find(name);
            cur = it == mat_ids.end() ? -1 : it->second;
        }
    }
    if (out.tris.empty()) return fail(VIRS_E_IO, std::string("no faces in OBJ file: ") + path);
    return VIRS_OK;
}

// simulator.cpp:288-310; the max corner starts at FLT_MIN as in the reference.
void mesh_bbox(const Mesh &m, float nudge, float bmin[3], float bmax[3])
{
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
    for (size_t i = 0; i + 2 < m.verts.size(); i += 3)
        for (int a = 0; a < 3; ++a) {
            const float v = m.verts[i + a];
            if (v < lo[a]) lo[a] = v;
            if (hi[a] < v) hi[a] = v;
        }
    for (int a = 0; a < 3; ++a) {
        bmin[a] = lo[a] - nudge;
        bmax[a] = hi[a] + nudge;
    }
}

// simulator.cpp:321-329
void grid_dims(const float bmin[3], const float bmax[3], float h, uint64_t dims[3])
{
    const float nvm = 1.f / h;
    for (int a = 0; a < 3; ++a) {
        const float s = (bmax[a] - bmin[a]) * nvm;
        dims[a] = s > 0.f ? (uint64_t)s : 0;
    }
}

} // namespace virs
