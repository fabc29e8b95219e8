// Mesh -> voxel grid on the host (the reference does this on the host too).
//
//   OBJ parsing                 replaces tinyobj::LoadObj at simulator.cpp:279
//   bounding box + nudge        simulator.cpp:288-310
//   grid sizing                 simulator.cpp:321-329
//   toVoxel                     simulator.h:39-45
//   triangle/box SAT test       simulator.cpp:45-141
//   triangle sweep, flags 1/3   simulator.cpp:396-452
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

struct V3 {
    float x, y, z;
};

V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
float min3(float a, float b, float c) { float m = a; if (b < m) m = b; if (c < m) m = c; return m; }
float max3(float a, float b, float c) { float m = a; if (m < b) m = b; if (m < c) m = c; return m; }

// simulator.cpp:73-86; the projection uses the .y and .z components for
// every edge/axis pair, as the reference does.
bool axis_test(float a, float b, float fa, float fb, V3 p0, V3 p1, V3 p2, float ex, float ey)
{
    const float p0p = a * p0.y - b * p0.z;
    const float p1p = a * p1.y - b * p1.z;
    const float p2p = a * p2.y - b * p2.z;
    const float mn = min3(p0p, p1p, p2p), mx = max3(p0p, p1p, p2p);
    const float rad = fa * ey + fb * ex;
    return !(mn > rad || mx < -rad);
}

bool tri_box(V3 v0w, V3 v1w, V3 v2w, V3 lo, V3 hi)
{
    const V3 c = {(lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f};
    const V3 e = {(hi.x - lo.x) * 0.5f, (hi.y - lo.y) * 0.5f, (hi.z - lo.z) * 0.5f};
    const V3 v0 = sub(v0w, c), v1 = sub(v1w, c), v2 = sub(v2w, c);
    const V3 f0 = sub(v1, v0), f1 = sub(v2, v1), f2 = sub(v0, v2);
    const V3 a0 = vabs(f0), a1 = vabs(f1), a2 = vabs(f2);
    if (!axis_test(f0.z, f0.y, a0.z, a0.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis_test(f0.z, f0.x, a0.z, a0.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis_test(f0.y, f0.x, a0.y, a0.x, v0, v1, v2, e.x, e.y)) return false;
    if (!axis_test(f1.z, f1.y, a1.z, a1.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis_test(f1.z, f1.x, a1.z, a1.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis_test(f1.y, f1.x, a1.y, a1.x, v0, v1, v2, e.x, e.y)) return false;
    if (!axis_test(f2.z, f2.y, a2.z, a2.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis_test(f2.z, f2.x, a2.z, a2.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis_test(f2.y, f2.x, a2.y, a2.x, v0, v1, v2, e.x, e.y)) return false;
    float mn = min3(v0.x, v1.x, v2.x), mx = max3(v0.x, v1.x, v2.x);
    if (mn > e.x || mx < -e.x) return false;
    mn = min3(v0.y, v1.y, v2.y); mx = max3(v0.y, v1.y, v2.y);
    if (mn > e.y || mx < -e.y) return false;
    mn = min3(v0.z, v1.z, v2.z); mx = max3(v0.z, v1.z, v2.z);
    if (mn > e.z || mx < -e.z) return false;
    const V3 n = {f0.y * f1.z - f0.z * f1.y, f0.z * f1.x - f0.x * f1.z, f0.x * f1.y - f0.y * f1.x};
    const float d = -(n.x * v0.x + n.y * v0.y + n.z * v0.z);
    const float r = e.x * std::fabs(n.x) + e.y * std::fabs(n.y) + e.z * std::fabs(n.z);
    return !(std::fabs(d) > r);
}

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

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

// simulator.cpp:396-452 with the material-role table.
void voxelize(const Mesh &m, const std::vector<uint8_t> &roles, float h, const float bmin[3], uint64_t nx,
              uint64_t ny, uint64_t nz, uint8_t *flags, uint8_t *wall_mat)
{
    auto vox = [&](uint32_t vi) {
        const float *p = &m.verts[3 * (size_t)vi];
        return V3{(p[0] - bmin[0]) / h, (p[1] - bmin[1]) / h, (p[2] - bmin[2]) / h};
    };
    for (size_t t = 0; t < m.tri_mat.size(); ++t) {
        const int mid = m.tri_mat[t];
        const uint8_t role = (mid >= 0 && (size_t)mid < roles.size()) ? roles[mid] : VIRS_ROLE_IGNORE;
        const V3 g0 = vox(m.tris[3 * t]), g1 = vox(m.tris[3 * t + 1]), g2 = vox(m.tris[3 * t + 2]);
        const int ix0 = clampi((int)std::floor(min3(g0.x, g1.x, g2.x)), 0, (int)nx - 1);
        const int iy0 = clampi((int)std::floor(min3(g0.y, g1.y, g2.y)), 0, (int)ny - 1);
        const int iz0 = clampi((int)std::floor(min3(g0.z, g1.z, g2.z)), 0, (int)nz - 1);
        const int ix1 = clampi((int)std::ceil(max3(g0.x, g1.x, g2.x)), 0, (int)nx - 1);
        const int iy1 = clampi((int)std::ceil(max3(g0.y, g1.y, g2.y)), 0, (int)ny - 1);
        const int iz1 = clampi((int)std::ceil(max3(g0.z, g1.z, g2.z)), 0, (int)nz - 1);
        for (int k = iz0; k <= iz1; ++k)
            for (int j = iy0; j <= iy1; ++j)
                for (int i = ix0; i <= ix1; ++i) {
                    const V3 lo = {(float)i, (float)j, (float)k};
                    const V3 hi = {(float)i + 1.f, (float)j + 1.f, (float)k + 1.f};
                    if (!tri_box(g0, g1, g2, lo, hi)) continue;
                    const size_t idx = ((size_t)k * ny + (size_t)j) * nx + (size_t)i;
                    if (role == VIRS_ROLE_SOURCE) {
                        flags[idx] = 3;
                    } else if (role != VIRS_ROLE_IGNORE) {
                        flags[idx] = 1;
                        wall_mat[idx] = role;
                    }
                }
    }
}

} // namespace virs
