/*
 * Triangle meshes (OBJ) as Akinci boundary particles: the host side.
 *
 *   - load_obj restates Utilities::OBJLoader::loadObj
 *     (extern/OBJLoader/OBJLoader.h:31-158) for triangulated meshes:
 *     "v x y z" lines, each coordinate times the per-axis scale; "f" lines
 *     whose first three entries give the position index (1-based) as their
 *     first '/'-separated field; other lines are ignored;
 *   - placement builds AkinciBoundaryObject::sampleGeometry's matrix
 *     (src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:194-208):
 *     glm::rotate(I, rx, X), then (.., ry, Y), then (.., rz, Z), in float
 *     and in glm's operation order (glm/ext/matrix_transform.inl:18-46);
 *   - the sampling itself and the placement of every sample run on the GPU
 *     (csrc/sph_mesh.cu).
 * Compiled with -ffp-contract=off: the matrix entries must round as glm's.
 *
 * Where the reference's behaviour is undefined this code reports an error:
 * an unreadable file, a vertex index outside the mesh or a non-finite
 * coordinate (the reference reads past its vectors or samples NaN).
 */
#include "geometry.h"

#include "../../include/sph2o_cuda.h"
#include "../csrc/sph_mesh.h"

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace sphgeo {
namespace {

struct M4 {
    float m[4][4]; /* columns: m[col][row] */
};

M4 identity()
{
    M4 r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
}

/* glm::rotate(m, angle, axis) */
M4 rotate(const M4& m, float angle, float vx, float vy, float vz)
{
    const float c = std::cos(angle), s = std::sin(angle);
    /* glm::normalize: v * (1 / sqrt(dot(v, v))), glm's dot summed left to right */
    const float inv = 1.0f / std::sqrt(vx * vx + vy * vy + vz * vz);
    const float a[3] = {vx * inv, vy * inv, vz * inv};
    const float t[3] = {(1.0f - c) * a[0], (1.0f - c) * a[1], (1.0f - c) * a[2]};
    float R[3][3];
    R[0][0] = c + t[0] * a[0];
    R[0][1] = t[0] * a[1] + s * a[2];
    R[0][2] = t[0] * a[2] - s * a[1];
    R[1][0] = t[1] * a[0] - s * a[2];
    R[1][1] = c + t[1] * a[1];
    R[1][2] = t[1] * a[2] + s * a[0];
    R[2][0] = t[2] * a[0] + s * a[1];
    R[2][1] = t[2] * a[1] - s * a[0];
    R[2][2] = c + t[2] * a[2];
    M4 r;
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 4; ++k) r.m[j][k] = m.m[0][k] * R[j][0] + m.m[1][k] * R[j][1] + m.m[2][k] * R[j][2];
    for (int k = 0; k < 4; ++k) r.m[3][k] = m.m[3][k];
    return r;
}

/* Position index of one face entry: the first '/'-separated field, read as
   std::stoi reads it */
long face_index(const std::string& tok)
{
    const std::string head = tok.substr(0, tok.find('/'));
    char* end = nullptr;
    const long v = std::strtol(head.c_str(), &end, 10);
    if (end == head.c_str()) throw std::invalid_argument("OBJ face entry without a vertex index: " + tok);
    return v;
}

std::vector<std::string> split_ws(const std::string& s)
{
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r')) ++i;
        size_t j = i;
        while (j < s.size() && s[j] != ' ' && s[j] != '\t' && s[j] != '\r') ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

void check(int rc, const std::string& err)
{
    if (rc != SPH_OK) throw StatusError(rc, err);
}

} // namespace

void load_obj(const std::string& path, const float scale[3], std::vector<float>& verts, std::vector<unsigned>& faces)
{
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot read OBJ file " + path);
    verts.clear();
    faces.clear();
    std::vector<long> raw;
    std::string line;
    while (std::getline(in, line)) {
        const std::vector<std::string> tok = split_ws(line);
        if (tok.empty()) continue;
        if (tok[0] == "v") {
            if (tok.size() < 4) throw std::invalid_argument("OBJ vertex with fewer than three coordinates");
            for (int k = 0; k < 3; ++k) {
                char* end = nullptr;
                const float x = std::strtof(tok[1 + k].c_str(), &end);
                if (end == tok[1 + k].c_str() || !std::isfinite(x))
                    throw std::invalid_argument("OBJ vertex coordinate is not a finite number: " + tok[1 + k]);
                verts.push_back(x * scale[k]);
            }
        } else if (tok[0] == "f") {
            if (tok.size() < 4) throw std::invalid_argument("OBJ face with fewer than three vertices");
            for (int k = 0; k < 3; ++k) raw.push_back(face_index(tok[1 + k]));
        }
    }
    const size_t nv = verts.size() / 3;
    faces.reserve(raw.size());
    for (long r : raw) {
        if (r < 1 || (size_t)r > nv) throw std::invalid_argument("OBJ face index outside the vertex list");
        faces.push_back((unsigned)(r - 1));
    }
}

void placement(const float rotate_xyz[3], float m16[16])
{
    M4 r = rotate(identity(), rotate_xyz[0], 1.0f, 0.0f, 0.0f);
    r = rotate(r, rotate_xyz[1], 0.0f, 1.0f, 0.0f);
    r = rotate(r, rotate_xyz[2], 0.0f, 0.0f, 1.0f);
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 4; ++k) m16[4 * c + k] = r.m[c][k];
}

void sample_mesh(const float* verts, unsigned nv, const unsigned* faces, unsigned nf, float max_distance,
                 std::vector<float>& out)
{
    std::string err;
    check(sph::sample_mesh_device(verts, nv, faces, nf, max_distance, nullptr, nullptr, out, err), err);
}

void sample_geometry(const std::string& path, float max_distance, const float scale[3], const float translate[3],
                     const float rotate_xyz[3], std::vector<float>& out)
{
    std::vector<float> verts;
    std::vector<unsigned> faces;
    load_obj(path, scale, verts, faces);
    float m16[16];
    placement(rotate_xyz, m16);
    std::string err;
    check(sph::sample_mesh_device(verts.data(), (unsigned)(verts.size() / 3), faces.data(),
                                  (unsigned)(faces.size() / 3), max_distance, m16, translate, out, err),
          err);
}

} // namespace sphgeo
