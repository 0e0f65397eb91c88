/*
 * CPU restatement of SPH2O's triangle mesh sampling -- TEST INFRASTRUCTURE.
 *
 * Only tests/ load this (through libsph2o_oracle.so), as the checker of the
 * GPU sampler in sph2o_b200/csrc/sph_mesh.cu. It restates, operation by
 * operation in float:
 *   - SPH::RegularTriangleSampling::sampleMesh
 *     (extern/RegularTriangleSampling/RegularTriangleSampling.cpp:12-117)
 *     with its default skip flags: every vertex, then the interior stops of
 *     each unique edge (sorted (min, max) pairs) at ceil(l / d) + 1 even
 *     stops, then for each face the interior stops of the interior lines
 *     parallel to its longest edge (ceil(h / d) + 1 lines over the height h,
 *     each at ceil(len / d) + 1 stops);
 *   - the placement of AkinciBoundaryObject::sampleGeometry
 *     (src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:194-210): the 4x4
 *     matrix glm::rotate(I, rx, X), then (.., ry, Y), then (.., rz, Z),
 *     applied to (x, y, z, 1), then the translation.
 * Eigen's fixed-size reductions sum a 3-vector as x + (y + z); glm sums
 * left to right and applies a matrix as (m0 x + m1 y) + (m2 z + m3 w).
 * Compiled with -ffp-contract=off (oracle/Makefile).
 *
 * Parity pinned: tests/test_geometry.py checks its samples bit for bit
 * against the boundary particles the reference itself generated for the
 * OBJ meshes of tests/golden/ (geometry_*.npz, written by make_golden.py).
 *
 * A face whose three vertices coincide adds no face samples (the
 * reference reads uninitialised vectors there).
 */
#include "sph_oracle.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace oracle_mesh {

constexpr unsigned kMaxSamples = 1u << 30;

namespace {

struct F3 {
    float x, y, z;
};

F3 at(const float* v, unsigned i) { return {v[3ull * i], v[3ull * i + 1], v[3ull * i + 2]}; }
F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
/* a + s * d, component by component */
F3 axpy(F3 a, float s, F3 d) { return {a.x + s * d.x, a.y + s * d.y, a.z + s * d.z}; }
/* Eigen's unrolled sum of three terms: x + (y + z) */
float sum3(float a, float b, float c) { return a + (b + c); }
float sqnorm(F3 a) { return sum3(a.x * a.x, a.y * a.y, a.z * a.z); }
float dot(F3 a, F3 b) { return sum3(a.x * b.x, a.y * b.y, a.z * b.z); }

void push(std::vector<float>& out, F3 p)
{
    if (out.size() / 3 >= kMaxSamples) throw std::length_error("mesh sampling exceeds the particle limit");
    out.push_back(p.x);
    out.push_back(p.y);
    out.push_back(p.z);
}

/* ceil(len / d) + 1 stops; lengths so long that the count leaves the
   unsigned range are refused instead of converted */
unsigned stops(float len, float d)
{
    const float q = std::ceil(len / d);
    if (!(q < (float)kMaxSamples)) throw std::length_error("mesh sampling exceeds the particle limit");
    return (unsigned)q + 1u;
}

/* RegularTriangleSampling::uniqueEdges (:96-117): (min, max) index pairs,
   sorted lexicographically, duplicates removed */
std::vector<std::pair<unsigned, unsigned>> unique_edges(unsigned nf, const unsigned* faces)
{
    std::vector<std::pair<unsigned, unsigned>> e;
    e.reserve(3ull * nf);
    for (unsigned t = 0; t < nf; ++t)
        for (unsigned c = 0; c < 3; ++c) {
            const unsigned a = faces[3ull * t + c], b = faces[3ull * t + (c + 1) % 3];
            e.emplace_back(std::min(a, b), std::max(a, b));
        }
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
    return e;
}

/* RegularTriangleSampling::appendEdgeSamples (:25-44), interior stops only;
   a zero-length edge contributes its first vertex once */
void edge_samples(const float* v, const std::vector<std::pair<unsigned, unsigned>>& edges, float d,
                  std::vector<float>& out)
{
    for (const auto& e : edges) {
        const F3 v0 = at(v, e.first);
        const F3 dir = sub(at(v, e.second), v0);
        const float l = std::sqrt(sqnorm(dir));
        const unsigned n = stops(l, d);
        if (n == 1u) {
            push(out, v0);
            continue;
        }
        for (unsigned i = 1; i < n - 1u; ++i) push(out, axpy(v0, (float)i / (float)(n - 1u), dir));
    }
}

/* RegularTriangleSampling::appendFaceSamples (:46-94), interior lines and
   interior stops only */
void face_samples(const float* v, unsigned nf, const unsigned* faces, float d, std::vector<float>& out)
{
    for (unsigned t = 0; t < nf; ++t) {
        const unsigned* f = faces + 3ull * t;
        float l2 = 0.0f;
        F3 v0{}, base{}, to_top{};
        for (unsigned c = 0; c < 3; ++c) {
            const F3 p = at(v, f[c]);
            const F3 e = sub(at(v, f[(c + 1) % 3]), p);
            const float le2 = sqnorm(e);
            if (le2 > l2) { /* strict: the first longest edge wins */
                l2 = le2;
                v0 = p;
                base = e;
                to_top = sub(at(v, f[(c + 2) % 3]), p);
            }
        }
        if (!(l2 > 0.0f)) continue; /* three coincident vertices */
        const float l = std::sqrt(l2);
        const F3 bn{base.x / l, base.y / l, base.z / l};
        const float along = dot(bn, to_top);
        const F3 perp{to_top.x - along * bn.x, to_top.y - along * bn.y, to_top.z - along * bn.z};
        const float h = std::sqrt(sqnorm(perp));
        const unsigned lines = stops(h, d);
        for (unsigned line = 1; line + 1u < lines; ++line) {
            const float alpha = (float)line / (float)(lines - 1u);
            const F3 start = axpy(v0, alpha, to_top);
            const float len = (1.0f - alpha) * l;
            const unsigned n = stops(len, d);
            for (unsigned i = 1; i + 1u < n; ++i) push(out, axpy(start, ((float)i * len) / (float)(n - 1u), bn));
        }
    }
}

/* glm matrices are arrays of columns: m[col][row] */
struct M4 {
    float m[4][4];
};

M4 identity()
{
    M4 r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
}

/* glm::rotate(m, angle, axis) (glm/ext/matrix_transform.inl:18-46) */
M4 rotate(const M4& m, float angle, F3 v)
{
    const float c = std::cos(angle), s = std::sin(angle);
    /* glm::normalize: v * (1 / sqrt(dot(v, v))), glm's dot summed left to right */
    const float inv = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    const F3 a{v.x * inv, v.y * inv, v.z * inv};
    const F3 t{(1.0f - c) * a.x, (1.0f - c) * a.y, (1.0f - c) * a.z};
    float R[3][3];
    R[0][0] = c + t.x * a.x;
    R[0][1] = t.x * a.y + s * a.z;
    R[0][2] = t.x * a.z - s * a.y;
    R[1][0] = t.y * a.x - s * a.z;
    R[1][1] = c + t.y * a.y;
    R[1][2] = t.y * a.z + s * a.x;
    R[2][0] = t.z * a.x + s * a.y;
    R[2][1] = t.z * a.y - s * a.x;
    R[2][2] = c + t.z * a.z;
    M4 r;
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 4; ++k) r.m[j][k] = m.m[0][k] * R[j][0] + m.m[1][k] * R[j][1] + m.m[2][k] * R[j][2];
    for (int k = 0; k < 4; ++k) r.m[3][k] = m.m[3][k];
    return r;
}

/* glm's mat4 * vec4 (glm/detail/type_mat4x4.inl:536-583) with w = 1 */
F3 apply(const M4& m, F3 p)
{
    float o[3];
    for (int k = 0; k < 3; ++k) o[k] = (m.m[0][k] * p.x + m.m[1][k] * p.y) + (m.m[2][k] * p.z + m.m[3][k] * 1.0f);
    return {o[0], o[1], o[2]};
}

} // namespace

void sample_mesh(const float* verts, unsigned nv, const unsigned* faces, unsigned nf, float max_distance,
                 std::vector<float>& out)
{
    if (!(max_distance > 0.0f) || !std::isfinite(max_distance))
        throw std::invalid_argument("mesh sampling distance must be positive and finite");
    for (size_t i = 0; i < 3ull * nf; ++i)
        if (faces[i] >= nv) throw std::invalid_argument("face index outside the vertex list");
    for (size_t i = 0; i < 3ull * nv; ++i)
        if (!std::isfinite(verts[i])) throw std::invalid_argument("non-finite mesh vertex");
    out.clear();
    for (unsigned i = 0; i < nv; ++i) push(out, at(verts, i)); /* appendVertexSamples (:19-23) */
    edge_samples(verts, unique_edges(nf, faces), max_distance, out);
    face_samples(verts, nf, faces, max_distance, out);
}

void transform_points(std::vector<float>& pts, const float translate[3], const float rotate_xyz[3])
{
    M4 r = rotate(identity(), rotate_xyz[0], {1.0f, 0.0f, 0.0f});
    r = rotate(r, rotate_xyz[1], {0.0f, 1.0f, 0.0f});
    r = rotate(r, rotate_xyz[2], {0.0f, 0.0f, 1.0f});
    for (size_t i = 0; i + 2 < pts.size(); i += 3) {
        const F3 p = apply(r, {pts[i], pts[i + 1], pts[i + 2]});
        pts[i] = p.x + translate[0];
        pts[i + 1] = p.y + translate[1];
        pts[i + 2] = p.z + translate[2];
    }
}

} // namespace oracle_mesh

extern "C" int sph_oracle_sample_mesh(const float* vertices, unsigned nv, const unsigned* faces, unsigned nf,
                                      float max_distance, const float rotate_xyz[3], const float translate[3],
                                      float* out, size_t capacity, size_t* count)
{
    try {
        std::vector<float> pts;
        oracle_mesh::sample_mesh(vertices, nv, faces, nf, max_distance, pts);
        if (rotate_xyz || translate) {
            const float zero[3] = {0.0f, 0.0f, 0.0f};
            oracle_mesh::transform_points(pts, translate ? translate : zero, rotate_xyz ? rotate_xyz : zero);
        }
        if (count) *count = pts.size() / 3;
        if (!out) return SPH_OK;
        if (capacity < pts.size() / 3) return SPH_ERR_CAPACITY;
        std::copy(pts.begin(), pts.end(), out);
        return SPH_OK;
    } catch (const std::length_error&) {
        return SPH_ERR_CAPACITY;
    } catch (const std::exception&) {
        return SPH_ERR_ARG;
    }
}
