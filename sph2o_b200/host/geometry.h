/* Triangle meshes as Akinci boundary particles (geometry.cpp). Errors are
   thrown: std::runtime_error for an unreadable file, std::invalid_argument
   for a malformed mesh, std::length_error above kMaxSamples samples. */
#pragma once

#include <string>
#include <vector>

namespace sphgeo {

/* Upper bound on the samples of one mesh (about 12 GiB of float3). */
constexpr unsigned kMaxSamples = 1u << 30;

/* Vertices (xyz, scaled per axis) and 0-based triangle indices of an OBJ file. */
void load_obj(const std::string& path, const float scale[3], std::vector<float>& verts, std::vector<unsigned>& faces);

/* Regular triangle sampling at spacing max_distance: vertices, interior edge
   stops, interior face stops, in that order; out holds xyz triples. */
void sample_mesh(const float* verts, unsigned nv, const unsigned* faces, unsigned nf, float max_distance,
                 std::vector<float>& out);

/* p <- Rz(Ry(Rx(I))) * (p, 1) + translate, as glm builds and applies it. */
void transform_points(std::vector<float>& pts, const float translate[3], const float rotate_xyz[3]);

/* load_obj + sample_mesh + transform_points. */
void sample_geometry(const std::string& path, float max_distance, const float scale[3], const float translate[3],
                     const float rotate_xyz[3], std::vector<float>& out);

} // namespace sphgeo
