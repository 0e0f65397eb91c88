/* Triangle meshes as Akinci boundary particles (geometry.cpp; the sampling
   runs on the GPU, csrc/sph_mesh.cu). Errors are thrown: std::runtime_error
   for an unreadable file, std::invalid_argument for a malformed mesh,
   StatusError (an SPH status code) for a failure of the device sampler. */
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

namespace sphgeo {

struct StatusError : std::runtime_error {
    int code;
    StatusError(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

/* Vertices (xyz, scaled per axis) and 0-based triangle indices of an OBJ file. */
void load_obj(const std::string& path, const float scale[3], std::vector<float>& verts, std::vector<unsigned>& faces);

/* The column-major 4x4 matrix Rz(Ry(Rx(I))) of glm::rotate about x, y, z. */
void placement(const float rotate_xyz[3], float m16[16]);

/* Regular triangle sampling at spacing max_distance: vertices, interior edge
   stops, interior face stops, in that order; out holds xyz triples. */
void sample_mesh(const float* verts, unsigned nv, const unsigned* faces, unsigned nf, float max_distance,
                 std::vector<float>& out);

/* load_obj + sampling + p <- placement * (p, 1) + translate. */
void sample_geometry(const std::string& path, float max_distance, const float scale[3], const float translate[3],
                     const float rotate_xyz[3], std::vector<float>& out);

} // namespace sphgeo
