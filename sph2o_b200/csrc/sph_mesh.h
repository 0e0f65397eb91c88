/* Regular triangle sampling of a mesh on the current CUDA device
   (sph_mesh.cu); plain host declarations, usable from host-only sources. */
#ifndef SPH2O_MESH_H
#define SPH2O_MESH_H

#include <string>
#include <vector>

namespace sph {

/* vertices (xyz), 0-based faces, spacing d; m16 (NULL: none) is a 4x4
   column-major placement applied to every sample, then `translate` (NULL:
   0). Returns an SPH status; err explains a failure. */
int sample_mesh_device(const float* v, unsigned nv, const unsigned* f, unsigned nf, float d, const float* m16,
                       const float* translate, std::vector<float>& out, std::string& err);

} // namespace sph

#endif
