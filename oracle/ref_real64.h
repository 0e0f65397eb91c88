/*
 * Force-included (g++ -include) when oracle/Makefile builds the FP64 variant
 * of the reference. It defines the include guard of the reference's
 * inc/Common/numeric_types.h first, so that header is skipped, and declares
 * the same type names in double precision. The reference sources are
 * compiled unmodified; only Real and the glm vector/matrix types change.
 */
#ifndef _NUMERIC_TYPES_H_
#define _NUMERIC_TYPES_H_

#include <glm/glm.hpp>
#include <glm/gtc/type_ptr.hpp>
#include <glm/gtc/quaternion.hpp>
#include <glm/gtx/compatibility.hpp>
#include <glm/gtx/string_cast.hpp>

typedef double Real;
typedef glm::dvec3 Vector3r;
typedef glm::dvec4 Vector4r;
typedef glm::ivec3 Vector3i;
typedef glm::uvec3 Vector3u;
typedef glm::dmat4 Matrix4r;
typedef glm::dquat Quat4r;

#endif
