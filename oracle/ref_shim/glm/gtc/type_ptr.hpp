// Stand-in for glm/gtc/type_ptr.hpp (TEST INFRASTRUCTURE ONLY, see ../glm.hpp).
#pragma once
#include "../glm.hpp"
namespace glm {
inline const float* value_ptr(const mat4& m) { return &m[0].x; }
inline const float* value_ptr(const vec3& v) { return &v.x; }
}  // namespace glm
