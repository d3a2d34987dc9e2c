// GLSL built-ins of the oracle's restated shader passes.
//
// TEST INFRASTRUCTURE ONLY. Mode 0 (the default) is the host libm: the oracle
// is then pinned bit for bit against the reference's own shaders compiled in
// oracle/_ref, which call libm. Mode 1 is the product library's definition of
// the built-ins (myrt_b200/csrc/glmath.hpp), which its kernels compute: device
// images are then compared with the oracle bit for bit. GLSL itself leaves the
// precision of these functions to the implementation.
#pragma once
#include <cmath>

#include "../myrt_b200/csrc/glmath.hpp"

namespace orc_glsl {
extern int mode;  // 0 = libm, 1 = the library's built-ins (orc_set_glsl_math)
inline float sin(float x) { return mode ? myrt_glmath::sin(x) : std::sin(x); }
inline float cos(float x) { return mode ? myrt_glmath::cos(x) : std::cos(x); }
inline float atan(float x) { return mode ? myrt_glmath::atan(x) : std::atan(x); }
inline float pow(float x, float y) { return mode ? myrt_glmath::pow(x, y) : std::pow(x, y); }
inline float exp(float x) { return mode ? myrt_glmath::exp(x) : std::exp(x); }
}  // namespace orc_glsl
