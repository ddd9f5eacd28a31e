/* Force-included into every reference translation unit built by oracle/ref/build_ref.py.
 * Supplies what the reference's MSVC-oriented sources take for granted on Linux:
 * INT_MAX (Material.hpp), std::powf (the solvers' setConfig) and memcpy_s
 * (ObjectComponents.cpp). */
#pragma once
#ifdef __cplusplus
#include <climits>
#include <cmath>
#include <cstring>
namespace std {
inline float powf(float a, float b) { return ::powf(a, b); }
}
#define memcpy_s(dst, dst_size, src, src_size) memcpy((dst), (src), (src_size))
#endif
