/* Build shim: the one helper of FlowLB's src/math/math.h that the solver path
 * uses (cudaInitData.cu), without the glm dependency of the full header. */
#pragma once
#include <cmath>
namespace FLB::Math {
template <typename T>
bool essentiallyEqual(T a, T b, T epsilon) { return std::abs(a - b) <= epsilon; }
}
