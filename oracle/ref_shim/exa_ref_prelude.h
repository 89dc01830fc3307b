/* Pre-included into every translation unit of the reference build
 * (oracle/_ref, test infrastructure).  libstdc++ 13 has no function
 * template std::abs, but the reference passes std::abs<double> as a
 * functor (kernels/aderdg/generic/c/3d/riemannSolverNonlinear.cpph:77-78),
 * so provide one; ordinary std::abs(x) calls still bind the non-template
 * overloads. */
#pragma once
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <sstream>
#include <string>
namespace std {
template <typename T> inline T abs(T x) { return x < T(0) ? -x : x; }
}
