#pragma once
#include "tarch/la/Vector.h"
namespace peano { namespace utils {
inline int dLinearisedWithoutLookup(const tarch::la::Vector<DIMENSIONS, int>& c, int max) {
  int r = 0; for (int d = DIMENSIONS - 1; d >= 0; d--) r = r * max + c[d]; return r;
}
}}
