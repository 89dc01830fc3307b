#pragma once
#ifndef DIMENSIONS
#error DIMENSIONS must be defined
#endif
// 2 * DIMENSIONS, the number of faces of a cell (Peano's utils/Globals.h
// provides it; the limiter kernels use it)
#ifndef DIMENSIONS_TIMES_TWO
#define DIMENSIONS_TIMES_TWO (2 * DIMENSIONS)
#endif
