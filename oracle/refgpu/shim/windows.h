// Stand-in for the Windows header the reference's Common.h includes: the
// assert macros it uses, the C headers MSVC brings in with it, and an empty
// __declspec.  Test infrastructure for building the reference's own CUDA
// sources on Linux; nothing here changes their arithmetic.
#pragma once
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <algorithm>
#ifndef _ASSERT
#define _ASSERT(e) assert(e)
#endif
#ifndef _ASSERTE
#define _ASSERTE(e) assert(e)
#endif
#ifndef __declspec
#define __declspec(x)
#endif
#if defined(DOUBLE_REAL) && defined(__CUDACC__)
// The FP64 build (-DDOUBLE_REAL): CUDA has no atomicExch for double, which
// BoundaryTool.cu uses to store solid face velocities.  The exchange of the
// 64-bit pattern is the same operation.
__device__ inline double atomicExch(double* a, double v) {
  return __longlong_as_double(
      (long long)atomicExch((unsigned long long*)a, (unsigned long long)__double_as_longlong(v)));
}
#endif
#include <cusparse.h>
#if CUSPARSE_VER_MAJOR >= 12
// removed from cuSPARSE 12; named only by an off-path header (CuSparsePCG.h)
typedef struct csrsv2Info* csrsv2Info_t;
#endif
