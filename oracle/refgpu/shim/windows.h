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
#include <cusparse.h>
#if CUSPARSE_VER_MAJOR >= 12
// removed from cuSPARSE 12; named only by an off-path header (CuSparsePCG.h)
typedef struct csrsv2Info* csrsv2Info_t;
#endif
