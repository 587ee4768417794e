/*
 * Forced-include shim that lets the SolidCloth reference sources (written for
 * MSVC/Win32) compile unchanged with g++ on Linux, for use as a test oracle.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the shipped library includes this.
 *
 * What it papers over:
 *   - Geometry/SDF.h uses std::floorf, which libstdc++ does not declare;
 *   - Physics/ClothPatch.cpp and Physics/ClothModel.cpp include the Win32
 *     Engine/Engine.h only for Printf/rand, so ENGINE_H is pre-defined and the
 *     portable Engine/Types.h + Engine/Utils.h are included instead;
 *   - a few Win32 typedefs, __declspec and fopen_s.
 */
#pragma once

#include <cmath>
#include <cfloat>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <vector>
#include <memory>
#include <stack>
#include <set>
#include <functional>

namespace std { using ::floorf; }

#ifndef LINUX
#define LINUX
#endif
#ifndef DISABLE_PROFILER
#define DISABLE_PROFILER
#endif

#define __declspec(x)

typedef long LONG;
typedef unsigned int UINT;
typedef void* HWND;
typedef unsigned long WPARAM;
typedef long LPARAM;
typedef long LRESULT;
#define CALLBACK
struct POINT { LONG x, y; };

static inline int fopen_s(FILE** f, const char* path, const char* mode)
{
    *f = fopen(path, mode);
    return *f ? 0 : 1;
}

/* Engine/Engine.h is Win32-only; the physics sources need only Utils/Types. */
#define ENGINE_H
#include "Engine/Types.h"
#include "Engine/Utils.h"
