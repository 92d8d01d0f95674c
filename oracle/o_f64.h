// Test infrastructure: prelude of the oracle's all-FP64 instance (liboracle64.so).
//
// ORACLE ONLY. The all-FP64 instance is the precision reference for the FP32 path and for the
// FP32 path with the FP64 D^-1 / root-inertia branch (artwgsl.js:192-207, :342): the same
// sequential restatement, with every float variable, vector and buffer element widened to
// double. The build force-includes this file (g++ -include o_f64.h -DORC_F64): it pulls in every
// standard header the oracle uses, keeps the IEEE binary32 type as `f32_t` for the buffer
// boundary, and then widens `float` to `double`. Float literals (1e-6f and the like) keep their
// float32 values, as do the packed statF constants: the two instances differ only in the
// precision of the arithmetic. sin / cos / atan2 (smath_o.h) are evaluated in double already and
// are no longer rounded to float. Words of statF, contacts and rows that carry u32 bits go
// through fbits / bitsf, which the FP64 instance maps to a value conversion to and from binary32
// (exact for every such word: indices, counts, flags and the all-ones sentinel).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

typedef float f32_t;
#define float double
