// Additions to shim.h for the reference's shape-metric kernels
// (cl/kernelGetPatchHu2D.cl, cl/kernelGetHuMap.cl,
// cl/kernelGetPhaseCorrelationMap.cl), which also use double arithmetic,
// trigonometry, pow and min/max.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle).
//
//  - $BW$ and $BH$ become template parameters: these kernels size private
//    and local arrays with them.
//  - pow/cos/sin/min/max resolve to the C++ overloads of the argument type,
//    as OpenCL's builtins do; pow(int, float) (the weight of
//    cl/kernelGetHuMap.cl:141) takes the float overload like OpenCL's
//    implicit conversion does.
#pragma once
#include <algorithm>
#include <cfloat>

#include "shim.h"

using std::cos;
using std::max;
using std::min;
using std::pow;
using std::sin;

static inline float pow(int a, float b) { return std::pow((float)a, b); }

static int RS_PS;  // $PATCH_SIZE$ of the Hu patch kernel (ellipse count K)
