// Host shim that lets the reference's OpenCL C kernel sources compile as C++.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle). The kernel text itself is
// never copied into this repository: oracle/refshim/build.py reads it from the
// reference checkout, substitutes the $PLACEHOLDER$ tokens the way the
// reference's host code does (java/CLUtils.java:325-339 replaceFirst), and
// writes the result under oracle/_ref/, which is not committed.
//
// Substitution choices:
//  - $BLOCK_SIZE$ / $PATCH_SIZE$ become a template parameter, because the
//    kernels size local arrays with it; every ellipse size the oracle needs is
//    instantiated.
//  - Every other placeholder becomes a runtime variable of the same C type the
//    reference's string literal denotes for an FP32 kernel: ints for sizes and
//    float for FILTER_PARAM, THRESHOLD, EPSILON, BLOCK_STD and BLOCK_MEAN. A
//    float variable holds exactly the value Java's Float.toString() prints, so
//    this equals compiling the kernel with f-suffixed literals (FP32 semantics).
//  - get_global_id() reads a thread-local work-item coordinate; the driver
//    loops over work-items with OpenMP.
//  - exp/sqrt/fabs/fmax resolve to the C++ float overloads, as OpenCL's
//    builtins do for float arguments.
#pragma once
#include <cmath>
#include <cstdint>

using std::exp;
using std::fabs;
using std::fmax;
using std::sqrt;

#define global
#define __global
#define __local
#define local

static int RS_W, RS_H, RS_BW, RS_BH, RS_BRW, RS_BRH, RS_D, RS_BZ, RS_BRZ;
static float RS_FILTER, RS_THRESHOLD, RS_EPSILON, RS_BLOCK_STD, RS_BLOCK_MEAN;
static thread_local int rs_gid[3];

static inline int get_global_id(int d) { return rs_gid[d]; }
