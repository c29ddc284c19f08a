// Test infrastructure (oracle): stand-in for the header that `ispc` generates
// from src/ispc/triangle.ispc (ispc is not installed). Layout of the exported
// structs follows src/ispc/triangle.ispc:5-25; the body is restated in C++ in
// oracle/refshim/ispc_kernels.cpp.
#pragma once

#include <ispc/ispc_config.h>

namespace ispc {
struct IntersectionN
{
    float t[SIMD_WIDTH];
    float b0[SIMD_WIDTH];
    float b1[SIMD_WIDTH];
};

struct TriangleN
{
    float vx[SIMD_WIDTH];
    float vy[SIMD_WIDTH];
    float vz[SIMD_WIDTH];
    float ex0[SIMD_WIDTH];
    float ey0[SIMD_WIDTH];
    float ez0[SIMD_WIDTH];
    float ex1[SIMD_WIDTH];
    float ey1[SIMD_WIDTH];
    float ez1[SIMD_WIDTH];
};

extern "C" void intersectTriangleN(
    IntersectionN& isects,
    const float* rayOrg,
    const float* rayDir,
    const TriangleN& triN);
}
