// Test infrastructure (oracle): stand-in for the header that `ispc` generates
// from src/ispc/bounding_box.ispc. `ispc` is not installed, so the exported
// struct and function are declared here by hand with the layout and calling
// convention ispc gives them (uniform arrays -> pointers, references kept), and
// the body is restated in C++ in oracle/refshim/ispc_kernels.cpp.
// Reference: src/ispc/bounding_box.ispc:5-13 (BoundingBoxN), 45-61 (export).
#pragma once

#include <ispc/ispc_config.h>

namespace ispc {
struct BoundingBoxN
{
    float minX[SIMD_WIDTH];
    float minY[SIMD_WIDTH];
    float minZ[SIMD_WIDTH];
    float maxX[SIMD_WIDTH];
    float maxY[SIMD_WIDTH];
    float maxZ[SIMD_WIDTH];
};

extern "C" void intersectBoundingBoxN(
    bool* intersects,
    const float* rayOrg,
    const float* rayDir,
    const float* invRayDir,
    float tFar,
    const BoundingBoxN& bboxN);
}
