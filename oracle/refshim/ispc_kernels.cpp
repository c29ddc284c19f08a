// Test infrastructure (oracle): C++ restatement of the two ISPC kernels of the
// reference, so that the reference's WideBvh (src/accelerators/wide_bvh.cpp)
// links and runs without `ispc`. Each `foreach` lane becomes one iteration of
// a plain loop; ispc's `min`/`max` are `a < b ? a : b` / `a > b ? a : b`,
// `select(c, a, b)` is `c ? a : b`. Division is IEEE (`1.0f / det`), and the
// whole file is compiled with -ffp-contract=off so every product and sum is
// rounded separately, as in the ispc source.
#include <ispc/bounding_box.h>
#include <ispc/triangle.h>

#include <cmath>

namespace {
// src/ispc/bounding_box.ispc:3  CORRECTION = 1 + 2 * gamma(3)
constexpr float kBoxCorrection = 1.0000004f;
// src/ispc/triangle.ispc:3  EPSILON
constexpr float kDetEpsilon = 1e-6f;

inline float fmin2(float a, float b) { return a < b ? a : b; }
inline float fmax2(float a, float b) { return a > b ? a : b; }

// src/ispc/bounding_box.ispc:15-43
inline bool slabTest(const float* o, const float* inv, float tFar,
    float minX, float minY, float minZ, float maxX, float maxY, float maxZ)
{
    float tx0 = (minX - o[0]) * inv[0];
    float tx1 = (maxX - o[0]) * inv[0];
    float ty0 = (minY - o[1]) * inv[1];
    float ty1 = (maxY - o[1]) * inv[1];
    float tz0 = (minZ - o[2]) * inv[2];
    float tz1 = (maxZ - o[2]) * inv[2];

    float tMin = fmax2(fmax2(fmin2(tx0, tx1), fmin2(ty0, ty1)), fmin2(tz0, tz1));
    float tMax = fmin2(fmin2(fmax2(tx0, tx1), fmax2(ty0, ty1)), fmax2(tz0, tz1));
    tMax *= kBoxCorrection;
    return (tMin <= tMax) & (tMax > 0.0f) & (tMin < tFar);
}
}

namespace ispc {
// src/ispc/bounding_box.ispc:45-61
extern "C" void intersectBoundingBoxN(
    bool* intersects, const float* rayOrg, const float* /*rayDir*/,
    const float* invRayDir, float tFar, const BoundingBoxN& b)
{
    for (int i = 0; i < SIMD_WIDTH; ++i)
    {
        intersects[i] = slabTest(rayOrg, invRayDir, tFar,
            b.minX[i], b.minY[i], b.minZ[i], b.maxX[i], b.maxY[i], b.maxZ[i]);
    }
}

// src/ispc/triangle.ispc:46-87
extern "C" void intersectTriangleN(
    IntersectionN& out, const float* o, const float* d, const TriangleN& tri)
{
    for (int i = 0; i < SIMD_WIDTH; ++i)
    {
        float sx = o[0] - tri.vx[i];
        float sy = o[1] - tri.vy[i];
        float sz = o[2] - tri.vz[i];

        // s1 = d x e1
        float s1x = d[1] * tri.ez1[i] - d[2] * tri.ey1[i];
        float s1y = d[2] * tri.ex1[i] - d[0] * tri.ez1[i];
        float s1z = d[0] * tri.ey1[i] - d[1] * tri.ex1[i];
        // s2 = s x e0
        float s2x = sy * tri.ez0[i] - sz * tri.ey0[i];
        float s2y = sz * tri.ex0[i] - sx * tri.ez0[i];
        float s2z = sx * tri.ey0[i] - sy * tri.ex0[i];

        float det = s1x * tri.ex0[i] + s1y * tri.ey0[i] + s1z * tri.ez0[i];
        bool hit = std::fabs(det) >= kDetEpsilon;

        float rcpDet = 1.0f / det;
        float t = (s2x * tri.ex1[i] + s2y * tri.ey1[i] + s2z * tri.ez1[i]) * rcpDet;
        float b0 = (s1x * sx + s1y * sy + s1z * sz) * rcpDet;
        float b1 = (d[0] * s2x + d[1] * s2y + d[2] * s2z) * rcpDet;

        hit &= t >= 0.0f;
        hit &= (b0 >= 0.0f) & (b1 >= 0.0f) & (b0 + b1 <= 1.0f);

        out.t[i] = hit ? t : NO_INTERSECT;
        out.b0[i] = hit ? b0 : NO_INTERSECT;
        out.b1[i] = hit ? b1 : NO_INTERSECT;
    }
}
}
