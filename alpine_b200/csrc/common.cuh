// Shared device/host helpers for the alpine_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#define AG_HD __host__ __device__ __forceinline__
#define AG_D __device__ __forceinline__

namespace ag {

// ---------------------------------------------------------------------------
// Error reporting from device code. Kernels never trap: a failed check sets a
// bit in a device status word and the host turns it into an error code.
enum DeviceError : uint32_t {
    kErrNone = 0,
    kErrStackOverflow = 1u << 0,   // traversal stack deeper than its capacity
    kErrBadIndex = 1u << 1,        // child/triangle index outside the arrays
    kErrIterations = 1u << 2,      // traversal visit cap reached
    kErrBuildDepth = 1u << 3,      // BVH build exceeded its level cap
    kErrQueueOverflow = 1u << 4,   // wavefront queue full
    kErrTensorWait = 1u << 5,      // a tensor-core (tcgen05) completion wait ran out
};

// ---------------------------------------------------------------------------
// Minimal float3 math.
AG_HD float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
AG_HD float3 operator+(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
AG_HD float3 operator-(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
AG_HD float3 operator-(float3 a) { return mk3(-a.x, -a.y, -a.z); }
AG_HD float3 operator*(float3 a, float3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
AG_HD float3 operator*(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
AG_HD float3 operator*(float s, float3 a) { return mk3(a.x * s, a.y * s, a.z * s); }
AG_HD float3 operator/(float3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
AG_HD float3 operator/(float3 a, float3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
AG_HD float3& operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
AG_HD float3& operator*=(float3& a, float3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
AG_HD float3& operator*=(float3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
AG_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AG_HD float3 cross(float3 a, float3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
AG_HD float3 fmin3(float3 a, float3 b) { return mk3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
AG_HD float3 fmax3(float3 a, float3 b) { return mk3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
AG_HD float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
AG_HD float maxc(float3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }

// Surface area of a box given its extent, as BoundingBox::computeSurfaceArea
// (src/utils/bounding_box.h:13-17).
AG_HD float half_area(float3 e) { return e.x * e.y + e.y * e.z + e.z * e.x; }

// ---------------------------------------------------------------------------
// Order-preserving float <-> uint32 mapping, so that atomicMin/atomicMax on
// unsigned words implement float min/max (exact, order independent).
AG_HD uint32_t f2ord(float f)
{
#ifdef __CUDA_ARCH__
    uint32_t b = __float_as_uint(f);
#else
    uint32_t b;
    __builtin_memcpy(&b, &f, 4);
#endif
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
AG_HD float ord2f(uint32_t u)
{
    uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    __builtin_memcpy(&f, &b, 4);
    return f;
#endif
}

// ---------------------------------------------------------------------------
// Warp helpers.
AG_D uint32_t lane_id() { return threadIdx.x & 31u; }
AG_D uint32_t lanemask_lt()
{
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace ag
