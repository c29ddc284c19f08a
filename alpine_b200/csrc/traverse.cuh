// Wide-BVH traversal (closest hit and any hit) for one ray per thread.
//
// Semantics follow the reference's wide traversal
// (src/accelerators/wide_bvh.cpp:487-619) and its triangle kernel
// (src/ispc/triangle.ispc:46-87): a hit is accepted when |det| >= 1e-6,
// t >= tmin (0 in the reference), b1 >= 0, b2 >= 0, b1 + b2 <= 1 and
// t < current tmax (the reference's `t >= tNear -> reject`). The triangle
// arithmetic is the reference's, with every product, sum and the reciprocal
// rounded separately (__fmul_rn / __fadd_rn / __frcp_rn), so t, b1 and b2 are
// bit-identical to the reference's FP32 values for the same triangle.
// The binary-BVH rule (kBinary, src/accelerators/bvh_common.cpp:66-103) is
// selectable per launch: |det| >= FLT_EPSILON, t, b1, b2 by IEEE division,
// b1 <= 1 and b2 <= 1 - b1, with the reference's order of tests. Child
// boxes are tested conservatively (quantised boxes are rounded outwards and
// the exit distance is scaled by 1 + 4e-7 as bounding_box.ispc:29 does).
//
// Traversal order: a node group {childBase, hits | imask} holds the pending
// internal children of one node in bits 24-31 (position = slot ^ octant of
// the ray direction, so the lowest bit is the nearest octant), and the
// triangle group {triBase, bits 0-23} the pending triangles. Groups with
// pending children are pushed to a per-thread stack in shared memory.
#pragma once

#include "bvh.cuh"

namespace ag {

constexpr float kBoxExitScale = 1.0000004f;

AG_D float dot_rn(float ax, float ay, float az, float bx, float by, float bz)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

AG_D bool opposite_nonzero(float a, float det)
{
    return ((__float_as_uint(a) ^ __float_as_uint(det)) & 0x80000000u) && a != 0.0f;
}

// Reference ray/triangle test with explicit rounding. Returns true for an
// accepted hit in [tmin, tmax) and writes t, b1, b2.
AG_D bool tri_test(float3 o, float3 d, float4 v0, float4 e0, float4 e1, float tmin, float tmax, float& t,
                   float& b1, float& b2)
{
    float sx = __fsub_rn(o.x, v0.x), sy = __fsub_rn(o.y, v0.y), sz = __fsub_rn(o.z, v0.z);
    float s1x = __fsub_rn(__fmul_rn(d.y, e1.z), __fmul_rn(d.z, e1.y));
    float s1y = __fsub_rn(__fmul_rn(d.z, e1.x), __fmul_rn(d.x, e1.z));
    float s1z = __fsub_rn(__fmul_rn(d.x, e1.y), __fmul_rn(d.y, e1.x));
    float det = dot_rn(s1x, s1y, s1z, e0.x, e0.y, e0.z);
    if (!(fabsf(det) >= 1e-6f)) return false;
    float nb1 = dot_rn(s1x, s1y, s1z, sx, sy, sz);
    // b1 = nb1 * (1/det) >= 0 needs nb1 == 0 or the sign of det (exact).
    if (opposite_nonzero(nb1, det)) return false;
    float s2x = __fsub_rn(__fmul_rn(sy, e0.z), __fmul_rn(sz, e0.y));
    float s2y = __fsub_rn(__fmul_rn(sz, e0.x), __fmul_rn(sx, e0.z));
    float s2z = __fsub_rn(__fmul_rn(sx, e0.y), __fmul_rn(sy, e0.x));
    float nb2 = dot_rn(d.x, d.y, d.z, s2x, s2y, s2z);
    if (opposite_nonzero(nb2, det)) return false;
    float nt = dot_rn(s2x, s2y, s2z, e1.x, e1.y, e1.z);
    if (tmin >= 0.0f && opposite_nonzero(nt, det)) return false;
    float rcp = __frcp_rn(det);
    float tt = __fmul_rn(nt, rcp);
    float u = __fmul_rn(nb1, rcp);
    float v = __fmul_rn(nb2, rcp);
    if (!(tt >= tmin) || !(tt < tmax)) return false;
    if (!(u >= 0.0f) || !(v >= 0.0f) || !(__fadd_rn(u, v) <= 1.0f)) return false;
    t = tt;
    b1 = u;
    b2 = v;
    return true;
}

// The reference binary BVH's Primitive::intersect
// (src/accelerators/bvh_common.cpp:66-103) with explicit rounding: divisions
// instead of one reciprocal, det rejected below FLT_EPSILON, and the tests in
// the reference's order. tmin / tmax bound the accepted t as in tri_test
// (tmin = 0 is the reference's own t >= 0 test); a NaN t is rejected there.
AG_D bool tri_test_binary(float3 o, float3 d, float4 v0, float4 e0, float4 e1, float tmin, float tmax, float& t,
                          float& b1, float& b2)
{
    float sx = __fsub_rn(o.x, v0.x), sy = __fsub_rn(o.y, v0.y), sz = __fsub_rn(o.z, v0.z);
    float s1x = __fsub_rn(__fmul_rn(d.y, e1.z), __fmul_rn(d.z, e1.y));
    float s1y = __fsub_rn(__fmul_rn(d.z, e1.x), __fmul_rn(d.x, e1.z));
    float s1z = __fsub_rn(__fmul_rn(d.x, e1.y), __fmul_rn(d.y, e1.x));
    float det = dot_rn(s1x, s1y, s1z, e0.x, e0.y, e0.z);
    if (fabsf(det) < 1.1920928955078125e-7f) return false;  // FLT_EPSILON
    float s2x = __fsub_rn(__fmul_rn(sy, e0.z), __fmul_rn(sz, e0.y));
    float s2y = __fsub_rn(__fmul_rn(sz, e0.x), __fmul_rn(sx, e0.z));
    float s2z = __fsub_rn(__fmul_rn(sx, e0.y), __fmul_rn(sy, e0.x));
    float tt = __fdiv_rn(dot_rn(s2x, s2y, s2z, e1.x, e1.y, e1.z), det);
    if (tt < 0.0f) return false;
    float u = __fdiv_rn(dot_rn(s1x, s1y, s1z, sx, sy, sz), det);
    if (u < 0.0f || u > 1.0f) return false;
    float v = __fdiv_rn(dot_rn(d.x, d.y, d.z, s2x, s2y, s2z), det);
    if (v < 0.0f || v > __fsub_rn(1.0f, u)) return false;
    if (!(tt >= tmin) || !(tt < tmax)) return false;
    t = tt;
    b1 = u;
    b2 = v;
    return true;
}

// Ray / sphere: the geometric form (the projection of the centre on the
// ray and the squared distance of the ray from it), front hit first, then the
// back hit for a ray starting inside, each accepted in [tmin, tmax).
// Embree's point-sphere intersector (Embree 4.3, the reference's only sphere
// path, src/accelerators/embree.cpp:107-122) publishes this method; it is
// restated here.
AG_D bool sphere_test(float3 o, float3 d, float4 c, float r, float tmin, float tmax, float& t)
{
    const float cx = c.x - o.x, cy = c.y - o.y, cz = c.z - o.z;
    const float rd2 = 1.0f / (d.x * d.x + d.y * d.y + d.z * d.z);
    const float proj = (cx * d.x + cy * d.y + cz * d.z) * rd2;
    const float px = cx - proj * d.x, py = cy - proj * d.y, pz = cz - proj * d.z;
    const float l2 = px * px + py * py + pz * pz;
    const float r2 = r * r;
    if (!(l2 <= r2)) return false;
    const float td = sqrtf((r2 - l2) * rd2);
    const float tf = proj - td, tb = proj + td;
    if (tf >= tmin && tf < tmax) { t = tf; return true; }
    if (tb >= tmin && tb < tmax) { t = tb; return true; }
    return false;
}

struct TraceResult {
    uint32_t prim;
    float t, b1, b2;
};

AG_D float safe_rcp(float d)
{
    float a = fabsf(d) < 1e-20f ? copysignf(1e-20f, d) : d;
    return __frcp_rn(a);
}

AG_D uint4 ldg4(const void* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// Exact float value of byte k of w, by the conversion unit (I2F, XU pipe) or
// by placing the byte under the exponent of 2^23 (PRMT) and subtracting 2^23
// (FADD), which runs on the ALU and FMA pipes. Bit i of AG_CVT_PRMT_MASK
// selects the second form for plane group i (near x, y, z, far x, y, z), so
// the 48 conversions of a node can be split between the pipes.
#ifndef AG_CVT_PRMT_MASK
#define AG_CVT_PRMT_MASK 0x12  // measured best on B200: y planes on ALU + FMA, the rest on XU
#endif
template <int kGroup>
AG_D float byte_to_float(uint32_t w, uint32_t k)
{
    if ((AG_CVT_PRMT_MASK >> kGroup) & 1)
        return __uint_as_float(__byte_perm(w, 0x4b000000u, 0x7440u | k)) - 8388608.0f;
    return float((w >> (8 * k)) & 0xffu);
}

AG_D float max3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
AG_D float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Intersects the 8 child boxes of a node; returns the hit mask (internal
// children at bits 24 + (slot ^ oct), triangles at their offsets).
AG_D uint32_t intersect_children(const uint4& w0, const uint4& w1, const uint4& w2, const uint4& w3, const uint4& w4,
                                 float3 o, float3 id, uint32_t oct, float tmin, float tmax)
{
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t e = w0.w;
    const float sx = __fmul_rn(__uint_as_float((e & 0xffu) << 23), id.x);
    const float sy = __fmul_rn(__uint_as_float(((e >> 8) & 0xffu) << 23), id.y);
    const float sz = __fmul_rn(__uint_as_float(((e >> 16) & 0xffu) << 23), id.z);
    const float ox = __fmul_rn(__fsub_rn(px, o.x), id.x);
    const float oy = __fmul_rn(__fsub_rn(py, o.y), id.y);
    const float oz = __fmul_rn(__fsub_rn(pz, o.z), id.z);
    // near / far planes per axis chosen by the direction sign
    const bool nx = oct & 1u, ny = oct & 2u, nz = oct & 4u;
    const uint32_t nearX[2] = {nx ? w3.z : w2.x, nx ? w3.w : w2.y};
    const uint32_t farX[2] = {nx ? w2.x : w3.z, nx ? w2.y : w3.w};
    const uint32_t nearY[2] = {ny ? w4.x : w2.z, ny ? w4.y : w2.w};
    const uint32_t farY[2] = {ny ? w2.z : w4.x, ny ? w2.w : w4.y};
    const uint32_t nearZ[2] = {nz ? w4.z : w3.x, nz ? w4.w : w3.y};
    const uint32_t farZ[2] = {nz ? w3.x : w4.z, nz ? w3.y : w4.w};
    const uint32_t meta[2] = {w1.z, w1.w};
    uint32_t hits = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            float tnx = fmaf(byte_to_float<0>(nearX[h], k), sx, ox);
            float tny = fmaf(byte_to_float<1>(nearY[h], k), sy, oy);
            float tnz = fmaf(byte_to_float<2>(nearZ[h], k), sz, oz);
            float tfx = fmaf(byte_to_float<3>(farX[h], k), sx, ox);
            float tfy = fmaf(byte_to_float<4>(farY[h], k), sy, oy);
            float tfz = fmaf(byte_to_float<5>(farZ[h], k), sz, oz);
            float tn = max3f(tnx, tny, fmaxf(tnz, tmin));
            float tf = min3f(tfx, tfy, tfz) * kBoxExitScale;
            if (tn <= tf && tn <= tmax) {
                uint32_t m = (meta[h] >> (8 * k)) & 0xffu;
                uint32_t low = m & 0x1fu;
                uint32_t pos = low >= 24u ? (low ^ oct) : low;
                hits |= (m >> 5) << pos;
            }
        }
    }
    return hits;
}

// Traversal state of one ray (kept in registers; the stack is in shared memory).
struct RayState {
    float3 o, d, id;
    float tmin, tmax;
    uint32_t oct;
    uint2 ngroup, tgroup;
    int sp;
    uint32_t visits;
    TraceResult res;
    bool found;
};

AG_D void ray_init(RayState& s, float3 o, float3 d, float tmin, float tmax)
{
    s.o = o;
    s.d = d;
    s.id = mk3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    s.tmin = tmin;
    s.tmax = tmax;
    s.oct = (s.id.x < 0.0f ? 1u : 0u) | (s.id.y < 0.0f ? 2u : 0u) | (s.id.z < 0.0f ? 4u : 0u);
    s.ngroup = make_uint2(0u, (1u << (24u + s.oct)) | 1u);  // the root as slot 0 of a virtual parent
    s.tgroup = make_uint2(0u, 0u);
    s.sp = 0;
    s.visits = 0;
    s.res.prim = 0xffffffffu;
    s.res.t = 3.402823466e38f;
    s.res.b1 = 0.0f;
    s.res.b2 = 0.0f;
    s.found = false;
}

// One traversal step: tests the pending triangles, then fetches and
// intersects the next node. Returns true when the ray is finished (s.found
// tells whether it hit; on a device-side error the ray ends as a miss).
// stack: this thread's first entry in shared memory, entries `stride` apart.
// nodeVisits / triVisits count wide nodes fetched and triangles tested (the
// reference's BvhStats counters, src/accelerators/bvh_common.h:19-61).
template <bool kAny, bool kBinary = false>
AG_D bool ray_step(const BvhView& bvh, RayState& s, uint2* stack, int stride, uint32_t& err, uint32_t& nodeVisits,
                   uint32_t& triVisits)
{
    // all pending triangles before the next node (measured on B200: testing
    // at most 1, 2 or 4 per step is 25-30 % slower)
    while (s.tgroup.y != 0u) {
        uint32_t k = __ffs(s.tgroup.y) - 1u;
        s.tgroup.y &= s.tgroup.y - 1u;
        uint32_t ti = s.tgroup.x + k;
        if (ti >= bvh.triCount) { err |= kErrBadIndex; s.found = false; return true; }
        ++triVisits;
        const TriRecord* r = bvh.tris + ti;
        float4 v0 = __ldg(&r->v0), e0 = __ldg(&r->e0), e1 = __ldg(&r->e1);
        float t, b1, b2;
        bool accepted;
        if (__float_as_uint(e0.w) == kSphereTag) {
            accepted = sphere_test(s.o, s.d, v0, e0.x, s.tmin, s.tmax, t);
            b1 = b2 = 0.0f;
        } else {
            accepted = kBinary ? tri_test_binary(s.o, s.d, v0, e0, e1, s.tmin, s.tmax, t, b1, b2)
                               : tri_test(s.o, s.d, v0, e0, e1, s.tmin, s.tmax, t, b1, b2);
        }
        if (accepted) {
            s.res.prim = __float_as_uint(v0.w);
            s.res.t = t;
            s.res.b1 = b1;
            s.res.b2 = b2;
            s.found = true;
            if (kAny) return true;
            s.tmax = t;
        }
    }
    if ((s.ngroup.y & 0xff000000u) == 0u) {
        if (s.sp == 0) return true;
        s.ngroup = stack[--s.sp * stride];
    }
    uint32_t p = __ffs(s.ngroup.y >> 24) - 1u;
    s.ngroup.y &= ~(1u << (24u + p));
    uint32_t slot = p ^ s.oct;
    uint32_t child = s.ngroup.x + __popc(s.ngroup.y & 0xffu & ((1u << slot) - 1u));
    if (s.ngroup.y & 0xff000000u) {
        if (s.sp >= (int)bvh.stackLimit) { err |= kErrStackOverflow; s.found = false; return true; }
        stack[s.sp++ * stride] = s.ngroup;
    }
    if (child >= bvh.nodeCount) { err |= kErrBadIndex; s.found = false; return true; }
    if (++s.visits > bvh.maxVisits) { err |= kErrIterations; s.found = false; return true; }
    ++nodeVisits;
    const uint4* np = reinterpret_cast<const uint4*>(bvh.nodes + child);
    uint4 w0 = ldg4(np), w1 = ldg4(np + 1), w2 = ldg4(np + 2), w3 = ldg4(np + 3), w4 = ldg4(np + 4);
    uint32_t hits = intersect_children(w0, w1, w2, w3, w4, s.o, s.id, s.oct, s.tmin, s.tmax);
    s.ngroup = make_uint2(w1.x, (hits & 0xff000000u) | (w0.w >> 24));
    s.tgroup = make_uint2(w1.y, hits & 0x00ffffffu);
    return false;
}

// Traces one ray to completion. Returns true when something was hit
// (closest: res filled; any: the first hit found).
template <bool kAny, bool kBinary = false>
AG_D bool trace(const BvhView& bvh, float3 o, float3 d, float tmin, float tmax, TraceResult& res, uint2* stack,
                int stride, uint32_t& err, uint32_t& nodeVisits, uint32_t& triVisits)
{
    RayState s;
    ray_init(s, o, d, tmin, tmax);
    if (bvh.nodeCount != 0) {
        while (!ray_step<kAny, kBinary>(bvh, s, stack, stride, err, nodeVisits, triVisits)) {
        }
    }
    if (!s.found) {
        s.res.prim = 0xffffffffu;
        s.res.t = 3.402823466e38f;
        s.res.b1 = 0.0f;
        s.res.b2 = 0.0f;
    }
    res = s.res;
    return s.found;
}

}  // namespace ag
