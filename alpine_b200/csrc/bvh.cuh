// BVH layouts in HBM.
//
// Wide node (80 bytes, five 16-byte words, read with five 128-bit loads):
//   word0: float px, py, pz          quantisation origin = node box minimum
//          u8 ex, ey, ez             biased exponents: child box quantum 2^(e-127)
//          u8 imask                  bit s set <=> slot s holds an internal child
//   word1: u32 childBase             index of the first internal child node
//          u32 triBase               index of the first triangle record
//          u8 meta[8]                per slot: empty = 0;
//                                    internal = 0x20 | (24 + slot);
//                                    leaf = (unary count << 5) | triangle offset
//   word2: u8 qlox[8], qloy[8]       child box minima, in quanta, rounded down
//   word3: u8 qloz[8], qhix[8]
//   word4: u8 qhiy[8], qhiz[8]       child box maxima, in quanta, rounded up
// Internal children are stored contiguously from childBase in slot order, so
// slot s lives at childBase + popc(imask & ((1 << s) - 1)). Leaf children hold
// 1-3 triangles; the triangles of one node are contiguous from triBase (at
// most 24). Slot s is assigned, at build time, to the child whose centroid is
// best aligned with octant corner s of the node (bit k of s set = + side of
// axis k); a ray with direction-sign bits `oct` visits hit children in order
// of (s ^ oct), i.e. roughly front to back.
//
// Triangle record (48 bytes, three 128-bit loads): {v0.xyz, prim id},
// {e0.xyz, 0}, {e1.xyz, 0} with e0 = v1 - v0 and e1 = v2 - v0, the same FP32
// values the reference intersects (src/accelerators/bvh_common.cpp:105-125).
// A sphere (an analytic primitive, Sphere::Data vertices: centre + radius)
// shares the record: {centre.xyz, kSpherePrim | sphere index},
// {radius, 0, 0, tag kSphereTag}, unused; a triangle's e0.w is 0.
#pragma once

#include "common.cuh"

namespace ag {

struct alignas(16) WideNode {
    float px, py, pz;
    uint32_t e_imask;     // ex | ey << 8 | ez << 16 | imask << 24
    uint32_t childBase;
    uint32_t triBase;
    uint32_t meta[2];
    uint32_t qlo[3][2];   // [axis][bytes 0-3, 4-7]
    uint32_t qhi[3][2];
};
static_assert(sizeof(WideNode) == 80, "wide node is 80 bytes");

struct alignas(16) TriRecord {
    float4 v0;   // w = prim id (bits)
    float4 e0;
    float4 e1;
};
static_assert(sizeof(TriRecord) == 48, "triangle record is 48 bytes");

// Binary build node (internal representation of the binned-SAH build).
struct alignas(16) BinNode {
    float3 lo;
    uint32_t begin;     // first primitive reference of the subtree
    float3 hi;
    uint32_t count;     // primitives in the subtree
    int32_t left;       // child node ids, -1 for a leaf
    int32_t right;
    uint32_t pad[2];
};
static_assert(sizeof(BinNode) == 48, "binary node is 48 bytes");

constexpr uint32_t kSpherePrim = 0x80000000u;  // hit / record prim ids of spheres carry this bit
constexpr uint32_t kSphereTag = 1u;            // e0.w bits of a sphere record

constexpr int kWidth = 8;
constexpr int kMaxLeafTris = 3;          // unary count field holds 1..3
constexpr int kSahBins = 32;             // binned SAH resolution
#ifndef AG_TRAVERSAL_STACK
#define AG_TRAVERSAL_STACK 24
#endif
constexpr int kTraversalStack = AG_TRAVERSAL_STACK;  // node-group stack entries per ray
constexpr uint32_t kMaxVisits = 1u << 16;  // default per-ray wide-node visit cap

// Triangle acceptance rule of a traversal: the reference's 8-wide BVH
// (src/ispc/triangle.ispc:46-87) or its binary BVH
// (src/accelerators/bvh_common.cpp:66-103).
constexpr uint32_t kTriTestWide = 0;
constexpr uint32_t kTriTestBinary = 1;

struct BvhView {
    const WideNode* nodes = nullptr;
    const TriRecord* tris = nullptr;
    uint32_t nodeCount = 0;
    uint32_t triCount = 0;
    uint32_t maxVisits = kMaxVisits;                 // a ray fetching more nodes ends with kErrIterations
    uint32_t stackLimit = (uint32_t)kTraversalStack;  // stack entries a ray may use (<= kTraversalStack)
    uint32_t triTest = kTriTestWide;                 // selects the kernel instantiation at launch
};

}  // namespace ag
