/* Test infrastructure (oracle). CPU restatement, in plain C, of the reference
 * semantics of the traversal hot path. Only tests, smoke() and bench.py's CPU
 * baseline call it; the product never does.
 *
 * Ray layout everywhere: 8 floats {ox, oy, oz, tmin, dx, dy, dz, tmax}.
 * Triangle layout: 9 floats {v0.xyz, e0.xyz, e1.xyz} with e0 = v1 - v0,
 * e1 = v2 - v0, exactly the FP32 values the reference stores
 * (src/accelerators/bvh_common.cpp:105-125).
 * Hit layout: prim (uint32, 0xffffffff on miss), t, b1, b2 (b1, b2 are the
 * barycentrics of v1 and v2: src/shapes/mesh.cpp:61-63).
 */
#ifndef ALPINE_ORACLE_H
#define ALPINE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Semantics selector for the ray/triangle test. */
enum {
    ORC_TRI_ISPC = 0, /* src/ispc/triangle.ispc:46-87 (|det| >= 1e-6, rcp-multiply) */
    ORC_TRI_PRIM = 1  /* src/accelerators/bvh_common.cpp:66-103 (|det| >= FLT_EPSILON, divide) */
};

int orc_tri_test(int sem, const float* ray, const float* tri, float* t, float* b1, float* b2);

/* Slab tests. box: {minx, miny, minz, maxx, maxy, maxz}. inv: 1/dir. */
int orc_box_ispc(const float* org, const float* inv, float tfar, const float* box); /* bounding_box.ispc:15-43 */
int orc_box_ref(const float* org, const float* inv, float tfar, const float* box);  /* bounding_box.h:23-56 */

/* FP64 Moller-Trumbore on the FP32 triangle record. Returns 1 when the ray
 * plane intersection is finite; writes t, b1, b2 and, in cond[3], the forward
 * error scale of the FP32 evaluation of t, b1 and b2 (sum of absolute products
 * divided by |det|). An FP32 evaluation of the same formula is expected within
 * ORC_ULP_BOUND * FLT_EPSILON * cond[k] of the FP64 value. */
#define ORC_ULP_BOUND 16.0
int orc_tri_fp64(const float* ray, const float* tri, double* t, double* b1, double* b2, double* cond);

/* Canonical closest hit: minimal t in [tmin, tmax), ties broken by the lowest
 * primitive index. ntie[i] = number of primitives with exactly that t. */
void orc_closest_brute(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris,
                       uint32_t* prim, float* t, float* b1, float* b2, uint32_t* ntie);
/* Any hit in [tmin, tmax). */
void orc_any_brute(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris,
                   uint8_t* occluded);

/* The same canonical queries accelerated by a conservative CPU BVH (median
 * split, double-precision padded boxes), for inputs too large for brute force.
 * nthreads <= 0 uses all cores. */
void* orc_bvh_create(const float* tris, uint32_t ntris);
void orc_bvh_closest(void* h, int sem, const float* rays, uint64_t nrays, int nthreads,
                     uint32_t* prim, float* t, float* b1, float* b2, uint32_t* ntie);
void orc_bvh_any(void* h, int sem, const float* rays, uint64_t nrays, int nthreads, uint8_t* occluded);
void orc_bvh_destroy(void* h);

/* Re-evaluates ray i against triangle prim[i] (skipped when prim[i] is
 * 0xffffffff): hit[i] = 1 when accepted in [tmin, tmax) with t/b1/b2 written.
 * Used to verify every reported hit of a large query exactly. */
void orc_tri_test_batch(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris,
                        const uint32_t* prim, uint8_t* hit, float* t, float* b1, float* b2);

/* Triangle records from an indexed mesh (bvh_common.cpp:105-125). */
void orc_make_tris(const float* verts, const uint32_t* idx, uint32_t ntris, float* tris);

#ifdef __cplusplus
}
#endif
#endif
