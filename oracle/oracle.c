/* Test infrastructure (oracle): plain-C restatement of the reference's
 * ray/box/triangle semantics and canonical closest/any-hit queries.
 * See oracle.h for layouts. Compiled with -ffp-contract=off: every FP32 product
 * and sum is rounded separately, as in the reference sources.
 * Used only by tests, smoke() and bench.py's CPU baseline. */
#define _GNU_SOURCE
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------- */
/* Ray/triangle tests                                                         */

/* src/ispc/triangle.ispc:46-87 and src/accelerators/bvh_common.cpp:66-103.
 * Both evaluate s = o - v0, s1 = d x e1, s2 = s x e0, det = s1.e0,
 * t = s2.e1 / det, b1 = s1.s / det, b2 = d.s2 / det; they differ in the det
 * threshold (1e-6 vs FLT_EPSILON), in rcp-multiply vs divide, and in the order
 * of the rejection tests (which does not change the accepted set). */
int
orc_tri_test(int sem, const float* ray, const float* tri, float* tout, float* b1out, float* b2out)
{
    const float ox = ray[0], oy = ray[1], oz = ray[2], tmin = ray[3];
    const float dx = ray[4], dy = ray[5], dz = ray[6], tmax = ray[7];
    const float vx = tri[0], vy = tri[1], vz = tri[2];
    const float ax = tri[3], ay = tri[4], az = tri[5]; /* e0 */
    const float bx = tri[6], by = tri[7], bz = tri[8]; /* e1 */

    float sx = ox - vx, sy = oy - vy, sz = oz - vz;
    float s1x = dy * bz - dz * by;
    float s1y = dz * bx - dx * bz;
    float s1z = dx * by - dy * bx;
    float s2x = sy * az - sz * ay;
    float s2y = sz * ax - sx * az;
    float s2z = sx * ay - sy * ax;
    float det = s1x * ax + s1y * ay + s1z * az;
    float num_t = s2x * bx + s2y * by + s2z * bz;
    float num_b1 = s1x * sx + s1y * sy + s1z * sz;
    float num_b2 = dx * s2x + dy * s2y + dz * s2z;
    float t, b1, b2;

    if (sem == ORC_TRI_ISPC) {
        if (!(fabsf(det) >= 1e-6f)) return 0;
        float rcp = 1.0f / det;
        t = num_t * rcp;
        b1 = num_b1 * rcp;
        b2 = num_b2 * rcp;
        if (!(t >= 0.0f)) return 0;
        if (!((b1 >= 0.0f) & (b2 >= 0.0f) & (b1 + b2 <= 1.0f))) return 0;
    } else {
        if (fabsf(det) < FLT_EPSILON) return 0;
        t = num_t / det;
        if (t < 0.0f) return 0;
        b1 = num_b1 / det;
        if (b1 < 0.0f || b1 > 1.0f) return 0;
        b2 = num_b2 / det;
        if (b2 < 0.0f || b2 > 1.0f - b1) return 0;
    }
    /* tmin / tmax extend the reference (which has t >= 0 and tFar): with
     * tmin = 0 the lower bound is the reference's own t >= 0 test. */
    if (!(t >= tmin) || !(t < tmax)) return 0;
    *tout = t;
    *b1out = b1;
    *b2out = b2;
    return 1;
}

/* ------------------------------------------------------------------------- */
/* Slab tests                                                                 */

static inline float mn(float a, float b) { return a < b ? a : b; }
static inline float mx(float a, float b) { return a > b ? a : b; }

/* src/ispc/bounding_box.ispc:15-43 */
int
orc_box_ispc(const float* o, const float* inv, float tfar, const float* b)
{
    float tx0 = (b[0] - o[0]) * inv[0], tx1 = (b[3] - o[0]) * inv[0];
    float ty0 = (b[1] - o[1]) * inv[1], ty1 = (b[4] - o[1]) * inv[1];
    float tz0 = (b[2] - o[2]) * inv[2], tz1 = (b[5] - o[2]) * inv[2];
    float tmn = mx(mx(mn(tx0, tx1), mn(ty0, ty1)), mn(tz0, tz1));
    float tmx = mn(mn(mx(tx0, tx1), mx(ty0, ty1)), mx(tz0, tz1));
    tmx *= 1.0000004f;
    return (tmn <= tmx) & (tmx > 0.0f) & (tmn < tfar);
}

/* src/utils/bounding_box.h:23-56 (correction = 1 + 2 * gamma(3)) */
int
orc_box_ref(const float* o, const float* inv, float tfar, const float* b)
{
    const float eps = 0.5f * FLT_EPSILON;
    const float g3 = (3.0f * eps) / (1.0f - 3.0f * eps);
    const float corr = 1.0f + 2.0f * g3;
    float tMin = ((inv[0] >= 0.0f ? b[0] : b[3]) - o[0]) * inv[0];
    float tMax = ((inv[0] >= 0.0f ? b[3] : b[0]) - o[0]) * inv[0];
    tMax *= corr;
    float tyMin = ((inv[1] >= 0.0f ? b[1] : b[4]) - o[1]) * inv[1];
    float tyMax = ((inv[1] >= 0.0f ? b[4] : b[1]) - o[1]) * inv[1];
    tyMax *= corr;
    if (tMin > tyMax || tMax < tyMin) return 0;
    tMin = tMin > tyMin ? tMin : tyMin;
    tMax = tMax < tyMax ? tMax : tyMax;
    float tzMin = ((inv[2] >= 0.0f ? b[2] : b[5]) - o[2]) * inv[2];
    float tzMax = ((inv[2] >= 0.0f ? b[5] : b[2]) - o[2]) * inv[2];
    tzMax *= corr;
    if (tMin > tzMax || tMax < tzMin) return 0;
    tMin = tMin > tzMin ? tMin : tzMin;
    tMax = tMax < tzMax ? tMax : tzMax;
    return tMin < tfar && tMax > 0.0f;
}

/* ------------------------------------------------------------------------- */
/* FP64 Moller-Trumbore with forward-error scales                             */

int
orc_tri_fp64(const float* ray, const float* tri, double* t, double* b1, double* b2, double* cond)
{
    double o[3] = {ray[0], ray[1], ray[2]}, d[3] = {ray[4], ray[5], ray[6]};
    double v[3] = {tri[0], tri[1], tri[2]}, a[3] = {tri[3], tri[4], tri[5]}, b[3] = {tri[6], tri[7], tri[8]};
    double s[3] = {o[0] - v[0], o[1] - v[1], o[2] - v[2]};
    double s1[3] = {d[1] * b[2] - d[2] * b[1], d[2] * b[0] - d[0] * b[2], d[0] * b[1] - d[1] * b[0]};
    double s2[3] = {s[1] * a[2] - s[2] * a[1], s[2] * a[0] - s[0] * a[2], s[0] * a[1] - s[1] * a[0]};
    /* magnitudes of the terms of each product, for the error scale */
    double s1a[3] = {fabs(d[1] * b[2]) + fabs(d[2] * b[1]), fabs(d[2] * b[0]) + fabs(d[0] * b[2]),
                     fabs(d[0] * b[1]) + fabs(d[1] * b[0])};
    double sa[3] = {fabs(o[0]) + fabs(v[0]), fabs(o[1]) + fabs(v[1]), fabs(o[2]) + fabs(v[2])};
    double s2a[3] = {sa[1] * fabs(a[2]) + sa[2] * fabs(a[1]), sa[2] * fabs(a[0]) + sa[0] * fabs(a[2]),
                     sa[0] * fabs(a[1]) + sa[1] * fabs(a[0])};
    double det = s1[0] * a[0] + s1[1] * a[1] + s1[2] * a[2];
    if (det == 0.0) return 0;
    double ad = fabs(det);
    double detA = s1a[0] * fabs(a[0]) + s1a[1] * fabs(a[1]) + s1a[2] * fabs(a[2]);
    *t = (s2[0] * b[0] + s2[1] * b[1] + s2[2] * b[2]) / det;
    *b1 = (s1[0] * s[0] + s1[1] * s[1] + s1[2] * s[2]) / det;
    *b2 = (d[0] * s2[0] + d[1] * s2[1] + d[2] * s2[2]) / det;
    double tA = s2a[0] * fabs(b[0]) + s2a[1] * fabs(b[1]) + s2a[2] * fabs(b[2]);
    double b1A = s1a[0] * sa[0] + s1a[1] * sa[1] + s1a[2] * sa[2];
    double b2A = fabs(d[0]) * s2a[0] + fabs(d[1]) * s2a[1] + fabs(d[2]) * s2a[2];
    /* relative error of num/det is bounded by (|num terms| + |q| |det terms|) / |det| */
    cond[0] = (tA + fabs(*t) * detA) / ad;
    cond[1] = (b1A + fabs(*b1) * detA) / ad;
    cond[2] = (b2A + fabs(*b2) * detA) / ad;
    return 1;
}

void
orc_tri_test_batch(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris,
                   const uint32_t* prim, uint8_t* hit, float* t, float* b1, float* b2)
{
    for (uint64_t i = 0; i < nrays; ++i) {
        hit[i] = 0;
        t[i] = FLT_MAX;
        b1[i] = b2[i] = 0.0f;
        if (prim[i] == 0xffffffffu || prim[i] >= ntris) continue;
        float r[8];
        memcpy(r, rays + 8 * i, sizeof r);
        r[7] = FLT_MAX;
        hit[i] = (uint8_t)orc_tri_test(sem, r, tris + 9 * (uint64_t)prim[i], &t[i], &b1[i], &b2[i]);
    }
}

/* ------------------------------------------------------------------------- */
/* Brute force canonical queries                                              */

void
orc_make_tris(const float* verts, const uint32_t* idx, uint32_t ntris, float* tris)
{
    for (uint32_t i = 0; i < ntris; ++i) {
        const float* p0 = verts + 3 * (uint64_t)idx[3 * i];
        const float* p1 = verts + 3 * (uint64_t)idx[3 * i + 1];
        const float* p2 = verts + 3 * (uint64_t)idx[3 * i + 2];
        float* r = tris + 9 * (uint64_t)i;
        for (int k = 0; k < 3; ++k) {
            r[k] = p0[k];
            r[3 + k] = p1[k] - p0[k];
            r[6 + k] = p2[k] - p0[k];
        }
    }
}

static inline void
consider(int sem, const float* ray, const float* tri, uint32_t id,
         uint32_t* bp, float* bt, float* bb1, float* bb2, uint32_t* nt)
{
    float t, b1, b2;
    float r[8];
    memcpy(r, ray, sizeof r);
    r[7] = FLT_MAX; /* ties at the current best must still be seen */
    if (!orc_tri_test(sem, r, tri, &t, &b1, &b2)) return;
    if (!(t < ray[7])) return;
    if (t < *bt || *bp == 0xffffffffu) {
        *bt = t; *bp = id; *bb1 = b1; *bb2 = b2; *nt = 1;
    } else if (t == *bt) {
        *nt += 1;
        if (id < *bp) { *bp = id; *bb1 = b1; *bb2 = b2; }
    }
}

void
orc_closest_brute(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris,
                  uint32_t* prim, float* t, float* b1, float* b2, uint32_t* ntie)
{
    for (uint64_t i = 0; i < nrays; ++i) {
        uint32_t bp = 0xffffffffu, nt = 0;
        float bt = FLT_MAX, bb1 = 0.0f, bb2 = 0.0f;
        const float* r = rays + 8 * i;
        for (uint32_t k = 0; k < ntris; ++k) consider(sem, r, tris + 9 * (uint64_t)k, k, &bp, &bt, &bb1, &bb2, &nt);
        prim[i] = bp; t[i] = bp == 0xffffffffu ? FLT_MAX : bt; b1[i] = bb1; b2[i] = bb2;
        if (ntie) ntie[i] = nt;
    }
}

void
orc_any_brute(int sem, const float* rays, uint64_t nrays, const float* tris, uint32_t ntris, uint8_t* occ)
{
    for (uint64_t i = 0; i < nrays; ++i) {
        const float* r = rays + 8 * i;
        uint8_t hit = 0;
        for (uint32_t k = 0; k < ntris && !hit; ++k) {
            float t, b1, b2;
            hit = (uint8_t)orc_tri_test(sem, r, tris + 9 * (uint64_t)k, &t, &b1, &b2);
        }
        occ[i] = hit;
    }
}

/* ------------------------------------------------------------------------- */
/* Conservative CPU BVH (oracle-only acceleration; any correct structure gives
 * the same canonical answers because boxes are padded and ties are explored) */

typedef struct {
    double lo[3], hi[3];
    uint32_t left, right; /* right == 0 => leaf covering [left, left + count) */
    uint32_t count;
} onode;

typedef struct {
    const float* tris;
    uint32_t ntris;
    uint32_t* order;
    float* cent;
    onode* nodes;
    uint32_t nnodes;
} obvh;

static void
tri_bounds(const float* tr, double* lo, double* hi)
{
    for (int k = 0; k < 3; ++k) {
        double a = tr[k], b = (double)tr[k] + tr[3 + k], c = (double)tr[k] + tr[6 + k];
        double l = a < b ? a : b; l = l < c ? l : c;
        double h = a > b ? a : b; h = h > c ? h : c;
        double pad = 1e-6 * (h - l) + 1e-7 * (fabs(l) + fabs(h)) + 1e-12;
        lo[k] = l - pad; hi[k] = h + pad;
    }
}

static uint64_t
spread3(uint64_t x)
{
    x &= 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

static const uint64_t* g_sort_keys;
static int
cmp_key(const void* a, const void* b)
{
    uint64_t ka = g_sort_keys[*(const uint32_t*)a], kb = g_sort_keys[*(const uint32_t*)b];
    if (ka != kb) return ka < kb ? -1 : 1;
    return *(const uint32_t*)a < *(const uint32_t*)b ? -1 : 1;
}

static uint32_t
obuild(obvh* b, uint32_t begin, uint32_t end)
{
    uint32_t id = b->nnodes++;
    onode* n = &b->nodes[id];
    for (int k = 0; k < 3; ++k) { n->lo[k] = DBL_MAX; n->hi[k] = -DBL_MAX; }
    for (uint32_t i = begin; i < end; ++i) {
        double lo[3], hi[3];
        tri_bounds(b->tris + 9 * (uint64_t)b->order[i], lo, hi);
        for (int k = 0; k < 3; ++k) {
            if (lo[k] < n->lo[k]) n->lo[k] = lo[k];
            if (hi[k] > n->hi[k]) n->hi[k] = hi[k];
        }
    }
    if (end - begin <= 4) {
        n->left = begin; n->right = 0; n->count = end - begin;
        return id;
    }
    uint32_t mid = begin + (end - begin) / 2; /* order[] is Morton-sorted */
    uint32_t l = obuild(b, begin, mid);
    uint32_t r = obuild(b, mid, end);
    n = &b->nodes[id];
    n->left = l; n->right = r; n->count = 0;
    return id;
}

void*
orc_bvh_create(const float* tris, uint32_t ntris)
{
    obvh* b = (obvh*)calloc(1, sizeof(obvh));
    b->tris = tris;
    b->ntris = ntris;
    b->order = (uint32_t*)malloc(sizeof(uint32_t) * (ntris ? ntris : 1));
    b->cent = (float*)malloc(sizeof(float) * 3 * (ntris ? ntris : 1));
    b->nodes = (onode*)malloc(sizeof(onode) * (2 * (uint64_t)ntris + 1));
    for (uint32_t i = 0; i < ntris; ++i) {
        b->order[i] = i;
        const float* tr = tris + 9 * (uint64_t)i;
        for (int k = 0; k < 3; ++k) b->cent[3 * (uint64_t)i + k] = tr[k] + (tr[3 + k] + tr[6 + k]) / 3.0f;
    }
    if (ntris) {
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t i = 0; i < ntris; ++i)
            for (int k = 0; k < 3; ++k) {
                float c = b->cent[3 * (uint64_t)i + k];
                if (c < lo[k]) lo[k] = c;
                if (c > hi[k]) hi[k] = c;
            }
        uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * ntris);
        for (uint32_t i = 0; i < ntris; ++i) {
            uint64_t q[3];
            for (int k = 0; k < 3; ++k) {
                double e = (double)hi[k] - lo[k];
                double u = e > 0 ? ((double)b->cent[3 * (uint64_t)i + k] - lo[k]) / e : 0.0;
                if (!(u >= 0.0)) u = 0.0;
                if (u > 1.0) u = 1.0;
                q[k] = (uint64_t)(u * 2097151.0);
            }
            keys[i] = spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2;
        }
        g_sort_keys = keys;
        qsort(b->order, ntris, sizeof(uint32_t), cmp_key);
        free(keys);
        obuild(b, 0, ntris);
    }
    return b;
}

void
orc_bvh_destroy(void* h)
{
    obvh* b = (obvh*)h;
    if (!b) return;
    free(b->order); free(b->cent); free(b->nodes); free(b);
}

/* box entry/exit in double, returns 0 when the slab interval is empty */
static inline int
obox(const onode* n, const double* o, const double* inv, double* t0, double* t1)
{
    double a = -DBL_MAX, c = DBL_MAX;
    for (int k = 0; k < 3; ++k) {
        double x0 = (n->lo[k] - o[k]) * inv[k], x1 = (n->hi[k] - o[k]) * inv[k];
        if (isnan(x0) || isnan(x1)) continue; /* ray on a slab plane with zero dir: keep */
        double l = x0 < x1 ? x0 : x1, h = x0 > x1 ? x0 : x1;
        if (l > a) a = l;
        if (h < c) c = h;
    }
    *t0 = a; *t1 = c;
    return a <= c;
}

static void
oquery(const obvh* b, int sem, const float* ray, int any, uint32_t* bp, float* bt, float* bb1, float* bb2,
       uint32_t* nt, uint8_t* occ)
{
    *bp = 0xffffffffu; *bt = FLT_MAX; *bb1 = 0.0f; *bb2 = 0.0f; *nt = 0;
    if (occ) *occ = 0;
    if (!b->ntris) return;
    double o[3] = {ray[0], ray[1], ray[2]}, inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0 / (double)ray[4 + k];
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const onode* n = &b->nodes[stack[--sp]];
        double t0, t1;
        if (!obox(n, o, inv, &t0, &t1)) continue;
        double cur = *bp == 0xffffffffu ? (double)ray[7] : (double)*bt;
        double slack = 1e-3 * (fabs(cur) + fabs(t0) + fabs(t1)) + 1e-6;
        if (t1 < (double)ray[3] - slack || t0 > cur + slack) continue;
        if (n->right == 0) {
            for (uint32_t i = 0; i < n->count; ++i) {
                uint32_t id = b->order[n->left + i];
                const float* tr = b->tris + 9 * (uint64_t)id;
                if (any) {
                    float t, b1, b2;
                    if (orc_tri_test(sem, ray, tr, &t, &b1, &b2)) { *occ = 1; return; }
                } else {
                    consider(sem, ray, tr, id, bp, bt, bb1, bb2, nt);
                }
            }
        } else {
            if (sp + 2 > 128) abort(); /* oracle tree depth is ~2 log2(n): cannot overflow */
            stack[sp++] = n->right;
            stack[sp++] = n->left;
        }
    }
    if (*bp == 0xffffffffu) *bt = FLT_MAX;
}

typedef struct {
    const obvh* b; int sem; const float* rays; uint64_t n; int any;
    uint32_t* prim; float* t; float* b1; float* b2; uint32_t* ntie; uint8_t* occ;
    uint64_t next; pthread_mutex_t mu;
} ojob;

static void*
oworker(void* p)
{
    ojob* j = (ojob*)p;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        uint64_t s = j->next; j->next += 512;
        pthread_mutex_unlock(&j->mu);
        if (s >= j->n) break;
        uint64_t e = s + 512 < j->n ? s + 512 : j->n;
        for (uint64_t i = s; i < e; ++i) {
            uint32_t bp, nt; float bt, bb1, bb2; uint8_t oc;
            oquery(j->b, j->sem, j->rays + 8 * i, j->any, &bp, &bt, &bb1, &bb2, &nt, j->any ? &oc : 0);
            if (j->any) j->occ[i] = oc;
            else {
                j->prim[i] = bp; j->t[i] = bt; j->b1[i] = bb1; j->b2[i] = bb2;
                if (j->ntie) j->ntie[i] = nt;
            }
        }
    }
    return 0;
}

static void
orun(ojob* j, int nthreads)
{
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    pthread_mutex_init(&j->mu, 0);
    j->next = 0;
    for (int i = 1; i < nthreads; ++i) pthread_create(&th[i], 0, oworker, j);
    oworker(j);
    for (int i = 1; i < nthreads; ++i) pthread_join(th[i], 0);
    pthread_mutex_destroy(&j->mu);
}

void
orc_bvh_closest(void* h, int sem, const float* rays, uint64_t nrays, int nthreads,
                uint32_t* prim, float* t, float* b1, float* b2, uint32_t* ntie)
{
    ojob j;
    memset(&j, 0, sizeof j);
    j.b = (const obvh*)h; j.sem = sem; j.rays = rays; j.n = nrays; j.any = 0;
    j.prim = prim; j.t = t; j.b1 = b1; j.b2 = b2; j.ntie = ntie;
    orun(&j, nthreads);
}

void
orc_bvh_any(void* h, int sem, const float* rays, uint64_t nrays, int nthreads, uint8_t* occluded)
{
    ojob j;
    memset(&j, 0, sizeof j);
    j.b = (const obvh*)h; j.sem = sem; j.rays = rays; j.n = nrays; j.any = 1; j.occ = occluded;
    orun(&j, nthreads);
}
