// Device-side shading: sampling helpers, BSDFs, lights, light samplers,
// random numbers and the pinhole camera of the integrator.
//
// Every function restates the reference's math for the same quantity (cited
// per function) so that, compiled without multiply-add contraction, the FP32
// results follow the reference's operation order. Known reference quirks are
// kept on purpose:
//  * Microfacet::computePdf returns D / (4 wo.wh) although sample() draws the
//    visible-normal distribution (src/materials/microfacet.cpp:88-103 vs
//    14-46);
//  * the interpolated shading normal is not re-normalised
//    (src/shapes/mesh.cpp:85-101) and getBasis does not normalise its input
//    (src/math/vector.h:214-222);
//  * lights are not intersectable geometry.
#pragma once

#include "common.cuh"

namespace ag {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kOneMinusEpsilon = 0.99999988079071044921875f;  // 1 - FLT_EPSILON (src/utils/util.h:10)
constexpr float kRayOffset = 0.001f;                             // src/alpine_config.h:7

// ---------------------------------------------------------------------------
// vector helpers in the reference's operation order (src/math/vector.h)
AG_HD float len3(float3 v) { return sqrtf(dot(v, v)); }
AG_HD float3 normalize3(float3 v) { return v / len3(v); }
AG_HD float3 mul3(float3 a, float3 b) { return a * b; }

// getBasis (src/math/vector.h:214-222)
AG_HD void get_basis(float3 v, float3& b1, float3& b2)
{
    b1 = fabsf(v.x) > fabsf(v.y) ? normalize3(mk3(-v.z, 0.0f, v.x)) : normalize3(mk3(0.0f, v.z, -v.y));
    b2 = cross(v, b1);
}

// toLocal / toWorld (src/utils/util.h:30-38)
AG_HD float3 to_local(float3 v, float3 s, float3 t, float3 n) { return mk3(dot(s, v), dot(t, v), dot(n, v)); }
AG_HD float3 to_world(float3 v, float3 s, float3 t, float3 n) { return s * v.x + t * v.y + n * v.z; }

// trigonometric helpers (src/utils/util.h:17-34)
AG_HD float cos2_theta(float3 w) { return w.z * w.z; }
AG_HD float sin2_theta(float3 w) { return fmaxf(1.0f - cos2_theta(w), 0.0f); }
AG_HD float sin_theta(float3 w) { return sqrtf(sin2_theta(w)); }
AG_HD float tan2_theta(float3 w) { return sin2_theta(w) / cos2_theta(w); }
AG_HD float cos_phi(float3 w)
{
    float st = sin_theta(w);
    return st == 0.0f ? 1.0f : fminf(fmaxf(w.x / st, -1.0f), 1.0f);
}
AG_HD float sin_phi(float3 w)
{
    float st = sin_theta(w);
    return st == 0.0f ? 0.0f : fminf(fmaxf(w.y / st, -1.0f), 1.0f);
}
AG_HD bool same_hemisphere(float3 a, float3 b) { return a.z * b.z > 0.0f; }
AG_HD float3 reflect3(float3 v, float3 n) { return -v + n * 2.0f * dot(v, n); }

// powerHeuristic with one sample each (src/utils/util.h:49-54)
AG_HD float power_heuristic(float a, float b) { return (a * a) / (a * a + b * b); }

// schlickFresnel (src/utils/util.h:56-60)
AG_HD float3 schlick(float3 f0, float3 wi, float3 wh)
{
    float f = powf(fmaxf(0.0f, 1.0f - dot(wi, wh)), 5.0f);
    return mk3(f, f, f) + f0 * (1.0f - f);
}

// sampleConcentricDisk (src/utils/util.cpp:6-31)
AG_HD float2 concentric_disk(float ux, float uy)
{
    float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) return make_float2(0.0f, 0.0f);
    float theta, r;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        theta = 0.25f * kPi * (oy / ox);
    } else {
        r = oy;
        theta = 0.5f * kPi * (1.0f - 0.5f * (ox / oy));
    }
    return make_float2(r * cosf(theta), r * sinf(theta));
}

// ---------------------------------------------------------------------------
// Random numbers.
//
// Reference stream: per-pixel xorshift128 seeded by the pixel index
// (src/sampler.cpp:7-42), drawn in the reference's order. Counter mode: a
// stateless hash of (seed, pixel, sample, dimension), so samples of one pixel
// can run in parallel and every run is deterministic.
struct XorShift128 {
    uint32_t s[4];
};

AG_HD void xorshift_seed(XorShift128& r, uint32_t seed)
{
    for (uint32_t i = 1; i <= 4; ++i) r.s[i - 1] = seed = 1812433253u * (seed ^ (seed >> 30)) + i;
}

AG_HD uint32_t xorshift_next(XorShift128& r)
{
    uint32_t t = r.s[3];
    uint32_t s = r.s[0];
    r.s[3] = r.s[2];
    r.s[2] = r.s[1];
    r.s[1] = s;
    t ^= t << 11;
    t ^= t >> 8;
    return r.s[0] = t ^ s ^ (s >> 19);
}

// Sampler::get1D: u32 / UINT32_MAX in double, clamped to 1 - FLT_EPSILON.
AG_HD float xorshift_1d(XorShift128& r)
{
    uint32_t v = xorshift_next(r);
    double d = (double)v / 4294967295.0;
    return fminf((float)d, kOneMinusEpsilon);
}

// SplitMix64 finaliser (Steele, Lea, Flood 2014).
AG_HD uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct CounterRng {
    uint64_t key;  // hash of (seed, pixel, sample)
    uint32_t dim;
};

AG_HD void counter_init(CounterRng& r, uint32_t seed, uint32_t pixel, uint32_t sample)
{
    r.key = splitmix64(((uint64_t)sample << 32 | pixel) ^ splitmix64((uint64_t)seed));
    r.dim = 0;
}

AG_HD float counter_1d(CounterRng& r)
{
    uint64_t h = splitmix64(r.key + 0x632be59bd9b4e019ull * (uint64_t)(++r.dim));
    return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);  // 24 bits -> [0, 1)
}

// ---------------------------------------------------------------------------
// Materials.
enum MaterialKind : uint32_t { kMatDielectric = 0, kMatConductor = 1 };

// Per-triangle render attributes: material id and flags.
constexpr uint32_t kTriHasNormals = 0x80000000u;      // interpolate the vertex normals
constexpr uint32_t kTriMorphedNormals = 0x40000000u;  // the mesh has normal morph targets
constexpr uint32_t kTriHasUvs = 0x20000000u;          // interpolate the vertex texture coordinates
constexpr uint32_t kTriHasTangents = 0x10000000u;     // tangent-space shading normals (needs normals)
constexpr uint32_t kTriMaterialMask = 0x0fffffffu;

struct Material {
    uint32_t kind;
    float r, g, b;    // base colour (Dielectric: diffuse albedo; Conductor: F0)
    float ax, ay;     // microfacet alpha, already clamped to >= 0.001
    uint32_t lobes;   // Dielectric: 1 (Lambertian) or 2 (+ Microfacet, when ax^2 + ay^2 < 1 unclamped)
    uint32_t baseTex;    // base-colour texture id + 1 (0 = the constant colour above)
    uint32_t normalTex;  // normal-map texture id + 1 (0 = none: the tangent-space normal (0, 0, 1))
};

// One texture of the texel pool: texels [offset, offset + width * height),
// row-major float4 (the loader's Texture4f, src/texture.h).
struct TextureInfo {
    uint32_t offset, width, height, pad;
};

// Texture<T>::sample (src/texture.h:19-35): nearest texel, coordinates
// wrapped to [0, 1) by u - floor(u), scaled by the size, clamped.
AG_D float4 texture_sample(const TextureInfo& t, const float4* texels, float u, float v)
{
    u = u - floorf(u);
    v = v - floorf(v);
    uint32_t x = (uint32_t)(u * (float)t.width);
    uint32_t y = (uint32_t)(v * (float)t.height);
    x = min(x, t.width - 1u);
    y = min(y, t.height - 1u);
    return texels[t.offset + x + y * t.width];
}

// EnvironmentMap::sample (src/environment_map.cpp:14-37): the lat-long map
// at u = atan2(d.z, d.x) / 2pi + 0.5, v = acos(clamp(d.y)) / pi, nearest texel.
AG_D float3 environment_sample(const float* env, uint32_t w, uint32_t h, float3 d)
{
    float u = atan2f(d.z, d.x) / (2.0f * kPi) + 0.5f;
    float v = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) / kPi;
    u = u - floorf(u);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const uint32_t x = min((uint32_t)(u * (float)w), w - 1u);
    const uint32_t y = min((uint32_t)(v * (float)h), h - 1u);
    const float* t = env + 3ull * (y * (size_t)w + x);
    return mk3(t[0], t[1], t[2]);
}

struct BsdfSample {
    float3 estimator;  // bsdf * cos / pdf
    float3 wi;
    float pdf;
};

constexpr float kDielectricF0 = 0.16f * 0.5f * 0.5f;  // src/materials/dielectric.cpp:11-12

// Microfacet (src/materials/microfacet.cpp), alpha = (ax, ay)
AG_HD float mf_distribution(float3 wh, float ax, float ay)
{
    float cos4 = cos2_theta(wh) * cos2_theta(wh);
    float c2 = cos_phi(wh) * cos_phi(wh);
    float s2 = sin_phi(wh) * sin_phi(wh);
    float term = 1.0f + tan2_theta(wh) * (c2 / (ax * ax) + s2 / (ay * ay));
    float invD = kPi * ax * ay * cos4 * term * term;
    return invD != 0.0f ? 1.0f / invD : 0.0f;
}

AG_HD float mf_lambda(float3 v, float ax, float ay)
{
    float alpha = sqrtf(cos_phi(v) * cos_phi(v) * ax * ax + sin_phi(v) * sin_phi(v) * ay * ay);
    return (-1.0f + sqrtf(1.0f + alpha * alpha * tan2_theta(v))) / 2.0f;
}

AG_HD float mf_g2(float3 wo, float3 wi, float ax, float ay)
{
    return 1.0f / (1.0f + mf_lambda(wo, ax, ay) + mf_lambda(wi, ax, ay));
}

// Microfacet::sample with VNDF sampling (microfacet.cpp:10-46)
AG_HD bool mf_sample(float3 wo, float ux, float uy, float3 f0, float ax, float ay, BsdfSample& out)
{
    float3 woh = normalize3(mk3(ax * wo.x, ay * wo.y, wo.z));
    float2 t = concentric_disk(ux, uy);
    float s = 0.5f * (1.0f + woh.z);
    t.y = (1.0f - s) * sqrtf(1.0f - t.x * t.x) + s * t.y;
    float3 nhh = mk3(t.x, t.y, sqrtf(fmaxf(0.0f, 1.0f - t.x * t.x - t.y * t.y)));
    float3 b1, b2;
    get_basis(woh, b1, b2);
    float3 nh = b1 * nhh.x + b2 * nhh.y + woh * nhh.z;
    float3 wh = normalize3(mk3(ax * nh.x, ay * nh.y, fmaxf(0.0f, nh.z)));
    if (!same_hemisphere(wo, wh)) wh = -wh;
    float3 wi = reflect3(wo, wh);
    if (!same_hemisphere(wo, wi)) return false;
    float3 f = schlick(f0, wi, wh);
    float g1 = 1.0f / (1.0f + mf_lambda(wo, ax, ay));
    float g2 = mf_g2(wo, wi, ax, ay);
    float d = mf_distribution(wh, ax, ay);
    out.estimator = f * g2 / g1;
    out.wi = wi;
    out.pdf = d / (4.0f * dot(wo, wh));
    return true;
}

// Microfacet::computeBsdf (microfacet.cpp:48-70)
AG_HD float3 mf_bsdf(float3 wo, float3 wi, float3 f0, float ax, float ay)
{
    float cwo = fabsf(wo.z), cwi = fabsf(wi.z);
    if (cwo == 0.0f || cwi == 0.0f) return mk3(0.0f, 0.0f, 0.0f);
    float3 wh = wo + wi;
    float l = len3(wh);
    if (l == 0.0f) return mk3(0.0f, 0.0f, 0.0f);
    wh = wh / l;
    float3 f = schlick(f0, wi, wh);
    float d = mf_distribution(wh, ax, ay);
    float g2 = mf_g2(wo, wi, ax, ay);
    return f * d * g2 / (4.0f * cwo * cwi);
}

// Microfacet::computePdf (microfacet.cpp:72-90): D / (4 wo.wh)
AG_HD float mf_pdf(float3 wo, float3 wi, float ax, float ay)
{
    float3 wh = wo + wi;
    float l = len3(wh);
    if (l == 0.0f) return 0.0f;
    wh = wh / l;
    float d = mf_distribution(wh, ax, ay);
    return d / (4.0f * dot(wo, wh));
}

// Lambertian (src/materials/lambertian.cpp:8-36) with
// sampleCosineWeightedHemisphere (src/utils/util.cpp:33-41)
AG_HD bool lambert_sample(float ux, float uy, float3 bc, BsdfSample& out)
{
    float2 d = concentric_disk(ux, uy);
    float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    float3 wi = normalize3(mk3(d.x, d.y, z));
    float pdf = z / kPi;
    if (pdf == 0.0f) return false;
    out.estimator = bc;
    out.wi = wi;
    out.pdf = pdf;
    return true;
}
AG_HD float3 lambert_bsdf(float3 bc) { return bc / kPi; }
AG_HD float lambert_pdf(float3 wi) { return fmaxf(wi.z, 0.0f) / kPi; }

AG_HD float3 mat_color(const Material& m) { return mk3(m.r, m.g, m.b); }

// Material::sample: Dielectric (src/materials/dielectric.cpp:31-62) and
// Conductor (src/materials/conductor.cpp:18-25)
AG_HD bool mat_sample(const Material& m, float3 wo, float u0, float u1, BsdfSample& out)
{
    float3 bc = mat_color(m);
    if (m.kind == kMatConductor) return mf_sample(wo, u0, u1, bc, m.ax, m.ay, out);
    const uint32_t n = m.lobes;
    uint32_t idx = (uint32_t)(u0 * (float)n) & 0xffu;
    float uu = u0 * (float)n - (float)idx;
    const float3 f0 = mk3(kDielectricF0, kDielectricF0, kDielectricF0);
    bool ok = idx == 0 ? lambert_sample(uu, u1, bc, out) : mf_sample(wo, uu, u1, f0, m.ax, m.ay, out);
    if (!ok) return false;
    float cosTerm = out.wi.z;
    if (cosTerm <= 0.0f) return false;
    float3 bsdf = out.estimator * out.pdf / cosTerm;
    if (n == 2) {
        if (idx != 0) {
            out.pdf += lambert_pdf(out.wi);
            bsdf += lambert_bsdf(bc);
        } else {
            out.pdf += mf_pdf(wo, out.wi, m.ax, m.ay);
            bsdf += mf_bsdf(wo, out.wi, f0, m.ax, m.ay);
        }
    }
    out.pdf /= (float)n;
    out.estimator = bsdf * cosTerm / out.pdf;
    return true;
}

// Material::computeBsdf
AG_HD float3 mat_bsdf(const Material& m, float3 wo, float3 wi)
{
    float3 bc = mat_color(m);
    if (m.kind == kMatConductor) return mf_bsdf(wo, wi, bc, m.ax, m.ay);
    float3 sum = mk3(0.0f, 0.0f, 0.0f);
    sum += lambert_bsdf(bc);
    if (m.lobes == 2) sum += mf_bsdf(wo, wi, mk3(kDielectricF0, kDielectricF0, kDielectricF0), m.ax, m.ay);
    return sum;
}

// Material::computePdf
AG_HD float mat_pdf(const Material& m, float3 wo, float3 wi)
{
    if (m.kind == kMatConductor) return mf_pdf(wo, wi, m.ax, m.ay);
    float sum = 0.0f;
    sum += lambert_pdf(wi);
    if (m.lobes == 2) sum += mf_pdf(wo, wi, m.ax, m.ay);
    return sum / (float)m.lobes;
}

// ---------------------------------------------------------------------------
// The plain continuation procedure (Material::sample) as a density over
// directions, for one-sample MIS with another sampling technique. For wo and
// wi in the upper hemisphere, writes the true density p of the procedure's
// output direction and its effective integrand f_eff * cos = E[estimator | wi]
// * p, so that f_eff * cos / q for any mixture density q containing p
// estimates exactly what the plain estimator estimates, including the
// reference's pdf conventions (VNDF sampling with a D / (4 wo.wh) pdf in the
// dielectric mixture, dielectric.cpp:31-62).
//   VNDF density of the reflected direction: G1(wo) D(wh) / (4 cos(theta_o))
//   (Heitz 2018, "Sampling the GGX Distribution of Visible Normals"), times
//   the indicator of the half-space the reference's sampler actually covers.
//   Heitz's warp of the disk is exact when the frame's second axis T2 lies in
//   the vertical plane of the stretched view direction Vh; then the warped
//   half-disk is the projection of {N : N.z >= 0}. The reference builds the
//   frame with getBasis(Vh), whose b2 is tilted, so the warped half-disk is
//   the projection of {N : N . (r b2 + Vh.z Vh) >= 0}, r = sqrt(1 - Vh.z^2),
//   uniformly covered with the same density; normals outside it are never
//   produced (and those inside it below the horizon are clamped and then
//   rejected as wi.z <= 0).
AG_HD float mf_vndf_density(float3 wo, float3 wi, float ax, float ay)
{
    float3 wh = wo + wi;
    float l = len3(wh);
    if (l == 0.0f || wo.z <= 0.0f) return 0.0f;
    wh = wh / l;
    if (wh.z <= 0.0f || dot(wo, wh) <= 0.0f) return 0.0f;
    const float3 vh = normalize3(mk3(ax * wo.x, ay * wo.y, wo.z));
    float3 b1, b2;
    get_basis(vh, b1, b2);
    const float r = sqrtf(fmaxf(0.0f, 1.0f - vh.z * vh.z));
    const float3 n2 = b2 * r + vh * vh.z;
    const float3 nh = mk3(wh.x / ax, wh.y / ay, wh.z);  // un-stretched normal (unnormalised)
    if (dot(nh, n2) < 0.0f) return 0.0f;
    float g1 = 1.0f / (1.0f + mf_lambda(wo, ax, ay));
    return g1 * mf_distribution(wh, ax, ay) / (4.0f * wo.z);
}

// Microfacet::sample's estimator F G2 / G1 as a function of wi.
AG_HD float3 mf_estimator(float3 wo, float3 wi, float3 f0, float ax, float ay)
{
    float3 wh = wo + wi;
    float l = len3(wh);
    if (l == 0.0f) return mk3(0.0f, 0.0f, 0.0f);
    wh = wh / l;
    float3 f = schlick(f0, wi, wh);
    float g1 = 1.0f / (1.0f + mf_lambda(wo, ax, ay));
    return f * mf_g2(wo, wi, ax, ay) / g1;
}

AG_HD bool plain_eval(const Material& m, float3 wo, float3 wi, float& p, float3& fcos)
{
    p = 0.0f;
    fcos = mk3(0.0f, 0.0f, 0.0f);
    if (wo.z <= 0.0f || wi.z <= 0.0f) return false;
    const float3 bc = mat_color(m);
    if (m.kind == kMatConductor) {
        p = mf_vndf_density(wo, wi, m.ax, m.ay);
        fcos = mf_estimator(wo, wi, bc, m.ax, m.ay) * p;
        return p > 0.0f;
    }
    const float pc = wi.z / kPi;  // cosine-weighted hemisphere
    if (m.lobes == 1) {
        p = pc;
        fcos = bc * pc;  // estimator = base colour
        return p > 0.0f;
    }
    const float3 f0 = mk3(kDielectricF0, kDielectricF0, kDielectricF0);
    const float cosT = wi.z;
    const float pmRep = mf_pdf(wo, wi, m.ax, m.ay);     // reference's reported microfacet pdf
    const float3 fm = mf_bsdf(wo, wi, f0, m.ax, m.ay);
    const float pv = mf_vndf_density(wo, wi, m.ax, m.ay);
    // Lambertian lobe sampled wi: bsdf = bc/pi + f_m, pdf = (pc + pmRep) / 2
    const float3 estL = (lambert_bsdf(bc) + fm) * cosT / ((pc + pmRep) / 2.0f);
    fcos = estL * (0.5f * pc);
    // microfacet lobe sampled wi: bsdf = est_m pmRep / cos + bc/pi
    if (pv > 0.0f) {
        const float3 estMf = mf_estimator(wo, wi, f0, m.ax, m.ay);
        const float3 estM = (estMf * pmRep / cosT + lambert_bsdf(bc)) * cosT / ((pmRep + pc) / 2.0f);
        fcos += estM * (0.5f * pv);
    }
    p = 0.5f * pc + 0.5f * pv;
    return p > 0.0f;
}

// ---------------------------------------------------------------------------
// Lights.
enum LightKind : uint32_t { kLightPoint = 0, kLightDisk = 1, kLightQuad = 2 };

struct Light {
    uint32_t kind;
    float scale;        // LightHandle::setScale
    float3 position;    // point / disk centre / quad corner
    float3 radiance;    // emitted radiance (disk, quad) or intensity (point)
    float3 normal;      // disk / quad
    float3 axisU;       // disk: binormal, quad: first edge
    float3 axisV;       // disk: tangent,  quad: second edge
    float radius;       // disk
    float area;         // disk / quad
    float3 power;       // Light::getPower (colour * power)
    float3 bmin, bmax;  // Light::getBoundingBox
};

struct LightSample {
    float3 L;
    float3 wi;
    float distance;
    float pdf;
};

AG_HD bool light_is_delta(const Light& l) { return l.kind == kLightPoint; }

// Light::sample: PointLight (src/lights/point_light.cpp:22-38), DiskLight
// (src/lights/disk_light.cpp:30-53); QuadLight follows the DiskLight contract
// on a parallelogram (position + u * axisU + v * axisV).
AG_HD bool light_sample(const Light& l, float u0, float u1, float3 hit, LightSample& out)
{
    if (l.kind == kLightPoint) {
        float3 wi = l.position - hit;
        float d2 = dot(wi, wi);
        if (d2 == 0.0f) return false;
        float d = sqrtf(d2);
        wi = wi / d;
        out.L = l.radiance / d2 * l.scale;
        out.wi = wi;
        out.distance = d;
        out.pdf = 1.0f;
        return true;
    }
    float3 p;
    if (l.kind == kLightDisk) {
        float2 ds = concentric_disk(u0, u1);
        p = l.position + (l.axisU * ds.x + l.axisV * ds.y) * l.radius;
    } else {
        p = l.position + l.axisU * u0 + l.axisV * u1;
    }
    float3 wi = p - hit;
    float d = len3(wi);
    if (d == 0.0f) return false;
    wi = wi / d;
    float c = fmaxf(0.0f, dot(-wi, l.normal));
    if (c == 0.0f) return false;
    out.L = l.radiance * l.scale;
    out.wi = wi;
    out.distance = d;
    out.pdf = (d * d) / (l.area * c);
    return true;
}

// Light::computePdf (disk_light.cpp:55-81); returns pdf, writes distance.
AG_HD float light_pdf(const Light& l, float3 hit, float3 wi, float& dist)
{
    dist = 0.0f;
    if (l.kind == kLightPoint) return 0.0f;
    float c = fmaxf(0.0f, dot(-wi, l.normal));
    if (c == 0.0f) return 0.0f;
    float distance = dot(hit - l.position, l.normal) / c;
    if (distance < 0.0f) return 0.0f;
    float3 p = hit + wi * distance;
    bool inside;
    if (l.kind == kLightDisk) {
        float3 q = p - l.position;
        inside = dot(q, q) < l.radius * l.radius;
    } else {
        float3 q = p - l.position;
        float su = dot(q, l.axisU) / dot(l.axisU, l.axisU);
        float sv = dot(q, l.axisV) / dot(l.axisV, l.axisV);
        inside = su >= 0.0f && su <= 1.0f && sv >= 0.0f && sv <= 1.0f;
    }
    if (inside && c > 0.0f) {
        dist = distance;
        return (distance * distance) / (l.area * c);
    }
    return 0.0f;
}

AG_HD float3 light_emitted(const Light& l) { return l.kind == kLightPoint ? mk3(0.0f, 0.0f, 0.0f) : l.radiance * l.scale; }

// ---------------------------------------------------------------------------
// Light samplers.
enum LightSamplerKind : uint32_t { kSamplerNone = 0, kSamplerUniform = 1, kSamplerPower = 2, kSamplerBvh = 3 };

struct AliasBin {
    float q, p;
    uint32_t alias;
};

// Light BVH node (flattened LightNode, src/light_samplers/bvh_light_sampler.cpp:17-51):
// power = sum of |power| of the cluster, box of the cluster; interior nodes
// have child = index of the first child (the second is child + 1 ... stored
// explicitly), leaves have light >= 0.
struct LightNode {
    float power;
    float3 bmin, bmax;
    int32_t left, right;  // -1 for leaves
    int32_t light;        // light index for leaves, -1 otherwise
};

// LightNode::importance (bvh_light_sampler.cpp:24-51)
AG_HD float light_node_importance(const LightNode& n, float3 p, float3 nrm)
{
    float3 wi = 0.5f * (n.bmin + n.bmax) - p;
    float d2 = dot(wi, wi);
    float3 diag = n.bmax - n.bmin;
    float imp = n.power / fmaxf(d2, 0.5f * len3(diag));
    float br = 0.5f * len3(diag);
    float br2 = br * br;
    if (d2 > 0.0f && d2 > br2) {
        float sinB2 = br2 / d2;
        float sinB = sqrtf(sinB2);
        float cosB = sqrtf(1.0f - sinB2);
        wi = normalize3(wi);
        float cosI = fabsf(dot(wi, nrm));
        float sinI = sqrtf(1 - cosI * cosI);
        imp *= cosI <= cosB ? cosI * cosB + sinI * sinB : 1.0f;
    }
    return imp;
}

// The light BVH as the sampler descends it: per interior node, both
// children's bounds and power in one 64-byte record (one aligned load per
// level). ref: the child's interior node index, or -(light + 1) for a leaf.
struct LightPair {
    float4 lo0;  // child 0: bmin.xyz, power
    float4 hi0;  // child 0: bmax.xyz, ref (int bits)
    float4 lo1;  // child 1
    float4 hi1;
};
static_assert(sizeof(LightPair) == 64, "LightPair layout");

struct LightSamplerView {
    uint32_t kind;
    uint32_t count;
    const Light* lights;
    const AliasBin* alias;
    const LightNode* nodes;   // the tree (the root is read when it is a single leaf)
    const LightPair* pairs;   // the same tree packed for the descent
};

AG_HD int32_t float_bits(float f)
{
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    int32_t i;
    memcpy(&i, &f, sizeof i);
    return i;
#endif
}

AG_HD LightNode light_child(float4 lo, float4 hi)
{
    LightNode n;
    n.power = lo.w;
    n.bmin = mk3(lo.x, lo.y, lo.z);
    n.bmax = mk3(hi.x, hi.y, hi.z);
    n.left = n.right = -1;
    n.light = -1;
    return n;
}

// LightSampler::sample: uniform (uniform_light_sampler.cpp:15-27), power
// (power_light_sampler.cpp:25-35 + alias_table.cpp:71-81), BVH
// (bvh_light_sampler.cpp:267-319). Returns the light index or -1.
// kKind: the sampler kind when it is known at compile time (-1: read ls.kind),
// so that a kernel specialised for one sampler holds only its code.
template <int kKind = -1>
AG_HD int sample_light(const LightSamplerView& ls, float u, float3 hit, float3 ns, float& pdf)
{
    const uint32_t kind = kKind >= 0 ? (uint32_t)kKind : ls.kind;
    if (ls.count == 0 || kind == kSamplerNone) return -1;
    if (kind == kSamplerUniform) {
        uint32_t i = (uint32_t)(u * (float)ls.count);
        if (i > ls.count - 1) i = ls.count - 1;
        pdf = 1.0f / (float)ls.count;
        return (int)i;
    }
    if (kind == kSamplerPower) {
        uint32_t b = (uint32_t)(u * (float)ls.count);
        if (b > ls.count - 1) b = ls.count - 1;
        float up = fminf(u * (float)ls.count - (float)b, kOneMinusEpsilon);
        uint32_t idx = up < ls.alias[b].q ? b : ls.alias[b].alias;
        pdf = ls.alias[idx].p;
        return (int)idx;
    }
    // BVH: stochastic descent by importance with u remapping
    const LightNode& root = ls.nodes[0];
    if (root.left < 0 || root.right < 0) {  // a single light
        if (root.light >= 0 && light_node_importance(root, hit, ns) > 0.0f) {
            pdf = 1.0f;
            return root.light;
        }
        return -1;
    }
    int node = 0;
    float p = 1.0f;
    for (int guard = 0; guard < 128; ++guard) {
        const float4* q = reinterpret_cast<const float4*>(ls.pairs + node);
        const float4 lo0 = q[0], hi0 = q[1], lo1 = q[2], hi1 = q[3];
        const float w0 = light_node_importance(light_child(lo0, hi0), hit, ns);
        const float w1 = light_node_importance(light_child(lo1, hi1), hit, ns);
        if (w0 == 0.0f && w1 == 0.0f) return -1;
        float up = (w0 + w1) * u;
        int idx = up < w0 ? 0 : 1;
        const float wc = idx == 0 ? w0 : w1;
        p *= wc / (w0 + w1);
        u = idx == 0 ? fminf(up / w0, kOneMinusEpsilon) : fminf((up - w0) / w1, kOneMinusEpsilon);
        const int ref = float_bits(idx == 0 ? hi0.w : hi1.w);
        if (ref < 0) {
            // a leaf: its importance is wc (the same function of the same node)
            if (wc > 0.0f) {
                pdf = p;
                return -ref - 1;
            }
            return -1;
        }
        node = ref;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// Pinhole camera (src/camera.cpp:13-29, 73-96): film at distance 1.
struct Camera {
    float3 eye;
    float3 viewX, viewY, viewZ;
    float filmW, filmH;
};

AG_HD void camera_ray(const Camera& c, float x, float y, float3& org, float3& dir)
{
    float fx = (x - 0.5f) * c.filmW;
    float fy = (0.5f - y) * c.filmH;
    // mul(viewMatrix, (fx, fy, 1)) = col0 * fx + col1 * fy + col2 * 1
    float3 d = c.viewX * fx + c.viewY * fy + c.viewZ * 1.0f;
    dir = normalize3(d);
    org = c.eye;
}

}  // namespace ag
