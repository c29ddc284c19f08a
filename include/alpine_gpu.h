/*
 * alpine_gpu.h -- C ABI of the B200 (sm_100a) backend of alpine.
 *
 * Plain C types only: pointers, sizes and int status codes; no exceptions or
 * C++/torch types cross this boundary. One context owns one CUDA stream and
 * all device memory it allocates; calls on one context are not re-entrant
 * (use one context per host thread). Host arrays are caller-owned and copied.
 *
 * Each entry point names the reference interface it replaces (paths inside the
 * alpine source tree).
 */
#ifndef ALPINE_GPU_H
#define ALPINE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALPINE_GPU_ABI_VERSION 1

#if defined(__GNUC__)
#define ALPINE_GPU_API __attribute__((visibility("default")))
#else
#define ALPINE_GPU_API
#endif

/* Status codes. Every entry point returns one of these (0 on success); the
 * message of the last failure is available from alpine_gpu_last_error(). */
typedef enum alpine_gpu_status {
    ALPINE_GPU_OK = 0,
    ALPINE_GPU_ERR_INVALID_ARGUMENT = -1,
    ALPINE_GPU_ERR_CUDA = -2,
    ALPINE_GPU_ERR_INVALID_STATE = -3,
    ALPINE_GPU_ERR_LIMIT = -4,         /* a device-side limit was exceeded (stack, visits, queue) */
    ALPINE_GPU_ERR_OUT_OF_MEMORY = -5
} alpine_gpu_status;

typedef struct alpine_gpu_ctx alpine_gpu_ctx;

typedef struct alpine_gpu_config {
    int device;          /* CUDA device ordinal */
    uint32_t width;      /* framebuffer size for rendering; 0 for a trace-only context */
    uint32_t height;
    uint32_t max_depth;  /* path length limit, as alpine::initialize's maxDepth */
} alpine_gpu_config;

/* One ray: 32 bytes. The reference's Ray (src/ray.h:6-10) plus the parametric
 * range: hits are accepted for t in [tmin, tmax). Reference semantics are
 * tmin = 0 and tmax = FLT_MAX (closest hit) or tmax = tFar (any hit). */
typedef struct alpine_gpu_ray {
    float org[3];
    float tmin;
    float dir[3];
    float tmax;
} alpine_gpu_ray;

/* Closest hit: 16 bytes. prim is the global triangle index (triangles are
 * numbered across meshes in the order they were added); 0xffffffff and
 * t = FLT_MAX on a miss. b1, b2 are the barycentrics of the second and third
 * vertex (the reference's Intersection::barycentric, src/intersection.h:8-16). */
typedef struct alpine_gpu_hit {
    uint32_t prim;
    float t;
    float b1;
    float b2;
} alpine_gpu_hit;

typedef struct alpine_gpu_bvh_stats {
    uint32_t triangles;
    uint32_t binary_nodes;
    uint32_t binary_levels;
    uint32_t wide_nodes;
    uint32_t wide_depth;
    float sah_cost;      /* SAH cost of the wide tree, relative to the root area */
    float build_ms;      /* device time of the last build */
    uint32_t spheres;    /* analytic spheres in the BVH */
    uint32_t child_slots; /* filled child slots over all wide nodes (of 8 each) */
    uint32_t big_levels;  /* leading binary levels with a node of more than 512 primitives (split by the
                             block-wide kernels; the rest are split one warp per node) */
} alpine_gpu_bvh_stats;

/* Creates a context on cfg->device (replaces alpine::initialize,
 * include/alpine/alpine.h:10-14, for the GPU backend). */
ALPINE_GPU_API int alpine_gpu_create(const alpine_gpu_config* cfg, alpine_gpu_ctx** out);

/* Releases every resource of the context (alpine::shutdown, alpine.h:16). */
ALPINE_GPU_API void alpine_gpu_destroy(alpine_gpu_ctx* ctx);

/* Message of the last failed call on this context ("" if none). */
ALPINE_GPU_API const char* alpine_gpu_last_error(const alpine_gpu_ctx* ctx);

/* Removes all meshes, lights and the acceleration structure
 * (alpine::resetScene, alpine.h:23; Scene::reset, src/scenes/scene.h:21-26). */
ALPINE_GPU_API int alpine_gpu_reset_scene(alpine_gpu_ctx* ctx);

/* Appends one triangle mesh (Accelerator::appendMesh,
 * src/accelerators/accelerator.h:19-22): vertices float[3 * vertex_count],
 * indices uint32[3 * triangle_count] (local to this mesh). Writes the shape id
 * (0, 1, ... in call order). */
ALPINE_GPU_API int alpine_gpu_add_mesh(alpine_gpu_ctx* ctx, const float* vertices, uint32_t vertex_count, const uint32_t* indices,
                        uint32_t triangle_count, uint32_t* shape_id);

/* Appends analytic spheres (Accelerator::appendSphere,
 * src/accelerators/accelerator.h:24; Sphere::Data, src/shapes/sphere.h:14-18):
 * float[4 * count] = centre xyz, radius; a material id per sphere (NULL:
 * material 0). They share the BVH with the triangles (next build). A hit on
 * sphere k reports prim = 0x80000000 | k (spheres numbered across calls in
 * the order added), t, and b1 = b2 = 0. The ray / sphere test takes the
 * front hit, else the back hit of a ray starting inside, in [tmin, tmax);
 * rendering shades a sphere with its outward normal (Sphere::
 * getIntersectionAttributes, sphere.cpp:23-37: ns = ng). In the reference
 * only the Embree accelerator intersects spheres. Writes the index of the
 * first sphere added. */
ALPINE_GPU_API int alpine_gpu_add_spheres(alpine_gpu_ctx* ctx, const float* spheres, uint32_t count,
                                          const uint32_t* material, uint32_t* first_sphere);

/* Replaces the vertex positions of one mesh (Accelerator::getVertexBuffer +
 * updateShape, accelerator.h:27-29). Takes effect at the next build. */
ALPINE_GPU_API int alpine_gpu_update_vertices(alpine_gpu_ctx* ctx, uint32_t shape_id, const float* vertices);

/* Morph-target animation (glTF morph targets: Mesh::Data::targets,
 * src/shapes/mesh.h:27-33; Animation, src/animation.h).
 * alpine_gpu_set_morph_targets: `count` (1-32) targets of one mesh, vertex
 *   deltas float[count][3 * vertex_count] and optionally normal deltas of the
 *   same shape (the mesh must then have vertex normals, set by
 *   alpine_gpu_set_triangle_attributes). The mesh's current positions and
 *   normals become the base; the weights start at 0 (mesh.cpp:14-20).
 * alpine_gpu_add_animation_channel: one channel (Animation::Channel) of
 *   `keyframes` (>= 2) morph keyframes for that mesh: times[k] (not
 *   decreasing) and weights[k][count].
 * alpine_gpu_update_scene: Alpine::updateScene(time) (alpine.cpp:204-212):
 *   per channel, time clamped to the keyframe range, the segment found and
 *   the weights lerped (Animation::update, animation.cpp:10-39); the vertices
 *   (and normals) morphed on the GPU as Mesh::update does (mesh.cpp:29-55,
 *   the normals as mesh.cpp:86-101), then the BVH rebuilt (stats may be NULL).
 * alpine_gpu_get_vertices: the current positions (and vertex normals, zero
 *   for a mesh without) of one mesh; either pointer may be NULL. */
ALPINE_GPU_API int alpine_gpu_set_morph_targets(alpine_gpu_ctx* ctx, uint32_t shape_id, const float* vertex_deltas,
                                                const float* normal_deltas, uint32_t count);
ALPINE_GPU_API int alpine_gpu_add_animation_channel(alpine_gpu_ctx* ctx, uint32_t shape_id, const float* times,
                                                    const float* weights, uint32_t keyframes);
ALPINE_GPU_API int alpine_gpu_update_scene(alpine_gpu_ctx* ctx, float time, alpine_gpu_bvh_stats* stats);
ALPINE_GPU_API int alpine_gpu_get_vertices(alpine_gpu_ctx* ctx, uint32_t shape_id, float* vertices, float* normals);

/* Full (re)build of the BVH on the GPU: binned SAH with 32 bins, collapsed to
 * an 8-wide quantised BVH (Accelerator::updateScene, accelerator.h:31;
 * src/accelerators/wide_bvh.cpp:175-197). stats may be NULL. */
ALPINE_GPU_API int alpine_gpu_build(alpine_gpu_ctx* ctx, alpine_gpu_bvh_stats* stats);

/* Rebuild without host round trips (no counterpart in the reference, which
 * rebuilds synchronously in Accelerator::updateScene): the same tree as
 * alpine_gpu_build, bit for bit, enqueued on the context stream. Every count
 * of the level-by-level build stays in device memory, so nothing waits on
 * the host, and the fixed sequence of launches is captured in a CUDA graph
 * on the first call and replayed by later calls. It runs max_binary_levels
 * binned-SAH levels and max_wide_levels collapse levels; 0 takes the last
 * alpine_gpu_build's depths plus a margin (binary: +max(4, levels / 4); wide:
 * +2). A tree deeper than a cap is reported by the next alpine_gpu_synchronize
 * / render_wait as ALPINE_GPU_ERR_LIMIT ("BVH build level cap reached"): past
 * the binary cap nothing is written and the previous tree stays in place;
 * past the wide cap the tree is partly rewritten, so queries and renders
 * until the next build are not to be trusted. A synchronous build recovers
 * in both cases. Needs an alpine_gpu_build of the same scene first (it sizes
 * the buffers; the primitive count may not change). Host-buffer queries
 * (alpine_gpu_trace / _occluded) and renders of the context wait for it; a
 * *_device query on a caller's stream must be ordered after it by the caller
 * (alpine_gpu_synchronize, for instance).
 * alpine_gpu_update_scene_async: alpine_gpu_update_scene's morph followed by
 *   this rebuild with the default caps, all on the context stream, so that a
 *   frame's morph, rebuild and alpine_gpu_render_async are enqueued without
 *   any host wait.
 * alpine_gpu_read_build_stats: waits for the stream and reads the statistics
 *   of the last alpine_gpu_build_async from device memory (build_ms: its
 *   device time; triangles, spheres and big_levels: those of the last
 *   alpine_gpu_build); graph_captures / graph_launches (either may be NULL)
 *   count the captures and replays of its graph. The block-wide kernels for
 *   nodes of more than 512 primitives run on the first big_levels + 2 levels
 *   only; a larger node met below them is reported like a level cap. */
ALPINE_GPU_API int alpine_gpu_build_async(alpine_gpu_ctx* ctx, uint32_t max_binary_levels, uint32_t max_wide_levels);
ALPINE_GPU_API int alpine_gpu_update_scene_async(alpine_gpu_ctx* ctx, float time);
ALPINE_GPU_API int alpine_gpu_read_build_stats(alpine_gpu_ctx* ctx, alpine_gpu_bvh_stats* stats,
                                               uint32_t* graph_captures, uint32_t* graph_launches);

/* How the binary SAH tree is collapsed into 8-wide nodes (the next build):
 *   COLLAPSE_SAH (0, the default): SAH-optimal. A dynamic program over the
 *     binary tree picks, for every wide node, the binary nodes that fill its
 *     slots at least SAH cost (Ylitie, Karras and Laine, HPG 2017). Nodes
 *     are fuller than under the greedy rule, and rays fetch fewer of them.
 *   COLLAPSE_GREEDY (1): the reference's rule (src/accelerators/wide_bvh.cpp:
 *     200-243): open the internal child of largest surface area until the
 *     8 slots are used.
 * triangle_cost: SAH cost of one triangle test relative to one wide-node
 *   visit (COLLAPSE_SAH only); 0 = 1.0 (measured best on B200: a triangle
 *   test costs about 3.6 node visits of time in the traversal kernel, but
 *   costs above 1 change little).
 * Hits do not depend on the collapse, except which of two triangles at
 * exactly the same distance is reported. */
#define ALPINE_GPU_COLLAPSE_SAH 0u
#define ALPINE_GPU_COLLAPSE_GREEDY 1u
typedef struct alpine_gpu_build_options {
    uint32_t collapse;
    float triangle_cost;
} alpine_gpu_build_options;
ALPINE_GPU_API int alpine_gpu_set_build_options(alpine_gpu_ctx* ctx, const alpine_gpu_build_options* options);

/* Closest hit for `count` rays in HOST memory (Accelerator::intersect,
 * accelerator.h:33, batched). Pinned buffers are copied in chunks overlapped
 * with the traversal; pageable buffers are staged. Waits for the work already
 * enqueued on the context stream first, and blocks until done. */
ALPINE_GPU_API int alpine_gpu_trace(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count, alpine_gpu_hit* hits);

/* Any hit in [tmin, tmax) for rays in HOST memory (Accelerator::intersectAny,
 * accelerator.h:35, batched): occluded[i] = 1 when something is hit. */
ALPINE_GPU_API int alpine_gpu_occluded(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count, uint8_t* occluded);

/* The same two queries on DEVICE buffers, enqueued on `stream` (a
 * cudaStream_t; NULL = the context's stream). Asynchronous: errors raised by
 * the kernels are reported by the next alpine_gpu_synchronize(). */
ALPINE_GPU_API int alpine_gpu_trace_device(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count, alpine_gpu_hit* hits,
                            void* stream);
ALPINE_GPU_API int alpine_gpu_occluded_device(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count, uint8_t* occluded,
                               void* stream);

/* Closest hit for at most ALPINE_GPU_NOALLOC_MAX_RAYS rays in HOST memory,
 * allocating no memory. This entry point has no counterpart in the reference.
 * It is for callers that cannot call cudaMalloc at query time: a host
 * application that owns the device-memory budget through its own pools, or a
 * per-frame path that cannot accept an allocation's implicit synchronisation
 * or a late out-of-memory failure. alpine_gpu_trace grows device staging
 * buffers as needed; this variant stages through one fixed 3 MiB array in
 * device memory that every GPU loading the library holds until exit. Larger
 * batches are rejected with ALPINE_GPU_ERR_INVALID_ARGUMENT. The first call
 * on a device looks up the array's device address; with CUDA's lazy module
 * loading that first call may also load the module that holds the array. The
 * call is synchronous (it waits for its own copies) and copies through host
 * memory, so it must never be made while the context's stream, or a stream it
 * depends on, is being captured. All calls share the array, so calls are
 * serialised inside the library; calls that overlapped on one device would
 * race. Results are identical to alpine_gpu_trace. */
#define ALPINE_GPU_NOALLOC_MAX_RAYS 65536
ALPINE_GPU_API int alpine_gpu_trace_noalloc(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count,
                                            alpine_gpu_hit* hits);

/* Traversal options (no counterpart in the reference's API; default: all 0).
 * triangle_test selects the hit rule of every traversal of the context
 *   (queries and rendering), i.e. which reference accelerator's answers the
 *   GPU reproduces bit for bit:
 *   WIDE_BVH (0): the reference's 8-wide BVH and its ISPC triangle kernel
 *     (src/accelerators/wide_bvh.cpp:487-619, src/ispc/triangle.ispc:46-87):
 *     |det| >= 1e-6, t, b1, b2 by one reciprocal of det, b1 + b2 <= 1;
 *   BINARY_BVH (1): the reference's binary BVH (AcceleratorType::Bvh,
 *     Primitive::intersect, src/accelerators/bvh_common.cpp:66-103):
 *     |det| >= FLT_EPSILON, t, b1, b2 by division, b1 <= 1, b2 <= 1 - b1.
 *   The two rules disagree on near-degenerate triangles (about 0.2% of
 *   incoherent rays on a dense soup).
 * max_visits: per-ray cap on wide nodes fetched; 0 = 65536. A ray that reaches
 *   it ends as a miss and the call reports ALPINE_GPU_ERR_LIMIT.
 * stack_limit: traversal stack entries a ray may use, 1-24; 0 = 24. A ray that
 *   needs more ends as a miss and the call reports ALPINE_GPU_ERR_LIMIT. The
 *   reference's traversals stop on an assert instead
 *   (src/accelerators/bvh.cpp:231, wide_bvh.cpp:604).
 * The two limits exist so that the device-side failure path can be exercised
 * on purpose; the defaults are never reached by a BVH this library builds. */
#define ALPINE_GPU_TRIANGLE_TEST_WIDE_BVH 0u
#define ALPINE_GPU_TRIANGLE_TEST_BINARY_BVH 1u
typedef struct alpine_gpu_traversal_options {
    uint32_t triangle_test;
    uint32_t max_visits;
    uint32_t stack_limit;
} alpine_gpu_traversal_options;
ALPINE_GPU_API int alpine_gpu_set_traversal_options(alpine_gpu_ctx* ctx, const alpine_gpu_traversal_options* options);

/* Traversal statistics for `count` rays in DEVICE memory: runs the same
 * traversal as alpine_gpu_trace_device / alpine_gpu_occluded_device (any_hit
 * selects which) with counters, and writes the wide nodes fetched and the
 * triangles tested, summed over all rays. The reference's BvhStats
 * (src/accelerators/bvh_common.h:19-61, enabled by ENABLE_BVH_STATS).
 * Synchronous. */
ALPINE_GPU_API int alpine_gpu_traversal_stats(alpine_gpu_ctx* ctx, const alpine_gpu_ray* rays, uint64_t count,
                                              int any_hit, uint64_t* node_visits, uint64_t* triangle_visits);

/* ---------------------------------------------------------------------------
 * Rendering: the wavefront path tracer (alpine::render and its state,
 * src/alpine.cpp:259-483). The framebuffer size and path length come from
 * alpine_gpu_config (width, height, max_depth). */

/* Materials (src/materials/): DIELECTRIC is a uniform mixture of Lambertian
 * and GGX microfacet (F0 = 0.04), the latter only when 2 roughness^2 < 1
 * (dielectric.cpp:15-20); CONDUCTOR is GGX microfacet with F0 = base colour
 * (conductor.cpp:9-16). alpha = roughness, clamped to >= 0.001. The loaders
 * create exactly these two (gltf_loader.cpp:404-414; OBJ files yield
 * DIELECTRIC with roughness 1, obj_loader.cpp:73-75). */
#define ALPINE_GPU_MATERIAL_DIELECTRIC 0u
#define ALPINE_GPU_MATERIAL_CONDUCTOR 1u
typedef struct alpine_gpu_material {
    uint32_t kind;
    float base_color[3];
    float roughness;
} alpine_gpu_material;

/* Replaces the material table (the loaders' per-primitive Material objects,
 * src/shapes/mesh.h:16-36). Material 0 is used by triangles without one. */
ALPINE_GPU_API int alpine_gpu_set_materials(alpine_gpu_ctx* ctx, const alpine_gpu_material* materials,
                                            uint32_t count);

/* Material probes on the GPU, for arrays in HOST memory, directions in the
 * local shading frame (z = shading normal). Synchronous.
 * alpine_gpu_material_sample: Material::sample (src/materials/material.h:18-19;
 *   dielectric.cpp:31-62, conductor.cpp:18-25) for `count` (wo[3], u[2])
 *   pairs; writes wi[3], estimator[3] (bsdf * cos / pdf), pdf and ok (0 when
 *   the reference returns no sample; the other outputs are then 0).
 * alpine_gpu_material_eval: Material::computeBsdf / computePdf
 *   (material.h:21-24) at (wo[3], wi[3]) pairs, plus the true density of the
 *   direction that Material::sample outputs and its effective integrand
 *   E[estimator | wi] * density (3 floats): the quantities one-sample MIS with
 *   the learned guide uses. Output pointers may be NULL. */
ALPINE_GPU_API int alpine_gpu_material_sample(alpine_gpu_ctx* ctx, const alpine_gpu_material* material,
                                              const float* wo, const float* u, uint32_t count, float* wi,
                                              float* estimator, float* pdf, uint8_t* ok);
ALPINE_GPU_API int alpine_gpu_material_eval(alpine_gpu_ctx* ctx, const alpine_gpu_material* material,
                                            const float* wo, const float* wi, uint32_t count, float* bsdf,
                                            float* pdf, float* sample_density, float* sample_integrand);

/* Per-vertex shading normals (float[3 * vertex_count], may be NULL: the
 * geometric normal is used) and per-triangle material ids (may be NULL:
 * material 0) of one mesh (Mesh::Data normals / materials,
 * src/shapes/mesh.h:16-36; Mesh::getIntersectionAttributes, mesh.cpp:57-154). */
ALPINE_GPU_API int alpine_gpu_set_triangle_attributes(alpine_gpu_ctx* ctx, uint32_t shape_id, const float* normals,
                                                      const uint32_t* triangle_material);

/* Texture coordinates and tangents of one mesh (Mesh::Data uvs / tangents,
 * src/shapes/mesh.h:16-36), per vertex, indexed like the positions:
 * uvs float[2 * vertex_count] (NULL: none), tangents float[4 * vertex_count]
 * = xyz and the bitangent sign (NULL: none; needs uvs and the vertex normals
 * of alpine_gpu_set_triangle_attributes). With tangents the shading normal is
 * the reference's tangent-space normal (mesh.cpp:104-144):
 * normalize(B v.x + T v.y + N v.z), T and B = normalize(cross(n, t) sign)
 * interpolated per corner, v the material's normal map at uv or (0, 0, 1).
 * Tangent morph targets are not supported (the tangents stay as given). */
ALPINE_GPU_API int alpine_gpu_set_triangle_uvs(alpine_gpu_ctx* ctx, uint32_t shape_id, const float* uvs,
                                               const float* tangents);

/* Textures (Texture4f, src/texture.h): width x height float4 texels,
 * row-major, already converted as the loader does (sRGB base colours
 * linearised, normal maps remapped to [-1, 1]: gltf_loader.cpp:417-460).
 * Sampled with the reference's nearest lookup (texture.h:19-35). Writes the
 * texture id (0, 1, ... in call order). */
ALPINE_GPU_API int alpine_gpu_add_texture(alpine_gpu_ctx* ctx, const float* texels, uint32_t width, uint32_t height,
                                          uint32_t* texture_id);

/* Binds textures to one material of the table set by alpine_gpu_set_materials
 * (Dielectric / Conductor baseColorTex and normalTex, dielectric.cpp:14-21;
 * -1 = none). The base-colour texture replaces the constant colour in every
 * use (sampling, evaluation, the albedo AOV), as getBaseColor(uv) does.
 * alpine_gpu_set_materials resets the bindings. */
ALPINE_GPU_API int alpine_gpu_set_material_textures(alpine_gpu_ctx* ctx, uint32_t material,
                                                    int32_t base_color_texture, int32_t normal_texture);

/* alpine::loadEnvironmentMap (alpine.h:57; src/environment_map.cpp): a
 * lat-long map of width x height RGB texels (3 floats each, row-major) that
 * escaping rays read instead of the background colour (alpine.cpp:318-323),
 * with the reference's direction-to-texel mapping (environment_map.cpp:14-37).
 * rgb = NULL removes it. */
ALPINE_GPU_API int alpine_gpu_set_environment_map(alpine_gpu_ctx* ctx, const float* rgb, uint32_t width,
                                                  uint32_t height);

/* Binary glTF scenes (alpine::loadScene with FileType::Gltf, alpine.h:30;
 * src/loaders/gltf_loader.cpp). alpine_gpu_load_glb appends a .glb file's
 * scene to the context with the reference loader's semantics: its materials
 * (Conductor when metallicFactor > 0, else Dielectric; alpha =
 * roughnessFactor; base-colour and normal textures from 8-bit PNG images) to
 * the material table; one mesh per glTF mesh, in mesh order, with the
 * positions, normals and tangents transformed by the node's matrix, vertex
 * normals, texture coordinates and tangents; morph targets and LINEAR
 * "weights" animation channels (alpine_gpu_update_scene then animates them);
 * KHR_lights_punctual lights as point lights of intensity colour *
 * intensity. Call alpine_gpu_build afterwards. The file is read by the
 * project's own GLB parser (the reference uses tinygltf). Writes what was
 * added (info may be NULL).
 * alpine_gpu_glb_inspect parses a file without a context (no GPU needed) and
 * writes its counts (shapes = glTF meshes, first_* = 0). */
typedef struct alpine_gpu_glb_info {
    uint32_t shapes;          /* meshes added (shape ids first_shape, first_shape + 1, ...) */
    uint32_t first_shape;
    uint32_t triangles;
    uint32_t materials;       /* materials appended (ids first_material, ...) */
    uint32_t first_material;
    uint32_t textures;        /* textures created */
    uint32_t images;
    uint32_t lights;
    uint32_t channels;        /* animation channels (inspect: all; load: the ones applied) */
} alpine_gpu_glb_info;
ALPINE_GPU_API int alpine_gpu_load_glb(alpine_gpu_ctx* ctx, const char* path, alpine_gpu_glb_info* info);
ALPINE_GPU_API int alpine_gpu_glb_inspect(const char* path, alpine_gpu_glb_info* info);

/* Lights (alpine::addPointLight / addDiskLight, include/alpine/alpine.h:35-42;
 * src/lights/). A quad light is a one-sided emitting parallelogram
 * corner + [0,1] edge_u + [0,1] edge_v with constant radiance, emitting on the
 * side of cross(edge_u, edge_v); it has no counterpart in the reference and
 * follows DiskLight's sampling contract (src/lights/light.h:30-41). Lights are
 * not visible to camera rays, as in the reference. */
ALPINE_GPU_API int alpine_gpu_add_point_light(alpine_gpu_ctx* ctx, float power, const float color[3],
                                              const float position[3], uint32_t* light_id);
ALPINE_GPU_API int alpine_gpu_add_disk_light(alpine_gpu_ctx* ctx, float power, const float color[3],
                                             const float position[3], const float target[3], float radius,
                                             uint32_t* light_id);
ALPINE_GPU_API int alpine_gpu_add_quad_light(alpine_gpu_ctx* ctx, const float radiance[3], const float corner[3],
                                             const float edge_u[3], const float edge_v[3], uint32_t* light_id);
/* LightHandle::setScale (include/alpine/light.h:6-7). Rebuild the light
 * sampler afterwards for power- and BVH-based sampling. */
ALPINE_GPU_API int alpine_gpu_set_light_scale(alpine_gpu_ctx* ctx, uint32_t light_id, float scale);

/* alpine::buildLightSampler (alpine.h:44-51): call after all lights are added.
 * Same numbering as LightSamplerType. */
#define ALPINE_GPU_LIGHT_SAMPLER_UNIFORM 0
#define ALPINE_GPU_LIGHT_SAMPLER_POWER 1
#define ALPINE_GPU_LIGHT_SAMPLER_BVH 2
ALPINE_GPU_API int alpine_gpu_build_light_sampler(alpine_gpu_ctx* ctx, int type);

/* alpine::setBackgroundColor (alpine.h:53): radiance of rays that escape. */
ALPINE_GPU_API int alpine_gpu_set_background(alpine_gpu_ctx* ctx, float r, float g, float b);

/* CameraHandle::setLookAt (include/alpine/camera.h:6-12): pinhole camera,
 * fovy in radians, film at distance 1. */
ALPINE_GPU_API int alpine_gpu_set_camera(alpine_gpu_ctx* ctx, const float eye[3], const float target[3],
                                         const float up[3], float fovy, float aspect);

/* Render options (no counterpart in the reference's API).
 * sampler: REFERENCE_STREAM reproduces the reference's per-pixel xorshift128
 *   stream (src/sampler.cpp), drawn in the reference's order, one sample per
 *   pixel at a time, with FP32 arithmetic rounded like the reference;
 *   COUNTER (default) hashes (seed, pixel, sample, dimension), so all samples
 *   of a pixel run in parallel and every run is deterministic.
 * max_paths_per_wave: 0 = 2^21.
 * russian_roulette_depth: 0 = off (the reference has none); d > 0 applies
 *   roulette to continuations from depth d on (COUNTER sampler only).
 * accumulate_fp64: per-pixel sums in FP64 (long convergence runs).
 * guide: 1 = learned path guiding of the continuation direction (COUNTER
 *   sampler only). At every vertex with the view direction above the shading
 *   surface the direction comes from the guide's mixture with probability
 *   guide_fraction, else from the material's own sampling procedure, and is
 *   weighted by the one-sample MIS estimator f / (a p_guide + (1 - a) p_mat),
 *   where f and p_mat are the effective integrand and the true density of the
 *   material's procedure: the image converges to the same expectation as
 *   without guiding.
 * guide_fraction: a in (0, 1]; 0 = 0.5.
 * guide_train: 1 = record path vertices and train the guide (Adam) between
 *   waves on the radiance they received.
 * guide_batch: samples per Adam step; 0 = 16384.
 * guide_lr: Adam learning rate; 0 = 0.01.
 * guide_warmup_steps: the guide is sampled only after this many Adam steps
 *   (before that, vertices use the material's procedure and are recorded for
 *   training).
 * guide_spp_per_wave: samples per pixel per wave while the guide trains
 *   (training happens between waves); 0 = 1. Later waves are as large as
 *   unguided ones.
 * guide_steps_per_wave: at most this many Adam steps after a wave; 0 = 8.
 * guide_min_roughness: vertices whose microfacet alpha is below this use the
 *   material's procedure only and are not recorded for training (a
 *   near-specular lobe is already sampled well and is narrower than the
 *   guide's lobes); 0 = guide every vertex.
 * guide_train_steps: stop training after this many Adam steps since the
 *   guide's last reset (the guide is then used as it is); 0 = no limit.
 * cuda_graph: 1 = capture the whole wave loop of an unguided render as a CUDA
 *   graph and replay it while the launch configuration (spp, sizes, device
 *   buffers, camera, lights, options) stays the same; a rebuilt BVH of the
 *   same scene replays the same graph. Results are identical either way.
 * guide_max_depth: vertices at this depth and deeper use the material's
 *   procedure only and are not recorded (their throughput is small, their
 *   inference costs the same); 0 = guide every depth.
 * shade_order: QUEUE (0) shades the hits in the order the traversal queue
 *   holds them; BY_MATERIAL (1) first groups them (a two-pass counting sort on
 *   the GPU) by miss / material kind and lobes / guided, so that the threads of
 *   a warp take the same shading branches. Results are identical either way
 *   (each path's arithmetic does not depend on its queue position); only the
 *   selection among more training records than fit the guide's buffer
 *   depends on the order. */
#define ALPINE_GPU_SAMPLER_REFERENCE_STREAM 0u
#define ALPINE_GPU_SAMPLER_COUNTER 1u
#define ALPINE_GPU_SHADE_ORDER_QUEUE 0u
#define ALPINE_GPU_SHADE_ORDER_BY_MATERIAL 1u
typedef struct alpine_gpu_render_options {
    uint32_t sampler;
    uint32_t max_paths_per_wave;
    uint32_t russian_roulette_depth;
    uint32_t seed;
    uint32_t accumulate_fp64;
    uint32_t guide;
    float guide_fraction;
    uint32_t guide_train;
    uint32_t guide_batch;
    float guide_lr;
    uint32_t guide_warmup_steps;
    uint32_t guide_spp_per_wave;
    uint32_t guide_steps_per_wave;
    float guide_min_roughness;
    uint32_t guide_train_steps;
    uint32_t cuda_graph;
    uint32_t guide_max_depth;
    uint32_t shade_order;
} alpine_gpu_render_options;
ALPINE_GPU_API int alpine_gpu_set_render_options(alpine_gpu_ctx* ctx, const alpine_gpu_render_options* options);

/* alpine::resetAccumulation (alpine.h:60): zero the sums, restart the
 * per-pixel reference streams (Sampler::reset(pixel index)). */
ALPINE_GPU_API int alpine_gpu_reset_accumulation(alpine_gpu_ctx* ctx);

/* alpine::render(spp) (alpine.h:61, alpine.cpp:271-288): adds spp samples
 * per pixel to the accumulation. Synchronous. */
ALPINE_GPU_API int alpine_gpu_render(alpine_gpu_ctx* ctx, uint32_t spp);

/* The same without waiting: the render is enqueued on the context's stream
 * (an unguided render never waits for the GPU; a training guided render
 * waits between waves). alpine_gpu_render_wait waits for it and reports
 * device-side errors. Contexts are independent, so renders of several
 * contexts enqueued from one thread run concurrently on the GPU. Reading the
 * accumulation waits as well. */
ALPINE_GPU_API int alpine_gpu_render_async(alpine_gpu_ctx* ctx, uint32_t spp);
ALPINE_GPU_API int alpine_gpu_render_wait(alpine_gpu_ctx* ctx);
/* Number of render graphs captured and launched on this context. */
ALPINE_GPU_API int alpine_gpu_render_graph_stats(alpine_gpu_ctx* ctx, uint32_t* captures, uint32_t* launches);

/* Autotuner (no counterpart in the reference): renders probe_spp samples per
 * pixel (0 = 4) for each wave size (2^18 ... 2^22 paths) and traversal block
 * size (64, 128, 256 threads), keeps the fastest pair for this context and
 * writes it. When the render options enable guiding, it then times each of
 * the guide's inference kernels (ALPINE_GPU_GUIDE_KERNEL_*, identical
 * outputs) with training paused and keeps the faster (guide_kernel; otherwise
 * guide_kernel reports the current one). The guide's weights and Adam steps
 * are left as they were; the accumulation is reset. */
typedef struct alpine_gpu_tuning {
    uint32_t max_paths_per_wave;
    uint32_t trace_block;
    float samples_per_second;
    uint32_t guide_kernel;
} alpine_gpu_tuning;
ALPINE_GPU_API int alpine_gpu_autotune(alpine_gpu_ctx* ctx, uint32_t probe_spp, alpine_gpu_tuning* result);

/* Per-pixel sums of colour, albedo and normal (9 floats per pixel, the
 * reference's RenderTarget layout, src/denoisers/denoiser.h:7-12) and the
 * number of samples accumulated. Either pointer may be NULL. */
ALPINE_GPU_API int alpine_gpu_read_accumulation(alpine_gpu_ctx* ctx, float* sums, uint32_t* total_samples);
ALPINE_GPU_API int alpine_gpu_read_accumulation_f64(alpine_gpu_ctx* ctx, double* sums, uint32_t* total_samples);

/* Checkpoint / resume of a long render (alpine::render accumulates into
 * mAccumBuffer / mTotalSamples and continues each pixel's Sampler stream,
 * src/alpine.cpp:259-288; the reference keeps them in memory only). Restores
 * the sums (the layout of alpine_gpu_read_accumulation, converted to the
 * context's accumulation precision) and the sample count, and, for the
 * REFERENCE_STREAM sampler, the per-pixel stream states of
 * alpine_gpu_read_sampler_state. The next render continues exactly as the
 * interrupted run would have: the COUNTER sampler numbers samples from
 * total_samples on. Set the render options first. */
ALPINE_GPU_API int alpine_gpu_write_accumulation(alpine_gpu_ctx* ctx, const float* sums, uint32_t total_samples);
ALPINE_GPU_API int alpine_gpu_write_accumulation_f64(alpine_gpu_ctx* ctx, const double* sums,
                                                     uint32_t total_samples);
ALPINE_GPU_API int alpine_gpu_write_sampler_state(alpine_gpu_ctx* ctx, const uint32_t* state);

/* alpine::postProcess + getFrameBuffer (alpine.h:63-65, alpine.cpp:446-483)
 * without the denoiser: mean colour (3 floats per pixel, may be NULL) and the
 * tone-mapped (ACES when tonemap != 0), clamped, sRGB-encoded 8-bit image
 * (3 bytes per pixel, may be NULL). */
ALPINE_GPU_API int alpine_gpu_post_process(alpine_gpu_ctx* ctx, int tonemap, float* mean_rgb, uint8_t* rgb8);

/* ---------------------------------------------------------------------------
 * Learned path guiding (no counterpart in the reference): a hash-grid encoded
 * MLP predicting an 8-lobe von Mises-Fisher mixture over incident directions,
 * trained online. These entry points expose the model for tests and tools;
 * the integrator uses it when alpine_gpu_render_options.guide is set.
 * Query record: 12 floats {pos[3], roughness, wo[3], 0, normal[3], 0}.
 * Sample record: 16 floats {query[12], dir[3], weight}.
 * Raw output: 40 floats = 8 lobes x {direction[3], log kappa, logit}.
 * alpine_gpu_guide_dims: resolutions receives one grid resolution per level
 * (8 levels of 4 features; room for 16 entries), the grid parameters are
 * [level][entry][feature]. */
ALPINE_GPU_API int alpine_gpu_guide_dims(uint32_t* weight_count, uint64_t* grid_params, uint32_t* table_size,
                                         uint32_t* resolutions);
ALPINE_GPU_API int alpine_gpu_guide_reset(alpine_gpu_ctx* ctx, uint32_t seed, const float scene_lo[3],
                                          const float scene_hi[3]);
ALPINE_GPU_API int alpine_gpu_guide_infer(alpine_gpu_ctx* ctx, const float* queries, uint32_t count, float* raw);
/* The same on DEVICE buffers (queries: 12 floats each, raw: 40 floats each),
 * launched on `stream` (NULL: the context's stream) without synchronising;
 * device-side errors are reported by the next alpine_gpu_synchronize. */
ALPINE_GPU_API int alpine_gpu_guide_infer_device(alpine_gpu_ctx* ctx, const float* queries, uint32_t count, float* raw,
                                                 void* stream);
/* Inference kernel of the guide (rendering and alpine_gpu_guide_infer):
 * WARP_MMA (default): each warp runs 32 queries through the MLP with
 *   warp-level mma.sync tiles; TENSOR_MEMORY: tiles of 128 queries run
 *   through tcgen05 MMAs with the accumulators in tensor memory (sm_100a).
 * Both compute the same BF16 x BF16 -> FP32 products; sums may differ in the
 * last bits (accumulation order). */
#define ALPINE_GPU_GUIDE_KERNEL_WARP_MMA 0
#define ALPINE_GPU_GUIDE_KERNEL_TENSOR_MEMORY 1
ALPINE_GPU_API int alpine_gpu_guide_set_kernel(alpine_gpu_ctx* ctx, int kernel);
/* Weight-gradient kernel of the guide's training, dW_l = dY_l^T X_l over a
 * slice of samples per layer: TENSOR_MEMORY (default) runs it as tcgen05
 * MMAs (M 128 with the layer's output rows zero-padded, N 64, K 16 per
 * instruction over 64-sample stages) accumulating in tensor memory, one CTA
 * per (split of the samples, layer); WARP_MMA runs mma.sync tiles, one warp
 * per (layer, 16 rows, split). Both sum BF16 x BF16 products in FP32; the
 * sums differ in the last bits (order). */
ALPINE_GPU_API int alpine_gpu_guide_set_gradient_kernel(alpine_gpu_ctx* ctx, int kernel);
/* Adam steps taken since the last reset, waves rendered with guiding, and the
 * mean training loss (KL divergence up to a constant) of the last trained
 * wave's steps (0 before any). Any pointer may be NULL. */
ALPINE_GPU_API int alpine_gpu_guide_steps(alpine_gpu_ctx* ctx, uint32_t* adam_steps, uint32_t* guided_waves,
                                          float* last_loss);
ALPINE_GPU_API int alpine_gpu_guide_gradients(alpine_gpu_ctx* ctx, const float* samples, uint32_t count, float* dW,
                                              const uint64_t* grid_index, uint32_t grid_count, float* grid_grad,
                                              float* loss);
ALPINE_GPU_API int alpine_gpu_guide_train(alpine_gpu_ctx* ctx, const float* samples, uint32_t count, float lr,
                                          float* loss);
ALPINE_GPU_API int alpine_gpu_guide_get_weights(alpine_gpu_ctx* ctx, float* weights);
ALPINE_GPU_API int alpine_gpu_guide_set_weights(alpine_gpu_ctx* ctx, const float* weights);
ALPINE_GPU_API int alpine_gpu_guide_grid(alpine_gpu_ctx* ctx, const uint64_t* index, uint32_t count, float* read,
                                         const float* write);
ALPINE_GPU_API int alpine_gpu_guide_sample_mixture(alpine_gpu_ctx* ctx, const float* raw, const float* u,
                                                   uint32_t count, float* dirs, float* pdfs);

/* Per-pixel state of the reference random stream (4 words per pixel, the
 * reference's Sampler state, src/sampler.h; src/alpine.cpp:108), as left by
 * the last render in REFERENCE_STREAM mode. For parity checks of the draw
 * order. */
ALPINE_GPU_API int alpine_gpu_read_sampler_state(alpine_gpu_ctx* ctx, uint32_t* state);

/* Waits for all work of the context and reports device-side errors. */
ALPINE_GPU_API int alpine_gpu_synchronize(alpine_gpu_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
