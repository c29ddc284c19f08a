"""ctypes binding of the C ABI (include/alpine_gpu.h) and a thin Python wrapper.

The CUDA library must have been built (``python -m alpine_b200.build``); there
is no fallback: importing this module without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

# ALPINE_GPU_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("ALPINE_GPU_LIB", _build.LIB)

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_CUDA = -2
ERR_INVALID_STATE = -3
ERR_LIMIT = -4
ERR_OUT_OF_MEMORY = -5

RAY_DTYPE = np.dtype([("org", np.float32, 3), ("tmin", np.float32), ("dir", np.float32, 3), ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("prim", np.uint32), ("t", np.float32), ("b1", np.float32), ("b2", np.float32)])
MISS = 0xFFFFFFFF
NOALLOC_MAX_RAYS = 65536
GUIDE_KERNEL_WARP_MMA = 0
GUIDE_KERNEL_TENSOR_MEMORY = 1
TRIANGLE_TEST_WIDE_BVH = 0
TRIANGLE_TEST_BINARY_BVH = 1
SHADE_ORDER_QUEUE = 0
SHADE_ORDER_BY_MATERIAL = 1
SHADE_ORDER_DEFAULT = SHADE_ORDER_BY_MATERIAL
COLLAPSE_SAH = 0
COLLAPSE_GREEDY = 1


class GpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"alpine_gpu error {code}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("width", C.c_uint32), ("height", C.c_uint32), ("max_depth", C.c_uint32)]


class BvhStats(C.Structure):
    _fields_ = [("triangles", C.c_uint32), ("binary_nodes", C.c_uint32), ("binary_levels", C.c_uint32),
                ("wide_nodes", C.c_uint32), ("wide_depth", C.c_uint32), ("sah_cost", C.c_float),
                ("build_ms", C.c_float), ("spheres", C.c_uint32), ("child_slots", C.c_uint32),
                ("big_levels", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RenderOptions(C.Structure):
    _fields_ = [("sampler", C.c_uint32), ("max_paths_per_wave", C.c_uint32), ("russian_roulette_depth", C.c_uint32),
                ("seed", C.c_uint32), ("accumulate_fp64", C.c_uint32), ("guide", C.c_uint32),
                ("guide_fraction", C.c_float), ("guide_train", C.c_uint32), ("guide_batch", C.c_uint32),
                ("guide_lr", C.c_float), ("guide_warmup_steps", C.c_uint32), ("guide_spp_per_wave", C.c_uint32),
                ("guide_steps_per_wave", C.c_uint32), ("guide_min_roughness", C.c_float),
                ("guide_train_steps", C.c_uint32), ("cuda_graph", C.c_uint32),
                ("guide_max_depth", C.c_uint32), ("shade_order", C.c_uint32)]


class TraversalOptions(C.Structure):
    _fields_ = [("triangle_test", C.c_uint32), ("max_visits", C.c_uint32), ("stack_limit", C.c_uint32)]


class BuildOptions(C.Structure):
    _fields_ = [("collapse", C.c_uint32), ("triangle_cost", C.c_float)]


class GlbInfo(C.Structure):
    _fields_ = [("shapes", C.c_uint32), ("first_shape", C.c_uint32), ("triangles", C.c_uint32),
                ("materials", C.c_uint32), ("first_material", C.c_uint32), ("textures", C.c_uint32),
                ("images", C.c_uint32), ("lights", C.c_uint32), ("channels", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("max_paths_per_wave", C.c_uint32), ("trace_block", C.c_uint32), ("samples_per_second", C.c_float),
                ("guide_kernel", C.c_uint32)]


MATERIAL_DTYPE = np.dtype([("kind", np.uint32), ("base_color", np.float32, 3), ("roughness", np.float32)])
DIELECTRIC = 0
CONDUCTOR = 1
SAMPLER_UNIFORM, SAMPLER_POWER, SAMPLER_BVH = 0, 1, 2
RNG_REFERENCE_STREAM, RNG_COUNTER = 0, 1

_lib = None


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def lib():
    """Loads libalpine_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m alpine_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.alpine_gpu_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
        L.alpine_gpu_destroy.argtypes = [vp]
        L.alpine_gpu_destroy.restype = None
        L.alpine_gpu_last_error.argtypes = [vp]
        L.alpine_gpu_last_error.restype = C.c_char_p
        L.alpine_gpu_reset_scene.argtypes = [vp]
        L.alpine_gpu_add_mesh.argtypes = [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(C.c_uint32)]
        L.alpine_gpu_add_spheres.argtypes = [vp, vp, C.c_uint32, vp, C.POINTER(C.c_uint32)]
        L.alpine_gpu_update_vertices.argtypes = [vp, C.c_uint32, vp]
        L.alpine_gpu_build.argtypes = [vp, C.POINTER(BvhStats)]
        L.alpine_gpu_set_morph_targets.argtypes = [vp, C.c_uint32, vp, vp, C.c_uint32]
        L.alpine_gpu_add_animation_channel.argtypes = [vp, C.c_uint32, vp, vp, C.c_uint32]
        L.alpine_gpu_update_scene.argtypes = [vp, C.c_float, C.POINTER(BvhStats)]
        L.alpine_gpu_build_async.argtypes = [vp, C.c_uint32, C.c_uint32]
        L.alpine_gpu_update_scene_async.argtypes = [vp, C.c_float]
        L.alpine_gpu_read_build_stats.argtypes = [vp, C.POINTER(BvhStats), C.POINTER(C.c_uint32),
                                                  C.POINTER(C.c_uint32)]
        L.alpine_gpu_get_vertices.argtypes = [vp, C.c_uint32, vp, vp]
        L.alpine_gpu_trace.argtypes = [vp, vp, C.c_uint64, vp]
        L.alpine_gpu_occluded.argtypes = [vp, vp, C.c_uint64, vp]
        L.alpine_gpu_trace_device.argtypes = [vp, vp, C.c_uint64, vp, vp]
        L.alpine_gpu_occluded_device.argtypes = [vp, vp, C.c_uint64, vp, vp]
        L.alpine_gpu_synchronize.argtypes = [vp]
        L.alpine_gpu_trace_noalloc.argtypes = [vp, vp, C.c_uint64, vp]
        L.alpine_gpu_set_traversal_options.argtypes = [vp, C.POINTER(TraversalOptions)]
        L.alpine_gpu_set_build_options.argtypes = [vp, C.POINTER(BuildOptions)]
        f3 = C.POINTER(C.c_float)
        u32p = C.POINTER(C.c_uint32)
        L.alpine_gpu_set_materials.argtypes = [vp, vp, C.c_uint32]
        L.alpine_gpu_material_sample.argtypes = [vp, vp, vp, vp, C.c_uint32, vp, vp, vp, vp]
        L.alpine_gpu_material_eval.argtypes = [vp, vp, vp, vp, C.c_uint32, vp, vp, vp, vp]
        L.alpine_gpu_set_triangle_attributes.argtypes = [vp, C.c_uint32, vp, vp]
        L.alpine_gpu_set_triangle_uvs.argtypes = [vp, C.c_uint32, vp, vp]
        L.alpine_gpu_add_texture.argtypes = [vp, vp, C.c_uint32, C.c_uint32, u32p]
        L.alpine_gpu_set_material_textures.argtypes = [vp, C.c_uint32, C.c_int32, C.c_int32]
        L.alpine_gpu_set_environment_map.argtypes = [vp, vp, C.c_uint32, C.c_uint32]
        L.alpine_gpu_load_glb.argtypes = [vp, C.c_char_p, C.POINTER(GlbInfo)]
        L.alpine_gpu_glb_inspect.argtypes = [C.c_char_p, C.POINTER(GlbInfo)]
        L.alpine_gpu_add_point_light.argtypes = [vp, C.c_float, f3, f3, u32p]
        L.alpine_gpu_add_disk_light.argtypes = [vp, C.c_float, f3, f3, f3, C.c_float, u32p]
        L.alpine_gpu_add_quad_light.argtypes = [vp, f3, f3, f3, f3, u32p]
        L.alpine_gpu_set_light_scale.argtypes = [vp, C.c_uint32, C.c_float]
        L.alpine_gpu_build_light_sampler.argtypes = [vp, C.c_int]
        L.alpine_gpu_set_background.argtypes = [vp, C.c_float, C.c_float, C.c_float]
        L.alpine_gpu_set_camera.argtypes = [vp, f3, f3, f3, C.c_float, C.c_float]
        L.alpine_gpu_set_render_options.argtypes = [vp, C.POINTER(RenderOptions)]
        L.alpine_gpu_reset_accumulation.argtypes = [vp]
        L.alpine_gpu_render.argtypes = [vp, C.c_uint32]
        L.alpine_gpu_render_async.argtypes = [vp, C.c_uint32]
        L.alpine_gpu_render_wait.argtypes = [vp]
        L.alpine_gpu_render_graph_stats.argtypes = [vp, u32p, u32p]
        L.alpine_gpu_autotune.argtypes = [vp, C.c_uint32, C.POINTER(Tuning)]
        L.alpine_gpu_read_accumulation.argtypes = [vp, vp, u32p]
        L.alpine_gpu_read_accumulation_f64.argtypes = [vp, vp, u32p]
        L.alpine_gpu_post_process.argtypes = [vp, C.c_int, vp, vp]
        L.alpine_gpu_read_sampler_state.argtypes = [vp, vp]
        L.alpine_gpu_write_accumulation.argtypes = [vp, vp, C.c_uint32]
        L.alpine_gpu_write_accumulation_f64.argtypes = [vp, vp, C.c_uint32]
        L.alpine_gpu_write_sampler_state.argtypes = [vp, vp]
        L.alpine_gpu_guide_dims.argtypes = [u32p, C.POINTER(C.c_uint64), u32p, u32p]
        L.alpine_gpu_guide_reset.argtypes = [vp, C.c_uint32, f3, f3]
        L.alpine_gpu_guide_infer.argtypes = [vp, vp, C.c_uint32, vp]
        L.alpine_gpu_guide_infer_device.argtypes = [vp, vp, C.c_uint32, vp, vp]
        L.alpine_gpu_guide_steps.argtypes = [vp, u32p, u32p, C.POINTER(C.c_float)]
        L.alpine_gpu_guide_set_kernel.argtypes = [vp, C.c_int]
        L.alpine_gpu_guide_set_gradient_kernel.argtypes = [vp, C.c_int]
        L.alpine_gpu_guide_gradients.argtypes = [vp, vp, C.c_uint32, vp, vp, C.c_uint32, vp, vp]
        L.alpine_gpu_guide_train.argtypes = [vp, vp, C.c_uint32, C.c_float, f3]
        L.alpine_gpu_guide_get_weights.argtypes = [vp, vp]
        L.alpine_gpu_guide_set_weights.argtypes = [vp, vp]
        L.alpine_gpu_guide_grid.argtypes = [vp, vp, C.c_uint32, vp, vp]
        L.alpine_gpu_guide_sample_mixture.argtypes = [vp, vp, vp, C.c_uint32, vp, vp]
        L.alpine_gpu_traversal_stats.argtypes = [vp, vp, C.c_uint64, C.c_int, C.POINTER(C.c_uint64),
                                                 C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def glb_inspect(path) -> dict:
    """Counts of a .glb file's contents (no context or GPU needed)."""
    info = GlbInfo()
    rc = lib().alpine_gpu_glb_inspect(str(path).encode(), C.byref(info))
    if rc != OK:
        raise GpuError(rc, f"cannot read {path} as binary glTF")
    return info.as_dict()


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Context:
    """One alpine_gpu context (one device, one stream)."""

    def __init__(self, device=0, width=0, height=0, max_depth=8):
        self.L = lib()
        self.h = C.c_void_p()
        cfg = Config(device, width, height, max_depth)
        rc = self.L.alpine_gpu_create(C.byref(cfg), C.byref(self.h))
        if rc != OK:
            raise GpuError(rc, "alpine_gpu_create failed")
        self.stats = None

    def _check(self, rc):
        if rc != OK:
            raise GpuError(rc, self.L.alpine_gpu_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self.L.alpine_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset_scene(self):
        self._check(self.L.alpine_gpu_reset_scene(self.h))

    def add_mesh(self, verts, idx) -> int:
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
        sid = C.c_uint32()
        self._check(self.L.alpine_gpu_add_mesh(self.h, _ptr(v), v.shape[0], _ptr(i), i.shape[0], C.byref(sid)))
        return sid.value

    def add_spheres(self, spheres, material=None) -> int:
        """Analytic spheres float[N, 4] (centre, radius), material id per
        sphere; returns the index of the first (hits report 0x80000000 | index)."""
        s = np.ascontiguousarray(spheres, np.float32).reshape(-1, 4)
        m = None if material is None else np.ascontiguousarray(material, np.uint32)
        first = C.c_uint32()
        self._check(self.L.alpine_gpu_add_spheres(self.h, _ptr(s), s.shape[0], None if m is None else _ptr(m),
                                                  C.byref(first)))
        return first.value

    def update_vertices(self, shape, verts):
        v = np.ascontiguousarray(verts, np.float32)
        self._check(self.L.alpine_gpu_update_vertices(self.h, shape, _ptr(v)))

    def set_morph_targets(self, shape, vertex_deltas, normal_deltas=None):
        """vertex_deltas (and normal_deltas): float[T, V, 3] morph targets."""
        vd = np.ascontiguousarray(vertex_deltas, np.float32)
        nd = None if normal_deltas is None else np.ascontiguousarray(normal_deltas, np.float32)
        t = vd.shape[0] if vd.ndim == 3 else 1
        self._check(self.L.alpine_gpu_set_morph_targets(self.h, shape, _ptr(vd), None if nd is None else _ptr(nd), t))

    def add_animation_channel(self, shape, times, weights):
        """times: float[K]; weights: float[K, T]."""
        tt = np.ascontiguousarray(times, np.float32)
        ww = np.ascontiguousarray(weights, np.float32)
        self._check(self.L.alpine_gpu_add_animation_channel(self.h, shape, _ptr(tt), _ptr(ww), tt.size))

    def update_scene(self, time) -> dict:
        """Alpine::updateScene: morph on the GPU, then rebuild the BVH."""
        s = BvhStats()
        self._check(self.L.alpine_gpu_update_scene(self.h, float(time), C.byref(s)))
        self.stats = s.as_dict()
        return self.stats

    def get_vertices(self, shape, count):
        """(positions float[count, 3], vertex normals float[count, 3]) of one mesh."""
        v = np.empty((count, 3), np.float32)
        n = np.empty((count, 3), np.float32)
        self._check(self.L.alpine_gpu_get_vertices(self.h, shape, _ptr(v), _ptr(n)))
        return v, n

    def build(self) -> dict:
        s = BvhStats()
        self._check(self.L.alpine_gpu_build(self.h, C.byref(s)))
        self.stats = s.as_dict()
        return self.stats

    def build_async(self, max_binary_levels=0, max_wide_levels=0):
        """Rebuild enqueued on the context stream with no host wait (the same
        tree as build(); a captured graph replayed). 0 = the last build()'s
        depths plus a margin. Device-side errors surface at synchronize()."""
        self._check(self.L.alpine_gpu_build_async(self.h, max_binary_levels, max_wide_levels))

    def update_scene_async(self, time):
        """update_scene's morph and build_async, enqueued without a host wait."""
        self._check(self.L.alpine_gpu_update_scene_async(self.h, float(time)))

    def read_build_stats(self) -> dict:
        """Statistics of the last build_async (waits for the stream), with the
        number of captures and replays of its graph."""
        s = BvhStats()
        cap, lau = C.c_uint32(), C.c_uint32()
        self._check(self.L.alpine_gpu_read_build_stats(self.h, C.byref(s), C.byref(cap), C.byref(lau)))
        d = s.as_dict()
        d["graph_captures"] = cap.value
        d["graph_launches"] = lau.value
        return d

    def trace(self, rays: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.empty(r.shape[0], HIT_DTYPE) if out is None else out
        self._check(self.L.alpine_gpu_trace(self.h, _ptr(r), r.shape[0], _ptr(hits)))
        return hits

    def trace_noalloc(self, rays: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """Closest hit through the entry point that allocates no memory
        (at most NOALLOC_MAX_RAYS rays per call)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.empty(r.shape[0], HIT_DTYPE) if out is None else out
        self._check(self.L.alpine_gpu_trace_noalloc(self.h, _ptr(r), r.shape[0], _ptr(hits)))
        return hits

    def occluded(self, rays: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.empty(r.shape[0], np.uint8) if out is None else out
        self._check(self.L.alpine_gpu_occluded(self.h, _ptr(r), r.shape[0], _ptr(occ)))
        return occ

    def trace_device(self, rays_ptr: int, n: int, hits_ptr: int, stream: int = 0):
        self._check(self.L.alpine_gpu_trace_device(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr),
                                                   C.c_void_p(stream or None)))

    def occluded_device(self, rays_ptr: int, n: int, occ_ptr: int, stream: int = 0):
        self._check(self.L.alpine_gpu_occluded_device(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(occ_ptr),
                                                      C.c_void_p(stream or None)))

    def set_traversal_options(self, triangle_test=TRIANGLE_TEST_WIDE_BVH, max_visits=0, stack_limit=0):
        """Triangle rule of every traversal (the reference's 8-wide or binary
        BVH) and the per-ray device-side limits (0 = defaults)."""
        o = TraversalOptions(triangle_test, max_visits, stack_limit)
        self._check(self.L.alpine_gpu_set_traversal_options(self.h, C.byref(o)))

    def set_build_options(self, collapse=COLLAPSE_SAH, triangle_cost=0.0):
        """Collapse rule of the next builds (COLLAPSE_SAH: SAH-optimal, the
        default; COLLAPSE_GREEDY: the reference's rule) and the SAH cost of a
        triangle test per wide-node visit (0 = 1.0)."""
        o = BuildOptions(collapse, triangle_cost)
        self._check(self.L.alpine_gpu_set_build_options(self.h, C.byref(o)))

    def traversal_stats(self, rays_ptr: int, n: int, any_hit: bool):
        """(wide nodes fetched, triangles tested) summed over n device rays."""
        nv, tv = C.c_uint64(), C.c_uint64()
        self._check(self.L.alpine_gpu_traversal_stats(self.h, C.c_void_p(rays_ptr), n, int(any_hit), C.byref(nv),
                                                      C.byref(tv)))
        return nv.value, tv.value

    # ---- rendering -------------------------------------------------------
    def set_materials(self, materials):
        """materials: sequence of (kind, (r, g, b), roughness[, base texture,
        normal texture]); texture ids from add_texture, None / -1 = none."""
        m = np.zeros(len(materials), MATERIAL_DTYPE)
        for i, (k, col, r, *_) in enumerate(materials):
            m[i] = (k, col, r)
        self._check(self.L.alpine_gpu_set_materials(self.h, _ptr(m) if len(m) else None, len(m)))
        for i, mat in enumerate(materials):
            if len(mat) > 3:
                bt = -1 if mat[3] is None else mat[3]
                nt = -1 if len(mat) < 5 or mat[4] is None else mat[4]
                if bt >= 0 or nt >= 0:
                    self.set_material_textures(i, bt, nt)

    @staticmethod
    def _material(material):
        k, col, r = material
        m = np.zeros(1, MATERIAL_DTYPE)
        m[0] = (k, col, r)
        return m

    def material_sample(self, material, wo, u):
        """Material::sample on the GPU. material: (kind, (r, g, b), roughness);
        wo: (n, 3), u: (n, 2). Returns wi (n, 3), estimator (n, 3), pdf (n,),
        ok (n,) bool."""
        m = self._material(material)
        wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
        u = np.ascontiguousarray(u, np.float32).reshape(-1, 2)
        n = wo.shape[0]
        if u.shape[0] != n:
            raise ValueError("wo and u differ in length")
        wi = np.zeros((n, 3), np.float32)
        est = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        ok = np.zeros(n, np.uint8)
        self._check(self.L.alpine_gpu_material_sample(self.h, _ptr(m), _ptr(wo), _ptr(u), n, _ptr(wi), _ptr(est),
                                                      _ptr(pdf), _ptr(ok)))
        return wi, est, pdf, ok.astype(bool)

    def material_eval(self, material, wo, wi):
        """computeBsdf, computePdf and the sampling procedure's true density
        and effective integrand at (wo, wi) pairs. Returns bsdf (n, 3),
        pdf (n,), density (n,), integrand (n, 3)."""
        m = self._material(material)
        wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
        wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
        n = wo.shape[0]
        if wi.shape[0] != n:
            raise ValueError("wo and wi differ in length")
        bsdf = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        dens = np.zeros(n, np.float32)
        integ = np.zeros((n, 3), np.float32)
        self._check(self.L.alpine_gpu_material_eval(self.h, _ptr(m), _ptr(wo), _ptr(wi), n, _ptr(bsdf), _ptr(pdf),
                                                    _ptr(dens), _ptr(integ)))
        return bsdf, pdf, dens, integ

    def set_triangle_attributes(self, shape, normals=None, tri_material=None):
        n = None if normals is None else np.ascontiguousarray(normals, np.float32)
        t = None if tri_material is None else np.ascontiguousarray(tri_material, np.uint32)
        self._check(self.L.alpine_gpu_set_triangle_attributes(self.h, shape, None if n is None else _ptr(n),
                                                              None if t is None else _ptr(t)))

    def set_triangle_uvs(self, shape, uvs=None, tangents=None):
        """Per-vertex texture coordinates float[V, 2] and tangents float[V, 4]."""
        u = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
        t = None if tangents is None else np.ascontiguousarray(tangents, np.float32)
        self._check(self.L.alpine_gpu_set_triangle_uvs(self.h, shape, None if u is None else _ptr(u),
                                                       None if t is None else _ptr(t)))

    def add_texture(self, rgba) -> int:
        """float32 [H, W, 4] texels; returns the texture id."""
        t = np.ascontiguousarray(rgba, np.float32)
        i = C.c_uint32()
        self._check(self.L.alpine_gpu_add_texture(self.h, _ptr(t), t.shape[1], t.shape[0], C.byref(i)))
        return i.value

    def set_material_textures(self, material, base_color=-1, normal=-1):
        self._check(self.L.alpine_gpu_set_material_textures(self.h, material, base_color, normal))

    def load_glb(self, path) -> dict:
        """Appends a binary glTF scene (alpine::loadScene, FileType::Gltf)."""
        info = GlbInfo()
        self._check(self.L.alpine_gpu_load_glb(self.h, str(path).encode(), C.byref(info)))
        return info.as_dict()

    def set_environment_map(self, rgb):
        """float32 [H, W, 3] lat-long map (None removes it)."""
        if rgb is None:
            self._check(self.L.alpine_gpu_set_environment_map(self.h, None, 0, 0))
            return
        e = np.ascontiguousarray(rgb, np.float32)
        self._check(self.L.alpine_gpu_set_environment_map(self.h, _ptr(e), e.shape[1], e.shape[0]))

    def add_point_light(self, power, color, position):
        i = C.c_uint32()
        self._check(self.L.alpine_gpu_add_point_light(self.h, power, _f3(color), _f3(position), C.byref(i)))
        return i.value

    def add_disk_light(self, power, color, position, target, radius):
        i = C.c_uint32()
        self._check(self.L.alpine_gpu_add_disk_light(self.h, power, _f3(color), _f3(position), _f3(target), radius,
                                                     C.byref(i)))
        return i.value

    def add_quad_light(self, radiance, corner, edge_u, edge_v):
        i = C.c_uint32()
        self._check(self.L.alpine_gpu_add_quad_light(self.h, _f3(radiance), _f3(corner), _f3(edge_u), _f3(edge_v),
                                                     C.byref(i)))
        return i.value

    def set_light_scale(self, light, scale):
        self._check(self.L.alpine_gpu_set_light_scale(self.h, light, scale))

    def build_light_sampler(self, kind):
        self._check(self.L.alpine_gpu_build_light_sampler(self.h, kind))

    def set_background(self, r, g, b):
        self._check(self.L.alpine_gpu_set_background(self.h, r, g, b))

    def set_camera(self, eye, target, up, fovy, aspect):
        self._check(self.L.alpine_gpu_set_camera(self.h, _f3(eye), _f3(target), _f3(up), fovy, aspect))

    def set_render_options(self, sampler=RNG_COUNTER, max_paths_per_wave=0, russian_roulette_depth=0, seed=0,
                           accumulate_fp64=False, guide=False, guide_fraction=0.5, guide_train=True,
                           guide_batch=16384, guide_lr=1e-2, guide_warmup_steps=0, guide_spp_per_wave=1,
                           guide_steps_per_wave=8, guide_min_roughness=0.0, guide_train_steps=0, cuda_graph=False,
                           guide_max_depth=0, shade_order=None):
        """Options of alpine_gpu_render_options; the guide_* fields apply when
        guide is set (learned path guiding, counter sampler only)."""
        o = RenderOptions(sampler, max_paths_per_wave, russian_roulette_depth, seed, int(accumulate_fp64),
                          int(guide), guide_fraction, int(guide_train), guide_batch, guide_lr, guide_warmup_steps,
                          guide_spp_per_wave, guide_steps_per_wave, guide_min_roughness, guide_train_steps,
                          int(cuda_graph), guide_max_depth,
                          SHADE_ORDER_DEFAULT if shade_order is None else shade_order)
        self._check(self.L.alpine_gpu_set_render_options(self.h, C.byref(o)))

    def reset_accumulation(self):
        self._check(self.L.alpine_gpu_reset_accumulation(self.h))

    def render(self, spp):
        self._check(self.L.alpine_gpu_render(self.h, spp))

    def render_async(self, spp):
        """Enqueues a render on the context's stream (see alpine_gpu_render_async)."""
        self._check(self.L.alpine_gpu_render_async(self.h, spp))

    def render_wait(self):
        self._check(self.L.alpine_gpu_render_wait(self.h))

    def graph_stats(self):
        """(render graphs captured, render graphs launched)."""
        a, b = C.c_uint32(), C.c_uint32()
        self._check(self.L.alpine_gpu_render_graph_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, probe_spp=4):
        """Picks the wave size and traversal block size for this scene, and the
        guide's inference kernel when guiding is on; resets the accumulation."""
        t = Tuning()
        self._check(self.L.alpine_gpu_autotune(self.h, probe_spp, C.byref(t)))
        return {"max_paths_per_wave": t.max_paths_per_wave, "trace_block": t.trace_block,
                "samples_per_second": t.samples_per_second, "guide_kernel": t.guide_kernel}

    def read_accumulation(self, width, height, fp64=False):
        """(sums float[H, W, 9] = colour, albedo, normal sums; total samples)."""
        out = np.empty((height, width, 9), np.float64 if fp64 else np.float32)
        n = C.c_uint32()
        f = self.L.alpine_gpu_read_accumulation_f64 if fp64 else self.L.alpine_gpu_read_accumulation
        self._check(f(self.h, _ptr(out), C.byref(n)))
        return out, n.value

    def read_sampler_state(self, width, height):
        out = np.empty((height, width, 4), np.uint32)
        self._check(self.L.alpine_gpu_read_sampler_state(self.h, _ptr(out)))
        return out

    def write_accumulation(self, sums, total_samples):
        """Checkpoint restore: sums float32 or float64 [H, W, 9] and the sample count."""
        a = np.ascontiguousarray(sums)
        if a.dtype == np.float64:
            self._check(self.L.alpine_gpu_write_accumulation_f64(self.h, _ptr(a), total_samples))
        else:
            a = np.ascontiguousarray(a, np.float32)
            self._check(self.L.alpine_gpu_write_accumulation(self.h, _ptr(a), total_samples))

    def write_sampler_state(self, state):
        s = np.ascontiguousarray(state, np.uint32)
        self._check(self.L.alpine_gpu_write_sampler_state(self.h, _ptr(s)))

    def post_process(self, width, height, tonemap=True):
        mean = np.empty((height, width, 3), np.float32)
        ldr = np.empty((height, width, 3), np.uint8)
        self._check(self.L.alpine_gpu_post_process(self.h, int(tonemap), _ptr(mean), _ptr(ldr)))
        return mean, ldr

    # ---- learned guide ----------------------------------------------------
    def guide_dims(self):
        wc, gp, ts = C.c_uint32(), C.c_uint64(), C.c_uint32()
        res = (C.c_uint32 * 16)()
        self._check(self.L.alpine_gpu_guide_dims(C.byref(wc), C.byref(gp), C.byref(ts), res))
        return {"weights": wc.value, "grid_params": gp.value, "table_size": ts.value, "res": [r for r in res if r]}

    def guide_reset(self, seed, lo, hi):
        self._check(self.L.alpine_gpu_guide_reset(self.h, seed, _f3(lo), _f3(hi)))

    def guide_steps(self, with_loss=False):
        """(Adam steps since the last reset, waves rendered with guiding[, mean
        loss of the last trained wave])."""
        a, b, l = C.c_uint32(), C.c_uint32(), C.c_float()
        self._check(self.L.alpine_gpu_guide_steps(self.h, C.byref(a), C.byref(b), C.byref(l)))
        return (a.value, b.value, l.value) if with_loss else (a.value, b.value)

    def guide_set_kernel(self, kernel):
        """GUIDE_KERNEL_WARP_MMA (mma.sync) or GUIDE_KERNEL_TENSOR_MEMORY (tcgen05)."""
        self._check(self.L.alpine_gpu_guide_set_kernel(self.h, kernel))

    def guide_set_gradient_kernel(self, kernel):
        """Training's weight-gradient kernel: GUIDE_KERNEL_TENSOR_MEMORY
        (tcgen05, default) or GUIDE_KERNEL_WARP_MMA (mma.sync)."""
        self._check(self.L.alpine_gpu_guide_set_gradient_kernel(self.h, kernel))

    def guide_infer(self, queries):
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 12)
        raw = np.empty((q.shape[0], 40), np.float32)
        self._check(self.L.alpine_gpu_guide_infer(self.h, _ptr(q), q.shape[0], _ptr(raw)))
        return raw

    def guide_infer_device(self, queries_ptr: int, n: int, raw_ptr: int, stream: int = 0):
        """Inference on device buffers (float32[n, 12] in, float32[n, 40] out)
        on `stream`, without synchronising."""
        self._check(self.L.alpine_gpu_guide_infer_device(self.h, C.c_void_p(queries_ptr), n, C.c_void_p(raw_ptr),
                                                         C.c_void_p(stream or None)))

    def guide_gradients(self, samples, grid_index=None):
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 16)
        dW = np.empty(self.guide_dims()["weights"], np.float32)
        gi = None if grid_index is None else np.ascontiguousarray(grid_index, np.uint64)
        gg = None if gi is None else np.empty(gi.size, np.float32)
        self._check(self.L.alpine_gpu_guide_gradients(self.h, _ptr(s), s.shape[0], _ptr(dW),
                                                      None if gi is None else _ptr(gi), 0 if gi is None else gi.size,
                                                      None if gg is None else _ptr(gg), None))
        return dW, gg

    def guide_train(self, samples, lr=1e-2):
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 16)
        loss = (C.c_float * 3)()
        self._check(self.L.alpine_gpu_guide_train(self.h, _ptr(s), s.shape[0], lr, loss))
        return loss[0]

    def guide_get_weights(self):
        w = np.empty(self.guide_dims()["weights"], np.float32)
        self._check(self.L.alpine_gpu_guide_get_weights(self.h, _ptr(w)))
        return w

    def guide_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.L.alpine_gpu_guide_set_weights(self.h, _ptr(w)))

    def guide_grid(self, index, write=None):
        idx = np.ascontiguousarray(index, np.uint64)
        out = np.empty(idx.size, np.float32)
        wv = None if write is None else np.ascontiguousarray(write, np.float32)
        self._check(self.L.alpine_gpu_guide_grid(self.h, _ptr(idx), idx.size, _ptr(out),
                                                 None if wv is None else _ptr(wv)))
        return out

    def guide_sample_mixture(self, raw, u):
        r = np.ascontiguousarray(raw, np.float32).reshape(40)
        uu = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
        dirs = np.empty((uu.shape[0], 3), np.float32)
        pdfs = np.empty(uu.shape[0], np.float32)
        self._check(self.L.alpine_gpu_guide_sample_mixture(self.h, _ptr(r), _ptr(uu), uu.shape[0], _ptr(dirs),
                                                           _ptr(pdfs)))
        return dirs, pdfs

    def synchronize(self):
        self._check(self.L.alpine_gpu_synchronize(self.h))
