"""Test infrastructure: the oracle.

ctypes bindings to two CPU libraries built by ``oracle/Makefile``:

* ``liboracle.so`` -- the project's plain-C restatement of the reference's
  ray/box/triangle semantics (src/ispc/triangle.ispc:46-87,
  src/accelerators/bvh_common.cpp:66-103, src/ispc/bounding_box.ispc:15-43,
  src/utils/bounding_box.h:23-56), canonical brute-force / BVH-accelerated
  closest and any-hit queries and an FP64 Moller-Trumbore.
* ``_ref/libalpine_ref.so`` -- the unmodified reference sources (Bvh, WideBvh,
  integrator) behind a C-ABI harness (``refshim/ref_harness.cpp``), built for
  parity (IEEE FP32, no FMA contraction).
* ``_ref/libalpine_ref_plugin.so`` -- the parity build plus the GPU plug-in a
  maintainer adds to the reference (``alpine_b200/plugin``: GpuAccelerator
  and the GpuBackend render branch), for the boundary tests (``plugin=True``).
* ``_ref/libalpine_ref_fast_v3.so`` / ``_v4.so`` -- the same sources built with
  the host's vector ISA (AVX2 / AVX-512, no FMA contraction); used only by the
  timed CPU arms (``timing=True``).

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference arms use this package. The product (``alpine_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libalpine_ref.so")
REF_PLUGIN_SO = os.path.join(_HERE, "_ref", "libalpine_ref_plugin.so")
REF_FAST_SO = {3: os.path.join(_HERE, "_ref", "libalpine_ref_fast_v3.so"),
               4: os.path.join(_HERE, "_ref", "libalpine_ref_fast_v4.so")}

TRI_ISPC = 0
TRI_PRIM = 1

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        L = C.CDLL(ORACLE_SO)
        L.orc_tri_test.argtypes = [C.c_int, _f32p, _f32p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]
        L.orc_tri_test.restype = C.c_int
        L.orc_tri_fp64.argtypes = [_f32p, _f32p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), _f64p]
        L.orc_tri_fp64.restype = C.c_int
        L.orc_box_ispc.argtypes = [_f32p, _f32p, C.c_float, _f32p]
        L.orc_box_ref.argtypes = [_f32p, _f32p, C.c_float, _f32p]
        L.orc_closest_brute.argtypes = [C.c_int, _f32p, C.c_uint64, _f32p, C.c_uint32, _u32p, _f32p, _f32p,
                                        _f32p, _u32p]
        L.orc_any_brute.argtypes = [C.c_int, _f32p, C.c_uint64, _f32p, C.c_uint32, _u8p]
        L.orc_bvh_create.argtypes = [_f32p, C.c_uint32]
        L.orc_bvh_create.restype = C.c_void_p
        L.orc_bvh_closest.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_uint64, C.c_int, _u32p, _f32p, _f32p,
                                      _f32p, _u32p]
        L.orc_bvh_any.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_uint64, C.c_int, _u8p]
        L.orc_bvh_destroy.argtypes = [C.c_void_p]
        L.orc_tri_test_batch.argtypes = [C.c_int, _f32p, C.c_uint64, _f32p, C.c_uint32, _u32p, _u8p, _f32p,
                                         _f32p, _f32p]
        L.orc_make_tris.argtypes = [_f32p, _u32p, C.c_uint32, _f32p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = line.split()
                    return all(x in flags for x in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))
    except OSError:
        pass
    return False


def timing_build() -> str:
    """Path of the speed build of the reference for this host (AVX-512 when
    the host has it), else the parity build."""
    for level in ((4, 3) if _host_has_avx512() else (3,)):
        if os.path.exists(REF_FAST_SO[level]):
            return REF_FAST_SO[level]
    return REF_SO


def plugin_available() -> bool:
    return os.path.exists(REF_PLUGIN_SO)


def ref(timing: bool = False, plugin: bool = False):
    """The compiled reference: the parity build (``oracle/_ref/libalpine_ref.so``),
    with timing=True the speed build for this host, with plugin=True the
    parity build with the GPU plug-in installed."""
    path = REF_PLUGIN_SO if plugin else (timing_build() if timing else REF_SO)
    if path not in _ref:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = C.CDLL(path)
        L.ref_accel_create.argtypes = [C.c_int, C.c_uint64]
        L.ref_accel_create.restype = C.c_void_p
        L.ref_accel_add_mesh.argtypes = [C.c_void_p, _f32p, C.c_uint32, _u32p, C.c_uint32]
        L.ref_accel_add_mesh.restype = C.c_uint32
        L.ref_accel_build.argtypes = [C.c_void_p]
        L.ref_accel_build.restype = C.c_double
        L.ref_accel_intersect.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_int, _u32p, _f32p, _f32p, _f32p]
        L.ref_accel_occluded.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_int, _u8p]
        L.ref_accel_update_vertices.argtypes = [C.c_void_p, C.c_uint32, _f32p, C.c_uint32]
        L.ref_accel_intersect_ng.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_int, _u32p, _f32p, _f32p, _f32p,
                                             _f32p, _u8p]
        if plugin:
            L.ref_render_gpu_branch.argtypes = [C.c_int, C.c_uint32, C.c_int]
            L.ref_render_gpu_branch.restype = C.c_int
        L.ref_accel_destroy.argtypes = [C.c_void_p]
        L.ref_render_init.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        L.ref_render_init.restype = C.c_int
        L.ref_render_reset_scene.argtypes = [C.c_int]
        L.ref_render_add_mesh.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, C.c_void_p, _u32p, _f32p,
                                          C.c_uint32]
        L.ref_render_add_mesh.restype = C.c_int
        L.ref_render_add_morph_mesh.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, C.c_void_p, _u32p, _f32p,
                                                C.c_uint32, _f32p, C.c_void_p, C.c_uint32, _f32p, _f32p, C.c_uint32]
        L.ref_render_add_morph_mesh.restype = C.c_int
        L.ref_morph_vertices.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, _f32p, C.c_uint32, _f32p, _f32p,
                                         C.c_uint32, C.c_float, _f32p]
        L.ref_render_add_texture.argtypes = [_f32p, C.c_uint32, C.c_uint32]
        L.ref_render_add_texture.restype = C.c_int
        L.ref_render_add_mesh_ex.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, C.c_void_p, C.c_void_p,
                                             C.c_void_p, _u32p, _f32p, C.c_uint32]
        L.ref_render_add_mesh_ex.restype = C.c_int
        L.ref_render_set_environment.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.ref_render_load_obj.argtypes = [C.c_char_p]
        L.ref_render_load_glb.argtypes = [C.c_char_p]
        L.ref_render_load_glb.restype = C.c_int
        L.ref_render_shape_count.restype = C.c_uint32
        L.ref_render_mesh_data.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_render_mesh_data.restype = C.c_uint32
        L.ref_render_light_count.restype = C.c_uint32
        L.ref_render_light_info.argtypes = [C.c_uint32, _f32p, _f32p]
        L.ref_render_load_obj.restype = C.c_int
        L.ref_render_add_disk_light.argtypes = [C.c_float, _f32p, _f32p, _f32p, C.c_float]
        L.ref_render_add_point_light.argtypes = [C.c_float, _f32p, _f32p]
        L.ref_render_add_quad_light.argtypes = [_f32p, _f32p, _f32p, _f32p]
        L.ref_render_update_scene.argtypes = [C.c_float]
        L.ref_render_build_light_sampler.argtypes = [C.c_int]
        L.ref_render_set_background.argtypes = [C.c_float, C.c_float, C.c_float]
        L.ref_render_set_camera.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_float]
        L.ref_render.argtypes = [C.c_uint32]
        L.ref_render.restype = C.c_double
        L.ref_render_read_accum.argtypes = [_f32p]
        L.ref_render_read_accum.restype = C.c_uint32
        L.ref_render_post_process.argtypes = [C.c_int, _u8p]
        L.ref_render_read_sampler_state.argtypes = [_u32p]
        L.ref_material_sample.argtypes = [_f32p, _f32p, _f32p, C.c_uint32, _f32p, _f32p, _f32p, _u8p]
        L.ref_material_eval.argtypes = [_f32p, _f32p, _f32p, C.c_uint32, _f32p, _f32p]
        _ref[path] = L
    return _ref[path]


# ---------------------------------------------------------------------------
def make_tris(verts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Triangle records {v0, e0, e1} (bvh_common.cpp:105-125)."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1)
    i = np.ascontiguousarray(idx, np.uint32).reshape(-1)
    out = np.empty((i.size // 3, 9), np.float32)
    lib().orc_make_tris(v, i, i.size // 3, out.reshape(-1))
    return out


def tri_test(ray, tri, sem=TRI_ISPC):
    t, b1, b2 = C.c_float(), C.c_float(), C.c_float()
    hit = lib().orc_tri_test(sem, np.ascontiguousarray(ray, np.float32), np.ascontiguousarray(tri, np.float32),
                             C.byref(t), C.byref(b1), C.byref(b2))
    return bool(hit), t.value, b1.value, b2.value


def tri_test_batch(rays, tris, prim, sem=TRI_ISPC):
    """Exact re-evaluation of ray i against triangle prim[i] (tmax ignored)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    prim = np.ascontiguousarray(prim, np.uint32)
    n = rays.shape[0]
    hit = np.empty(n, np.uint8)
    t = np.empty(n, np.float32)
    b1 = np.empty(n, np.float32)
    b2 = np.empty(n, np.float32)
    lib().orc_tri_test_batch(sem, rays.reshape(-1), n, tris.reshape(-1), tris.shape[0], prim, hit, t, b1, b2)
    return hit.astype(bool), t, b1, b2


def sphere_hits_fp64(rays, spheres):
    """Analytic ray / sphere intersections in FP64 (numpy): for rays [N, 8]
    and spheres [M, 4] (centre, radius), the front hit, else the back hit of
    a ray starting inside, in [tmin, tmax). Returns t [N, M] (inf on a miss)
    and the tangency margin |r^2 - l^2| / r^2 (l the ray's distance from the
    centre), small where FP32 and FP64 may disagree on hit or miss."""
    r = np.asarray(rays, np.float64)
    sp = np.asarray(spheres, np.float64)
    o, tmin, d, tmax = r[:, None, 0:3], r[:, None, 3], r[:, None, 4:7], r[:, None, 7]
    c = sp[None, :, 0:3] - o
    rad = np.abs(sp[None, :, 3])
    dd = np.sum(d * d, -1)
    proj = np.sum(c * d, -1) / dd
    perp = c - proj[..., None] * d
    l2 = np.sum(perp * perp, -1)
    r2 = rad * rad
    with np.errstate(invalid="ignore"):
        td = np.sqrt(np.maximum(r2 - l2, 0.0) / dd)
    tf, tb = proj - td, proj + td
    hit = l2 <= r2
    front = hit & (tf >= tmin) & (tf < tmax)
    back = hit & ~front & (tb >= tmin) & (tb < tmax)
    t = np.where(front, tf, np.where(back, tb, np.inf))
    margin = np.abs(r2 - l2) / np.maximum(r2, 1e-300)
    return t, margin


def tri_fp64(ray, tri):
    t, b1, b2 = C.c_double(), C.c_double(), C.c_double()
    cond = np.zeros(3, np.float64)
    ok = lib().orc_tri_fp64(np.ascontiguousarray(ray, np.float32), np.ascontiguousarray(tri, np.float32),
                            C.byref(t), C.byref(b1), C.byref(b2), cond)
    return bool(ok), t.value, b1.value, b2.value, cond


def closest_brute(rays, tris, sem=TRI_ISPC):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = rays.shape[0]
    prim = np.empty(n, np.uint32)
    t = np.empty(n, np.float32)
    b1 = np.empty(n, np.float32)
    b2 = np.empty(n, np.float32)
    ntie = np.empty(n, np.uint32)
    lib().orc_closest_brute(sem, rays.reshape(-1), n, tris.reshape(-1), tris.shape[0], prim, t, b1, b2, ntie)
    return prim, t, b1, b2, ntie


def any_brute(rays, tris, sem=TRI_ISPC):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    occ = np.empty(rays.shape[0], np.uint8)
    lib().orc_any_brute(sem, rays.reshape(-1), rays.shape[0], tris.reshape(-1), tris.shape[0], occ)
    return occ


class OracleBvh:
    """Canonical closest / any-hit queries over a conservative CPU BVH."""

    def __init__(self, tris):
        self.tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        self.h = lib().orc_bvh_create(self.tris.reshape(-1), self.tris.shape[0])

    def closest(self, rays, sem=TRI_ISPC, nthreads=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        b1 = np.empty(n, np.float32)
        b2 = np.empty(n, np.float32)
        ntie = np.empty(n, np.uint32)
        lib().orc_bvh_closest(self.h, sem, rays.reshape(-1), n, nthreads, prim, t, b1, b2, ntie)
        return prim, t, b1, b2, ntie

    def any(self, rays, sem=TRI_ISPC, nthreads=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.empty(rays.shape[0], np.uint8)
        lib().orc_bvh_any(self.h, sem, rays.reshape(-1), rays.shape[0], nthreads, occ)
        return occ

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_destroy(self.h)
            self.h = None


class RefRenderer:
    """The reference integrator (class Alpine, src/alpine.cpp) through the
    harness: one process-wide instance, as the reference is a singleton."""

    ACC_BVH, ACC_WIDE_BVH = 0, 1
    # plug-in build only: the GpuAccelerator installed as the Alpine's
    # accelerator (8-wide / binary triangle rule)
    ACC_GPU, ACC_GPU_BINARY = 3, 4

    def __init__(self, width, height, max_depth, accelerator=ACC_BVH, arena_bytes=1 << 30, timing=False,
                 plugin=False, gpu_branch=False, seed=0):
        """plugin: use the plug-in build; gpu_branch: route the Alpine
        methods through the GpuBackend render branch (counter RNG, `seed`)."""
        self.L = ref(timing, plugin or gpu_branch)
        self.w, self.h = width, height
        if not self.L.ref_render_init(width, height, max_depth, arena_bytes):
            raise RuntimeError("ref_render_init failed")
        self.L.ref_render_reset_scene(accelerator)
        if gpu_branch and not self.L.ref_render_gpu_branch(1, seed, int(accelerator == self.ACC_BVH)):
            raise RuntimeError("ref_render_gpu_branch failed")

    def add_texture(self, rgba):
        """Texture4f from float32 [H, W, 4]; returns its id."""
        t = np.ascontiguousarray(rgba, np.float32)
        return self.L.ref_render_add_texture(t.reshape(-1), t.shape[1], t.shape[0])

    def load_glb(self, path):
        """alpine::loadScene(path, FileType::Gltf): the reference's GltfLoader."""
        if not self.L.ref_render_load_glb(str(path).encode()):
            raise RuntimeError(f"reference loader failed on {path}")

    def meshes(self):
        """The loaded scene's meshes as the reference holds them: dicts of
        positions, normals, uvs, tangents (Mesh::Data), prims and the current
        (possibly morphed) vertex buffer."""
        out = []
        for i in range(self.L.ref_render_shape_count()):
            nt = C.c_uint32()
            nv = self.L.ref_render_mesh_data(i, C.byref(nt), None, None, None, None, None, None)
            d = {k: np.zeros((nv, c), np.float32) for k, c in (("pos", 3), ("nrm", 3), ("uv", 2), ("tan", 4),
                                                                 ("current", 3))}
            d["prims"] = np.zeros((nt.value, 3), np.uint32)
            self.L.ref_render_mesh_data(i, C.byref(nt), d["pos"].ctypes.data, d["nrm"].ctypes.data,
                                        d["uv"].ctypes.data, d["tan"].ctypes.data, d["prims"].ctypes.data,
                                        d["current"].ctypes.data)
            out.append(d)
        return out

    def lights(self):
        """(power RGB, position) of every light of the loaded scene."""
        res = []
        for i in range(self.L.ref_render_light_count()):
            p, q = np.zeros(3, np.float32), np.zeros(3, np.float32)
            self.L.ref_render_light_info(i, p, q)
            res.append((p, q))
        return res

    def set_environment_map(self, rgb):
        """Alpine::mEnvironmentMap from float32 [H, W, 3] (None removes it)."""
        if rgb is None:
            self.L.ref_render_set_environment(None, 0, 0)
            return
        self._env = np.ascontiguousarray(rgb, np.float32)
        self.L.ref_render_set_environment(self._env.ctypes.data, self._env.shape[1], self._env.shape[0])

    def add_mesh(self, verts, idx, normals=None, tri_material=None, materials=((0, (0.5, 0.5, 0.5), 1.0),),
                 uvs=None, tangents=None):
        """materials: (kind, (r, g, b), roughness[, base texture, normal texture])."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1)
        i = np.ascontiguousarray(idx, np.uint32).reshape(-1)
        nt = i.size // 3
        tm = np.zeros(nt, np.uint32) if tri_material is None else np.ascontiguousarray(tri_material, np.uint32)
        nptr = None
        if normals is not None:
            self._normals = np.ascontiguousarray(normals, np.float32).reshape(-1)
            nptr = self._normals.ctypes.data
        textured = uvs is not None or tangents is not None or any(len(m) > 3 for m in materials)
        if not textured:
            mats = np.array([[k, *c, r] for k, c, r, *_ in materials], np.float32).reshape(-1)
            if not self.L.ref_render_add_mesh(v, v.size // 3, i, nt, nptr, tm, mats, len(materials)):
                raise RuntimeError("ref_render_add_mesh failed")
            return
        recs = []
        for m in materials:
            k, c, r = m[:3]
            bt = m[3] if len(m) > 3 and m[3] is not None else -1
            ntex = m[4] if len(m) > 4 and m[4] is not None else -1
            recs.append([k, *c, r, bt, ntex])
        mats = np.array(recs, np.float32).reshape(-1)
        self._uvs = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1)
        self._tangents = None if tangents is None else np.ascontiguousarray(tangents, np.float32).reshape(-1)
        if not self.L.ref_render_add_mesh_ex(v, v.size // 3, i, nt, nptr,
                                             None if self._uvs is None else self._uvs.ctypes.data,
                                             None if self._tangents is None else self._tangents.ctypes.data,
                                             tm, mats, len(materials)):
            raise RuntimeError("ref_render_add_mesh_ex failed")

    def add_morph_mesh(self, verts, idx, normals, tri_material, materials, deltas, normal_deltas, times, weights):
        """A mesh with morph targets deltas float[T, V, 3] (and normal deltas)
        and one animation channel (times float[K], weights float[K, T]);
        update_scene(time) applies it (Alpine::updateScene)."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1)
        i = np.ascontiguousarray(idx, np.uint32).reshape(-1)
        nt = i.size // 3
        tm = np.zeros(nt, np.uint32) if tri_material is None else np.ascontiguousarray(tri_material, np.uint32)
        mats = np.array([[k, *c, r] for k, c, r in materials], np.float32).reshape(-1)
        keep = []
        nptr = None
        if normals is not None:
            keep.append(np.ascontiguousarray(normals, np.float32).reshape(-1))
            nptr = keep[-1].ctypes.data
        d = np.ascontiguousarray(deltas, np.float32)
        ndptr = None
        if normal_deltas is not None:
            keep.append(np.ascontiguousarray(normal_deltas, np.float32).reshape(-1))
            ndptr = keep[-1].ctypes.data
        t = np.ascontiguousarray(times, np.float32)
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        if not self.L.ref_render_add_morph_mesh(v, v.size // 3, i, nt, nptr, tm, mats, len(materials), d.reshape(-1),
                                                ndptr, d.shape[0], t, w, t.size):
            raise RuntimeError("ref_render_add_morph_mesh failed")
        self._keep = getattr(self, "_keep", []) + keep

    def add_disk_light(self, power, color, position, target, radius):
        self.L.ref_render_add_disk_light(power, np.asarray(color, np.float32), np.asarray(position, np.float32),
                                         np.asarray(target, np.float32), radius)

    def add_point_light(self, power, color, position):
        self.L.ref_render_add_point_light(power, np.asarray(color, np.float32), np.asarray(position, np.float32))

    def add_quad_light(self, radiance, corner, edge_u, edge_v):
        """The oracle's project-written QuadLight (not in the reference)."""
        self.L.ref_render_add_quad_light(np.asarray(radiance, np.float32), np.asarray(corner, np.float32),
                                         np.asarray(edge_u, np.float32), np.asarray(edge_v, np.float32))

    def build(self):
        self.L.ref_render_update_scene(0.0)

    def update_scene(self, time):
        """Alpine::updateScene(time): animations, then the accelerator rebuild."""
        self.L.ref_render_update_scene(float(time))

    def build_light_sampler(self, kind):
        self.L.ref_render_build_light_sampler(kind)

    def set_background(self, r, g, b):
        self.L.ref_render_set_background(r, g, b)

    def set_camera(self, eye, target, up, fovy, aspect):
        self.L.ref_render_set_camera(np.asarray(eye, np.float32), np.asarray(target, np.float32),
                                     np.asarray(up, np.float32), fovy, aspect)

    def reset_accumulation(self):
        self.L.ref_render_reset_accumulation()

    def render(self, spp):
        ms = self.L.ref_render(spp)
        if ms < 0:
            raise RuntimeError("render failed (GPU render branch)")
        return ms

    def read_accumulation(self):
        out = np.empty((self.h, self.w, 9), np.float32)
        n = self.L.ref_render_read_accum(out.reshape(-1))
        return out, n

    def post_process(self, tonemap=True):
        out = np.empty((self.h, self.w, 3), np.uint8)
        self.L.ref_render_post_process(int(tonemap), out.reshape(-1))
        return out

    def read_sampler_state(self):
        out = np.empty((self.h, self.w, 4), np.uint32)
        self.L.ref_render_read_sampler_state(out.reshape(-1))
        return out

    def close(self):
        self.L.ref_render_shutdown()


def _material_record(material):
    kind, col, rough = material
    return np.array([float(kind), col[0], col[1], col[2], rough], np.float32)


def ref_material_sample(material, wo, u):
    """The reference's Material::sample (src/materials/material.h:18-19) for
    (wo, u) pairs in the local frame. material: (kind, (r, g, b), roughness),
    kind 0 = Dielectric, 1 = Conductor. Returns wi, estimator, pdf, ok."""
    wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
    u = np.ascontiguousarray(u, np.float32).reshape(-1, 2)
    n = wo.shape[0]
    wi = np.empty((n, 3), np.float32)
    est = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    ok = np.empty(n, np.uint8)
    ref().ref_material_sample(_material_record(material), wo.reshape(-1), u.reshape(-1), n, wi.reshape(-1),
                              est.reshape(-1), pdf, ok)
    return wi, est, pdf, ok.astype(bool)


def ref_material_eval(material, wo, wi):
    """The reference's Material::computeBsdf / computePdf (material.h:21-24)."""
    wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
    wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
    n = wo.shape[0]
    bsdf = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    ref().ref_material_eval(_material_record(material), wo.reshape(-1), wi.reshape(-1), n, bsdf.reshape(-1), pdf)
    return bsdf, pdf


def ref_morph_vertices(verts, idx, deltas, times, weights, time):
    """The reference's Animation::update + Mesh::update (src/animation.cpp:
    10-39, src/shapes/mesh.cpp:29-55) of one mesh on its Bvh accelerator:
    the morphed positions at `time`. deltas float[T, V, 3]; times float[K];
    weights float[K, T]."""
    v = np.ascontiguousarray(verts, np.float32)
    i = np.ascontiguousarray(idx, np.uint32)
    d = np.ascontiguousarray(deltas, np.float32)
    t = np.ascontiguousarray(times, np.float32)
    w = np.ascontiguousarray(weights, np.float32)
    out = np.empty_like(v)
    ref().ref_morph_vertices(v.reshape(-1), v.shape[0], i.reshape(-1), i.shape[0], d.reshape(-1), d.shape[0], t,
                             w.reshape(-1), t.size, float(time), out.reshape(-1))
    return out


class RefAccel:
    """The reference's own Bvh (kind 0) or WideBvh (kind 1) accelerator."""

    BVH = 0
    WIDE_BVH = 1
    # plug-in build only: the GpuAccelerator (8-wide / binary triangle rule)
    GPU = 2
    GPU_BINARY = 3

    def __init__(self, kind, verts, idx, arena_bytes=1 << 30, timing=False, plugin=False):
        self.L = ref(timing, plugin or kind >= self.GPU)
        self.h = self.L.ref_accel_create(kind, arena_bytes)
        v = np.ascontiguousarray(verts, np.float32).reshape(-1)
        i = np.ascontiguousarray(idx, np.uint32).reshape(-1)
        self.L.ref_accel_add_mesh(self.h, v, v.size // 3, i, i.size // 3)
        self.build_ms = self.L.ref_accel_build(self.h)

    def intersect(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        b1 = np.empty(n, np.float32)
        b2 = np.empty(n, np.float32)
        self.L.ref_accel_intersect(self.h, rays.reshape(-1), n, nthreads, prim, t, b1, b2)
        return prim, t, b1, b2

    def occluded(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.empty(rays.shape[0], np.uint8)
        self.L.ref_accel_occluded(self.h, rays.reshape(-1), rays.shape[0], nthreads, occ)
        return occ

    def update_vertices(self, shape, verts):
        """Mesh::update's path: write the shape's vertex buffer
        (getVertexBuffer), updateShape, then updateScene (rebuild)."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1)
        self.L.ref_accel_update_vertices(self.h, shape, v, v.size // 3)

    def intersect_ng(self, rays, nthreads=0):
        """intersect() plus Intersection::ng (float[n, 3]) and whether the hit
        carries the mesh's shape pointer."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        b1 = np.empty(n, np.float32)
        b2 = np.empty(n, np.float32)
        ng = np.empty((n, 3), np.float32)
        ok = np.empty(n, np.uint8)
        self.L.ref_accel_intersect_ng(self.h, rays.reshape(-1), n, nthreads, prim, t, b1, b2, ng.reshape(-1), ok)
        return prim, t, b1, b2, ng, ok.astype(bool)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_accel_destroy(self.h)
            self.h = None
