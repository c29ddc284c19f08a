"""Test infrastructure: the oracle.

ctypes bindings to two CPU libraries built by ``oracle/Makefile``:

* ``liboracle.so`` -- the project's plain-C restatement of the reference's
  ray/box/triangle semantics (src/ispc/triangle.ispc:46-87,
  src/accelerators/bvh_common.cpp:66-103, src/ispc/bounding_box.ispc:15-43,
  src/utils/bounding_box.h:23-56), canonical brute-force / BVH-accelerated
  closest and any-hit queries and an FP64 Moller-Trumbore.
* ``_ref/libalpine_ref.so`` -- the unmodified reference sources (Bvh, WideBvh,
  integrator) behind a C-ABI harness (``refshim/ref_harness.cpp``).

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

TRI_ISPC = 0
TRI_PRIM = 1

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_lib = None
_ref = None


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


def ref():
    """The compiled reference (``oracle/_ref/libalpine_ref.so``)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"{REF_SO} missing: run `make -C oracle ref` where the reference tree exists")
        L = C.CDLL(REF_SO)
        L.ref_accel_create.argtypes = [C.c_int, C.c_uint64]
        L.ref_accel_create.restype = C.c_void_p
        L.ref_accel_add_mesh.argtypes = [C.c_void_p, _f32p, C.c_uint32, _u32p, C.c_uint32]
        L.ref_accel_add_mesh.restype = C.c_uint32
        L.ref_accel_build.argtypes = [C.c_void_p]
        L.ref_accel_build.restype = C.c_double
        L.ref_accel_intersect.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_int, _u32p, _f32p, _f32p, _f32p]
        L.ref_accel_occluded.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_int, _u8p]
        L.ref_accel_destroy.argtypes = [C.c_void_p]
        L.ref_render_init.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        L.ref_render_init.restype = C.c_int
        L.ref_render_reset_scene.argtypes = [C.c_int]
        L.ref_render_add_mesh.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, C.c_void_p, _u32p, _f32p,
                                          C.c_uint32]
        L.ref_render_add_mesh.restype = C.c_int
        L.ref_render_load_obj.argtypes = [C.c_char_p]
        L.ref_render_load_obj.restype = C.c_int
        L.ref_render_add_disk_light.argtypes = [C.c_float, _f32p, _f32p, _f32p, C.c_float]
        L.ref_render_add_point_light.argtypes = [C.c_float, _f32p, _f32p]
        L.ref_render_update_scene.argtypes = [C.c_float]
        L.ref_render_build_light_sampler.argtypes = [C.c_int]
        L.ref_render_set_background.argtypes = [C.c_float, C.c_float, C.c_float]
        L.ref_render_set_camera.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_float]
        L.ref_render.argtypes = [C.c_uint32]
        L.ref_render.restype = C.c_double
        L.ref_render_read_accum.argtypes = [_f32p]
        L.ref_render_read_accum.restype = C.c_uint32
        L.ref_render_post_process.argtypes = [C.c_int, _u8p]
        _ref = L
    return _ref


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


class RefAccel:
    """The reference's own Bvh (kind 0) or WideBvh (kind 1) accelerator."""

    BVH = 0
    WIDE_BVH = 1

    def __init__(self, kind, verts, idx, arena_bytes=1 << 30):
        self.L = ref()
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

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_accel_destroy(self.h)
            self.h = None
