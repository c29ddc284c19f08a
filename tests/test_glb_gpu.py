"""GPU tests of alpine_gpu_load_glb against the reference's own loader
(src/loaders/gltf_loader.cpp running in oracle/_ref on the same file):

* every mesh's positions and normals after loading are bit-identical to the
  reference's Mesh::Data (node transforms, primitive concatenation, the
  later of two nodes referencing one mesh);
* after Alpine::updateScene(t) at several times (LINEAR weights channels,
  dense and sparse morph targets; STEP and translation channels skipped),
  the morphed positions equal the reference's vertex buffers bit for bit;
* a render of the loaded scene (Conductor / textured normal-mapped
  Dielectric / default materials, punctual lights) follows the reference
  path by path in reference-stream mode.
"""
import math

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu

import glb_writer

pytestmark = pytest.mark.gpu

W = H = 40
CAM = ((0.0, 2.5, -6.0), (0.0, 0.6, 0.0), (0.0, 1.0, 0.0), math.radians(50.0))


@pytest.fixture(scope="module")
def scene_path(tmp_path_factory):
    p = tmp_path_factory.mktemp("glbgpu") / "scene.glb"
    glb_writer.make_scene(p)
    return p


def _ref(path, depth=4):
    r = oracle.RefRenderer(W, H, depth, accelerator=oracle.RefRenderer.ACC_WIDE_BVH)
    r.load_glb(path)
    r.set_camera(*CAM, W / H)
    return r


def _gpu(path, depth=4, sampler=gpu.RNG_REFERENCE_STREAM):
    c = gpu.Context(0, W, H, depth)
    c.set_materials([])
    info = c.load_glb(path)
    c.set_camera(*CAM, W / H)
    c.set_render_options(sampler=sampler)
    return c, info


def test_loaded_geometry_and_animation_match_reference(scene_path):
    r = _ref(scene_path)
    c, info = _gpu(scene_path)
    try:
        assert info["shapes"] == 4 and info["lights"] == 2 and info["channels"] == 2 and info["textures"] == 2
        ref_meshes = r.meshes()
        for k, m in enumerate(ref_meshes):
            v, n = c.get_vertices(info["first_shape"] + k, m["pos"].shape[0])
            assert v.tobytes() == m["pos"].tobytes(), f"mesh {k} positions"
            assert n.tobytes() == m["nrm"].tobytes(), f"mesh {k} normals"
        for t in (0.3, 1.0, 1.7, 2.2, 3.0):
            r.update_scene(t)
            c.update_scene(t)
            for k, m in enumerate(r.meshes()):
                v, _ = c.get_vertices(info["first_shape"] + k, m["pos"].shape[0])
                assert v.tobytes() == m["current"].tobytes(), f"mesh {k} morphed positions at t = {t}"
    finally:
        c.close()
        r.close()


def test_loaded_scene_render_stream_parity(scene_path):
    r = _ref(scene_path)
    r.build()
    r.build_light_sampler(gpu.SAMPLER_POWER)
    r.reset_accumulation()
    r.render(2)
    ra, rn = r.read_accumulation()
    rs = r.read_sampler_state()
    r.close()
    c, _ = _gpu(scene_path)
    try:
        c.build()
        c.build_light_sampler(gpu.SAMPLER_POWER)
        c.reset_accumulation()
        c.render(2)
        ga, gn = c.read_accumulation(W, H)
        gs = c.read_sampler_state(W, H)
    finally:
        c.close()
    assert rn == gn == 2
    rc, gc = ra[..., :3].astype(np.float64), ga[..., :3].astype(np.float64)
    rel = np.abs(gc - rc).max(-1) / np.maximum(np.abs(rc).max(-1), 1e-3)
    close = (rel < 1e-3).mean()
    same = (rs == gs).all(-1).mean()
    aov = np.abs(ga[..., 3:] - ra[..., 3:]).max()
    print(f"GLB scene stream parity: {close:.4f} within 1e-3, {same:.4f} identical streams, AOV {aov:.2e}")
    assert rc.mean() > 0.0
    assert close > 0.95 and same > 0.95 and aov < 1e-3
