"""GPU tests of morph-target animation (Alpine::updateScene).

* The morphed positions equal the reference's own Animation::update +
  Mesh::update (oracle/_ref) bit for bit, at times before, between, on and
  after the keyframes: the weights follow the same clamp, segment search and
  std::lerp, and the device morph rounds every product and sum separately in
  the reference's order.
* After the morph the BVH is rebuilt: closest hits on the morphed geometry
  match the oracle bit-exactly.
* An animated scene renders like the reference's animated scene
  (reference-stream mode).
"""
import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes

from parity import compare_closest

pytestmark = pytest.mark.gpu


def _mesh():
    v, t, n = scenes.uv_sphere((0.1, -0.2, 0.3), 0.7, 24, 12)
    return v, t, n


def _animation(nv, targets=3, keys=5, seed=1):
    rng = np.random.default_rng(seed)
    deltas = rng.normal(0, 0.05, (targets, nv, 3)).astype(np.float32)
    times = np.cumsum(rng.uniform(0.2, 1.0, keys)).astype(np.float32)
    weights = rng.uniform(-1.5, 1.5, (keys, targets)).astype(np.float32)
    weights[1, 0] = 0.0  # a sign change across a segment (lerp's first branch)
    return deltas, times, weights


@pytest.mark.parametrize("where", ["before", "on", "mid", "after", "last"])
def test_morph_matches_reference(where):
    v, t, _ = _mesh()
    deltas, times, weights = _animation(v.shape[0])
    time = {"before": times[0] - 1.0, "on": times[2], "mid": 0.37 * times[1] + 0.63 * times[2],
            "after": times[-1] + 3.0, "last": times[-1]}[where]
    ref = oracle.ref_morph_vertices(v, t, deltas, times, weights, time)
    ctx = gpu.Context(0)
    sid = ctx.add_mesh(v, t)
    ctx.set_morph_targets(sid, deltas)
    ctx.add_animation_channel(sid, times, weights)
    ctx.update_scene(time)
    got, _ = ctx.get_vertices(sid, v.shape[0])
    ctx.close()
    assert got.view(np.uint32).tolist() == ref.view(np.uint32).tolist()


def test_rebuild_after_morph_traces_like_the_oracle():
    v, t, _ = _mesh()
    deltas, times, weights = _animation(v.shape[0], seed=4)
    ctx = gpu.Context(0)
    other = scenes.triangle_soup(3000, seed=9)
    ctx.add_mesh(*other)
    sid = ctx.add_mesh(v, t)
    ctx.set_morph_targets(sid, deltas)
    ctx.add_animation_channel(sid, times, weights)
    rng = np.random.default_rng(3)
    for frame, time in enumerate([0.0, 1.3, 2.9]):
        ctx.update_scene(time)
        mv, _ = ctx.get_vertices(sid, v.shape[0])
        verts = np.concatenate([other[0], mv])
        idx = np.concatenate([other[1], t + other[0].shape[0]])
        tris = oracle.make_tris(verts, idx)
        rays = np.zeros((20000, 8), np.float32)
        rays[:, 0:3] = rng.uniform(-1.2, 1.2, (20000, 3))
        d = rng.normal(size=(20000, 3))
        rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
        rays[:, 7] = 3.4e38
        hits = ctx.trace(rays)
        rp, rt, rb1, rb2, _ = oracle.closest_brute(rays, tris)
        rep = compare_closest(rays, tris, hits, rp, rt, rb1, rb2)
        assert rep["hits"] > 1000
    ctx.close()


def test_animated_room_stream_parity():
    """The room with its sphere breathing (positions and normals morphed),
    rendered at time 7.3 by the reference and the GPU, one sample per pixel."""
    scene = scenes.room_scene(seed=8)
    sphere = scene["meshes"][-1]
    sphere["morph"] = scenes.sinusoid_morph(sphere["verts"], sphere["normals"], amplitude=0.05, with_normals=True)
    scene["time"] = 7.3
    W = H = 40
    ref = oracle.RefRenderer(W, H, 3, accelerator=oracle.RefRenderer.ACC_WIDE_BVH)
    scenes.load_scene(ref, scene, W, H)
    ref.build_light_sampler(gpu.SAMPLER_POWER)
    ref.reset_accumulation()
    ref.render(1)
    ra, _ = ref.read_accumulation()
    rs = ref.read_sampler_state()
    ref.close()
    ctx = gpu.Context(0, W, H, 3)
    scenes.load_scene(ctx, scene, W, H)
    ctx.build_light_sampler(gpu.SAMPLER_POWER)
    ctx.set_render_options(sampler=gpu.RNG_REFERENCE_STREAM)
    ctx.reset_accumulation()
    ctx.render(1)
    ga, _ = ctx.read_accumulation(W, H)
    gs = ctx.read_sampler_state(W, H)
    ctx.close()
    rc, gc = ra[..., :3].astype(np.float64), ga[..., :3].astype(np.float64)
    rel = np.abs(gc - rc).max(-1) / np.maximum(np.abs(rc).max(-1), 1e-3)
    close = (rel < 1e-3).mean()
    same = (rs == gs).all(-1).mean()
    print(f"animated room: {close:.4f} of pixels within 1e-3, {same:.4f} with identical stream state")
    assert close > 0.95 and same > 0.95


def test_animation_errors():
    v, t, _ = _mesh()
    ctx = gpu.Context(0)
    sid = ctx.add_mesh(v, t)
    with pytest.raises(RuntimeError):
        ctx.add_animation_channel(sid, [0.0, 1.0], [[0.0], [1.0]])  # no targets yet
    with pytest.raises(RuntimeError):
        ctx.set_morph_targets(sid, np.zeros((1, v.shape[0], 3)), np.zeros((1, v.shape[0], 3)))  # no normals
    ctx.set_morph_targets(sid, np.zeros((1, v.shape[0], 3)))
    with pytest.raises(RuntimeError):
        ctx.add_animation_channel(sid, [0.0], [[1.0]])  # one keyframe
    with pytest.raises(RuntimeError):
        ctx.add_animation_channel(sid, [1.0, 0.0], [[0.0], [1.0]])  # decreasing times
    ctx.close()
