"""GPU parity tests of the path tracer against the reference integrator.

The reference (oracle/_ref: class Alpine of src/alpine.cpp with its materials,
lights and light samplers) renders the same seeded scenes on the CPU.

* Reference-stream mode: the GPU draws the reference's per-pixel xorshift128
  stream in the reference's order with the same FP32 operation order, so
  per-pixel sums agree closely. They differ only where a libm-vs-CUDA ulp
  difference (cos, sin, pow) flips a branch and the stream diverges for the
  rest of that sample.
* Counter mode: independent random numbers; per-pixel means agree within the
  statistical error measured from the reference's own batches (z-test).
"""
import math

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes

pytestmark = pytest.mark.gpu

W = H = 40
DEPTH = 8


def _gpu_ctx(scene, sampler_kind, rng_mode, w=W, h=H, depth=DEPTH, triangle_test=gpu.TRIANGLE_TEST_WIDE_BVH,
             **opts):
    ctx = gpu.Context(0, w, h, depth)
    ctx.set_traversal_options(triangle_test)
    scenes.load_scene(ctx, scene, w, h)
    ctx.build_light_sampler(sampler_kind)
    ctx.set_render_options(sampler=rng_mode, **opts)
    ctx.reset_accumulation()
    return ctx


def _ref(scene, sampler_kind, w=W, h=H, depth=DEPTH, accelerator=oracle.RefRenderer.ACC_WIDE_BVH):
    # WideBvh by default: the reference traversal whose triangle test
    # (triangle.ispc) the GPU's default rule reproduces bit-exactly; ACC_BVH
    # pairs with the GPU's binary-BVH rule
    r = oracle.RefRenderer(w, h, depth, accelerator=accelerator)
    scenes.load_scene(r, scene, w, h)
    r.build_light_sampler(sampler_kind)
    r.reset_accumulation()
    return r


def _stream_compare(scene, sampler_kind, spp=1, depth=DEPTH, binary=False):
    acc = oracle.RefRenderer.ACC_BVH if binary else oracle.RefRenderer.ACC_WIDE_BVH
    ref = _ref(scene, sampler_kind, depth=depth, accelerator=acc)
    ref.render(spp)
    ra, rn = ref.read_accumulation()
    rs = ref.read_sampler_state()
    ref.close()
    mode = gpu.TRIANGLE_TEST_BINARY_BVH if binary else gpu.TRIANGLE_TEST_WIDE_BVH
    ctx = _gpu_ctx(scene, sampler_kind, gpu.RNG_REFERENCE_STREAM, depth=depth, triangle_test=mode)
    ctx.render(spp)
    ga, gn = ctx.read_accumulation(W, H)
    gs = ctx.read_sampler_state(W, H)
    ctx.close()
    assert rn == gn == spp
    rc, gc = ra[..., :3].astype(np.float64), ga[..., :3].astype(np.float64)
    rel = np.abs(gc - rc).max(-1) / np.maximum(np.abs(rc).max(-1), 1e-3)
    close = (rel < 1e-3).mean()
    same_stream = (rs == gs).all(-1).mean()
    mean_rel = abs(gc.mean() - rc.mean()) / max(rc.mean(), 1e-9)
    aov = np.abs(ga[..., 3:] - ra[..., 3:]).max()
    print(f"stream parity: {close:.4f} of pixels within 1e-3, {same_stream:.4f} with identical random stream "
          f"state, image mean rel diff {mean_rel:.2e}, AOV max diff {aov:.2e}")
    return close, same_stream, mean_rel, aov


def test_stream_parity_room_power_sampler():
    """One sample per pixel, depth 8: the GPU follows the reference path by path."""
    close, same, mean_rel, aov = _stream_compare(scenes.room_scene(), gpu.SAMPLER_POWER)
    assert close > 0.95 and same > 0.95
    assert mean_rel < 0.02
    assert aov < 1e-3


def test_stream_parity_room_binary_bvh():
    """The room as the reference renders it with its binary BVH
    (AcceleratorType::Bvh, the accelerator of the small-room configuration):
    the GPU's binary-BVH triangle rule follows it path by path."""
    close, same, mean_rel, aov = _stream_compare(scenes.room_scene(), gpu.SAMPLER_POWER, binary=True)
    assert close > 0.95 and same > 0.95
    assert mean_rel < 0.02
    assert aov < 1e-3


def test_stream_parity_depth_two_four_samples():
    close, same, mean_rel, _ = _stream_compare(scenes.room_scene(seed=7), gpu.SAMPLER_POWER, spp=4, depth=2)
    assert close > 0.97 and same > 0.97


@pytest.mark.parametrize("kind", [gpu.SAMPLER_UNIFORM, gpu.SAMPLER_POWER, gpu.SAMPLER_BVH])
def test_stream_parity_many_lights(kind):
    """48 disk / point lights: the alias table and the light BVH select the
    same lights with the same pdfs as the reference's samplers."""
    scene = scenes.add_random_lights(scenes.room_scene(seed=3), 48, seed=7)
    close, same, mean_rel, _ = _stream_compare(scene, kind, spp=2, depth=3)
    assert close > 0.97 and same > 0.97
    assert mean_rel < 0.01


def test_stream_parity_quad_light():
    close, same, mean_rel, _ = _stream_compare(scenes.room_scene(seed=2, light="quad"), gpu.SAMPLER_POWER,
                                               spp=2, depth=3)
    assert close > 0.97 and same > 0.97
    assert mean_rel < 0.01


def _gpu_batches(scene, kind, w, h, batches, per, depth=DEPTH, seed=11):
    ctx = _gpu_ctx(scene, kind, gpu.RNG_COUNTER, w, h, depth=depth, seed=seed)
    means, prev = [], np.zeros((h, w, 3), np.float64)
    for _ in range(batches):
        ctx.render(per)
        a, _ = ctx.read_accumulation(w, h)
        cur = a[..., :3].astype(np.float64)
        means.append((cur - prev) / per)
        prev = cur
    ctx.close()
    return np.array(means)


@pytest.mark.parametrize("kind,light", [(gpu.SAMPLER_POWER, "disk"), (gpu.SAMPLER_BVH, "quad")])
def test_counter_mode_unbiased_vs_reference(kind, light):
    """Per-pixel z-test of the reference mean (256 spp) against the GPU mean
    (counter RNG, 16 x 1024 spp); the per-sample variance is estimated from
    the GPU batches and scaled to each side's sample count."""
    scene = scenes.room_scene(seed=4, light=light)
    w = h = 24
    ref = _ref(scene, kind, w, h)
    ref.render(256)
    a, n = ref.read_accumulation()
    ref.close()
    rmean = a[..., :3].astype(np.float64) / n
    gb = _gpu_batches(scene, kind, w, h, 16, 1024)
    gmean = gb.mean(0)
    var1 = gb.var(0, ddof=1) * 1024  # per-sample variance
    se = np.sqrt(var1 / 256 + var1 / (16 * 1024))
    ok = se > 1e-7
    z = (rmean - gmean)[ok] / se[ok]
    rel = abs(rmean.mean() - gmean.mean()) / gmean.mean()
    print(f"counter-mode z-test: |z|>5 fraction {(np.abs(z) > 5).mean():.4f}, mean z {z.mean():.3f}, "
          f"image mean ref {rmean.mean():.5f} gpu {gmean.mean():.5f} (rel {rel:.2e})")
    assert (np.abs(z) > 5).mean() < 0.02
    assert abs(z.mean()) < 0.25
    assert rel < 0.02


def test_counter_mode_deterministic():
    scene = scenes.room_scene(seed=5)
    out = []
    for _ in range(2):
        ctx = _gpu_ctx(scene, gpu.SAMPLER_BVH, gpu.RNG_COUNTER, seed=3)
        ctx.render(16)
        out.append(ctx.read_accumulation(W, H)[0].tobytes())
        ctx.close()
    assert out[0] == out[1]


def test_post_process_matches_reference():
    """postProcess (mean, ACES, clamp, sRGB, 8 bits) on matching accumulations."""
    scene = scenes.room_scene(seed=6)
    ref = _ref(scene, gpu.SAMPLER_POWER, depth=3)
    ref.render(1)
    rimg = ref.post_process(True)
    ref.close()
    ctx = _gpu_ctx(scene, gpu.SAMPLER_POWER, gpu.RNG_REFERENCE_STREAM, depth=3)
    ctx.render(1)
    _, gimg = ctx.post_process(W, H, True)
    ctx.close()
    diff = np.abs(gimg.astype(int) - rimg.astype(int))
    print(f"LDR: {(diff <= 1).mean():.4f} of channels within 1 code, {(diff == 0).mean():.4f} identical")
    assert (diff <= 1).mean() > 0.98


@pytest.mark.parametrize("kind", [gpu.SAMPLER_UNIFORM, gpu.SAMPLER_POWER, gpu.SAMPLER_BVH])
def test_stream_parity_city(kind):
    """A small many-light city (60 buildings, 600 window quad lights, GGX /
    metallic facades): the three light samplers select the same lights with
    the same pdfs as the reference's samplers."""
    scene = scenes.city_scene(seed=5, buildings=60, lights=600, extent=200.0)
    eye = (0.0, 60.0, -95.0)
    scene["camera"] = (eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), scene["camera"][3])
    close, same, mean_rel, _ = _stream_compare(scene, kind, spp=2, depth=3)
    assert close > 0.95 and same > 0.97
    assert mean_rel < 0.02


def test_fp64_accumulators_match_fp32_and_reference():
    """FP64 per-pixel accumulators (for convergence runs): the same samples as
    the FP32 path (counter RNG, same seed) summed in double precision. The
    sums agree with the FP32 sums to FP32 rounding, the FP64 read-back of the
    FP32 path and the FP32 read-back of the FP64 path are consistent, and the
    FP64 image passes the z-test against the reference renderer."""
    scene = scenes.room_scene(seed=4)
    w = h = 24
    sums = {}
    for fp64 in (False, True):
        ctx = _gpu_ctx(scene, gpu.SAMPLER_POWER, gpu.RNG_COUNTER, w, h, seed=5, accumulate_fp64=fp64)
        for _ in range(4):
            ctx.render(256)
        s64, n64 = ctx.read_accumulation(w, h, fp64=True)
        s32, n32 = ctx.read_accumulation(w, h)
        ctx.close()
        assert n64 == n32 == 1024
        if fp64:
            assert (s32 == s64.astype(np.float32)).all()
        else:
            assert (s64 == s32.astype(np.float64)).all()
        sums[fp64] = s64
    a, b = sums[False][..., :3], sums[True][..., :3]
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * np.abs(b).mean())
    print(f"fp32 vs fp64 sums: max rel diff {rel.max():.2e}, mean {rel.mean():.2e}")
    assert rel.max() < 1e-3 and rel.mean() < 1e-5
    assert not (a == b).all()  # the FP64 path does sum differently
    ref = _ref(scene, gpu.SAMPLER_POWER, w, h)
    ref.render(256)
    ra, rn = ref.read_accumulation()
    ref.close()
    rmean = ra[..., :3].astype(np.float64) / rn
    gb = _gpu_batches(scene, gpu.SAMPLER_POWER, w, h, 16, 256, seed=6)
    var1 = gb.var(0, ddof=1) * 256
    gmean = b[..., :3] / 1024
    se = np.sqrt(var1 / 256 + var1 / 1024)
    ok = se > 1e-7
    z = (rmean - gmean)[ok] / se[ok]
    print(f"fp64 z-test: |z|>5 fraction {(np.abs(z) > 5).mean():.4f}, mean z {z.mean():.3f}")
    assert (np.abs(z) > 5).mean() < 0.02
    assert abs(z.mean()) < 0.25


@pytest.mark.parametrize("rng,fp64", [(gpu.RNG_REFERENCE_STREAM, False), (gpu.RNG_COUNTER, False),
                                      (gpu.RNG_COUNTER, True)])
def test_checkpoint_resume_continues_exactly(rng, fp64):
    """A render interrupted after 8 spp and resumed in a new context from the
    read-back sums, sample count (and reference streams) gives the same sums,
    bit for bit, as one uninterrupted 8 + 8 spp run."""
    scene = scenes.room_scene(seed=6)
    w = h = 24
    opts = dict(seed=7, accumulate_fp64=fp64)
    a = _gpu_ctx(scene, gpu.SAMPLER_POWER, rng, w, h, depth=4, **opts)
    a.render(8)
    sums, n = a.read_accumulation(w, h, fp64=fp64)
    state = a.read_sampler_state(w, h)
    a.render(8)
    full, nf = a.read_accumulation(w, h, fp64=fp64)
    a.close()
    b = _gpu_ctx(scene, gpu.SAMPLER_POWER, rng, w, h, depth=4, **opts)
    b.write_accumulation(sums, n)
    b.write_sampler_state(state)
    b.render(8)
    resumed, nr = b.read_accumulation(w, h, fp64=fp64)
    b.close()
    assert n == 8 and nf == nr == 16
    assert resumed.tobytes() == full.tobytes()


def test_stream_parity_textures_normal_maps_environment():
    """Base-colour textures (wrapping coordinates), a tangent-space normal map
    and the lat-long environment map, against the reference's Texture4f,
    Mesh::getIntersectionAttributes and EnvironmentMap: path-by-path parity
    in reference-stream mode, including the albedo / normal AOVs."""
    close, same, mean_rel, aov = _stream_compare(scenes.textured_scene(), gpu.SAMPLER_POWER, spp=2, depth=4)
    assert close > 0.95 and same > 0.95
    assert mean_rel < 0.02
    assert aov < 1e-3


def test_textured_scene_counter_mode_unbiased_vs_reference():
    scene = scenes.textured_scene(seed=2)
    w, h = 32, 24
    ref = _ref(scene, gpu.SAMPLER_POWER, w, h, depth=5)
    ref.render(256)
    a, n = ref.read_accumulation()
    ref.close()
    rmean = a[..., :3].astype(np.float64) / n
    gb = _gpu_batches(scene, gpu.SAMPLER_POWER, w, h, 16, 1024, depth=5)
    gmean = gb.mean(0)
    var1 = gb.var(0, ddof=1) * 1024
    se = np.sqrt(var1 / 256 + var1 / (16 * 1024))
    ok = se > 1e-7
    z = (rmean - gmean)[ok] / se[ok]
    det = ~ok  # sky seen directly: deterministic, must match
    print(f"textured z-test: |z|>5 fraction {(np.abs(z) > 5).mean():.4f}, mean z {z.mean():.3f}")
    assert (np.abs(z) > 5).mean() < 0.02 and abs(z.mean()) < 0.25
    assert np.allclose(rmean[det], gmean[det], rtol=1e-4, atol=1e-6)
    # the environment map is what escaping rays see: a background-only render differs
    ctx = _gpu_ctx(dict(scene, environment=None), gpu.SAMPLER_POWER, gpu.RNG_COUNTER, w, h, depth=5, seed=3)
    ctx.render(64)
    plain = ctx.read_accumulation(w, h)[0][..., :3] / 64
    ctx.close()
    assert abs(plain.mean() - gmean.mean()) > 0.1 * gmean.mean()
