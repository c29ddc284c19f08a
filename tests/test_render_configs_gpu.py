"""Image parity at the BASELINE render configurations, against the reference
renderer (oracle/_ref: class Alpine of src/alpine.cpp, src/alpine.cpp:290-432).

Every case keeps the configuration's full scene geometry, lights, materials,
light sampler and path depth; only the image is smaller where the reference's
CPU time demands it (same camera, fewer pixels), and the spp are the test's.

Test: per-pixel z-test of the reference mean (R spp) against the GPU mean
(counter RNG, 16 batches of B spp); the per-sample variance of each pixel is
estimated from the GPU batches and scaled to each side's sample count. Pass:
at most 2% of pixels with |z| > 5 and |mean z| < 0.25 (the bar of the
existing small-scene z-tests), the same on 4x4-pixel block means, where
heavy-tailed per-pixel estimates average out, and |z| < 5 for the image mean
itself (its standard error from the summed per-pixel variances). Pixels whose
GPU variance is 0 (deterministic, e.g. sky seen directly) must agree to 1e-4
relative. relMSE of the GPU image against the reference image is printed
beside the statistics (it is dominated by the reference's own noise at R spp).

The uniform and power samplers over the city's 131,011 lights are extremely
heavy-tailed estimators (a rare nearby light carries most of a pixel's
value), so their image means scatter by tens of percent between runs even at
tens of thousands of spp; the test's bar for them is statistical, as above.
"""
from __future__ import annotations

import functools

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

BATCHES = 16


def _relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2 * ref.mean() ** 2)))


def _zstats(rmean, gb, r_spp, b_spp, block=4):
    """z statistics of the reference mean against GPU batch means gb[k]."""
    gmean = gb.mean(0)
    var1 = gb.var(0, ddof=1) * b_spp  # per-sample variance per pixel and channel
    se = np.sqrt(var1 / r_spp + var1 / (BATCHES * b_spp))
    det = var1 == 0
    scale = np.maximum(np.abs(gmean), 1e-6)
    det_bad = int((det & (np.abs(rmean - gmean) > 1e-4 * scale)).sum())
    ok = ~det
    z = (rmean - gmean)[ok] / se[ok]
    # block means: per-batch block means give the block variance directly
    h, w = rmean.shape[:2]
    hb, wb = h // block, w // block

    def blocks(x):
        x = x[..., :hb * block, :wb * block, :]
        return x.reshape(*x.shape[:-3], hb, block, wb, block, 3).mean(axis=(-4, -2))

    rb, gbb = blocks(rmean), blocks(gb)
    gbm = gbb.mean(0)
    vb = gbb.var(0, ddof=1) * b_spp
    seb = np.sqrt(vb / r_spp + vb / (BATCHES * b_spp))
    okb = vb > 0
    zb = (rb - gbm)[okb] / seb[okb]
    return {
        "pixels": int(ok.sum()), "frac_z5": float((np.abs(z) > 5).mean()), "mean_z": float(z.mean()),
        "block_frac_z5": float((np.abs(zb) > 5).mean()), "block_mean_z": float(zb.mean()),
        "deterministic": int(det.sum()), "deterministic_bad": det_bad,
        "relmse": _relmse(gmean, rmean), "image_mean_ref": float(rmean.mean()), "image_mean_gpu": float(gmean.mean()),
        "image_mean_z": float((rmean.mean() - gmean.mean()) /
                              max(np.sqrt(var1.sum() / r_spp + var1.sum() / (BATCHES * b_spp)) / var1.size, 1e-30)),
    }


def _check(st):
    print(f"z-test: {st}")
    assert st["deterministic_bad"] == 0
    assert st["frac_z5"] < 0.02 and abs(st["mean_z"]) < 0.25
    assert st["block_frac_z5"] < 0.02 and abs(st["block_mean_z"]) < 0.25
    assert abs(st["image_mean_z"]) < 5


def _gpu_batches(ctx, w, h, b_spp):
    means, prev = [], np.zeros((h, w, 3), np.float64)
    ctx.reset_accumulation()
    for _ in range(BATCHES):
        ctx.render(b_spp)
        a, _ = ctx.read_accumulation(w, h, fp64=True)
        cur = a[..., :3].astype(np.float64)
        means.append((cur - prev) / b_spp)
        prev = cur
    return np.array(means)


def _ref_mean(r, spp):
    r.reset_accumulation()
    r.render(spp)
    a, n = r.read_accumulation()
    return a[..., :3].astype(np.float64) / n


# ---------------------------------------------------------------------------
# Config 1: the small room, 256x256, depth 8, power light sampler, binary BVH
# (the reference renders it with AcceleratorType::Bvh; the GPU uses its
# binary-BVH triangle rule). The GPU runs both without Russian roulette (the
# reference has none) and with roulette from depth 3 as the configuration
# asks: roulette is unbiased, so both means match the reference.

@pytest.mark.parametrize("rr", [0, 3])
def test_room_config_vs_reference(rr):
    w = h = 256
    scene = scenes.room_scene(light="quad")
    r = oracle.RefRenderer(w, h, 8, accelerator=oracle.RefRenderer.ACC_BVH)
    scenes.load_scene(r, scene, w, h)
    r.build_light_sampler(gpu.SAMPLER_POWER)
    r_spp = 64
    rmean = _ref_mean(r, r_spp)
    r.close()
    ctx = gpu.Context(0, w, h, 8)
    try:
        ctx.set_traversal_options(gpu.TRIANGLE_TEST_BINARY_BVH)
        scenes.load_scene(ctx, scene, w, h)
        ctx.build_light_sampler(gpu.SAMPLER_POWER)
        ctx.set_render_options(sampler=gpu.RNG_COUNTER, russian_roulette_depth=rr, seed=21 + rr)
        gb = _gpu_batches(ctx, w, h, 256)
    finally:
        ctx.close()
    _check(_zstats(rmean, gb, r_spp, 256))


# ---------------------------------------------------------------------------
# Config 3: the many-light city, full geometry (about 1.2M triangles) and all
# 131,011 window quad lights, depth 8, each of the three light samplers. The
# image is 96x54 (1920x1080 / 20, same camera).

CITY_W, CITY_H = 96, 54
CITY_REF_SPP = 1024
CITY_GPU_SPP = 4096  # per batch


@functools.lru_cache(maxsize=1)
def _city():
    return scenes.city_scene()


@pytest.fixture(scope="module")
def city_reference():
    scene = _city()
    r = oracle.RefRenderer(CITY_W, CITY_H, 8, accelerator=oracle.RefRenderer.ACC_WIDE_BVH)
    scenes.load_scene(r, scene, CITY_W, CITY_H)
    out = {}
    for kind in (gpu.SAMPLER_UNIFORM, gpu.SAMPLER_POWER, gpu.SAMPLER_BVH):
        r.build_light_sampler(kind)
        out[kind] = _ref_mean(r, CITY_REF_SPP)
    r.close()
    return out


@pytest.mark.parametrize("kind", [gpu.SAMPLER_UNIFORM, gpu.SAMPLER_POWER, gpu.SAMPLER_BVH])
def test_city_config_vs_reference(city_reference, kind):
    scene = _city()
    assert sum(m["idx"].shape[0] for m in scene["meshes"]) > 1_200_000 and len(scene["lights"]) > 130_000
    ctx = gpu.Context(0, CITY_W, CITY_H, 8)
    try:
        scenes.load_scene(ctx, scene, CITY_W, CITY_H)
        ctx.build_light_sampler(kind)
        ctx.set_render_options(sampler=gpu.RNG_COUNTER, seed=31 + kind)
        gb = _gpu_batches(ctx, CITY_W, CITY_H, CITY_GPU_SPP)
    finally:
        ctx.close()
    _check(_zstats(city_reference[kind], gb, CITY_REF_SPP, CITY_GPU_SPP))


# ---------------------------------------------------------------------------
# Config 5: the glossy interior, full geometry (2.0M triangles, 70% GGX with
# roughness in [0.02, 0.4], sky of radiance 5 through two window openings),
# depth 12, plain MIS. The image is 96x54 (1920x1080 / 20, same camera).

def test_interior_config_vs_reference():
    w, h = 96, 54
    scene = scenes.glossy_interior_scene()
    assert sum(m["idx"].shape[0] for m in scene["meshes"]) > 1_900_000
    r = oracle.RefRenderer(w, h, 12, accelerator=oracle.RefRenderer.ACC_WIDE_BVH)
    scenes.load_scene(r, scene, w, h)
    r_spp = 256
    rmean = _ref_mean(r, r_spp)
    r.close()
    ctx = gpu.Context(0, w, h, 12)
    try:
        scenes.load_scene(ctx, scene, w, h)
        ctx.set_render_options(sampler=gpu.RNG_COUNTER, seed=41)
        gb = _gpu_batches(ctx, w, h, 1024)
    finally:
        ctx.close()
    _check(_zstats(rmean, gb, r_spp, 1024))
