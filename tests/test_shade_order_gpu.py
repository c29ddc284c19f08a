"""The shading queue grouped by material (alpine_gpu_render_options.
shade_order = BY_MATERIAL, a two-pass counting sort between the closest-hit
traversal and shading) renders exactly the image the queue order renders:
every path's arithmetic depends on the path only. Checked bit for bit on
scenes that fill every bin: misses (the city's sky), Lambertian-only and
two-lobe dielectrics, conductors, guided vertices; in both RNG modes.
"""
import numpy as np
import pytest

from alpine_b200 import gpu, scenes

pytestmark = pytest.mark.gpu


def _render(scene, w, h, depth, kind, order, spp, **opts):
    ctx = gpu.Context(0, w, h, depth)
    try:
        scenes.load_scene(ctx, scene, w, h)
        ctx.build_light_sampler(kind)
        ctx.set_render_options(shade_order=order, **opts)
        ctx.reset_accumulation()
        ctx.render(spp)
        return ctx.read_accumulation(w, h)[0]
    finally:
        ctx.close()


def _city():
    scene = scenes.city_scene(seed=5, buildings=60, lights=600, extent=200.0)
    scene["camera"] = ((0.0, 60.0, -95.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), scene["camera"][3])
    return scene


@pytest.mark.parametrize("rng", [gpu.RNG_REFERENCE_STREAM, gpu.RNG_COUNTER])
@pytest.mark.parametrize("which", ["room", "city"])
def test_shade_order_gives_identical_images(rng, which):
    if which == "room":
        scene, kind = scenes.add_random_lights(scenes.room_scene(seed=3), 16, seed=7), gpu.SAMPLER_POWER
    else:
        scene, kind = _city(), gpu.SAMPLER_BVH
    spp = 2 if rng == gpu.RNG_REFERENCE_STREAM else 16
    imgs = [_render(scene, 48, 32, 6, kind, order, spp, sampler=rng, seed=4, russian_roulette_depth=0)
            for order in (gpu.SHADE_ORDER_QUEUE, gpu.SHADE_ORDER_BY_MATERIAL)]
    assert imgs[0].tobytes() == imgs[1].tobytes()
    assert imgs[0][..., :3].sum() > 0


def test_shade_order_guided_identical():
    """Guided shading (fixed guide: training off) in both orders."""
    scene = scenes.room_scene(seed=5)
    imgs = [_render(scene, 24, 24, 5, gpu.SAMPLER_POWER, order, 32, sampler=gpu.RNG_COUNTER, seed=9, guide=True,
                    guide_train=False, guide_spp_per_wave=8)
            for order in (gpu.SHADE_ORDER_QUEUE, gpu.SHADE_ORDER_BY_MATERIAL)]
    assert imgs[0].tobytes() == imgs[1].tobytes()
